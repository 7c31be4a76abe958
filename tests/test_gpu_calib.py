"""Calibration callers of the NUFFT on the GPU against fixtures of the
reference (tests/golden/make_golden.py ``calib``): non-Cartesian ``find_acs``
(src/deepmr/recon/calib/acs.py:117-152: central samples, adjoint NUFFT at
oversampling 2, centred FFT) in 2D and 3D, and ``espirit_cal``
(src/deepmr/recon/calib/espirit.py:14-148) on 2D radial data, all with the data
on the GPU so the adjoint NUFFT is this library's kernel.

Tolerance: 1e-5 relative L2 (float32), ESPIRiT maps included: their SVDs run
in LAPACK on the host as in the reference's CPU path, so even the per-voxel
phases (which the Fourier resampling to the image grid mixes) agree.
"""

import os

import numpy as np
import pytest
import torch

from deepmr_b200 import calib

pytestmark = pytest.mark.gpu

HERE = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
TOL = 1e-5


def rel(a, b):
    a = np.asarray(torch.as_tensor(a).cpu(), dtype=np.complex128)
    b = np.asarray(torch.as_tensor(b).cpu(), dtype=np.complex128)
    return float(np.linalg.norm((a - b).ravel()) / np.linalg.norm(b.ravel()))


def _case(name):
    d = np.load(os.path.join(HERE, name + ".npz"))
    return {k: (torch.as_tensor(d[k]).cuda() if d[k].ndim else d[k]) for k in d.files}


def test_noncartesian_acs_2d():
    d = _case("calib2d")
    out = calib.find_acs(d["kspace"], [64, 64], d["coord"], d["dcf"])
    assert out.is_cuda and tuple(out.shape) == tuple(d["acs"].shape)
    assert rel(out, d["acs"]) < TOL


def test_noncartesian_acs_3d():
    d = _case("calib3d")
    out = calib.find_acs(d["kspace"], [16, 16, 16], d["coord"], None)
    assert tuple(out.shape) == tuple(d["acs"].shape)
    assert rel(out, d["acs"]) < TOL


def test_espirit_maps_2d_radial():
    d = _case("calib2d")
    maps, cal = calib.espirit_cal(d["kspace"], coord=d["coord"], dcf=d["dcf"], shape=int(d["shape"]))
    ref = d["maps"]
    assert maps.is_cuda and tuple(maps.shape) == tuple(ref.shape)
    assert rel(cal, d["cal"]) < TOL
    assert rel(maps, ref) < TOL
    pm = maps * maps[:, :, :1].conj()
    pr = ref * ref[:, :, :1].conj()
    assert rel(pm, pr) < TOL
    assert rel(maps.abs(), ref.abs()) < TOL
    # the maps are unit-norm over coils (rss normalisation)
    norm = (maps.abs() ** 2).sum(2).sqrt()
    assert torch.allclose(norm, torch.ones_like(norm), atol=1e-5)
