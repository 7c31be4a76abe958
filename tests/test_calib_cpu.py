"""Calibration helpers on the CPU against fixtures of the reference
(tests/golden/make_golden.py ``calib``): Cartesian ``find_acs``
(src/deepmr/recon/calib/acs.py:54-114), the signal helpers ``resample``,
``rss``, ``fermi`` (src/deepmr/_signal/resize.py:105-211, subspace.py:9-70,
filter.py:8-100), and the ESPIRiT stage (espirit.py:152-223) run on the
reference's own calibration data, so only the NUFFT is left for the GPU test.

Tolerance: 1e-5 relative L2 (float32), for the ESPIRiT maps directly (phases
included: the SVDs are LAPACK's, as the reference's) and through the
phase-invariant products m_c * conj(m_0).
"""

import os

import numpy as np
import torch

from deepmr_b200 import calib

HERE = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
TOL = 1e-5


def rel(a, b):
    a = np.asarray(torch.as_tensor(a).cpu(), dtype=np.complex128)
    b = np.asarray(torch.as_tensor(b).cpu(), dtype=np.complex128)
    return float(np.linalg.norm((a - b).ravel()) / np.linalg.norm(b.ravel()))


def phase_free(maps, coil_axis):
    m = torch.as_tensor(maps)
    return m * m.narrow(coil_axis, 0, 1).conj()


def test_cartesian_acs():
    d = np.load(os.path.join(HERE, "calib_cart.npz"))
    out = calib.find_acs(torch.as_tensor(d["kspace"]))
    assert tuple(out.shape) == d["acs"].shape
    assert rel(out, d["acs"]) < TOL


def test_signal_helpers():
    d = np.load(os.path.join(HERE, "calib_cart.npz"))
    x, xr = torch.as_tensor(d["x"]), torch.as_tensor(d["xr"])
    assert rel(calib.resample(x, [24, 24]), d["x_up"]) < TOL
    assert rel(calib.resample(x, [12, 14]), d["x_down"]) < TOL
    up = calib.resample(xr, [24, 24])
    assert not up.is_complex() and rel(up, d["xr_up"]) < TOL
    assert rel(calib.rss(x, axis=0), d["x_rss"]) < TOL
    assert rel(calib.fermi(2, 24, 10), d["fermi"]) < TOL
    # numpy in, numpy out
    assert isinstance(calib.resample(d["x"], [24, 24]), np.ndarray)


def test_resize_pad_crop():
    x = torch.arange(5.0)
    assert calib.resize(torch.tensor([0, 1, 0]), [5]).tolist() == [0, 0, 1, 0, 0]
    assert calib.resize(x, [3]).tolist() == [1.0, 2.0, 3.0]
    assert calib.resize(x[None], [3]).shape == (1, 3)


def test_espirit_stage_on_reference_calibration_data():
    d = np.load(os.path.join(HERE, "calib2d.npz"))
    n = int(d["shape"])
    maps = calib._espirit(torch.as_tensor(d["acs"]).clone(), 6, 24, 0.02, 0.0)[[0]]
    maps = calib.resample(maps, [n, n])
    maps = (maps / calib.rss(maps, axis=1, keepdim=True)[[0]]).swapaxes(1, 2)
    ref = d["maps"]
    assert tuple(maps.shape) == ref.shape
    assert rel(maps, ref) < TOL
    assert rel(phase_free(maps, 2), phase_free(ref, 2)) < TOL
    assert rel(maps.abs(), np.abs(ref)) < TOL
