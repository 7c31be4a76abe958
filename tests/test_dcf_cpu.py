"""Voronoi density compensation on the CPU against fixtures of the reference
(tests/golden/make_golden.py ``dcf``; src/deepmr/_design/grad/utils/dcf.py:75-160):
2D radial with the centre sampled by every spoke (repeated points), one
spiral interleaf as uniformly rotated shots, rotated interleaves with edge
extrapolation, and a 3D kooshball (the reference's 3D cell measure).

Tolerance: 1e-6 relative L2 (float32; the Voronoi diagram is Qhull's in both,
the measured restatement agrees bitwise on these cases).
"""

import numpy as np
import pytest
import torch

from conftest import golden_cases
from deepmr_b200 import dcf

TOL = 1e-6


def rel(a, b):
    a, b = np.asarray(a, np.float64), np.asarray(b, np.float64)
    return float(np.linalg.norm(a - b) / np.linalg.norm(b))


@pytest.mark.parametrize("name", golden_cases(kind="dcf"))
def test_voronoi_vs_reference(load_golden, name):
    d = load_golden(name)
    w = dcf.voronoi(d["coord"], nshots=int(d["nshots"]), fix_edge=bool(d["fix_edge"]), ratio=float(d["ratio"]))
    assert w.dtype == np.float32 and w.shape == d["dcf"].shape
    assert rel(w, d["dcf"]) < TOL


def test_voronoi_torch_and_complex_inputs(load_golden):
    d = load_golden("dcf_radial2d")
    ref = d["dcf"]
    w = dcf.voronoi(torch.as_tensor(d["coord"]))
    assert isinstance(w, torch.Tensor) and w.dtype == torch.float32
    assert rel(w.numpy(), ref) < TOL
    c = d["coord"][..., 0] + 1j * d["coord"][..., 1]
    assert rel(dcf.voronoi(c), ref) < TOL


def test_voronoi_centre_weight_and_repeated_points(load_golden):
    """The sample nearest k = 0 weighs 1 / nshots; repeated centre samples
    other than the first are weighted as the reference weights them."""
    d = load_golden("dcf_spiral_shots")
    w = dcf.voronoi(d["coord"], nshots=6)
    k0 = np.argmin((d["coord"] ** 2).sum(-1))
    assert abs(float(w[k0]) - 1.0 / 6) < 1e-6
    assert np.all(np.isfinite(w)) and np.all(w > 0)


def test_analytical_and_angular():
    rng = np.random.default_rng(0)
    c = rng.standard_normal((3, 5, 3))
    np.testing.assert_allclose(dcf.analytical_dcf(c), np.sqrt((c**2).sum(-1)))
    wi = rng.random(5)
    axes = np.array([0, 1, 2])
    out = dcf.angular_compensation(wi, c, axes)
    expect = np.stack([wi * np.linalg.norm(np.delete(c[n], axes[n], axis=-1), axis=-1) for n in range(3)])
    np.testing.assert_allclose(out, expect / expect.sum(), rtol=1e-12)
