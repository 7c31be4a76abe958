"""Pin the oracle (CPU restatement) against golden outputs of the reference.

The golden vectors were produced by running the reference implementation
itself (tests/golden/make_golden.py). The oracle is only trusted as a checker
for the CUDA library because these tests pass.
"""

import numpy as np
import pytest
import torch

from conftest import golden_cases
from oracle import nufft_ref as R

# The oracle sums in the reference's loop order without fastmath contraction;
# the remaining differences are fp32 rounding.
TOL = 2e-6


def _width(g):
    w = g["width"]
    return int(w) if w.ndim == 0 else tuple(int(v) for v in w)


def _os(g):
    o = g["oversamp"]
    return float(o) if o.ndim == 0 else tuple(float(v) for v in o)


def _shape(g):
    s = g["shape"]
    return int(s) if s.ndim == 0 else tuple(int(v) for v in s)


@pytest.mark.parametrize("name", golden_cases())
def test_oracle_plan_params(name, load_golden):
    g = load_golden(name)
    plan = R.plan_nufft(torch.as_tensor(g["coord"]), _shape(g), _width(g), _os(g))
    np.testing.assert_array_equal(np.asarray(plan.os_shape, np.int32), g["plan_os_shape"])
    np.testing.assert_array_equal(np.asarray(plan.width, np.int32), g["plan_width"])
    np.testing.assert_array_equal(np.asarray(plan.beta, np.float32), g["plan_beta"])
    np.testing.assert_array_equal(np.asarray(plan.oversamp, np.float32), g["plan_oversamp"])
    assert plan.interpolator.scale == pytest.approx(float(g["plan_scale"]), rel=1e-14)


@pytest.mark.parametrize("name", golden_cases())
def test_oracle_forward_adjoint(name, load_golden):
    g = load_golden(name)
    plan = R.plan_nufft(torch.as_tensor(g["coord"]), _shape(g), _width(g), _os(g))
    w = g.get("weight")
    y = R.apply_nufft(torch.as_tensor(g["image"]), plan, weight=w)
    x = R.apply_nufft_adj(torch.as_tensor(g["kspace"]), plan, weight=w)
    assert tuple(y.shape) == g["fwd"].shape
    assert tuple(x.shape) == g["adj"].shape
    assert R.rel_l2(y, g["fwd"]) < TOL
    assert R.rel_l2(x, g["adj"]) < TOL


@pytest.mark.parametrize("name", golden_cases(kind="toeplitz"))
def test_oracle_toeplitz(name, load_golden):
    g = load_golden(name)
    T = R.plan_toeplitz(torch.as_tensor(g["coord"]), _shape(g), dcf=g.get("dcf"), width=_width(g))
    assert tuple(T.value.shape) == g["kernel"].shape
    assert R.rel_l2(T.value, g["kernel"]) < TOL
    out = R.apply_selfadj(torch.as_tensor(g["image"]), T)
    assert R.rel_l2(out, g["selfadj"]) < TOL


@pytest.mark.parametrize("name", golden_cases(kind="lowrank"))
def test_oracle_lowrank(name, load_golden):
    """Low-rank subspace NUFFT (square basis: the reference runs only then)."""
    g = load_golden(name)
    plan = R.plan_nufft(torch.as_tensor(g["coord"]), _shape(g), _width(g), _os(g))
    w = g.get("weight")
    y = R.apply_nufft_lowrank(torch.as_tensor(g["image"]), plan, g["basis_adjoint"], weight=w)
    x = R.apply_nufft_adj_lowrank(torch.as_tensor(g["kspace"]), plan, g["basis"], weight=w)
    assert tuple(y.shape) == g["fwd"].shape and tuple(x.shape) == g["adj"].shape
    assert R.rel_l2(y, g["fwd"]) < TOL
    assert R.rel_l2(x, g["adj"]) < TOL


@pytest.mark.parametrize("name", golden_cases(kind="sparse"))
def test_oracle_sparse_fft(name, load_golden):
    """Cartesian sparse FFT: forward, adjoint (repeated indexes), self-adjoint."""
    g = load_golden(name)
    shape = int(g["shape"]) if g["shape"].ndim == 0 else tuple(int(s) for s in g["shape"])
    w = g.get("weight")
    y = R.sparse_fft(g["image"], g["indexes"], shape, g.get("basis_adjoint"), weight=w)
    x = R.sparse_ifft(g["kspace"], g["indexes"], shape, g.get("basis"), weight=w)
    assert y.shape == g["fwd"].shape and x.shape == g["adj"].shape
    assert R.rel_l2(y, g["fwd"]) < TOL
    assert R.rel_l2(x, g["adj"]) < TOL
    if "kernel" in g:
        k = R.sparse_toeplitz_kernel(g["indexes"], shape)
        np.testing.assert_allclose(k, g["kernel"], rtol=1e-6, atol=1e-7)
        assert R.rel_l2(R.sparse_selfadj(g["image"], k, int(g["ndim"])), g["selfadj"]) < TOL


def test_oracle_vs_nudft_small():
    """The reference operator approximates the exact NUDFT (expected error ~1e-2 at W3/os2)."""
    from deepmr_b200 import synth

    c = synth.radial_2d(8, 16, 16)
    img = synth.complex_gaussian((16, 16), seed=1).numpy()
    plan = R.plan_nufft(torch.as_tensor(c), 16, 6, 2.0)
    y = R.apply_nufft(torch.as_tensor(img), plan).numpy()
    yd = R.nudft(img, c.reshape(-1, 2), (16, 16)).reshape(y.shape)
    # fit the global scale the reference leaves unnormalised
    s = np.vdot(y.ravel(), yd.ravel()) / np.vdot(y.ravel(), y.ravel())
    assert abs(abs(s) - 1) < 0.02
    assert R.rel_l2(s * y, yd) < 1e-4


@pytest.mark.parametrize("name", golden_cases(kind="cgsense"))
def test_oracle_cgsense(name, load_golden):
    """The oracle's CG-SENSE (oracle/cg_ref.py) against the reference's own
    EncodingOp + cg_solve: AHy to float32 rounding, the 20-iteration solution
    within 1e-5 (CG steps amplify float32 rounding differences)."""
    from oracle import cg_ref

    g = load_golden(name)
    x, ahy, _ = cg_ref.cg_sense(torch.as_tensor(g["kspace"]), g["coord"], int(g["shape"]),
                                torch.as_tensor(g["maps"]), g["dcf"], int(g["niter"]))
    assert R.rel_l2(ahy, g["ahy"]) < TOL
    assert R.rel_l2(x, g["x_cg"]) < 1e-5
