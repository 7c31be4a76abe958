"""GPU parity of the drop-in NUFFT against the reference (golden vectors) and the oracle.

Tolerance: relative L2 error <= 1e-5 in float32 (the accuracy bar of the
B200 NUFFT); the golden vectors were produced by the reference itself.
"""

import numpy as np
import pytest
import torch

from conftest import golden_cases

pytestmark = pytest.mark.gpu

TOL = 1e-5


def rel(a, b):
    a = np.asarray(a.detach().cpu() if isinstance(a, torch.Tensor) else a, dtype=np.complex128)
    b = np.asarray(b.detach().cpu() if isinstance(b, torch.Tensor) else b, dtype=np.complex128)
    nb = np.linalg.norm(b.ravel())
    return float(np.linalg.norm((a - b).ravel()) / (nb if nb > 0 else 1.0))


def _p(g, k):
    v = g[k]
    if k == "oversamp":
        return float(v) if v.ndim == 0 else tuple(float(x) for x in v)
    return int(v) if v.ndim == 0 else tuple(int(x) for x in v)


@pytest.fixture(scope="module")
def F():
    import deepmr_b200.fft as F

    return F


@pytest.fixture(params=[True, False], ids=["det", "atomic"])
def grid_mode(request):
    import deepmr_b200.fft as F

    old = F.set_deterministic_gridding(request.param)
    yield request.param
    F.set_deterministic_gridding(old)


@pytest.mark.parametrize("name", golden_cases())
def test_golden_forward_adjoint(name, load_golden, F, grid_mode):
    g = load_golden(name)
    plan = F.plan_nufft(torch.as_tensor(g["coord"]), _p(g, "shape"), _p(g, "width"), _p(g, "oversamp"),
                        device="cuda")
    assert tuple(int(s) for s in plan.os_shape) == tuple(g["plan_os_shape"])
    assert tuple(int(w) for w in plan.width) == tuple(g["plan_width"])
    np.testing.assert_array_equal(np.asarray(plan.beta, np.float32), g["plan_beta"])
    assert plan.interpolator.scale == pytest.approx(float(g["plan_scale"]), rel=1e-12)
    w = g.get("weight")
    img = torch.as_tensor(g["image"]).cuda()
    ksp = torch.as_tensor(g["kspace"]).cuda()
    y = F.apply_nufft(img, plan, weight=w)
    x = F.apply_nufft_adj(ksp, plan, weight=w)
    assert tuple(y.shape) == g["fwd"].shape and y.device.type == "cuda"
    assert tuple(x.shape) == g["adj"].shape
    assert rel(y, g["fwd"]) < TOL, rel(y, g["fwd"])
    assert rel(x, g["adj"]) < TOL, rel(x, g["adj"])


@pytest.mark.parametrize("name", golden_cases(kind="toeplitz"))
def test_golden_toeplitz(name, load_golden, F):
    g = load_golden(name)
    T = F.plan_toeplitz_nufft(torch.as_tensor(g["coord"]), _p(g, "shape"), dcf=g.get("dcf"),
                              width=_p(g, "width"), device="cuda")
    assert tuple(T.value.shape) == g["kernel"].shape
    assert tuple(int(s) for s in T.shape) == tuple(g["kshape"])
    assert rel(T.value, g["kernel"]) < TOL, rel(T.value, g["kernel"])
    out = F.apply_nufft_selfadj(torch.as_tensor(g["image"]).cuda(), T)
    assert rel(out, g["selfadj"]) < TOL, rel(out, g["selfadj"])


def test_numpy_and_cpu_roundtrip(load_golden, F):
    """numpy in -> numpy out; CPU tensor in -> CPU tensor out (nufft.py:517-523)."""
    g = load_golden("radial2d_w4_os125")
    y = F.nufft(g["image"], torch.as_tensor(g["coord"]), width=4, oversamp=1.25)
    assert isinstance(y, np.ndarray) and rel(y, g["fwd"]) < TOL
    x = F.nufft_adj(torch.as_tensor(g["kspace"]), torch.as_tensor(g["coord"]), 24)
    assert isinstance(x, torch.Tensor) and x.device.type == "cpu" and rel(x, g["adj"]) < TOL


def _seeded_case(ndim, n, ncoils, width, os, seed=0):
    from deepmr_b200 import synth

    if ndim == 2:
        c = synth.radial_2d(n * 2, n * 2, n)
    else:
        c = synth.kooshball_3d(n * n // 2, n * 2, n)
    img = synth.complex_gaussian((ncoils,) + (n,) * ndim, seed=seed)
    return c, img


@pytest.mark.parametrize("ndim,n,ncoils,width,os", [(2, 128, 8, 3, 2.0), (2, 64, 3, 4, 1.25),
                                                    (3, 24, 4, 4, 1.25), (3, 16, 2, 6, 2.0),
                                                    (2, 48, 1, 8, 1.5)])
def test_seeded_vs_oracle(ndim, n, ncoils, width, os, F, grid_mode):
    from oracle import nufft_ref as R
    from deepmr_b200 import synth

    c, img = _seeded_case(ndim, n, ncoils, width, os)
    dcf = synth.ramp_dcf(c)
    plan = F.plan_nufft(torch.as_tensor(c), n, width, os, device="cuda")
    oplan = R.plan_nufft(torch.as_tensor(c), n, width, os)
    y = F.apply_nufft(img.cuda(), plan)
    y_ref = R.apply_nufft(img, oplan)
    assert rel(y, y_ref) < TOL
    x = F.apply_nufft_adj(y_ref.cuda(), plan, weight=dcf)
    x_ref = R.apply_nufft_adj(y_ref, oplan, weight=dcf)
    assert rel(x, x_ref) < TOL


def test_deterministic_gridding_is_bitwise_reproducible(F):
    from deepmr_b200 import synth

    c = synth.kooshball_3d(400, 48, 24)
    plan = F.plan_nufft(torch.as_tensor(c), 24, 4, 1.25, device="cuda")
    y = synth.complex_gaussian((3,) + c.shape[:-1], seed=3).cuda()
    old = F.set_deterministic_gridding(True)
    try:
        a = F.apply_nufft_adj(y, plan)
        b = F.apply_nufft_adj(y, plan)
    finally:
        F.set_deterministic_gridding(old)
    assert torch.equal(a, b)


def test_adjointness(F):
    """<A x, y> == <x, A^H y> * G (nufft_adj is the exact adjoint divided by prod(os_shape))."""
    from deepmr_b200 import synth

    c = synth.radial_2d(64, 96, 48)
    plan = F.plan_nufft(torch.as_tensor(c), 48, 4, 1.25, device="cuda")
    x = synth.complex_gaussian((2, 48, 48), seed=1).cuda()
    y = synth.complex_gaussian((2,) + c.shape[:-1], seed=2).cuda()
    G = float(np.prod([int(s) for s in plan.os_shape]))
    lhs = torch.vdot(F.apply_nufft(x, plan).flatten().to(torch.complex128), y.flatten().to(torch.complex128))
    rhs = torch.vdot(x.flatten().to(torch.complex128), F.apply_nufft_adj(y, plan).flatten().to(torch.complex128)) * G
    assert abs(lhs - rhs) / abs(lhs) < 1e-5


def test_frames_and_weights_per_batch(load_golden, F):
    g = load_golden("frames2d")
    plan = F.plan_nufft(torch.as_tensor(g["coord"]), 16, 4, 1.25, device="cuda")
    from oracle import nufft_ref as R

    oplan = R.plan_nufft(torch.as_tensor(g["coord"]), 16, 4, 1.25)
    w = torch.rand(g["kspace"].shape, generator=torch.Generator().manual_seed(0))
    y = F.apply_nufft(torch.as_tensor(g["image"]).cuda(), plan, weight=w)
    assert rel(y, R.apply_nufft(torch.as_tensor(g["image"]), oplan, weight=w)) < TOL
    x = F.apply_nufft_adj(torch.as_tensor(g["kspace"]).cuda(), plan, weight=w)
    assert rel(x, R.apply_nufft_adj(torch.as_tensor(g["kspace"]), oplan, weight=w)) < TOL


def test_empty_batch(F):
    from deepmr_b200 import synth

    c = synth.radial_2d(8, 16, 16)
    plan = F.plan_nufft(torch.as_tensor(c), 16, device="cuda")
    y = F.apply_nufft(torch.zeros(0, 16, 16, dtype=torch.complex64, device="cuda"), plan)
    assert tuple(y.shape) == (0, 8, 16)
    x = F.apply_nufft_adj(torch.zeros(0, 8, 16, dtype=torch.complex64, device="cuda"), plan)
    assert tuple(x.shape) == (0, 16, 16)


def test_nonfinite_coordinate_is_an_error(F):
    from deepmr_b200._lib import DmrError

    c = torch.zeros(1, 4, 2)
    c[0, 1, 0] = float("nan")
    c[0, 2, 1] = 0.3
    with pytest.raises(DmrError):
        F.plan_nufft(c, 8, device="cuda")


# --- ports of the reference's own assertions (tests/fft/test_nufft.py:28-640):
# integer coordinates make every axis Cartesian (width 1, no oversampling), so a
# centred delta maps to all-ones k-space, ones map back to the delta, and the
# Toeplitz self-adjoint of a delta is the delta (rtol = atol = 1e-4 there).
def _cart_coords(ndim, ncontrasts, npix):
    nodes = torch.arange(npix) - npix // 2
    grids = torch.meshgrid(*([nodes] * ndim), indexing="ij")
    coord = torch.stack([g.flatten() for g in grids], -1).to(torch.float32)[None]
    if ncontrasts > 1:
        coord = torch.repeat_interleave(coord[None], ncontrasts, 0)
    return coord


@pytest.mark.parametrize("ndim", [1, 2, 3])
@pytest.mark.parametrize("ncontrasts", [1, 2])
@pytest.mark.parametrize("ncoils,nslices", [(1, 1), (2, 2)])
def test_reference_delta_ones(ndim, ncontrasts, ncoils, nslices, F, npix=4):
    coord = _cart_coords(ndim, ncontrasts, npix)
    lead = [nslices, ncoils] + ([ncontrasts] if ncontrasts > 1 else [])
    img = torch.zeros(lead + [npix] * ndim, dtype=torch.complex64)
    img[(...,) + (npix // 2,) * ndim] = 1.0
    k = F.nufft(img.clone(), coord=coord, device="cuda", width=12)
    np.testing.assert_allclose(k.cpu().numpy(), np.ones(k.shape, np.complex64), rtol=1e-4, atol=1e-4)
    x = F.nufft_adj(torch.ones(k.shape, dtype=torch.complex64), coord=coord, shape=npix, device="cuda", width=12)
    np.testing.assert_allclose(x.cpu().numpy(), img.numpy(), rtol=1e-4, atol=1e-4)
    if ndim > 1:
        T = F.plan_toeplitz_nufft(coord, npix, width=12, device="cuda")
        out = F.apply_nufft_selfadj(img.clone(), T, device="cuda")
        np.testing.assert_allclose(out.cpu().numpy(), img.numpy(), rtol=1e-4, atol=1e-4)


def test_autograd_image_gradient(F):
    """Backward of apply_nufft is apply_nufft_adj (nufft.py:188-209)."""
    from deepmr_b200 import synth

    c = synth.radial_2d(16, 32, 16)
    plan = F.plan_nufft(torch.as_tensor(c), 16, device="cuda")
    x = synth.complex_gaussian((2, 16, 16), seed=4).cuda().requires_grad_(True)
    y = F.apply_nufft(x, plan)
    g = synth.complex_gaussian(tuple(y.shape), seed=5).cuda()
    (y * g.conj()).real.sum().backward()
    expect = F.apply_nufft_adj(g, plan)
    assert rel(x.grad, expect) < 1e-6
