"""GPU parity of the low-rank subspace NUFFT (basis / basis_adjoint).

Square bases are pinned against vectors produced by the reference itself
(tests/golden/lowrank*.npz; the reference runs only when ncoeff equals the
frame count). Fewer coefficients than frames — the case subspace MRF uses and
the reference cannot run — is checked against the oracle, which restates the
reference's kernels through the linearity of the pipeline, and by the adjoint
identity. Tolerance: relative L2 error <= 1e-5 in float32.
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


@pytest.fixture(scope="module")
def F():
    import deepmr_b200.fft as F

    return F


@pytest.fixture(params=[True, False], ids=["det", "atomic"])
def grid_mode(request, F):
    old = F.set_deterministic_gridding(request.param)
    yield request.param
    F.set_deterministic_gridding(old)


def _p(g, k):
    v = g[k]
    if k == "oversamp":
        return float(v) if v.ndim == 0 else tuple(float(x) for x in v)
    return int(v) if v.ndim == 0 else tuple(int(x) for x in v)


@pytest.mark.parametrize("name", golden_cases(kind="lowrank"))
def test_lowrank_golden(name, load_golden, F, grid_mode):
    g = load_golden(name)
    plan = F.plan_nufft(torch.as_tensor(g["coord"]), _p(g, "shape"), _p(g, "width"), _p(g, "oversamp"),
                        device="cuda")
    w = g.get("weight")
    y = F.apply_nufft(torch.as_tensor(g["image"]).cuda(), plan, basis_adjoint=g["basis_adjoint"], weight=w)
    x = F.apply_nufft_adj(torch.as_tensor(g["kspace"]).cuda(), plan, basis=g["basis"], weight=w)
    assert tuple(y.shape) == g["fwd"].shape and tuple(x.shape) == g["adj"].shape
    assert rel(y, g["fwd"]) < TOL
    assert rel(x, g["adj"]) < TOL


def _frames_2d(nf, n):
    from deepmr_b200 import synth

    return np.stack([synth.radial_2d(8, 2 * n, n, angle_offset=0.37 * f) for f in range(nf)]).astype(np.float32)


def _frames_3d(nf, n):
    from deepmr_b200 import synth

    return np.stack([synth.kooshball_3d(n * n // 2, 2 * n, n) * (1.0 - 0.05 * f) for f in range(nf)]).astype(
        np.float32)


@pytest.mark.parametrize("ndim,nf,ncoeff,nbatch", [(2, 6, 2, 3), (2, 5, 5, 1), (3, 4, 3, 9), (3, 3, 1, 2)])
def test_lowrank_fewer_coefficients_vs_oracle(ndim, nf, ncoeff, nbatch, F, grid_mode):
    from oracle import nufft_ref as R
    from deepmr_b200 import synth

    n = 24 if ndim == 2 else 20
    coord = _frames_2d(nf, n) if ndim == 2 else _frames_3d(nf, n)
    g = torch.Generator().manual_seed(ndim * 10 + nf)
    basis = torch.complex(torch.randn(ncoeff, nf, generator=g), torch.randn(ncoeff, nf, generator=g))
    ba = basis.conj().t()
    img = synth.complex_gaussian((nbatch, ncoeff) + (n,) * ndim, seed=1)
    ksp = synth.complex_gaussian((nbatch, nf) + coord.shape[1:-1], seed=2)
    dcf = torch.as_tensor(synth.ramp_dcf(coord.reshape(-1, ndim)).reshape(coord.shape[:-1]))
    c = torch.as_tensor(coord)
    plan = F.plan_nufft(c, n, 4, 1.25, device="cuda")
    oplan = R.plan_nufft(c, n, 4, 1.25)
    y = F.apply_nufft(img.cuda(), plan, basis_adjoint=ba)
    assert tuple(y.shape) == (nbatch, nf) + coord.shape[1:-1]
    assert rel(y, R.apply_nufft_lowrank(img, oplan, ba)) < TOL
    x = F.apply_nufft_adj(ksp.cuda(), plan, basis=basis, weight=dcf.cuda())
    assert tuple(x.shape) == (nbatch, ncoeff) + (n,) * ndim
    assert rel(x, R.apply_nufft_adj_lowrank(ksp, oplan, basis, weight=dcf)) < TOL


def test_lowrank_adjoint_identity(F):
    """<A x, y> = G <x, A^H y> with basis = basis_adjoint^H (nufft_adj = adjoint / G)."""
    from deepmr_b200 import synth

    n, nf, ncoeff = 20, 5, 3
    coord = _frames_2d(nf, n)
    g = torch.Generator().manual_seed(11)
    ba = torch.complex(torch.randn(nf, ncoeff, generator=g), torch.randn(nf, ncoeff, generator=g))
    plan = F.plan_nufft(torch.as_tensor(coord), n, 4, 1.25, device="cuda")
    x = synth.complex_gaussian((2, ncoeff, n, n), seed=3).cuda()
    y = synth.complex_gaussian((2, nf) + coord.shape[1:-1], seed=4).cuda()
    ax = F.apply_nufft(x, plan, basis_adjoint=ba)
    ahy = F.apply_nufft_adj(y, plan, basis=ba.conj().t())
    G = float(np.prod([int(s) for s in plan.os_shape]))
    lhs = torch.vdot(ax.flatten().to(torch.complex128), y.flatten().to(torch.complex128))
    rhs = G * torch.vdot(x.flatten().to(torch.complex128), ahy.flatten().to(torch.complex128))
    assert abs(lhs - rhs) / abs(lhs) < 1e-5


def test_lowrank_identity_basis_equals_frames(F):
    """An identity basis reproduces the plain multi-frame NUFFT."""
    from deepmr_b200 import synth

    n, nf = 16, 4
    coord = _frames_2d(nf, n)
    plan = F.plan_nufft(torch.as_tensor(coord), n, 4, 1.25, device="cuda")
    x = synth.complex_gaussian((3, nf, n, n), seed=5).cuda()
    eye = np.eye(nf, dtype=np.float32)  # real basis, numpy input
    assert rel(F.apply_nufft(x, plan, basis_adjoint=eye), F.apply_nufft(x, plan)) < 1e-6
    y = synth.complex_gaussian((3, nf) + coord.shape[1:-1], seed=6).cuda()
    assert rel(F.apply_nufft_adj(y, plan, basis=eye), F.apply_nufft_adj(y, plan)) < 1e-6


def test_lowrank_bad_basis_shape(F):
    n, nf = 16, 4
    plan = F.plan_nufft(torch.as_tensor(_frames_2d(nf, n)), n, 4, 1.25, device="cuda")
    x = torch.zeros((1, 2, n, n), dtype=torch.complex64, device="cuda")
    with pytest.raises(ValueError):
        F.apply_nufft(x, plan, basis_adjoint=np.ones((nf, 3), np.float32))
