"""Host logic of the drop-in operator algebra and CG (deepmr_b200.linops /
deepmr_b200.optim), on the CPU with small dense operators.

The reference's semantics (src/deepmr/linops/base.py:10-247,
src/deepmr/optim/cg.py:16-221): composition applies right to left, the
adjoint of a sum / product is the sum / reversed product of adjoints, and
cg_solve runs niter CG iterations from zero with complex64 inner products
over all but the batch axes, stopping once every residual norm is below tol.
"""

import numpy as np
import torch

from deepmr_b200 import linops, optim


class MatOp(linops.Linop):
    """y = M x over the last axis (ndim = 1)."""

    def __init__(self, m):
        super().__init__(1)
        self.m = torch.as_tensor(m)

    def forward(self, x):
        return x @ self.m.T

    def _adjoint_linop(self):
        return MatOp(self.m.conj().T)


def _rand(shape, seed):
    g = torch.Generator().manual_seed(seed)
    return torch.complex(torch.randn(shape, generator=g), torch.randn(shape, generator=g))


def test_algebra_matches_matrices():
    a, b = _rand((5, 5), 0), _rand((5, 5), 1)
    A, B = MatOp(a), MatOp(b)
    x = _rand((3, 5), 2)
    torch.testing.assert_close((A * B)(x), x @ (a @ b).T)
    torch.testing.assert_close((A + B)(x), x @ (a + b).T)
    torch.testing.assert_close((A - B)(x), x @ (a - b).T)
    torch.testing.assert_close((2.0 * A)(x), x @ (2 * a).T)
    torch.testing.assert_close((A * B).H(x), x @ (a @ b).conj())
    torch.testing.assert_close((A + B).H(x), x @ (a + b).conj())
    torch.testing.assert_close(((1j) * A).H(x), x @ ((1j) * a).conj())
    torch.testing.assert_close(linops.Identity(1)(x), x)
    torch.testing.assert_close((A * x), A(x))


def test_cg_solve_generic_path():
    """cg_solve with a Linop normal operator solves the Hermitian system; batch
    elements are independent and lamda adds a Tikhonov term."""
    m = _rand((6, 6), 3)
    h = m.conj().T @ m + 6.0 * torch.eye(6)
    AHA = MatOp(h.to(torch.complex64))
    rhs = _rand((2, 6), 4).to(torch.complex64)
    # (past exact convergence the residual is 0 and the next step divides 0 / 0,
    # as in the reference, so the iteration count stays near the system size)
    x, hist = optim.cg_solve(rhs, AHA, niter=8, tol=0.0, save_history=True)
    ref = torch.linalg.solve(h.to(torch.complex128), rhs.to(torch.complex128).T).T
    assert np.allclose(x.numpy(), ref.numpy(), rtol=1e-4, atol=1e-5)
    assert len(hist) == 8
    x2, _ = optim.cg_solve(rhs, AHA, niter=8, tol=0.0, lamda=0.5)
    ref2 = torch.linalg.solve((h + 0.5 * torch.eye(6)).to(torch.complex128), rhs.to(torch.complex128).T).T
    assert np.allclose(x2.numpy(), ref2.numpy(), rtol=1e-4, atol=1e-5)


def test_cg_solve_stops_at_tol_and_numpy_roundtrip():
    h = torch.diag(torch.tensor([1.0, 2.0, 3.0, 4.0], dtype=torch.complex64))
    rhs = np.ones((1, 4), np.complex64)
    x, _ = optim.cg_solve(rhs, MatOp(h), niter=50, tol=1e-3)
    assert isinstance(x, np.ndarray)
    assert np.allclose(x, [[1.0, 0.5, 1.0 / 3.0, 0.25]], atol=1e-3)
    # the reference's CGStep iterate after one step from x = 0: alpha r
    step = optim.CGStep(MatOp(h), torch.as_tensor(rhs), ndim=1)
    x1 = step(torch.zeros((1, 4), dtype=torch.complex64))
    r = torch.as_tensor(rhs)
    alpha = (r.conj() * r).sum() / (r.conj() * (r @ h.T)).sum()
    torch.testing.assert_close(x1, r * alpha)


def test_sense_ops_shapes_2d_and_fusion_detection():
    maps = _rand((1, 1, 3, 4, 4), 5).to(torch.complex64)
    C = linops.SenseOp(2, maps, multicontrast=False)
    x = _rand((1, 4, 4), 6).to(torch.complex64)
    y = C(x)
    assert tuple(y.shape) == (1, 1, 3, 4, 4)
    torch.testing.assert_close(C.H(y), (maps.conj() * maps * x[None, :, None]).sum(-3).sum(0))
    # <C x, y> = <x, C^H y>
    yy = _rand(tuple(y.shape), 7).to(torch.complex64)
    lhs = torch.vdot(C(x).flatten(), yy.flatten())
    rhs = torch.vdot(x.flatten(), C.H(yy).flatten())
    assert abs(lhs - rhs) < 1e-4 * abs(lhs)
    # a chain that is not C^H T C stays unfused
    assert linops.Compose([C.H, linops.Identity(2), C]).fused is None
