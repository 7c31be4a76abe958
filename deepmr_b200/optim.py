"""Conjugate gradient of the reference's CG-SENSE callers, on this library.

Drop-in for ``deepmr.optim.cg_solve`` / ``CGStep`` (src/deepmr/optim/cg.py:16-221):
same arguments, same iteration (x0 = 0, r = p = AHy, alpha = rsold / <p, AHA p>,
beta = rsnew / rsold), same stopping rule (every batch element's residual
norm sqrt(rsnew) below ``tol``) and the same ``(output, history)`` return.

When the normal operator is the fused SENSE + Toeplitz operator of
``deepmr_b200.linops`` (what ``EncodingOp(..., toeplitz=True)`` builds for one
set of coil maps) and no history is recorded, the whole solve stays on the
GPU: ``dmr_cg_init`` / ``dmr_cg_step`` with float64 inner products reduced in a
fixed order (the reference uses complex64 sums), the host reading the
residual only when ``tol`` asks for it. Any other operator runs the same
iteration with torch operations on the operator's device.
"""

__all__ = ["cg_solve", "CGStep"]

import math

import numpy as np
import torch
import torch.nn as nn

from . import linops as _linops
from . import recon as _recon


class CGStep(nn.Module):
    """One CG iteration (src/deepmr/optim/cg.py:150-221); ``forward(x)`` returns
    the next iterate, ``check_convergence()`` the stopping test."""

    def __init__(self, AHA, AHy, ndim=None, tol=None):
        super().__init__()
        self.ndim = getattr(AHA, "ndim", None) or ndim
        self.AHA = AHA
        self.AHy = AHy
        self.r = AHy.clone()
        self.p = self.r
        self.rsold = self.dot(self.r, self.r)
        self.rsnew = None
        self.tol = tol

    def dot(self, a, b):
        d = (a.conj() * b).reshape(*a.shape[: -self.ndim], -1).sum(-1)
        for _ in range(self.ndim):
            d = d[..., None]
        return d

    def forward(self, x):
        q = self.AHA(self.p)
        alpha = self.rsold / self.dot(self.p, q)
        out = x + self.p * alpha
        self.r = self.r + q * (-alpha)
        self.rsnew = torch.real(self.dot(self.r, self.r))
        self.p = self.r + self.p * (self.rsnew / self.rsold)
        self.rsold = self.rsnew
        return out

    def check_convergence(self):
        return self.tol is not None and bool((self.rsnew.sqrt() < self.tol).all())


def _fused_normal(AHA):
    """The fused SENSE + Toeplitz operator behind AHA (plain or plus lamda I), else None."""
    if isinstance(AHA, _linops.SenseGramOp):
        return AHA
    if isinstance(AHA, _linops.Compose) and AHA.fused is not None:
        return AHA.fused
    return None


@torch.no_grad()
def cg_solve(input, AHA, niter=10, device=None, tol=1e-4, lamda=0.0, ndim=None, save_history=False,
             verbose=False):
    """Solve AHA x = input (input = A^H y) by ``niter`` CG iterations from x = 0
    (src/deepmr/optim/cg.py:16-147). Returns ``(output, history)``."""
    isnumpy = isinstance(input, np.ndarray)
    x_in = torch.as_tensor(input)
    idevice = x_in.device
    fused = _fused_normal(AHA)
    if fused is not None and not save_history:
        op = fused.with_lamda(lamda) if lamda else fused
        dev = _recon._nufft.compute_device(device if device is not None and torch.device(device).type == "cuda"
                                           else (idevice if idevice.type == "cuda" else None))
        normal = op.normal(dev)
        ahy = x_in.to(dev, torch.complex64).reshape(normal.ishape).contiguous()
        cg = _recon.CGState(ahy, normal)
        cg.init()
        for _ in range(niter):
            cg.step()
            if tol is not None and tol > 0 and math.sqrt(max(cg.residual(), 0.0)) < tol:
                break
        out = cg.x.reshape(x_in.shape).to(idevice if device is None else device)
        return (out.numpy(force=True) if isnumpy else out), []
    dev = idevice if device is None else torch.device(device)
    x_in = x_in.to(dev)
    if isinstance(AHA, _linops.Linop):
        AHA = AHA.to(dev)
    elif not callable(AHA):
        AHA = torch.as_tensor(AHA, dtype=x_in.dtype, device=dev)
    ahy = x_in.clone()
    if lamda != 0.0:
        if isinstance(AHA, _linops.Linop):
            op = AHA + lamda * _linops.Identity(AHA.ndim)
        elif callable(AHA):
            op = lambda v: AHA(v) + lamda * v  # noqa: E731
        else:
            op = lambda v: AHA @ v + lamda * v  # noqa: E731
    else:
        op = AHA if callable(AHA) else (lambda v: AHA @ v)  # noqa: E731
    step = CGStep(op, ahy, ndim, tol)
    x = 0 * x_in
    out = x
    history = []
    for _ in range(niter):
        out = step(x)
        if step.check_convergence():
            break
        x = out.clone()
        if save_history:
            r = out - ahy
            history.append(0.5 * torch.linalg.norm(r).item() ** 2 + lamda * torch.linalg.norm(out).item() ** 2)
    out = out.to(dev)
    return (out.numpy(force=True) if isnumpy else out), history
