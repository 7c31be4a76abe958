"""ORACLE — test infrastructure only, never part of the product path.

CPU restatement of the reference's CG-SENSE with a Toeplitz normal operator:
CGStep / cg_solve (src/deepmr/optim/cg.py:16-221, complex64 torch arithmetic
as in the reference), SenseOp / SenseAdjointOp (src/deepmr/linops/coil.py:11-205),
NUFFTGramOp (src/deepmr/linops/nufft.py:189-241, width 6) and the zero-filled
AHy = E^H(dcf**0.5 y) of recon_lstsq (src/deepmr/recon/alg/classic_recon.py:153-156),
built on the oracle NUFFT of nufft_ref.py.
"""

import torch

from . import nufft_ref as R


def _dot(a, b):
    # CGStep.dot for one image (no batch axes): sum(conj(a) * b) in complex64
    return (a.conj() * b).reshape(-1).sum()


def cg_solve(ahy, AHA, niter):
    """cg_solve with tol disabled (cg.py:16-147): niter CG steps from x = 0."""
    r = ahy.clone()
    p = r
    rsold = _dot(r, r)
    x = 0 * ahy
    for _ in range(niter):
        q = AHA(p)
        alpha = rsold / _dot(p, q)
        x = x + p * alpha
        r = r + q * (-alpha)
        rsnew = torch.real(_dot(r, r))
        p = r + p * (rsnew / rsold)
        rsold = rsnew
    return x


def sense_normal(x, maps, gram, lamda=0.0):
    """C^H T C x (+ lamda x) with T the Toeplitz self-adjoint (linop.py:145-146)."""
    y = R.apply_selfadj(maps * x, gram)
    out = (maps.conj() * y).sum(0)
    return out + lamda * x if lamda else out


def cg_sense(kspace, coord, shape, maps, dcf, niter, lamda=0.0, width=4, gram_width=6):
    plan = R.plan_nufft(torch.as_tensor(coord), shape, width, 1.25)
    gram = R.plan_toeplitz(torch.as_tensor(coord), shape, dcf=dcf, width=gram_width)
    w = torch.as_tensor(dcf, dtype=torch.float32) ** 0.5
    img = R.apply_nufft_adj(w * torch.as_tensor(kspace), plan, weight=w)
    ahy = (torch.as_tensor(maps).conj() * img).sum(0)
    return cg_solve(ahy, lambda v: sense_normal(v, torch.as_tensor(maps), gram, lamda), niter), ahy, gram
