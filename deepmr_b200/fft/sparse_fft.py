"""Cartesian sparse FFT on B200 — drop-in for ``deepmr.fft.sparse_fft``.

Reference: prepare_sampling / plan_toeplitz_fft / apply_sparse_fft /
apply_sparse_ifft / apply_sparse_fft_selfadj (src/deepmr/fft/sparse_fft.py:21-503)
and the sampling / zero-fill kernels (src/deepmr/fft/_sparse/dense2sparse.py,
sparse2dense.py, toeplitz.py).

A sparse FFT is a NUFFT whose every axis is Cartesian: sampled index ``i`` of
an axis of size ``N`` is the centred grid coordinate ``i - N//2``, which the
NUFFT plan detects as Cartesian (width 1, no oversampling, no apodisation,
unit kernel scale). So the forward is the centred FFT (unnormalised) followed
by sampling, the adjoint zero-fills (summing repeated indices) and applies
the centred inverse FFT (1/N), exactly the reference's order, and the
low-rank subspace variants come with the NUFFT's. The self-adjoint operator
multiplies the uncentred orthonormal FFT by the normalised sample count of
every k-space point (the ifftshifted zero-fill of ones,
src/deepmr/fft/_sparse/toeplitz.py).
"""

__all__ = [
    "prepare_sampling",
    "plan_toeplitz_fft",
    "apply_sparse_fft",
    "apply_sparse_ifft",
    "apply_sparse_fft_selfadj",
    "SparseSampling",
]

from dataclasses import dataclass

import numpy as np
import torch

from .. import _lib
from . import nufft as _nufft
from . import toeplitz as _toeplitz


@dataclass
class SparseSampling:
    """Sampling mask (fields of the reference's Sampling, _sparse/plan.py:101-107)."""

    index: tuple  # per axis (z, y, x) order, each (nframes, npts) int
    dshape: tuple
    ishape: tuple
    ndim: int
    device: str
    plan: object = None  # the all-Cartesian NUFFT plan that runs it

    def to(self, device):
        if device != self.device:
            self.plan.to(device)
            self.device = device
        return self


def _indexes(indexes):
    idx = torch.as_tensor(indexes)
    if idx.is_floating_point():
        idx = idx.round()
    return idx.to(torch.int64)


def prepare_sampling(indexes, shape, device="cpu"):
    """Sampling mask from integer k-space indexes (reference: sparse_fft.py:21-68).

    indexes ``(ncontrasts, nviews, nsamples, ndim)`` in ``[0, N_i)``, axes (x, y[, z]);
    shape: grid size, scalar or (z, y, x).
    """
    idx = _indexes(indexes)
    ndim = int(idx.shape[-1])
    shape = [int(shape)] * ndim if np.isscalar(shape) else [int(s) for s in shape][-ndim:]
    n_xyz = np.asarray(shape[::-1])
    if idx.numel() and (int(idx.min()) < 0 or bool((idx >= torch.as_tensor(n_xyz)).any())):
        raise ValueError(f"sampling indexes must lie in [0, N) for grid shape {tuple(shape)}")
    coord = (idx - torch.as_tensor(n_xyz // 2)).to(torch.float32)
    plan = _nufft.plan_nufft(coord, shape, width=4, oversamp=1.0, device=device)
    if any(int(w) != 1 for w in plan.width):
        raise RuntimeError("sparse sampling plan is not Cartesian on every axis")
    ishape = list(idx.shape[:-1])
    while len(ishape) < 3:
        ishape = [1] + ishape
    nframes = ishape[0]
    flat = idx.reshape(nframes, -1, ndim)
    index = tuple(flat[..., a] for a in range(ndim))[::-1]
    return SparseSampling(index, tuple(shape), tuple(ishape[1:]), ndim, device, plan)


def apply_sparse_fft(image, sampling_mask, basis_adjoint=None, weight=None, device=None, threadsperblock=128):
    """Sparse FFT (reference: sparse_fft.py:140-180): centred FFT, then sampling."""
    return _nufft.apply_nufft(image, sampling_mask.plan, basis_adjoint, weight, device, threadsperblock)


def apply_sparse_ifft(kspace, sampling_mask, basis=None, weight=None, device=None, threadsperblock=128):
    """Inverse sparse FFT (reference: sparse_fft.py:222-257): zero-fill, then centred inverse FFT."""
    return _nufft.apply_nufft_adj(kspace, sampling_mask.plan, basis, weight, device, threadsperblock)


def plan_toeplitz_fft(coord, shape, basis=None, device="cpu"):
    """Self-adjoint kernel of the sparse FFT (reference: sparse_fft.py:71-95,
    _sparse/toeplitz.py:15-113): the sample count at every k-space point,
    ifftshifted, divided by the mean non-zero count, NaN -> 0."""
    if basis is not None:
        raise NotImplementedError("low-rank subspace sparse Toeplitz (basis) is not implemented by deepmr_b200")
    mask = prepare_sampling(coord, shape, device)
    ip = mask.plan.interpolator
    dev = ip.device
    # zero-fill of ones (deterministic: counts are exact small integers either
    # way); the gridded array is stored in FFT order = the ifftshift of the
    # centred counts, and the all-Cartesian plan has unit kernel scale
    ones = torch.ones((int(ip.total),), dtype=torch.complex64, device=dev)
    counts = torch.empty((1, ip.nframes) + tuple(ip.dshape), dtype=torch.complex64, device=dev)
    with torch.cuda.device(dev):
        _lib.check(_lib.lib().dmr_grid(ip.handle, _lib.ptr(ones), 0, _lib.ptr(counts), 1, None, 0, 1,
                                       _lib.stream_ptr(dev)))
    kern = counts[0].real if ip.nframes > 1 else counts[0, 0].real
    # normalised by the mean non-zero magnitude, NaN -> 0 (_sparse/toeplitz.py:107-111)
    nz = kern[kern != 0]
    kern = torch.nan_to_num(kern / (nz.abs().mean() if nz.numel() else float("nan")))
    return _toeplitz.GramMatrix(kern, tuple(mask.dshape), mask.ndim, device, False)


def apply_sparse_fft_selfadj(image, toeplitz_kern, device=None, threadsperblock=128):
    """Self-adjoint sparse FFT (reference: sparse_fft.py:284-311, 453-503):
    uncentred orthonormal FFT, times the sample counts, inverse FFT."""
    isnumpy = isinstance(image, np.ndarray)
    image = _nufft._as_cfloat(image)
    if device is not None:
        toeplitz_kern.to(device)
    out = _toeplitz.apply_toeplitz(image, toeplitz_kern)
    return out.numpy(force=True) if isnumpy else out
