"""Non-Cartesian NUFFT on B200 — drop-in for ``deepmr.fft``'s NUFFT API.

One-shot ``nufft`` / ``nufft_adj`` and ``sparse_fft`` / ``sparse_ifft``
(reference: src/deepmr/fft/__init__.py:31-286), the plan/apply functions of
``deepmr.fft.nufft`` and of ``deepmr.fft.sparse_fft``.
"""

import torch

from . import nufft as _nufft
from . import toeplitz as _toeplitz
from .fft import fft, ifft  # noqa: F401
from .nufft import (  # noqa: F401
    NUFFTPlan,
    apply_nufft,
    apply_nufft_adj,
    apply_nufft_selfadj,
    plan_nufft,
    plan_toeplitz_nufft,
)
from .graphs import CapturedNUFFT, frames_concat, frames_split  # noqa: F401
from . import sparse_fft as _sparse_fft
from .sparse_fft import (  # noqa: F401
    SparseSampling,
    apply_sparse_fft,
    apply_sparse_fft_selfadj,
    apply_sparse_ifft,
    plan_toeplitz_fft,
    prepare_sampling,
)
from .nufft import traj_grad  # noqa: F401
from .toeplitz import GramMatrix  # noqa: F401

__all__ = [
    "fft",
    "ifft",
    "nufft",
    "nufft_adj",
    "plan_nufft",
    "apply_nufft",
    "apply_nufft_adj",
    "plan_toeplitz_nufft",
    "apply_nufft_selfadj",
    "NUFFTPlan",
    "GramMatrix",
    "set_deterministic_gridding",
    "deterministic_gridding",
    "release_scratch",
    "set_deterministic_scratch_limit",
    "set_status_check",
    "traj_grad",
    "CapturedNUFFT",
    "frames_split",
    "frames_concat",
    "sparse_fft",
    "sparse_ifft",
    "prepare_sampling",
    "plan_toeplitz_fft",
    "apply_sparse_fft",
    "apply_sparse_ifft",
    "apply_sparse_fft_selfadj",
    "SparseSampling",
]


def set_deterministic_gridding(flag=True):
    """Select the gridding kernel used by the adjoint NUFFT.

    True: bitwise reproducible — 3D plans grid on the tensor cores with
    every work item (a bin, or 2048 samples of a heavier one) storing its
    region's partial sums, which a gather then adds per grid point in a fixed
    order (the partial sums take 2 KB per work item and coil in the library's
    scratch pool: see release_scratch); other plans with one owner per grid
    point or per tile.
    False (default): grid-point additions with atomics (summation order may
    vary between runs, results agree to float32 rounding).
    Returns the previous setting.
    """
    old = _nufft.DETERMINISTIC_GRIDDING
    _nufft.DETERMINISTIC_GRIDDING = bool(flag)
    return old


def release_scratch(device=None):
    """Give the memory that the library's scratch pool holds beyond what is in
    use back to the device (default: the current CUDA device). Synchronises
    the device."""
    import torch

    from .. import _lib

    if isinstance(device, int):
        dev = device
    else:
        idx = None if device is None else torch.device(device).index
        dev = torch.cuda.current_device() if idx is None else idx
    _lib.check(_lib.lib().dmr_scratch_release(int(dev)))


def set_deterministic_scratch_limit(nbytes):
    """Largest scratch (bytes) that deterministic 3D tensor-core gridding may
    take (2 KB per gridding work item and coil); a call that would need more,
    or for which the device has no memory left, runs on the register-tile
    kernel instead (deterministic, slower, small scratch). 0 removes the
    limit (the default). Process-wide; returns the previous limit."""
    from .. import _lib

    if nbytes < 0:
        raise ValueError("nbytes must be >= 0")
    return int(_lib.lib().dmr_det_scratch_limit(int(nbytes)))


def deterministic_gridding():
    """Current gridding mode (see set_deterministic_gridding)."""
    return _nufft.DETERMINISTIC_GRIDDING


def set_status_check(flag=True):
    """Also check the gridding's device status (a bounded wait that ran out
    raises DmrError DMR_ERR_TIMEOUT) after adjoint calls whose result stays on
    the GPU, at one stream synchronisation per call. Calls whose result returns
    to the host are always checked. Returns the previous setting."""
    return _nufft.set_status_check(flag)


def nufft(image, coord, shape=None, basis_adjoint=None, device="cpu", threadsperblock=128,
          width=4, oversamp=1.25):
    """N-dimensional NUFFT, plan + apply (reference: src/deepmr/fft/__init__.py:145-218).

    image ``(..., [ncontrasts,] ny, nx)`` or ``(..., [ncontrasts,] nz, ny, nx)``;
    coord ``(ncontrasts, nviews, nsamples, ndim)`` in grid units, (x, y[, z]).
    Returns kspace ``(..., [ncontrasts,] nviews, nsamples)`` on the input's device.
    """
    ndim = coord.shape[-1] if not isinstance(coord, (list, tuple)) else coord[0].shape[-1]
    if shape is None:
        shape = image.shape[-ndim:]
    if isinstance(coord, torch.Tensor) and coord.requires_grad and torch.is_grad_enabled():
        # differentiable w.r.t. the trajectory as well (extension)
        if basis_adjoint is not None:
            raise NotImplementedError("trajectory gradient with a low-rank basis")
        return _nufft.NUFFTTraj.apply(_nufft._as_cfloat(image), coord, shape, width, oversamp, device, None)
    plan = _nufft.plan_nufft(coord, shape, width, oversamp, device)
    return _nufft.apply_nufft(image, plan, basis_adjoint, threadsperblock=threadsperblock)


def nufft_adj(kspace, coord, shape, basis=None, device="cpu", threadsperblock=128, width=4,
              oversamp=1.25):
    """N-dimensional adjoint NUFFT, plan + apply (reference: src/deepmr/fft/__init__.py:221-286)."""
    if isinstance(coord, torch.Tensor) and coord.requires_grad and torch.is_grad_enabled():
        if basis is not None:
            raise NotImplementedError("trajectory gradient with a low-rank basis")
        return _nufft.NUFFTAdjTraj.apply(_nufft._as_cfloat(kspace), coord, shape, width, oversamp, device, None)
    plan = _nufft.plan_nufft(coord, shape, width, oversamp, device)
    return _nufft.apply_nufft_adj(kspace, plan, basis, threadsperblock=threadsperblock)


def sparse_fft(image, indexes, basis_adjoint=None, device="cpu", threadsperblock=128):
    """Sparse FFT, plan + apply (reference: src/deepmr/fft/__init__.py:31-86)."""
    ndim = indexes.shape[-1]
    mask = _sparse_fft.prepare_sampling(indexes, image.shape[-ndim:], device)
    return _sparse_fft.apply_sparse_fft(image, mask, basis_adjoint, threadsperblock=threadsperblock)


def sparse_ifft(kspace, indexes, shape, basis=None, device="cpu", threadsperblock=128):
    """Inverse sparse FFT, plan + apply (reference: src/deepmr/fft/__init__.py:89-142)."""
    mask = _sparse_fft.prepare_sampling(indexes, shape, device)
    return _sparse_fft.apply_sparse_ifft(kspace, mask, basis, threadsperblock=threadsperblock)
