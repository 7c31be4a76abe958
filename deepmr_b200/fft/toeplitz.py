"""Toeplitz kernel planning and application — drop-in for ``deepmr.fft.toeplitz``.

Reference: plan_toeplitz (src/deepmr/fft/toeplitz.py:15-157), GramMatrix
(toeplitz.py:165-195) and the plain branch of apply_toeplitz
(src/deepmr/fft/_interp/toeplitz.py:84-87). The point-spread function comes
from this library's adjoint NUFFT on the 2x grid; the FFT, ifftshift,
normalisation by the mean non-zero magnitude and NaN removal run in one C ABI
call (dmr_toeplitz_finalize); the self-adjoint application is one call
(dmr_toeplitz_apply).
"""

__all__ = ["plan_toeplitz", "GramMatrix", "apply_toeplitz"]

import ctypes
from dataclasses import dataclass

import numpy as np
import torch

from .. import _lib


@dataclass
class GramMatrix:
    """Toeplitz kernel (fields of the reference's GramMatrix, toeplitz.py:165-171)."""

    value: torch.Tensor
    shape: tuple
    ndim: int
    device: str
    islowrank: bool

    def to(self, device):
        if device != self.device:
            d = torch.device(device)
            if d.type == "cuda":
                self.value = self.value.to(d)
            self.device = device
        return self


def _workspace(ndim, kshape, batch, dev):
    n = ctypes.c_size_t()
    with torch.cuda.device(dev):
        _lib.check(_lib.lib().dmr_toeplitz_workspace_bytes(
            ndim, _lib.i32_array(kshape), int(batch), ctypes.byref(n)))
    return torch.empty(int(n.value), dtype=torch.uint8, device=dev)


def plan_toeplitz(coord, shape, basis=None, dcf=None, width=6, device="cpu"):
    """Compute the Toeplitz kernel of A^H A (reference: toeplitz.py:15-157)."""
    # deferred import (nufft imports this module); import names from the
    # submodule: the package attribute `nufft` is the one-shot function
    from .nufft import _apply_nufft_adj, compute_device, detect_cartesian, plan_nufft

    if basis is not None:
        raise NotImplementedError(
            "low-rank subspace Toeplitz (basis) is not implemented by deepmr_b200"
        )
    dev = compute_device(device)
    coord = torch.as_tensor(coord, dtype=torch.float32)
    ndim = coord.shape[-1]
    oversamp = np.asarray([2.0] * ndim)
    if np.isscalar(shape):
        shape = np.asarray([shape] * ndim, dtype=np.int16)
    else:
        shape = np.asarray(shape, dtype=np.int16)[-ndim:]
    if dcf is None:
        dcf = torch.ones(coord.shape[:-1], dtype=torch.float32, device=dev)
    else:
        dcf = torch.as_tensor(dcf).to(dev)
    delta = torch.ones(list(coord.shape[:-1]), dtype=torch.float32, device=dev)

    is_cart = detect_cartesian(coord.reshape(-1, ndim).to(dev).contiguous(), shape)
    oversamp[is_cart] = 1.0
    kshape = np.ceil(oversamp * shape).astype(np.int16)

    # point-spread function on the 2x grid (toeplitz.py:122-129); the plan casts
    # the float64 product back to float32
    coord2 = coord * torch.as_tensor(oversamp)
    plan = plan_nufft(coord2, kshape, width, 1.25, dev)
    # deterministic gridding: the kernel (planned once) is bitwise reproducible
    psf = _apply_nufft_adj(dcf * delta, plan, None, None, None, 128, deterministic=True)
    psf = psf.to(dev).contiguous()

    K = [int(k) for k in kshape]
    nk = int(np.prod(psf.shape[:-ndim]))
    kern = torch.empty_like(psf)
    ws = _workspace(ndim, K, nk, dev)
    with torch.cuda.device(dev):
        _lib.check(_lib.lib().dmr_toeplitz_finalize(
            ndim, _lib.i32_array(K), nk, _lib.ptr(psf), _lib.ptr(kern), _lib.ptr(ws), ws.numel(),
            _lib.stream_ptr(dev)))
    if kern.shape[0] == 1:  # toeplitz.py:135-136
        kern = kern[0]
    return GramMatrix(kern, tuple(kshape), ndim, device, False)


def apply_toeplitz(image, toeplitz_kernel):
    """Self-adjoint NUFFT by Toeplitz convolution (nufft.py:609-669).

    image ``(..., [ncontrasts,] *shape)``; returned on the input's device.
    """
    ndim = toeplitz_kernel.ndim
    kval = toeplitz_kernel.value
    dev = kval.device
    if dev.type != "cuda":
        raise RuntimeError("Toeplitz kernel must live on a CUDA device")
    x = image.to(dev).contiguous()
    ishape = [int(s) for s in x.shape[-ndim:]]
    K = [int(k) for k in toeplitz_kernel.shape]
    nk = int(np.prod(kval.shape[:-ndim])) if kval.dim() > ndim else 1
    batch = int(np.prod(x.shape[:-ndim]))
    out = torch.empty(x.shape, dtype=torch.complex64, device=dev)
    if batch > 0:
        if nk > 1 and (x.dim() < ndim + 1 or x.shape[-ndim - 1] != nk):
            raise ValueError(f"image {tuple(x.shape)} does not broadcast against kernel {tuple(kval.shape)}")
        kv = kval.to(torch.complex64).contiguous()
        ws = _workspace(ndim, K, batch, dev)
        with torch.cuda.device(dev):
            _lib.check(_lib.lib().dmr_toeplitz_apply(
                ndim, _lib.i32_array(K), _lib.i32_array(ishape), _lib.ptr(kv), nk, _lib.ptr(x),
                int(not x.is_complex()), _lib.ptr(out), batch, _lib.ptr(ws), ws.numel(),
                _lib.stream_ptr(dev)))
    from .nufft import _to_origin

    return _to_origin(out, image)
