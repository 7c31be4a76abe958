"""Centred FFT / inverse FFT — ``deepmr.fft.fft`` / ``ifft`` (reference:
src/deepmr/fft/fft.py:9-180), so the reference's callers (calibration,
Cartesian recon) run unchanged when this package stands in for ``deepmr.fft``.
torch's FFT (cuFFT on CUDA tensors) with the fftshift pair around it."""

__all__ = ["fft", "ifft"]

import numpy as np
import torch


def _axes(axes, ndim):
    if axes is None:
        return tuple(range(ndim))
    return tuple(a % ndim for a in axes)


def _centred(x, axes, norm, centered, inverse):
    isnumpy = isinstance(x, np.ndarray)
    t = torch.as_tensor(x)
    ax = _axes(axes, t.ndim)
    op = torch.fft.ifftn if inverse else torch.fft.fftn
    if centered:
        out = torch.fft.fftshift(op(torch.fft.ifftshift(t, dim=ax), dim=ax, norm=norm), dim=ax)
    else:
        out = op(t, dim=ax, norm=norm)
    return np.asarray(out) if isnumpy else out


def fft(input, axes=None, norm="ortho", centered=True):
    """Centred FFT over `axes` (all if None)."""
    return _centred(input, axes, norm, centered, False)


def ifft(input, axes=None, norm="ortho", centered=True):
    """Centred inverse FFT over `axes` (all if None)."""
    return _centred(input, axes, norm, centered, True)
