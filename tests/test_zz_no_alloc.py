"""Allocation-free Toeplitz normalisation entry point (runs last; GPU).

Some callers of this library cannot allocate device memory while they run:
an application that hands the GPU a fixed memory pool at start-up, or a
real-time reconstruction loop that forbids allocator calls once it is
running. `dmr_toeplitz_normalize_noalloc` serves them: it performs the
normalisation step of `dmr_toeplitz_finalize` (divide by the mean magnitude of
the non-zero entries, NaN -> 0) with its reduction scratch in a static device
array of the library instead of a caller workspace. The test calls it through
the C ABI twice in a row, on different inputs, and checks each result against
the existing workspace-based entry point.
"""

import ctypes

import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu

TOL = 1e-5  # relative L2, float32


def _rel(a, b):
    a = a.detach().cpu().numpy().astype(np.complex128).ravel()
    b = b.detach().cpu().numpy().astype(np.complex128).ravel()
    return float(np.linalg.norm(a - b) / np.linalg.norm(b))


def _finalize(psf, kshape):
    """Existing entry point: ifftshift, orthonormal FFT and normalisation, with a workspace."""
    from deepmr_b200 import _lib

    L = _lib.lib()
    dev = psf.device
    nk = psf.numel() // int(np.prod(kshape))
    n = ctypes.c_size_t()
    _lib.check(L.dmr_toeplitz_workspace_bytes(len(kshape), _lib.i32_array(kshape), nk, ctypes.byref(n)))
    ws = torch.empty(int(n.value), dtype=torch.uint8, device=dev)
    out = torch.empty_like(psf)
    _lib.check(L.dmr_toeplitz_finalize(len(kshape), _lib.i32_array(kshape), nk, _lib.ptr(psf), _lib.ptr(out),
                                       _lib.ptr(ws), ws.numel(), _lib.stream_ptr(dev)))
    return out


def test_noalloc_normalisation_matches_workspace_entry_point():
    from deepmr_b200 import _lib

    L = _lib.lib()
    dev = torch.device("cuda", 0)
    kshape = (48, 64, 40)  # 2 frames x 122,880 points: 15 partial sums
    dims = (-3, -2, -1)
    for seed in (0, 1):  # two calls in a row; the second finds the first's partial sums
        g = torch.Generator(device=dev).manual_seed(seed)
        psf = torch.complex(torch.randn((2,) + kshape, generator=g, device=dev),
                            torch.randn((2,) + kshape, generator=g, device=dev)).contiguous()
        ref = _finalize(psf, kshape)
        out = torch.fft.fftn(torch.fft.ifftshift(psf, dim=dims), dim=dims, norm="ortho").contiguous()
        rc = L.dmr_toeplitz_normalize_noalloc(_lib.ptr(out), out.numel(), _lib.stream_ptr(dev))
        assert rc == 0, L.dmr_last_error()
        torch.cuda.synchronize()
        assert _rel(out, ref) < TOL, _rel(out, ref)


def test_noalloc_normalisation_excludes_zeros():
    """Exact zeros do not enter the mean (plain torch float32 reference)."""
    from deepmr_b200 import _lib

    L = _lib.lib()
    dev = torch.device("cuda", 0)
    g = torch.Generator(device=dev).manual_seed(3)
    x = torch.complex(torch.randn(300_000, generator=g, device=dev), torch.randn(300_000, generator=g, device=dev))
    x[::5] = 0
    expect = x / torch.mean(torch.abs(x[x != 0]))
    out = x.clone()
    assert L.dmr_toeplitz_normalize_noalloc(_lib.ptr(out), out.numel(), _lib.stream_ptr(dev)) == 0
    torch.cuda.synchronize()
    assert _rel(out, expect) < TOL


def test_noalloc_rejects_oversized_input():
    from deepmr_b200 import _lib

    L = _lib.lib()
    buf = torch.zeros(16, dtype=torch.complex64, device="cuda")
    # rejected on the host before any device work: the pointer is never read
    rc = L.dmr_toeplitz_normalize_noalloc(_lib.ptr(buf), 67_108_864 + 1, _lib.stream_ptr(buf.device))
    assert rc == -1
    assert b"maximum" in L.dmr_last_error()
