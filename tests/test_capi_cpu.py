"""CPU-only checks of the C ABI library and the host-side logic (no GPU calls)."""

import ctypes
import os
import re

import numpy as np
import pytest
import torch

from conftest import ROOT, golden_cases

HEADER = os.path.join(ROOT, "include", "deepmr_b200.h")


def declared_symbols():
    text = open(HEADER).read()
    return sorted(set(re.findall(r"\b(dmr_[a-z0-9_]+)\s*\(", text)))


def test_header_matches_binding_table():
    from deepmr_b200 import _lib

    assert declared_symbols() == sorted(_lib.SYMBOLS)


def test_library_loads_and_exports_every_symbol():
    from deepmr_b200 import _lib

    L = _lib.lib()  # loads without a GPU (CUDA runtime is linked statically)
    for name in declared_symbols():
        assert hasattr(L, name), name
    assert L.dmr_version() >= 100
    assert L.dmr_launch_count() >= 0


def test_error_strings_without_device():
    from deepmr_b200 import _lib

    L = _lib.lib()
    # argument validation happens before any device work
    rc = L.dmr_plan_create(4, None, None, None, None, None, None, None, 1, None, None,
                           ctypes.byref(ctypes.c_void_p()))
    assert rc == -1
    assert b"ndim" in L.dmr_last_error()
    with pytest.raises(_lib.DmrError):
        _lib.check(rc)


def test_frames_layout():
    from deepmr_b200.fft.nufft import _frames

    c = torch.zeros(3, 5, 7, 2)
    flat, offs, ishape, ndim = _frames(c)
    assert flat.shape == (105, 2) and ishape == (5, 7) and ndim == 2
    assert offs.tolist() == [0, 35, 70, 105]
    flat, offs, ishape, ndim = _frames(torch.zeros(9, 3))
    assert ishape == (1, 9) and offs.tolist() == [0, 9]
    flat, offs, ishape, ndim = _frames([torch.zeros(4, 2), torch.zeros(2, 3, 2), torch.zeros(1, 2)])
    assert ishape is None and offs.tolist() == [0, 4, 10, 11]


@pytest.mark.parametrize("name", golden_cases())
def test_plan_parameters_match_reference(name, load_golden):
    """Host-side plan arithmetic (beta, Cartesian override, os_shape) vs the reference."""
    from oracle import nufft_ref as R

    g = load_golden(name)
    ndim = int(g["ndim"])
    width = g["width"]
    oversamp = g["oversamp"]
    w = np.asarray([int(width)] * ndim if width.ndim == 0 else width, dtype=np.int16)
    o = np.asarray([float(oversamp)] * ndim if oversamp.ndim == 0 else oversamp, dtype=np.float32)
    beta = np.pi * (((w / o) * (o - 0.5)) ** 2 - 0.8) ** 0.5
    s = g["shape"]
    shape = np.asarray([int(s)] * ndim if s.ndim == 0 else s, dtype=np.int16)[-ndim:]
    is_cart = R.cartesian_axes(g["coord"], shape)
    o[is_cart] = 1.0
    w[is_cart] = 1
    np.testing.assert_array_equal(np.ceil(o * shape).astype(np.int32), g["plan_os_shape"])
    np.testing.assert_array_equal(w.astype(np.int32), g["plan_width"])
    np.testing.assert_array_equal(np.asarray(beta, np.float32), g["plan_beta"])


def test_synthetic_generators_are_seeded():
    from deepmr_b200 import synth

    a = synth.kooshball_3d(10, 8, 16)
    b = synth.kooshball_3d(10, 8, 16)
    assert np.array_equal(a, b) and a.shape == (10, 8, 3)
    assert np.abs(a).max() <= 8.0
    r = synth.radial_2d(4, 6, 32)
    assert r.shape == (4, 6, 2) and np.all(r >= -16) and np.all(r < 16)
    x = synth.complex_gaussian((3, 4), seed=1)
    assert torch.equal(x, synth.complex_gaussian((3, 4), seed=1))
    m = synth.coil_maps(4, (8, 8), seed=0)
    np.testing.assert_allclose((np.abs(m) ** 2).sum(0), 1.0, rtol=1e-5)


@pytest.mark.skipif(torch.cuda.is_available(), reason="checks the no-GPU behaviour")
def test_public_api_fails_loudly_without_cuda():
    """Every entry point reaches the CUDA requirement and raises (no CPU fallback)."""
    import deepmr_b200.fft as F

    c = torch.zeros(1, 4, 2)
    img = torch.zeros(2, 8, 8, dtype=torch.complex64)
    calls = [
        lambda: F.plan_nufft(c, 8),
        lambda: F.nufft(img, c),
        lambda: F.nufft_adj(torch.zeros(2, 1, 4, dtype=torch.complex64), c, 8),
        lambda: F.plan_toeplitz_nufft(c, 8),
        lambda: F.plan_toeplitz_nufft(c, 8, dcf=torch.ones(1, 4)),
    ]
    for call in calls:
        with pytest.raises(RuntimeError, match="CUDA"):
            call()


def test_modules_bind_the_nufft_submodule():
    """deepmr_b200.fft.nufft is the one-shot function (as in the reference);
    internal users must hold the submodule."""
    import types

    from deepmr_b200 import recon
    from deepmr_b200.fft import graphs, toeplitz  # noqa: F401

    assert isinstance(recon._nufft, types.ModuleType)
    assert callable(recon._nufft.plan_nufft)
