"""Centred fft / ifft of the package (the reference's src/deepmr/fft/fft.py
semantics: fftshift(fftn(ifftshift(x))) with norm, over the given axes), and
the chunking of the pinned-host pipeline."""

import numpy as np
import pytest
import torch


def test_centred_fft_matches_numpy_and_round_trips():
    import deepmr_b200.fft as F

    rng = np.random.default_rng(0)
    x = (rng.standard_normal((3, 6, 5)) + 1j * rng.standard_normal((3, 6, 5))).astype(np.complex64)
    ax = (-2, -1)
    ref = np.fft.fftshift(np.fft.fftn(np.fft.ifftshift(x, axes=ax), axes=ax, norm="ortho"), axes=ax)
    y = F.fft(x, axes=ax)
    assert isinstance(y, np.ndarray)
    np.testing.assert_allclose(y, ref, rtol=1e-5, atol=1e-5)
    np.testing.assert_allclose(F.ifft(y, axes=ax), x, rtol=1e-5, atol=1e-5)
    t = F.fft(torch.as_tensor(x), axes=(1,), norm=None, centered=False)
    np.testing.assert_allclose(t.numpy(), np.fft.fft(x, axis=1), rtol=1e-4, atol=1e-4)


@pytest.mark.parametrize("batch,min_chunk,expect", [(32, 1, (16, 2)), (32, 2, (16, 2)), (32, 8, (4, 8)),
                                                     (5, 1, (5, 1)), (40, 1, (14, 3)), (16, 8, (2, 8)),
                                                     (12, 8, (1, 12)), (1, 1, (1, 1))])
def test_host_pipeline_chunks(batch, min_chunk, expect):
    """Chunking of the pinned-host pipeline: at most 16 chunks, at least
    min_chunk items each (3D adjoints use 2, deterministic ones 8), the last
    one possibly shorter."""
    import importlib

    N = importlib.import_module("deepmr_b200.fft.nufft")
    nch, cb = N._pipeline_chunks(batch, min_chunk)
    assert (nch, cb) == expect
    assert (nch - 1) * cb < batch <= nch * cb and nch <= N.PIPELINE_CHUNKS
