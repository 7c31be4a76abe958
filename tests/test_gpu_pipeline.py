"""Chunked host pipeline of apply_nufft / apply_nufft_adj for pinned CPU inputs.

A pinned, contiguous host input is split along its flattened batch; copies in,
compute and copies out of successive chunks overlap on three streams. The
result must equal the same call on a device-resident input (float32 rounding:
relative L2 error <= 1e-6; the chunked adjoint may pick a different gridding
schedule for a smaller batch), come back pinned on the host, and handle the
last short chunk, frames, real inputs and per-batch weights.
"""

import importlib

import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu

TOL = 1e-6


def rel(a, b):
    a = a.detach().cpu().to(torch.complex128)
    b = b.detach().cpu().to(torch.complex128)
    return float(torch.linalg.norm((a - b).flatten()) / torch.linalg.norm(b.flatten()))


@pytest.fixture(scope="module")
def F():
    import deepmr_b200.fft as F

    return F


@pytest.fixture
def spy(F, monkeypatch):
    """Force the pipeline at any size and count the chunked calls."""
    N = importlib.import_module("deepmr_b200.fft.nufft")

    calls = []
    orig = N._pipelined

    def wrapped(x_h, out_h, batch, dev, run, ws_bytes, *rest):
        calls.append(batch)
        return orig(x_h, out_h, batch, dev, run, ws_bytes, *rest)

    monkeypatch.setattr(N, "PIPELINE_MIN_BYTES", 0)
    monkeypatch.setattr(N, "_pipelined", wrapped)
    return calls


def _plan2d(F, nf=1, n=32):
    from deepmr_b200 import synth

    if nf == 1:
        coord = synth.radial_2d(24, 2 * n, n)
    else:
        coord = np.stack([synth.radial_2d(12, 2 * n, n, angle_offset=0.3 * f) for f in range(nf)])
    return F.plan_nufft(torch.as_tensor(coord.astype(np.float32)), n, 4, 1.25, device="cuda"), coord


@pytest.mark.parametrize("nbatch", [2, 5, 11, 16])
@pytest.mark.parametrize("det", [False, True], ids=["atomic", "det"])
def test_pipeline_matches_device_path(F, spy, nbatch, det):
    from deepmr_b200 import synth

    plan, coord = _plan2d(F)
    n = 32
    img = synth.complex_gaussian((nbatch, n, n), seed=nbatch)
    ksp = synth.complex_gaussian((nbatch,) + coord.shape[:-1], seed=nbatch + 1)
    dcf = torch.as_tensor(synth.ramp_dcf(coord.reshape(-1, 2)).reshape(coord.shape[:-1]))
    old = F.set_deterministic_gridding(det)
    try:
        y_h = F.apply_nufft(img.pin_memory(), plan)
        x_h = F.apply_nufft_adj(ksp.pin_memory(), plan, weight=dcf)
        y_d = F.apply_nufft(img.cuda(), plan)
        x_d = F.apply_nufft_adj(ksp.cuda(), plan, weight=dcf.cuda())
    finally:
        F.set_deterministic_gridding(old)
    assert spy == [nbatch, nbatch]
    for h, d in ((y_h, y_d), (x_h, x_d)):
        assert h.device.type == "cpu" and h.is_pinned() and h.shape == d.shape
        assert rel(h, d) < TOL


def test_pipeline_frames_real_and_batch_weights(F, spy):
    from deepmr_b200 import synth

    nf, n = 3, 32
    plan, coord = _plan2d(F, nf, n)
    img = synth.complex_gaussian((2, 3, nf, n, n), seed=7).real.contiguous()  # real input, batch (2, 3)
    wb = torch.rand((2, 3, nf) + coord.shape[1:-1], generator=torch.Generator().manual_seed(8))
    y_h = F.apply_nufft(img.pin_memory(), plan, weight=wb)
    y_d = F.apply_nufft(img.cuda(), plan, weight=wb.cuda())
    assert tuple(y_h.shape) == (2, 3, nf) + coord.shape[1:-1]
    assert rel(y_h, y_d) < TOL
    ksp = synth.complex_gaussian((2, 3, nf) + coord.shape[1:-1], seed=9)
    x_h = F.apply_nufft_adj(ksp.pin_memory(), plan, weight=wb)
    x_d = F.apply_nufft_adj(ksp.cuda(), plan, weight=wb.cuda())
    assert tuple(x_h.shape) == (2, 3, nf, n, n)
    assert rel(x_h, x_d) < TOL
    assert spy == [6, 6]


def test_pipeline_not_taken_for_pageable_or_single(F, spy):
    from deepmr_b200 import synth

    plan, coord = _plan2d(F)
    img = synth.complex_gaussian((4, 32, 32), seed=3)
    y = F.apply_nufft(img, plan)  # pageable
    y1 = F.apply_nufft(img[:1].clone().pin_memory(), plan)  # batch 1
    assert spy == []
    assert y.device.type == "cpu" and rel(y1, y[:1]) < TOL


def test_pipeline_default_threshold_3d(F):
    """3D calls above the default size run chunked (the adjoint in chunks of at
    least 8 coils) and match the device-input calls."""
    from deepmr_b200 import synth
    N = importlib.import_module("deepmr_b200.fft.nufft")

    n = 64
    coord = synth.kooshball_3d(8192, 2 * n, n).astype(np.float32)
    plan = F.plan_nufft(torch.as_tensor(coord), n, 4, 1.25, device="cuda")
    ksp = synth.complex_gaussian((16,) + coord.shape[:-1], seed=5)
    assert ksp.numel() * 8 >= N.PIPELINE_MIN_BYTES
    x_h = F.apply_nufft_adj(ksp.pin_memory(), plan)
    x_d = F.apply_nufft_adj(ksp.cuda(), plan)
    assert x_h.is_pinned() and rel(x_h, x_d) < TOL
    img = synth.complex_gaussian((8, n, n, n), seed=6)
    y_h = F.apply_nufft(img.pin_memory(), plan)
    assert y_h.is_pinned() and rel(y_h, F.apply_nufft(img.cuda(), plan)) < TOL
