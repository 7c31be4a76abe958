"""Frames of uneven length in one plan / one launch, and CUDA-graph capture (GPU).

Uneven frames have no reference counterpart (the reference needs rectangular
(ncontrasts, nviews, nsamples) coordinates, src/deepmr/fft/_interp/plan.py:66-77);
each frame is checked against the oracle run on that frame alone.
"""

import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu

TOL = 1e-5


def rel(a, b):
    a = np.asarray(torch.as_tensor(a).detach().cpu(), dtype=np.complex128).ravel()
    b = np.asarray(torch.as_tensor(b).detach().cpu(), dtype=np.complex128).ravel()
    return float(np.linalg.norm(a - b) / np.linalg.norm(b))


def _spiral_frames(nframes, n, seed=0):
    from deepmr_b200 import synth

    rng = np.random.default_rng(seed)
    lengths = rng.integers(80, 121, nframes)
    return [synth.spiral_2d(int(L), n, rotation=f * synth.GOLDEN_ANGLE)[0] for f, L in enumerate(lengths)]


@pytest.mark.parametrize("deterministic", [False, True])
def test_uneven_frames_vs_oracle_per_frame(deterministic):
    import deepmr_b200.fft as F
    from deepmr_b200 import synth
    from oracle import nufft_ref as R

    n, ncoils, nframes = 48, 3, 20
    coords = _spiral_frames(nframes, n)
    plan = F.plan_nufft(coords, n, 4, 1.25, device="cuda")
    img = synth.complex_gaussian((ncoils, nframes, n, n), seed=1)
    old = F.set_deterministic_gridding(deterministic)
    try:
        y = F.apply_nufft(img.cuda(), plan)
        total = sum(c.shape[0] for c in coords)
        assert tuple(y.shape) == (ncoils, total)
        ks = synth.complex_gaussian((ncoils, total), seed=2)
        x = F.apply_nufft_adj(ks.cuda(), plan)
    finally:
        F.set_deterministic_gridding(old)
    assert tuple(x.shape) == (ncoils, nframes, n, n)
    parts_y = F.frames_split(y, plan)
    parts_k = F.frames_split(ks, plan)
    for f, c in enumerate(coords):
        op = R.plan_nufft(torch.as_tensor(c), n, 4, 1.25)
        assert rel(parts_y[f], R.apply_nufft(img[:, f], op)) < TOL
        # the oracle takes one frame's samples as (coils, nviews=1, nsamples)
        assert rel(x[:, f], R.apply_nufft_adj(parts_k[f].reshape(ncoils, 1, -1), op)) < TOL


def test_captured_graph_matches_eager():
    import deepmr_b200.fft as F
    from deepmr_b200 import synth

    c = synth.radial_2d(64, 96, 48)
    plan = F.plan_nufft(torch.as_tensor(c), 48, 4, 1.25, device="cuda")
    dcf = torch.as_tensor(synth.ramp_dcf(c)).reshape(-1)
    op = F.CapturedNUFFT(plan, batch=4, weight=dcf, deterministic=True)
    img = synth.complex_gaussian((4, 48, 48), seed=3).cuda()
    ksp = synth.complex_gaussian((4,) + c.shape[:-1], seed=4).cuda()
    old = F.set_deterministic_gridding(True)
    try:
        for _ in range(2):  # replays are repeatable
            y = op.forward(img).clone()
            x = op.adjoint(ksp).clone()
            assert torch.equal(y, F.apply_nufft(img, plan, weight=dcf.reshape(c.shape[:-1])))
            assert torch.equal(x, F.apply_nufft_adj(ksp, plan, weight=dcf.reshape(c.shape[:-1])))
        # inputs written into the static buffers by the caller: no copy, same results
        op.x_in.copy_(img)
        op.y_in.copy_(ksp)
        assert torch.equal(op.forward().clone(), y)
        assert torch.equal(op.adjoint(op.y_in).clone(), x)
    finally:
        F.set_deterministic_gridding(old)
