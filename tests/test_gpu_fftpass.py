"""GPU parity of the fused, pruned 3D FFT passes of the NUFFT pipelines
(apodise + zero-pad + forward FFT; inverse FFT + crop + 1/G + apodisation)
against the oracle, on grids whose extents have compiled transforms (so the
passes run instead of cuFFT): odd and even image extents, anisotropic grids
from per-axis oversampling, several coils, frames, real images, density
weights, and both gridding modes. Forward and adjoint are also checked for
adjointness, <A x, y> = G <x, A^H y>.

Tolerance: relative L2 error <= 1e-5 in float32.
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


def _coord(shape, nviews, nsamples, seed, nframes=None):
    rng = np.random.default_rng(seed)
    n = np.asarray(shape[::-1], dtype=np.float32)  # (x, y, z) extents for coordinates (x, y, z)
    lead = (nviews, nsamples) if nframes is None else (nframes, nviews, nsamples)
    return (rng.uniform(-0.5, 0.5, lead + (3,)) * n).astype(np.float32)


# image shape and oversampling, both (z, y, x), chosen so that every grid extent
# ceil(os * n) has a compiled transform
CASES = [
    ((24, 20, 16), 2.0),                      # grid (48, 40, 32)
    ((19, 37, 25), (2.1, 1.29, 1.27)),        # odd extents, grid (40, 48, 32)
    ((32, 32, 32), 1.25),                     # grid 40^3
    ((48, 40, 64), (2.0, 1.19, 1.25)),        # grid (96, 48, 80)
]


@pytest.mark.parametrize("shape,os", CASES)
@pytest.mark.parametrize("det", [False, True], ids=["atomic", "deterministic"])
def test_fused_fft_nufft_vs_oracle(shape, os, det):
    import deepmr_b200.fft as F
    from deepmr_b200 import _lib, synth
    from oracle import nufft_ref as R

    coord = _coord(shape, 60, 24, seed=sum(shape))
    c = torch.as_tensor(coord)
    plan = F.plan_nufft(c, shape, 4, os, device="cuda")
    assert _lib.lib().dmr_fft3_fused(plan.interpolator.handle) == 1
    oplan = R.plan_nufft(c, shape, 4, os)
    img = synth.complex_gaussian((5,) + tuple(shape), seed=1)
    ksp = synth.complex_gaussian((5,) + tuple(c.shape[:-1]), seed=2)
    w = torch.rand(tuple(c.shape[:-1]), generator=torch.Generator().manual_seed(3))
    old = F.set_deterministic_gridding(det)
    try:
        y = F.apply_nufft(img.cuda(), plan)
        x = F.apply_nufft_adj(ksp.cuda(), plan, weight=w.cuda())
    finally:
        F.set_deterministic_gridding(old)
    assert rel(y, R.apply_nufft(img, oplan)) < TOL
    assert rel(x, R.apply_nufft_adj(ksp, oplan, weight=w)) < TOL


def test_fused_fft_frames_real_image_and_adjointness():
    import deepmr_b200.fft as F
    from deepmr_b200 import _lib
    from oracle import nufft_ref as R

    shape = (20, 24, 16)  # grid (40, 48, 32) at oversampling 2
    coord = _coord(shape, 30, 20, seed=9, nframes=3)
    c = torch.as_tensor(coord)
    plan = F.plan_nufft(c, shape, 4, 2.0, device="cuda")
    assert _lib.lib().dmr_fft3_fused(plan.interpolator.handle) == 1
    oplan = R.plan_nufft(c, shape, 4, 2.0)
    g = torch.Generator().manual_seed(4)
    img = torch.randn((2, 3) + shape, generator=g)  # real image, 2 coils, 3 frames
    y = F.apply_nufft(img.cuda(), plan)
    assert rel(y, R.apply_nufft(img, oplan)) < TOL
    yy = torch.complex(torch.randn(y.shape, generator=g), torch.randn(y.shape, generator=g))
    x = F.apply_nufft_adj(yy.cuda(), plan)
    assert rel(x, R.apply_nufft_adj(yy, oplan)) < TOL
    xc = torch.complex(torch.randn(x.shape, generator=g), torch.randn(x.shape, generator=g)).cuda()
    lhs = torch.vdot(F.apply_nufft(xc, plan).flatten(), yy.cuda().flatten())
    rhs = torch.vdot(xc.flatten(), F.apply_nufft_adj(yy.cuda(), plan).flatten()) * float(np.prod(plan.os_shape))
    assert abs(complex(lhs - rhs)) / abs(complex(lhs)) < 1e-5


def test_grid_outside_the_table_uses_cufft():
    import deepmr_b200.fft as F
    from deepmr_b200 import _lib

    shape = (12, 12, 12)  # grid 15^3: no compiled transform
    plan = F.plan_nufft(torch.as_tensor(_coord(shape, 20, 10, seed=5)), shape, 4, 1.25, device="cuda")
    assert _lib.lib().dmr_fft3_fused(plan.interpolator.handle) == 0


@pytest.mark.parametrize("frames", [1, 2])
def test_fused_toeplitz_selfadjoint_vs_oracle(frames):
    """3D Toeplitz self-adjoint through the fused passes (kernel grids 2N =
    32 x 40 x 48 have compiled transforms): zero-pad, FFT, kernel multiply and
    inverse FFT in one z pass, crop; with density weights, per-frame kernels."""
    import deepmr_b200.fft as F
    from oracle import nufft_ref as R

    shape = (16, 20, 24)
    coord = _coord(shape, 40, 20, seed=13, nframes=frames if frames > 1 else None)
    c = torch.as_tensor(coord)
    dcf = torch.rand(tuple(c.shape[:-1]), generator=torch.Generator().manual_seed(14)) + 0.5
    T = F.plan_toeplitz_nufft(c, shape, dcf=dcf, device="cuda")
    To = R.plan_toeplitz(c, shape, dcf=dcf)
    lead = (3,) + ((frames,) if frames > 1 else ())
    g = torch.Generator().manual_seed(15)
    img = torch.complex(torch.randn(lead + shape, generator=g), torch.randn(lead + shape, generator=g))
    out = F.apply_nufft_selfadj(img.cuda(), T)
    assert tuple(out.shape) == tuple(img.shape)
    assert rel(out, R.apply_selfadj(img, To)) < TOL


def _coord2(shape, nviews, nsamples, seed, nframes=None):
    rng = np.random.default_rng(seed)
    n = np.asarray(shape[::-1], dtype=np.float32)  # (x, y) extents
    lead = (nviews, nsamples) if nframes is None else (nframes, nviews, nsamples)
    return (rng.uniform(-0.5, 0.5, lead + (2,)) * n).astype(np.float32)


# 2D image shape and oversampling (y, x) -> grid extents with compiled transforms,
# including a factor 7 (56, 140, 280)
CASES_2D = [
    ((20, 24), 2.0, None),            # grid (40, 48)
    ((45, 37), (1.24, 1.5), None),    # odd extents, grid (56, 56)
    ((224, 112), 1.25, None),         # grid (280, 140)
    ((28, 40), 2.0, 3),               # grid (56, 80), 3 frames
]


@pytest.mark.parametrize("shape,os,frames", CASES_2D)
def test_fused_fft_2d_nufft_vs_oracle(shape, os, frames):
    import deepmr_b200.fft as F
    from deepmr_b200 import _lib, synth
    from oracle import nufft_ref as R

    coord = _coord2(shape, 40, 32, seed=sum(shape), nframes=frames)
    c = torch.as_tensor(coord)
    plan = F.plan_nufft(c, shape, 4, os, device="cuda")
    assert _lib.lib().dmr_fft3_fused(plan.interpolator.handle) == 1
    oplan = R.plan_nufft(c, shape, 4, os)
    lead = (4,) + ((frames,) if frames else ())
    img = synth.complex_gaussian(lead + tuple(shape), seed=1)
    ksp = synth.complex_gaussian(lead + tuple(c.shape[-3:-1]), seed=2)
    assert rel(F.apply_nufft(img.cuda(), plan), R.apply_nufft(img, oplan)) < TOL
    assert rel(F.apply_nufft_adj(ksp.cuda(), plan), R.apply_nufft_adj(ksp, oplan)) < TOL


@pytest.mark.parametrize("shape", [(16, 20), (28, 70)])
def test_fused_toeplitz_2d_vs_oracle(shape):
    """2D Toeplitz self-adjoint through the fused passes (kernel grids 2N with
    compiled transforms, one with a factor 7): the y pass is the fused
    forward FFT, kernel multiply and inverse FFT."""
    import deepmr_b200.fft as F
    from oracle import nufft_ref as R

    coord = _coord2(shape, 30, 40, seed=21)
    c = torch.as_tensor(coord)
    dcf = torch.rand(tuple(c.shape[:-1]), generator=torch.Generator().manual_seed(22)) + 0.5
    T = F.plan_toeplitz_nufft(c, shape, dcf=dcf, device="cuda")
    To = R.plan_toeplitz(c, shape, dcf=dcf)
    g = torch.Generator().manual_seed(23)
    img = torch.complex(torch.randn((5,) + shape, generator=g), torch.randn((5,) + shape, generator=g))
    out = F.apply_nufft_selfadj(img.cuda(), T)
    assert rel(out, R.apply_selfadj(img, To)) < TOL
