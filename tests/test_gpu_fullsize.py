"""GPU parity at the workloads' full sizes.

3D kooshball (the throughput workload): 192^3 image, 240^3 grid, 50,000
golden-means spokes x 384 samples (19.2 M samples), Kaiser-Bessel width 4,
oversampling 1.25, 32 coils on the GPU. Coils are independent, so coils 0 and
17 of the 32-coil GPU results are compared with the oracle run on those two
coils alone (the oracle restates the reference's CPU loops,
src/deepmr/fft/_interp/interp.py:124-227 and grid.py:181-284). Checked: the
forward (interpolation), the atomic adjoint (tensor-core gridding) and the
deterministic adjoint (tensor-core gridding into per-item partial sums, the
kooshball centre's bins as several 2048-sample items, gathered per grid point
in a fixed order; two calls bitwise equal), plus independence of the
result from the coil count (the tensor-core kernel's block shape depends on
it). This covers the kooshball centre's bins split into several work items,
the work-item order in 4x4x4-bin tiles and sample indices near 2^24.

Toeplitz at size: the self-adjoint of the same trajectory and density
weights (kernel grid 384^3), two coils, against the oracle with the kernel's
point-spread function summed in float64 (the reference's float32 sums are
7.4e-5 from it at this size).

Uneven frames at size: 224^2, 16 coils, 500 single-interleaf variable-density
spiral frames of U{800..1200} samples each (seeded), rotated by the golden
angle, width 4, oversampling 1.25; one plan and one call on the GPU; the
oracle runs on two coils as one 500-frame call padded to 1200 samples per
frame (zero data in the padding; padded forward outputs ignored).

Tolerance: relative L2 error <= 1e-5 in float32.
"""

import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu

TOL = 1e-5
COILS = (0, 17)


def rel(a, b):
    a = np.asarray(torch.as_tensor(a).detach().cpu(), dtype=np.complex128).ravel()
    b = np.asarray(torch.as_tensor(b).detach().cpu(), dtype=np.complex128).ravel()
    return float(np.linalg.norm(a - b) / np.linalg.norm(b))


@pytest.fixture(scope="module")
def koosh():
    import deepmr_b200.fft as F
    from deepmr_b200 import synth
    from oracle import nufft_ref as R

    n = 192
    coord = synth.kooshball_3d(50000, 384, n)
    c = torch.as_tensor(coord)
    dcf = torch.as_tensor(synth.ramp_dcf(coord))
    plan = F.plan_nufft(c, n, 4, 1.25, device="cuda")
    oplan = R.plan_nufft(c, n, 4, 1.25)
    img = synth.complex_gaussian((32, n, n, n), seed=11, device="cuda")
    ksp = synth.complex_gaussian((32,) + tuple(coord.shape[:-1]), seed=12, device="cuda")
    sel = list(COILS)
    out = dict(F=F, R=R, coord=c, plan=plan, oplan=oplan, dcf=dcf, img=img, ksp=ksp,
               img_sel=img[sel].cpu(), ksp_sel=ksp[sel].cpu())
    yield out
    del out
    torch.cuda.empty_cache()


def test_kooshball_fullsize_forward(koosh):
    F, R = koosh["F"], koosh["R"]
    y = F.apply_nufft(koosh["img"], koosh["plan"])
    assert tuple(y.shape) == (32, 50000, 384)
    ref = R.apply_nufft(koosh["img_sel"], koosh["oplan"])
    e = rel(y[list(COILS)], ref)
    print(f"forward rel err {e:.2e}")
    assert e < TOL


@pytest.mark.parametrize("deterministic", [False, True], ids=["atomic", "deterministic"])
def test_kooshball_fullsize_adjoint(koosh, deterministic):
    F, R = koosh["F"], koosh["R"]
    dcf = koosh["dcf"]
    old = F.set_deterministic_gridding(deterministic)
    try:
        x = F.apply_nufft_adj(koosh["ksp"], koosh["plan"], weight=dcf.cuda())
        koosh["plan"].interpolator.check_status()
    finally:
        F.set_deterministic_gridding(old)
    assert tuple(x.shape) == (32, 192, 192, 192)
    if deterministic:
        old = F.set_deterministic_gridding(True)
        try:
            again = F.apply_nufft_adj(koosh["ksp"], koosh["plan"], weight=dcf.cuda())
        finally:
            F.set_deterministic_gridding(old)
        assert torch.equal(x, again)
        del again
    key = "adj_ref"
    if key not in koosh:
        koosh[key] = R.apply_nufft_adj(koosh["ksp_sel"], koosh["oplan"], weight=dcf)
    e = rel(x[list(COILS)], koosh[key])
    print(f"adjoint ({'deterministic' if deterministic else 'atomic'}) rel err {e:.2e}")
    assert e < TOL


def test_kooshball_fullsize_coil_count_independent(koosh):
    """The same coils gridded in a 32-coil call and in a 2-coil call agree."""
    F = koosh["F"]
    dcf = koosh["dcf"].cuda()
    sel = list(COILS)
    x32 = F.apply_nufft_adj(koosh["ksp"], koosh["plan"], weight=dcf)[sel]
    x2 = F.apply_nufft_adj(koosh["ksp"][sel].contiguous(), koosh["plan"], weight=dcf)
    koosh["plan"].interpolator.check_status()
    assert rel(x2, x32) < TOL


def test_kooshball_fullsize_toeplitz(koosh):
    """Toeplitz self-adjoint at full size: the kernel from the whole trajectory
    with ramp density weights on the 384^3 grid, applied through the fused
    passes (pad, FFT, kernel multiply and inverse FFT in the z pass, crop) to
    two coils, against the oracle's self-adjoint with its point-spread
    function summed in float64 (`plan_toeplitz(exact=True)`). The reference's
    sequential float32 sums are not accurate enough here: its point-spread
    function is 7.4e-5 (relative L2) from the float64 sum of the same taps, the
    GPU's 2.0e-6, so against the float32 oracle the self-adjoint differs by
    1.35e-5, all of it the float32 oracle's own error (printed, not
    asserted)."""
    F, R = koosh["F"], koosh["R"]
    c, dcf = koosh["coord"], koosh["dcf"]
    T = F.plan_toeplitz_nufft(c, 192, dcf=dcf, device="cuda")
    x = F.apply_nufft_selfadj(koosh["img"][list(COILS)].contiguous(), T)
    del T
    ref = R.apply_selfadj(koosh["img_sel"], R.plan_toeplitz(c, 192, dcf=dcf, exact=True))
    e = rel(x, ref)
    e32 = rel(x, R.apply_selfadj(koosh["img_sel"], R.plan_toeplitz(c, 192, dcf=dcf)))
    print(f"toeplitz rel err {e:.2e} (float32 oracle: {e32:.2e})")
    assert e < TOL
    del x


def _spiral_frames(nframes, n, seed=0):
    from deepmr_b200 import synth

    rng = np.random.default_rng(seed)
    lengths = rng.integers(800, 1201, nframes)
    return [synth.spiral_2d(int(L), n, rotation=f * synth.GOLDEN_ANGLE)[0] for f, L in enumerate(lengths)]


@pytest.mark.parametrize("deterministic", [False, True], ids=["atomic", "deterministic"])
def test_uneven_frames_fullsize(deterministic):
    import deepmr_b200.fft as F
    from deepmr_b200 import synth
    from oracle import nufft_ref as R

    n, ncoils, nframes, lmax = 224, 16, 500, 1200
    coords = _spiral_frames(nframes, n, seed=3)
    plan = F.plan_nufft(coords, n, 4, 1.25, device="cuda")
    total = sum(c.shape[0] for c in coords)
    img = synth.complex_gaussian((ncoils, nframes, n, n), seed=21, device="cuda")
    ks = synth.complex_gaussian((ncoils, total), seed=22, device="cuda")
    old = F.set_deterministic_gridding(deterministic)
    try:
        y = F.apply_nufft(img, plan)
        x = F.apply_nufft_adj(ks, plan)
    finally:
        F.set_deterministic_gridding(old)
    assert tuple(y.shape) == (ncoils, total) and tuple(x.shape) == (ncoils, nframes, n, n)
    sel = [0, 9]
    # oracle: one 500-frame call padded to lmax samples per frame
    pad = np.zeros((nframes, 1, lmax, 2), np.float32)
    kpad = np.zeros((len(sel), nframes, 1, lmax), np.complex64)
    parts_k = F.frames_split(ks[sel].cpu(), plan)
    for f, c in enumerate(coords):
        pad[f, 0, : c.shape[0]] = c
        kpad[:, f, 0, : c.shape[0]] = parts_k[f].numpy()
    op = R.plan_nufft(torch.as_tensor(pad), n, 4, 1.25)
    y_ref = R.apply_nufft(img[sel].cpu(), op)  # (2, nframes, 1, lmax)
    x_ref = R.apply_nufft_adj(torch.as_tensor(kpad), op)  # (2, nframes, n, n)
    parts_y = F.frames_split(y[sel].cpu(), plan)
    yv = np.concatenate([parts_y[f].numpy().reshape(len(sel), -1) for f in range(nframes)], axis=1)
    yr = np.concatenate([np.asarray(y_ref)[:, f, 0, : c.shape[0]] for f, c in enumerate(coords)], axis=1)
    ey, ex = rel(yv, yr), rel(x[sel], x_ref)
    print(f"uneven frames: forward rel err {ey:.2e}, adjoint rel err {ex:.2e}")
    assert ey < TOL and ex < TOL
