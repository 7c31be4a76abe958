"""GPU parity of the tensor-core 3D gridding (atomic mode, tcgen05 TF32 with a
three-term split) against the oracle and against the deterministic gridding
kernels, which share no code with it.

Cases: coil counts below, at and above the 32 coils of one block (a partial
last coil chunk), one and several frames, real input, shared and per-batch
density weights, kernel widths 3..5 (bin regions of 216..512 points) and
width 6 at oversampling 2 (a larger region: the cell-cube kernels run). Tolerance: relative L2 error
<= 1e-5 in float32.
"""

import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu

TOL = 1e-5


def rel(a, b):
    a = np.asarray(a.detach().cpu() if isinstance(a, torch.Tensor) else a, dtype=np.complex128)
    b = np.asarray(b.detach().cpu() if isinstance(b, torch.Tensor) else b, dtype=np.complex128)
    return float(np.linalg.norm((a - b).ravel()) / np.linalg.norm(b.ravel()))


@pytest.fixture(scope="module")
def F():
    """The fft module, with atomic 3D gridding on the tensor cores for every
    coil count (by default batches under 20 coils run on the CUDA cores)."""
    import deepmr_b200.fft as F
    from deepmr_b200 import _lib

    old = _lib.lib().dmr_tc_min_coils(1)
    yield F
    _lib.lib().dmr_tc_min_coils(old)


def _grid(F, plan, ksp, weight=None, det=False):
    old = F.set_deterministic_gridding(det)
    try:
        return F.apply_nufft_adj(ksp, plan, weight=weight)
    finally:
        F.set_deterministic_gridding(old)


@pytest.mark.parametrize("ncoils", [1, 5, 32, 40])
def test_tc_grid_vs_oracle(F, ncoils):
    from oracle import nufft_ref as R
    from deepmr_b200 import synth

    n = 20
    coord = synth.kooshball_3d(300, 2 * n, n).astype(np.float32)
    c = torch.as_tensor(coord)
    plan = F.plan_nufft(c, n, 4, 1.25, device="cuda")
    ksp = synth.complex_gaussian((ncoils,) + coord.shape[:-1], seed=ncoils)
    dcf = torch.as_tensor(synth.ramp_dcf(coord.reshape(-1, 3)).reshape(coord.shape[:-1]))
    x = _grid(F, plan, ksp.cuda(), dcf.cuda())
    ref = R.apply_nufft_adj(ksp, R.plan_nufft(c, n, 4, 1.25), weight=dcf)
    assert rel(x, ref) < TOL


@pytest.mark.parametrize("det", [False, True], ids=["atomic", "deterministic"])
@pytest.mark.parametrize("width,os", [(2, 2.0), (3, 1.25), (4, 1.25), (5, 1.25), (6, 2.0)])
def test_tc_grid_widths_vs_oracle(F, width, os, det):
    """Widths 2..5 on the tensor cores (width 6 has no gridding bins and runs
    on the CUDA cores); deterministic width 5 (bins of 3 x 2 x 2 cells, regions
    of 7 x 6 x 6 points) has up to 3 covering bins per axis, the gather's
    general path."""
    from oracle import nufft_ref as R
    from deepmr_b200 import synth

    n = 20
    coord = synth.kooshball_3d(300, 2 * n, n).astype(np.float32)
    c = torch.as_tensor(coord)
    plan = F.plan_nufft(c, n, width, os, device="cuda")
    ksp = synth.complex_gaussian((6,) + coord.shape[:-1], seed=width)
    ref = R.apply_nufft_adj(ksp, R.plan_nufft(c, n, width, os))
    x = _grid(F, plan, ksp.cuda(), det=det)
    assert rel(x, ref) < TOL
    if det:
        assert torch.equal(x, _grid(F, plan, ksp.cuda(), det=True))


def test_tc_grid_vs_deterministic(F):
    from deepmr_b200 import synth

    n = 32
    coord = synth.kooshball_3d(1200, 2 * n, n).astype(np.float32)
    plan = F.plan_nufft(torch.as_tensor(coord), n, 4, 1.25, device="cuda")
    ksp = synth.complex_gaussian((12,) + coord.shape[:-1], seed=4).cuda()
    assert rel(_grid(F, plan, ksp), _grid(F, plan, ksp, det=True)) < TOL


def test_tc_grid_frames_real_batch_weights(F):
    from deepmr_b200 import synth

    n, nf = 24, 3
    coord = np.stack([synth.kooshball_3d(400, 2 * n, n) * (1.0 - 0.07 * f) for f in range(nf)]).astype(np.float32)
    plan = F.plan_nufft(torch.as_tensor(coord), n, 4, 1.25, device="cuda")
    ksp = synth.complex_gaussian((2, 17, nf) + coord.shape[1:-1], seed=3).real.contiguous().cuda()
    wb = torch.rand((2, 17, nf) + coord.shape[1:-1], generator=torch.Generator().manual_seed(4)).cuda()
    x = _grid(F, plan, ksp, wb)
    assert tuple(x.shape) == (2, 17, nf, n, n, n)
    assert rel(x, _grid(F, plan, ksp, wb, det=True)) < TOL


@pytest.mark.parametrize("ncoils", [3, 13, 37])
def test_tc_grid_deterministic_vs_oracle_and_release(F, ncoils):
    """Deterministic tensor-core gridding (per-item partial sums in the scratch
    pool, gathered per grid point) for coil counts that are not multiples of
    the 8-coil gather groups, one or two coil chunks, against the oracle;
    bitwise equal again after the pool gave its memory back."""
    from oracle import nufft_ref as R
    from deepmr_b200 import synth

    n = 20
    coord = synth.kooshball_3d(300, 2 * n, n).astype(np.float32)
    c = torch.as_tensor(coord)
    plan = F.plan_nufft(c, n, 4, 1.25, device="cuda")
    ksp = synth.complex_gaussian((ncoils,) + coord.shape[:-1], seed=20 + ncoils)
    dcf = torch.as_tensor(synth.ramp_dcf(coord.reshape(-1, 3)).reshape(coord.shape[:-1]))
    x = _grid(F, plan, ksp.cuda(), dcf.cuda(), det=True)
    ref = R.apply_nufft_adj(ksp, R.plan_nufft(c, n, 4, 1.25), weight=dcf)
    assert rel(x, ref) < TOL
    F.release_scratch()
    assert torch.equal(x, _grid(F, plan, ksp.cuda(), dcf.cuda(), det=True))


def test_tc_grid_deterministic_scratch_limit_falls_back(F):
    """A scratch limit below what deterministic tensor-core gridding needs
    sends the call to the register-tile kernel: within 1e-5 of the oracle,
    bitwise reproducible, and not bitwise equal to the tensor-core result
    (another summation order), which shows that the other kernel ran."""
    from oracle import nufft_ref as R
    from deepmr_b200 import synth

    n = 20
    coord = synth.kooshball_3d(300, 2 * n, n).astype(np.float32)
    c = torch.as_tensor(coord)
    plan = F.plan_nufft(c, n, 4, 1.25, device="cuda")
    ksp = synth.complex_gaussian((12,) + coord.shape[:-1], seed=31)
    ref = R.apply_nufft_adj(ksp, R.plan_nufft(c, n, 4, 1.25))
    old = F.set_deterministic_scratch_limit(1)
    try:
        assert F.set_deterministic_scratch_limit(1) == 1
        x = _grid(F, plan, ksp.cuda(), det=True)
        x2 = _grid(F, plan, ksp.cuda(), det=True)
    finally:
        F.set_deterministic_scratch_limit(old)
    xt = _grid(F, plan, ksp.cuda(), det=True)
    assert rel(x, ref) < TOL and rel(xt, ref) < TOL
    assert torch.equal(x, x2)
    assert not torch.equal(x, xt)


def test_tc_grid_adjoint_identity(F):
    """<A x, y> = G <x, A^H y> with the tensor-core adjoint."""
    from deepmr_b200 import synth

    n = 24
    coord = synth.kooshball_3d(600, 2 * n, n).astype(np.float32)
    plan = F.plan_nufft(torch.as_tensor(coord), n, 4, 1.25, device="cuda")
    x = synth.complex_gaussian((8, n, n, n), seed=5).cuda()
    y = synth.complex_gaussian((8,) + coord.shape[:-1], seed=6).cuda()
    ax = F.apply_nufft(x, plan)
    ahy = _grid(F, plan, y)
    G = float(np.prod([int(s) for s in plan.os_shape]))
    lhs = torch.vdot(ax.flatten().to(torch.complex128), y.flatten().to(torch.complex128))
    rhs = G * torch.vdot(x.flatten().to(torch.complex128), ahy.flatten().to(torch.complex128))
    assert abs(lhs - rhs) / abs(lhs) < 1e-5


def test_tc_grid_no_wait_ran_out(F):
    """The kernel's bounded mbarrier waits do not run out in normal runs."""
    import ctypes

    from deepmr_b200 import _lib, synth

    L = _lib.lib()
    count = ctypes.c_int64(-1)
    _lib.check(L.dmr_tc_timeouts(ctypes.byref(count), 1))  # reset
    n = 16
    coord = synth.kooshball_3d(200, 2 * n, n).astype(np.float32)
    plan = F.plan_nufft(torch.as_tensor(coord), n, 4, 1.25, device="cuda")
    _grid(F, plan, synth.complex_gaussian((4,) + coord.shape[:-1], seed=7).cuda())
    plan.interpolator.check_status()
    _lib.check(L.dmr_tc_timeouts(ctypes.byref(count), 0))
    assert count.value == 0


def test_tc_grid_timeout_reported(F):
    """A bounded wait that runs out is reported, not silent.

    The test hook dmr_tc_test_stall makes every gridding block wait on an
    mbarrier that nothing signals (bounded by 1 ms of global time): the call
    returns, dmr_plan_status reports DMR_ERR_TIMEOUT with the number of blocks
    that stopped, the device counter grows, the Python layer raises on a call
    whose result returns to the host, and the next normal call is correct."""
    import ctypes

    from deepmr_b200 import _lib, synth

    L = _lib.lib()
    n = 16
    coord = synth.kooshball_3d(200, 2 * n, n).astype(np.float32)
    plan = F.plan_nufft(torch.as_tensor(coord), n, 4, 1.25, device="cuda")
    ip = plan.interpolator
    ksp = synth.complex_gaussian((4,) + coord.shape[:-1], seed=8).cuda()
    grid = torch.empty((4,) + tuple(ip.dshape), dtype=torch.complex64, device="cuda")
    st = _lib.stream_ptr(torch.device("cuda", torch.cuda.current_device()))
    c0, c1 = ctypes.c_int64(-1), ctypes.c_int64(-1)
    _lib.check(L.dmr_tc_timeouts(ctypes.byref(c0), 0))
    _lib.check(L.dmr_tc_test_stall(1))
    try:
        rc = L.dmr_grid(ip.handle, _lib.ptr(ksp), 0, _lib.ptr(grid), 4, None, 0, 0, st)
        assert rc == 0  # the launch itself succeeds; the failure is in the status
        failed = ctypes.c_int32(-1)
        rc = L.dmr_plan_status(ip.handle, ctypes.byref(failed), 1, st)
        assert rc == -8, rc  # DMR_ERR_TIMEOUT
        assert failed.value > 0
        # the Python layer raises on a call whose result returns to the host
        with pytest.raises(_lib.DmrError) as ei:
            F.apply_nufft_adj(ksp.cpu(), plan)
        assert ei.value.code == -8
    finally:
        _lib.check(L.dmr_tc_test_stall(0))
    _lib.check(L.dmr_tc_timeouts(ctypes.byref(c1), 1))
    assert c1.value > c0.value
    # the status was reset by the reads above: a normal call is valid again
    rc = L.dmr_plan_status(ip.handle, None, 0, st)
    assert rc == 0
    x = _grid(F, plan, ksp)
    ip.check_status()
    assert rel(x, _grid(F, plan, ksp, det=True)) < TOL
