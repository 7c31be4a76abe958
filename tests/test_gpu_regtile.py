"""GPU parity of deterministic 3D gridding against the oracle: the tensor-core
kernel for widths 2..5 (every work item, a bin or a 2048-sample segment of a
heavier one, stores its region's partial sums; a gather adds them per grid
point in a fixed order), the register-tile kernel for
wider kernels and when the tensor-core path is switched off (DMR_NO_TC=1, in
a child process): regular and anisotropic grids (partial block regions at
the grid edge), several widths, coil counts that leave part of a 32-coil
block empty, frames, a trajectory dense enough to split the central regions
over several blocks, and bitwise reproducibility.

Tolerance: relative L2 error <= 1e-5 in float32.
"""

import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu

TOL = 1e-5


def rel(a, b):
    a = np.asarray(a.detach().cpu() if isinstance(a, torch.Tensor) else a, dtype=np.complex128)
    b = np.asarray(b.detach().cpu() if isinstance(b, torch.Tensor) else b, dtype=np.complex128)
    nb = np.linalg.norm(b.ravel())
    return float(np.linalg.norm((a - b).ravel()) / (nb if nb > 0 else 1.0))


@pytest.fixture(scope="module")
def F():
    import deepmr_b200.fft as F

    old = F.set_deterministic_gridding(True)
    yield F
    F.set_deterministic_gridding(old)


def _adjoint_case(F, coord, shape, ncoils, width, os, seed=0, dcf=True):
    from oracle import nufft_ref as R
    from deepmr_b200 import synth

    c = torch.as_tensor(coord)
    y = synth.complex_gaussian((ncoils,) + tuple(c.shape[:-1]), seed=seed)
    w = torch.as_tensor(synth.ramp_dcf(coord)) if dcf else None
    plan = F.plan_nufft(c, shape, width, os, device="cuda")
    oplan = R.plan_nufft(c, shape, width, os)
    x = F.apply_nufft_adj(y.cuda(), plan, weight=None if w is None else w.cuda())
    x_ref = R.apply_nufft_adj(y, oplan, weight=w)
    return x, x_ref, plan, y


@pytest.mark.parametrize("n,ncoils,width,os", [(24, 16, 4, 1.25), (24, 40, 4, 1.25), (16, 8, 6, 2.0),
                                               (20, 32, 3, 1.5), (12, 12, 4, 1.25)])
def test_regtile_isotropic(n, ncoils, width, os, F):
    from deepmr_b200 import synth

    coord = synth.kooshball_3d(n * n // 2, n * 2, n)
    x, x_ref, _, _ = _adjoint_case(F, coord, n, ncoils, width, os)
    assert rel(x, x_ref) < TOL


def test_regtile_anisotropic(F):
    from deepmr_b200 import synth

    shape = (20, 24, 28)
    c = synth.kooshball_3d(300, 56, shape)
    x, x_ref, _, _ = _adjoint_case(F, c, shape, 12, 4, 1.25, seed=1)
    assert x.shape[-3:] == shape
    assert rel(x, x_ref) < TOL


def test_regtile_split_regions(F):
    """Dense centre: the central windows hold more samples than one block takes."""
    from deepmr_b200 import synth

    coord = synth.kooshball_3d(3000, 48, 24)
    x, x_ref, _, _ = _adjoint_case(F, coord, 24, 16, 4, 1.25, seed=2)
    assert rel(x, x_ref) < TOL


def test_regtile_frames(F):
    from oracle import nufft_ref as R
    from deepmr_b200 import synth

    n, nf, nc = 16, 3, 10
    coord = np.stack([synth.kooshball_3d(150, 32, n) * (1.0 - 0.1 * f) for f in range(nf)]).astype(np.float32)
    c = torch.as_tensor(coord)
    y = synth.complex_gaussian((nc, nf) + tuple(coord.shape[1:-1]), seed=4)
    plan = F.plan_nufft(c, n, 4, 1.25, device="cuda")
    oplan = R.plan_nufft(c, n, 4, 1.25)
    x = F.apply_nufft_adj(y.cuda(), plan)
    x_ref = R.apply_nufft_adj(y, oplan)
    assert tuple(x.shape) == (nc, nf, n, n, n)
    assert rel(x, x_ref) < TOL


def test_regtile_real_kspace_and_weight_per_batch(F):
    from deepmr_b200 import _lib, synth

    n, nc = 16, 9
    coord = synth.kooshball_3d(200, 32, n)
    c = torch.as_tensor(coord)
    plan = F.plan_nufft(c, n, 4, 1.25, device="cuda")
    ip = plan.interpolator
    yr = torch.randn((nc,) + tuple(c.shape[:-1]), generator=torch.Generator().manual_seed(5))
    wb = torch.rand(yr.shape, generator=torch.Generator().manual_seed(6))
    L = _lib.lib()
    st = _lib.stream_ptr(torch.device("cuda"))
    g1 = torch.empty((nc,) + tuple(ip.dshape), dtype=torch.complex64, device="cuda")
    g2 = torch.empty_like(g1)
    yr_d, wb_d = yr.cuda(), wb.cuda()
    # real k-space with per-batch weights == complex k-space (imaginary 0) pre-multiplied
    # (deterministic gridding without a workspace: scratch from the library pool)
    _lib.check(L.dmr_grid(ip.handle, _lib.ptr(yr_d), 1, _lib.ptr(g1), nc, _lib.ptr(wb_d), 1, 1, st))
    yc = (yr * wb).to(torch.complex64).cuda()
    _lib.check(L.dmr_grid(ip.handle, _lib.ptr(yc), 0, _lib.ptr(g2), nc, None, 0, 1, st))
    torch.cuda.synchronize()
    assert rel(g1, g2) < 1e-6


def test_regtile_bitwise_reproducible_and_close_to_atomic(F):
    from deepmr_b200 import synth

    coord = synth.kooshball_3d(2000, 48, 24)
    plan = F.plan_nufft(torch.as_tensor(coord), 24, 4, 1.25, device="cuda")
    y = synth.complex_gaussian((20,) + coord.shape[:-1], seed=7).cuda()
    a = F.apply_nufft_adj(y, plan)
    b = F.apply_nufft_adj(y, plan)
    assert torch.equal(a, b)
    old = F.set_deterministic_gridding(False)
    try:
        c = F.apply_nufft_adj(y, plan)
    finally:
        F.set_deterministic_gridding(old)
    assert rel(a, c) < TOL  # summation order differs from the atomic kernel


def test_regtile_batch_slices_agree(F):
    """A coil's result does not depend on the other coils of its 32-coil block."""
    from deepmr_b200 import synth

    coord = synth.kooshball_3d(300, 40, 20)
    plan = F.plan_nufft(torch.as_tensor(coord), 20, 4, 1.25, device="cuda")
    y = synth.complex_gaussian((36,) + coord.shape[:-1], seed=8).cuda()
    full = F.apply_nufft_adj(y, plan)
    part = F.apply_nufft_adj(y[8:24].contiguous(), plan)
    assert torch.equal(full[8:24], part)


_RT_SCRIPT = r"""
import numpy as np, torch
import deepmr_b200.fft as F
from deepmr_b200 import synth
from oracle import nufft_ref as R
F.set_deterministic_gridding(True)
worst = 0.0
for n, nc, w, os, seed in [(24, 16, 4, 1.25, 0), (20, 32, 3, 1.5, 1), (24, 12, 5, 1.25, 2)]:
    coord = synth.kooshball_3d(2000, 48, n)
    c = torch.as_tensor(coord)
    y = synth.complex_gaussian((nc,) + tuple(c.shape[:-1]), seed=seed)
    plan = F.plan_nufft(c, n, w, os, device="cuda")
    a = F.apply_nufft_adj(y.cuda(), plan)
    b = F.apply_nufft_adj(y.cuda(), plan)
    assert torch.equal(a, b)
    ref = R.apply_nufft_adj(y[:2], R.plan_nufft(c, n, w, os))
    d = np.asarray(a[:2].cpu(), np.complex128) - np.asarray(ref, np.complex128)
    worst = max(worst, float(np.linalg.norm(d) / np.linalg.norm(np.asarray(ref, np.complex128))))
print("REL", worst)
"""


def test_register_tile_path_when_tensor_cores_off():
    """The register-tile kernel (the deterministic path without the tensor-core
    kernel) in a process started with DMR_NO_TC=1: oracle parity on dense
    kooshballs (split regions) and bitwise reproducibility."""
    import os
    import subprocess
    import sys

    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    env = dict(os.environ, DMR_NO_TC="1", PYTHONPATH=root + os.pathsep + os.environ.get("PYTHONPATH", ""))
    out = subprocess.run([sys.executable, "-c", _RT_SCRIPT], env=env, cwd=root, capture_output=True, text=True,
                         timeout=600)
    assert out.returncode == 0, out.stderr[-2000:]
    worst = float(out.stdout.split("REL")[-1])
    assert worst < TOL
