"""GPU parity of the Cartesian sparse FFT against vectors produced by the
reference itself (tests/golden/sparse*.npz): forward (centred FFT + sampling),
adjoint (zero-fill with repeated indexes + centred inverse FFT), per-sample
weights, frames, a square subspace basis, and the self-adjoint operator with
its normalised count kernel. Tolerance: relative L2 error <= 1e-5 in float32.
"""

import numpy as np
import pytest
import torch

from conftest import golden_cases

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

    return F


@pytest.fixture(params=[True, False], ids=["det", "atomic"])
def grid_mode(request, F):
    old = F.set_deterministic_gridding(request.param)
    yield request.param
    F.set_deterministic_gridding(old)


def _shape(g):
    return int(g["shape"]) if g["shape"].ndim == 0 else tuple(int(s) for s in g["shape"])


@pytest.mark.parametrize("name", golden_cases(kind="sparse"))
def test_sparse_golden(name, load_golden, F, grid_mode):
    g = load_golden(name)
    mask = F.prepare_sampling(g["indexes"], _shape(g), device="cuda")
    w = g.get("weight")
    y = F.apply_sparse_fft(torch.as_tensor(g["image"]).cuda(), mask, g.get("basis_adjoint"), weight=w)
    x = F.apply_sparse_ifft(torch.as_tensor(g["kspace"]).cuda(), mask, g.get("basis"), weight=w)
    assert tuple(y.shape) == g["fwd"].shape and tuple(x.shape) == g["adj"].shape
    assert rel(y, g["fwd"]) < TOL
    assert rel(x, g["adj"]) < TOL
    if "kernel" in g:
        T = F.plan_toeplitz_fft(g["indexes"], _shape(g), device="cuda")
        assert tuple(T.value.shape) == g["kernel"].shape
        assert rel(T.value, g["kernel"]) < 1e-6
        assert rel(F.apply_sparse_fft_selfadj(torch.as_tensor(g["image"]).cuda(), T), g["selfadj"]) < TOL


def test_sparse_one_shot_and_numpy(load_golden, F):
    g = load_golden("sparse3d")
    y = F.sparse_fft(g["image"], g["indexes"], device="cuda")
    assert isinstance(y, np.ndarray) and rel(y, g["fwd"]) < TOL
    x = F.sparse_ifft(g["kspace"], g["indexes"], _shape(g), device="cuda")
    assert isinstance(x, np.ndarray) and rel(x, g["adj"]) < TOL


def test_sparse_indexes_out_of_range(F):
    idx = np.array([[[0, 0], [12, 3]]])
    with pytest.raises(ValueError):
        F.prepare_sampling(idx, 12, device="cuda")
