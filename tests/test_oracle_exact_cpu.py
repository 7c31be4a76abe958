"""The oracle's float64-accumulation variant (`gridding_exact`,
`plan_toeplitz(exact=True)`), used as the parity reference where the
reference's sequential float32 sums lose precision (the full-size Toeplitz
point-spread function): on small cases, where float32 accumulation is
accurate, it agrees with the float32 oracle, in 2D, 3D, with frames and
complex data."""

import numpy as np
import torch

from deepmr_b200 import synth
from oracle import nufft_ref as R


def rel(a, b):
    a = torch.as_tensor(a).to(torch.complex128)
    b = torch.as_tensor(b).to(torch.complex128)
    return float(torch.linalg.norm(a - b) / torch.linalg.norm(b))


def test_gridding_exact_matches_float32_on_small_cases():
    c3 = torch.as_tensor(synth.kooshball_3d(60, 16, 12))
    p3 = R.plan_nufft(c3, 12, 4, 1.25)
    y3 = synth.complex_gaussian((2,) + tuple(c3.shape[:-1]), seed=1)
    assert rel(R.gridding_exact(y3, p3.interpolator), R.gridding(y3, p3.interpolator)) < 1e-6
    c2 = torch.as_tensor(np.stack([synth.radial_2d(12, 24, 16, angle_offset=0.3 * f) for f in range(3)]))
    p2 = R.plan_nufft(c2, 16, 3, 2.0)
    y2 = synth.complex_gaussian((2, 3) + tuple(c2.shape[1:-1]), seed=2)
    assert rel(R.gridding_exact(y2, p2.interpolator), R.gridding(y2, p2.interpolator)) < 1e-6
    assert rel(R.apply_nufft_adj(y2, p2, exact=True), R.apply_nufft_adj(y2, p2)) < 1e-6


def test_exact_toeplitz_matches_float32_on_small_cases():
    c = torch.as_tensor(synth.kooshball_3d(40, 16, 10))
    dcf = torch.as_tensor(synth.ramp_dcf(c.numpy()))
    a = R.plan_toeplitz(c, 10, dcf=dcf)
    b = R.plan_toeplitz(c, 10, dcf=dcf, exact=True)
    assert b.value.dtype == torch.complex64
    assert rel(b.value, a.value) < 1e-6
    img = synth.complex_gaussian((2, 10, 10, 10), seed=3)
    assert rel(R.apply_selfadj(img, b), R.apply_selfadj(img, a)) < 1e-6
