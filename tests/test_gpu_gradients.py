"""Gradients of the NUFFT on the GPU, checked against float64 finite differences.

Workload of the differentiable data-consistency configuration: 2D 256x256,
12 coils, 402 golden-angle spokes x 512 samples, width 4, oversampling 1.25,
loss ||A x - y||^2 with y from a seeded ellipse phantom plus complex Gaussian
noise (sigma 1e-2). The reference has no trajectory gradient (its backward
returns None for the plan), so the trajectory gradient is pinned only by the
finite differences; the image gradient follows the reference convention
(backward of apply_nufft is apply_nufft_adj = exact adjoint / prod(os_shape),
src/deepmr/fft/nufft.py:188-209).
"""

import math

import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu

EPS = 1e-3  # grid units for coordinates
TOL = 2e-3  # relative to the largest checked entry (float32 GPU vs float64 FD)


@pytest.fixture(scope="module")
def dc_problem():
    from deepmr_b200 import synth
    from oracle import nufft_ref as R

    N, C = 256, 12
    coord = synth.radial_2d(402, 512, N)
    phantom = torch.as_tensor(synth.ellipse_phantom(N, seed=0)).to(torch.complex64)
    maps = torch.as_tensor(synth.coil_maps(C, (N, N), seed=1))
    x_true = maps * phantom
    plan = R.plan_nufft(torch.as_tensor(coord), N, 4, 1.25)
    y = R.apply_nufft(x_true, plan)
    y = y + 1e-2 * synth.complex_gaussian(tuple(y.shape), seed=2)
    x = x_true + 0.05 * synth.complex_gaussian(tuple(x_true.shape), seed=3)  # evaluation point
    return dict(N=N, C=C, coord=coord, x=x, y=y)


def _safe_samples(coord, N, count, rng):
    """Samples whose tap set does not change within +-10*EPS on any axis."""
    g = math.ceil(1.25 * N)
    k = coord.reshape(-1, 2).astype(np.float64) * g / N + g // 2
    frac = np.abs((k - 2.0) - np.round(k - 2.0))
    ok = np.where((frac > 20 * EPS * g / N).all(1))[0]
    return rng.choice(ok, size=count, replace=False)


def test_trajectory_gradient_vs_fp64_fd(dc_problem):
    import deepmr_b200.fft as F
    from oracle import nufft_ref as R

    d = dc_problem
    coord = torch.as_tensor(d["coord"]).cuda().requires_grad_(True)
    x = d["x"].cuda()
    y = d["y"].cuda()
    r = F.nufft(x, coord, width=4, oversamp=1.25, device="cuda") - y
    loss = (r.real**2 + r.imag**2).sum()
    loss.backward()
    grad = coord.grad.reshape(-1, 2).cpu().numpy().astype(np.float64)

    f64 = R.Forward64(d["x"].numpy(), d["coord"], d["N"], 4, 1.25)
    flat = d["coord"].reshape(-1, 2).astype(np.float64)
    y64 = d["y"].numpy().reshape(d["C"], -1).astype(np.complex128)
    rng = np.random.default_rng(0)
    ps = _safe_samples(d["coord"], d["N"], 24, rng)
    num, ana = [], []
    for p in ps:
        for a in range(2):
            c_plus, c_minus = flat[p].copy(), flat[p].copy()
            c_plus[a] += EPS
            c_minus[a] -= EPS
            lp = np.sum(np.abs(f64.sample(c_plus) - y64[:, p]) ** 2)
            lm = np.sum(np.abs(f64.sample(c_minus) - y64[:, p]) ** 2)
            num.append((lp - lm) / (2 * EPS))
            ana.append(grad[p, a])
    num, ana = np.asarray(num), np.asarray(ana)
    err = np.max(np.abs(num - ana)) / np.max(np.abs(num))
    assert err < TOL, (err, num[:6], ana[:6])


def test_image_gradient_vs_fp64_fd(dc_problem):
    """G * x.grad == dL/dx from float64 central differences on a few pixels.

    Evaluated at x = 0.5 x_true (residual ~ -y/2, as early in a
    reconstruction): close to the data the residual is tiny, and A^H then
    amplifies the ~1e-6 systematic difference between the float32 operator
    (the reference's own float32 tables, which this library reproduces) and
    the float64 one used for the finite differences.
    """
    import deepmr_b200.fft as F
    from oracle import nufft_ref as R

    d = dict(dc_problem)
    N, C = d["N"], d["C"]
    d["x"] = 0.5 * (d["x"] - 0.05 * __import__("deepmr_b200").synth.complex_gaussian(tuple(d["x"].shape), seed=3))
    coord = torch.as_tensor(d["coord"])
    x = d["x"].cuda().requires_grad_(True)
    y = d["y"].cuda()
    plan = F.plan_nufft(coord, N, 4, 1.25, device="cuda")
    r = F.apply_nufft(x, plan) - y
    loss = (r.real**2 + r.imag**2).sum()
    loss.backward()
    G = float(np.prod([int(s) for s in plan.os_shape]))
    grad = x.grad.cpu().numpy().astype(np.complex128) * G

    # the loss is quadratic in x: central differences are exact up to rounding,
    # and only the perturbed coil changes, so use the float64 forward of that coil
    rng = np.random.default_rng(1)
    flat = d["coord"].reshape(-1, 2)
    y64 = d["y"].numpy().reshape(C, -1).astype(np.complex128)
    for _ in range(3):
        c, i, j = int(rng.integers(C)), int(rng.integers(N // 4, 3 * N // 4)), int(rng.integers(N // 4, 3 * N // 4))
        for part, unit in (("re", 1.0), ("im", 1j)):
            h = 1e-2
            xp = d["x"][c].numpy().astype(np.complex128).copy()
            xm = xp.copy()
            xp[i, j] += h * unit
            xm[i, j] -= h * unit
            fp = R.Forward64(xp, d["coord"], N, 4, 1.25)
            fm = R.Forward64(xm, d["coord"], N, 4, 1.25)
            # loss of coil c over all samples, through the float64 spectrum
            lp = _coil_loss(fp, flat, y64[c])
            lm = _coil_loss(fm, flat, y64[c])
            fd = (lp - lm) / (2 * h)
            g = grad[c, i, j].real if part == "re" else grad[c, i, j].imag
            assert abs(fd - g) <= 2e-3 * max(abs(fd), 1e-3), (part, fd, g)


def _coil_loss(f64, flat, yc):
    """sum_p |y_p - yc_p|^2 with all samples evaluated through the float64 spectrum,
    vectorised over taps (2D, width 4)."""
    N = f64.N_xyz
    G = f64.G_xyz
    kx = flat[:, 0].astype(np.float64) * G[0] / N[0] + G[0] // 2
    ky = flat[:, 1].astype(np.float64) * G[1] / N[1] + G[1] // 2
    from oracle.nufft_ref import kaiser_bessel

    x0 = np.ceil(kx - 2.0)
    y0 = np.ceil(ky - 2.0)
    kb = np.vectorize(kaiser_bessel)
    acc = np.zeros(flat.shape[0], dtype=np.complex128)
    wx = [kb(((x0 + i) - kx) / 2.0, f64.beta_xyz[0]) for i in range(4)]
    wy = [kb(((y0 + i) - ky) / 2.0, f64.beta_xyz[1]) for i in range(4)]
    K = f64.K
    for iy in range(4):
        yy = ((y0 + iy) % G[1]).astype(np.int64)
        for ix in range(4):
            xx = ((x0 + ix) % G[0]).astype(np.int64)
            acc += wy[iy] * wx[ix] * K[yy, xx]
    yhat = acc / f64.scale
    return float(np.sum(np.abs(yhat - yc) ** 2))


def test_adjoint_trajectory_gradient_consistent_with_forward():
    """d/dc Re<A^H(c) y, u> == d/dc Re<y, A(c) u> / G (adjoint identity)."""
    import deepmr_b200.fft as F
    from deepmr_b200 import synth

    N = 32
    c0 = torch.as_tensor(synth.radial_2d(20, 40, N, angle_offset=0.2)) + 0.013
    y = synth.complex_gaussian((3,) + tuple(c0.shape[:-1]), seed=5).cuda()
    u = synth.complex_gaussian((3, N, N), seed=6).cuda()
    c1 = c0.clone().cuda().requires_grad_(True)
    x = F.nufft_adj(y, c1, N, width=4, oversamp=1.25, device="cuda")
    (torch.vdot(x.flatten(), u.flatten()).real).backward()
    c2 = c0.clone().cuda().requires_grad_(True)
    k = F.nufft(u, c2, width=4, oversamp=1.25, device="cuda")
    G = math.ceil(1.25 * N) ** 2
    (torch.vdot(y.flatten(), k.flatten()).real / G).backward()
    a, b = c1.grad.cpu().numpy(), c2.grad.cpu().numpy()
    assert np.max(np.abs(a - b)) <= 1e-4 * np.max(np.abs(b)), np.max(np.abs(a - b))
