"""Generate golden NUFFT vectors by running the reference implementation.

Run where the reference project is available (read-only); its location is
the ``DEEPMR_REFERENCE`` environment variable (the project root, containing
``src/deepmr``), or ``--reference PATH``::

    DEEPMR_REFERENCE=/path/to/deep-mr python tests/golden/make_golden.py   # every case
    python tests/golden/make_golden.py lowrank    # only the low-rank cases
    python tests/golden/make_golden.py sparse     # only the sparse FFT cases
    python tests/golden/make_golden.py cgsense    # only the CG-SENSE case
    python tests/golden/make_golden.py calib      # only the calibration cases
    python tests/golden/make_golden.py dcf        # only the Voronoi density cases

The reference's top-level package import needs optional I/O dependencies that
are absent, so the script registers stub parent packages whose ``__path__``
points into the reference tree and imports ``deepmr.fft`` directly. Numba's
cache is redirected to a temporary directory so nothing is written into the
read-only tree. The CPU Toeplitz path of the reference needs its kernel value
as a numpy array (src/deepmr/fft/_interp/toeplitz.py:85 calls
``torch.from_numpy`` on it), so the script converts it after planning.

Each case is saved as ``tests/golden/<name>.npz`` with its inputs, plan
parameters and the reference outputs. Sizes are kept small (a few hundred KB
in total) so the fixtures can be committed and the GPU tests can use them on
machines without the reference.
"""

import os
import sys
import tempfile
import types

os.environ.setdefault("NUMBA_CACHE_DIR", tempfile.mkdtemp(prefix="numba_"))
sys.dont_write_bytecode = True

def _reference_root():
    if "--reference" in sys.argv:
        i = sys.argv.index("--reference")
        root = sys.argv[i + 1]
        del sys.argv[i:i + 2]
        return root
    root = os.environ.get("DEEPMR_REFERENCE")
    if not root:
        raise SystemExit("set DEEPMR_REFERENCE (or pass --reference) to the reference project's root")
    return root


REF_SRC = os.path.join(_reference_root(), "src", "deepmr")
HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.abspath(os.path.join(HERE, "..", "..")))

import numpy as np  # noqa: E402
import torch  # noqa: E402

from deepmr_b200 import synth  # noqa: E402


def import_reference():
    for name, path in [("deepmr", REF_SRC), ("deepmr._signal", REF_SRC + "/_signal")]:
        mod = types.ModuleType(name)
        mod.__path__ = [path]
        sys.modules[name] = mod
    import deepmr._signal.resize as resize_mod

    sys.modules["deepmr._signal"].resize = resize_mod.resize
    import deepmr.fft  # noqa: F401

    return sys.modules["deepmr.fft.nufft"], sys.modules["deepmr.fft"]


def import_reference_recon():
    """The reference's linear operators, CG and encoding-operator builder
    (deepmr.linops, deepmr.optim.cg, deepmr.recon.alg.linop) through the same
    stub parents. The Toeplitz kernel value is converted to numpy right after
    planning (the CPU path of apply_toeplitz needs it, toeplitz.py:85)."""
    import_reference()
    for name, sub in [("deepmr.optim", "/optim"), ("deepmr.recon", "/recon"), ("deepmr.recon.alg", "/recon/alg")]:
        mod = types.ModuleType(name)
        mod.__path__ = [REF_SRC + sub]
        sys.modules[name] = mod
    fft = sys.modules["deepmr.fft"]
    plan = fft.plan_toeplitz_nufft

    def plan_fixed(*args, **kwargs):
        T = plan(*args, **kwargs)
        T.value = T.value.numpy()
        return T

    fft.plan_toeplitz_nufft = plan_fixed
    import deepmr.optim.cg as cg  # noqa: E402
    import deepmr.recon.alg.linop as enc  # noqa: E402

    return cg, enc


def cgsense_case(name="cgsense2d", N=128, ncoils=8, nspokes=96, nsamples=256, niter=20, seed=0):
    """CG-SENSE of the reference (recon_lstsq with toeplitz=True: EncodingOp +
    zero-filled AHy + cg_solve, src/deepmr/recon/alg/classic_recon.py:133-174,
    without the intensity rescaling) on a 2D golden-angle radial acquisition:
    seeded phantom with a phase ramp, random-phase Gaussian coil maps, ramp
    density weights, data = E x + complex Gaussian noise. Saves the inputs, the
    reference's AHy and its solution after `niter` CG iterations (tol = 0)."""
    cg, enc = import_reference_recon()
    coord = torch.as_tensor(synth.radial_2d(nspokes, nsamples, N))
    dcf = torch.as_tensor(synth.ramp_dcf(coord.numpy()))
    maps = torch.as_tensor(synth.coil_maps(ncoils, (N, N), seed=seed + 5))
    ph = synth.ellipse_phantom(N, seed=seed + 2)
    x = torch.as_tensor(ph * np.exp(1j * 0.3 * np.linspace(-1, 1, N))[None, :]).to(torch.complex64)
    data = torch.zeros((ncoils, 1, nspokes, nsamples), dtype=torch.complex64)
    E, EHE = enc.EncodingOp(data, traj=coord, dcf=dcf, shape=(N, N), sensmap=maps[None, None],
                            toeplitz=True, device="cpu")
    y = E(x[None])[0, 0]  # (ncoils, nspokes, nsamples)
    g = torch.Generator().manual_seed(seed + 7)
    sigma = 1e-2 * float(y.abs().pow(2).mean().sqrt())
    y = y + sigma * torch.complex(torch.randn(y.shape, generator=g), torch.randn(y.shape, generator=g)) * 0.5**0.5
    y = y.to(torch.complex64)
    ahy = E.H(dcf**0.5 * y[None, None])  # (1, N, N)
    out, _ = cg.cg_solve(ahy, EHE, niter=niter, tol=0.0, ndim=2)
    np.savez_compressed(
        os.path.join(HERE, name + ".npz"), coord=_np(coord), dcf=_np(dcf), maps=_np(maps), kspace=_np(y),
        shape=np.int32(N), niter=np.int32(niter), ahy=_np(ahy[0]), x_cg=_np(out[0]),
    )
    print("wrote", name)


def _np(x):
    return x.detach().cpu().numpy() if isinstance(x, torch.Tensor) else np.asarray(x)


def import_reference_calib():
    """The reference's calibration callers of the NUFFT (deepmr.recon.calib.acs,
    .espirit) through stub parents; deepmr._signal gets the functions its
    package __init__ would re-export (resize, resample, rss)."""
    import_reference()
    for name, sub in [("deepmr.recon", "/recon"), ("deepmr.recon.calib", "/recon/calib")]:
        mod = types.ModuleType(name)
        mod.__path__ = [REF_SRC + sub]
        sys.modules[name] = mod
    import deepmr._signal.subspace  # noqa: F401

    resize_mod, subspace_mod = sys.modules["deepmr._signal.resize"], sys.modules["deepmr._signal.subspace"]
    sig = sys.modules["deepmr._signal"]
    sig.resize, sig.resample, sig.rss = resize_mod.resize, resize_mod.resample, subspace_mod.rss
    import deepmr.recon.calib.acs as acs  # noqa: E402
    import deepmr.recon.calib.espirit as espirit  # noqa: E402

    return acs, espirit


def import_reference_dcf():
    """The reference's density compensation module
    (src/deepmr/_design/grad/utils/dcf.py) through stub parents (its package
    __init__ files import the whole design toolbox)."""
    import_reference()
    for name, sub in [("deepmr._design", "/_design"), ("deepmr._design.grad", "/_design/grad"),
                      ("deepmr._design.grad.utils", "/_design/grad/utils")]:
        mod = types.ModuleType(name)
        mod.__path__ = [REF_SRC + sub]
        sys.modules[name] = mod
    import deepmr._design.grad.utils.dcf as dcf  # noqa: E402

    return dcf


def dcf_cases():
    """Voronoi density compensation (src/deepmr/_design/grad/utils/dcf.py:75-160)
    on float32 trajectories:
    dcf_radial2d: 2D radial, 24 spokes x 33 samples through k = 0 (the centre
    repeated 24 times), ratio 0.1;
    dcf_spiral_shots: one 400-sample spiral interleaf as 6 uniformly rotated
    shots (nshots = 6; the shots share k = 0);
    dcf_spiral_edge: 4 rotated 300-sample interleaves, fix_edge, ratio 0.2;
    dcf_koosh3d: 3D golden-means kooshball, 60 spokes x 12 samples."""
    dcf = import_reference_dcf()
    cases = {}
    ang = np.pi * np.arange(24) / 24
    r = np.linspace(-16, 16, 33)
    c = np.stack([np.outer(np.cos(ang), r), np.outer(np.sin(ang), r)], axis=-1).astype(np.float32)
    cases["dcf_radial2d"] = (c, dict(nshots=1, fix_edge=False, ratio=0.1))
    c = synth.spiral_2d(400, 48, nturns=6)[0]
    cases["dcf_spiral_shots"] = (c, dict(nshots=6, fix_edge=False, ratio=0.1))
    c = np.concatenate([synth.spiral_2d(300, 40, rotation=0.5 * np.pi * s, nturns=5) for s in range(4)])
    cases["dcf_spiral_edge"] = (c, dict(nshots=1, fix_edge=True, ratio=0.2))
    c = synth.kooshball_3d(60, 12, 16)
    cases["dcf_koosh3d"] = (c, dict(nshots=1, fix_edge=False, ratio=0.1))
    for name, (c, kw) in cases.items():
        w = dcf.voronoi(np.array(c, copy=True), **kw)
        np.savez_compressed(os.path.join(HERE, name + ".npz"), coord=c, dcf=np.asarray(w),
                            nshots=kw["nshots"], fix_edge=kw["fix_edge"], ratio=kw["ratio"])
        print("wrote", name, np.asarray(w).shape)


def calib_cases(seed=0):
    """Calibration callers of the reference on NUFFT data.

    calib2d: 2D golden-angle radial (128 spokes x 192 samples, 96^2 image,
    8 coils, ramp density weights), k-space = the reference's forward NUFFT of
    coil maps x phantom plus noise, in the 2D non-Cartesian layout (nslices=1,
    ncoils, ncontrasts=1, nviews, nsamples): find_acs (_find_noncart_acs,
    src/deepmr/recon/calib/acs.py:117-152, calibration grid 64^2) and
    espirit_cal (src/deepmr/recon/calib/espirit.py:14-223, k=6, r=24, t=0.02,
    c=0) maps and calibration data.
    calib3d: 3D golden-means kooshball (600 spokes x 48 samples, 24^3 image,
    4 coils): find_acs with a 16^3 calibration grid."""
    N, F = import_reference()
    acs, espirit = import_reference_calib()
    n, nc = 96, 8
    coord = torch.as_tensor(synth.radial_2d(128, 192, n))
    dcf = torch.as_tensor(synth.ramp_dcf(coord.numpy()))
    maps = torch.as_tensor(synth.coil_maps(nc, (n, n), seed=seed + 3))
    img = torch.as_tensor(synth.ellipse_phantom(n, seed=seed + 4)).to(torch.complex64) * maps
    y = F.nufft(img, coord, shape=n)  # (ncoils, nviews, nsamples)
    g = torch.Generator().manual_seed(seed + 9)
    y = (y + 1e-3 * torch.complex(torch.randn(y.shape, generator=g), torch.randn(y.shape, generator=g))).to(
        torch.complex64)
    data = y[None, :, None]  # (nslices, ncoils, ncontrasts, nviews, nsamples)
    cal = acs.find_acs(data, [64, 64], coord, dcf)
    emaps, ecal = espirit.espirit_cal(data, coord=coord, dcf=dcf, shape=n)
    np.savez_compressed(os.path.join(HERE, "calib2d.npz"), coord=_np(coord), dcf=_np(dcf), kspace=_np(data),
                        shape=np.int32(n), acs=_np(cal), maps=_np(emaps), cal=_np(ecal))
    print("wrote calib2d")

    n3, nc3 = 24, 4
    coord3 = torch.as_tensor(synth.kooshball_3d(600, 48, n3))
    img3 = torch.as_tensor(synth.complex_gaussian((nc3, n3, n3, n3), seed=seed + 11))
    y3 = F.nufft(img3, coord3, shape=n3)[:, None]  # (ncoils, ncontrasts, nviews, nsamples)
    cal3 = acs.find_acs(y3, [16, 16, 16], coord3, None)
    np.savez_compressed(os.path.join(HERE, "calib3d.npz"), coord=_np(coord3), kspace=_np(y3),
                        shape=np.int32(n3), acs=_np(cal3))
    print("wrote calib3d")

    # Cartesian find_acs (acs.py:54-114) on undersampled 2D multi-slice data
    # (fully sampled 10 x 8 centre, every other line outside), and the signal
    # helpers espirit_cal uses (resample up and down, rss, fermi)
    g = torch.Generator().manual_seed(seed + 13)
    cart = torch.complex(torch.randn(2, 4, 2, 32, 24, generator=g), torch.randn(2, 4, 2, 32, 24, generator=g))
    mask = torch.zeros(32, 24, dtype=torch.bool)
    mask[::2, :] = True
    mask[11:21, 8:16] = True
    cart = cart * mask
    cal_cart = acs.find_acs(cart)
    sig = sys.modules["deepmr._signal"]
    filt_mod = sys.modules["deepmr._signal.filter"]
    x = torch.complex(torch.randn(3, 16, 20, generator=g), torch.randn(3, 16, 20, generator=g))
    xr = torch.randn(3, 16, 20, generator=g)
    np.savez_compressed(os.path.join(HERE, "calib_cart.npz"), kspace=_np(cart), acs=_np(cal_cart),
                        x=_np(x), x_up=_np(sig.resample(x, [24, 24])), x_down=_np(sig.resample(x, [12, 14])),
                        xr=_np(xr), xr_up=_np(sig.resample(xr, [24, 24])), x_rss=_np(sig.rss(x, axis=0)),
                        fermi=_np(filt_mod.fermi(2, 24, 10)))
    print("wrote calib_cart")


def nufft_case(N, F, name, coord, shape, batch_shape, width, oversamp, weight=None,
               real_image=False, real_kspace=False, seed=0):
    """Run reference forward + adjoint on seeded inputs and save them."""
    coord = torch.as_tensor(coord, dtype=torch.float32)
    plan = N.plan_nufft(coord, shape, width=width, oversamp=oversamp)
    ndim = coord.shape[-1]
    nframes = coord.shape[0] if coord.ndim == 4 else 1
    img_shape = list(batch_shape) + ([nframes] if nframes > 1 else []) + list(plan.shape)
    g = torch.Generator().manual_seed(seed)
    if real_image:
        img = torch.randn(img_shape, generator=g, dtype=torch.float32)
    else:
        img = torch.complex(torch.randn(img_shape, generator=g), torch.randn(img_shape, generator=g))
    ksp_shape = list(batch_shape) + ([nframes] if nframes > 1 else []) + list(plan.interpolator.ishape)
    if real_kspace:
        ksp = torch.randn(ksp_shape, generator=g, dtype=torch.float32)
    else:
        ksp = torch.complex(torch.randn(ksp_shape, generator=g), torch.randn(ksp_shape, generator=g))
    w = None if weight is None else torch.as_tensor(weight, dtype=torch.float32)
    y = N.apply_nufft(img.clone(), plan, weight=w)
    x = N.apply_nufft_adj(ksp.clone(), plan, weight=w)
    out = dict(
        coord=_np(coord), shape=np.asarray(shape), width=np.asarray(width),
        oversamp=np.asarray(oversamp, dtype=np.float64), image=_np(img), kspace=_np(ksp),
        fwd=_np(y), adj=_np(x), plan_beta=np.asarray(plan.beta, dtype=np.float32),
        plan_os_shape=np.asarray(plan.os_shape, dtype=np.int32),
        plan_width=np.asarray(plan.width, dtype=np.int32),
        plan_oversamp=np.asarray(plan.oversamp, dtype=np.float32),
        plan_scale=np.float64(plan.interpolator.scale), ndim=np.int32(ndim),
    )
    if w is not None:
        out["weight"] = _np(w)
    np.savez_compressed(os.path.join(HERE, name + ".npz"), **out)
    print(f"{name}: fwd {tuple(y.shape)} adj {tuple(x.shape)} os {plan.os_shape} "
          f"w {plan.width} scale {plan.interpolator.scale:.6g}")


def toeplitz_case(N, name, coord, shape, batch_shape, dcf=None, width=4, seed=0):
    coord = torch.as_tensor(coord, dtype=torch.float32)
    d = None if dcf is None else torch.as_tensor(dcf, dtype=torch.float32)
    T = N.plan_toeplitz_nufft(coord, shape, dcf=d, width=width)
    T.value = T.value.numpy()  # CPU path needs a numpy value (toeplitz.py:85)
    ndim = coord.shape[-1]
    nframes = coord.shape[0] if coord.ndim == 4 else 1
    sh = [shape] * ndim if np.isscalar(shape) else list(shape)
    img_shape = list(batch_shape) + ([nframes] if nframes > 1 else []) + sh
    g = torch.Generator().manual_seed(seed)
    img = torch.complex(torch.randn(img_shape, generator=g), torch.randn(img_shape, generator=g))
    out_img = N.apply_nufft_selfadj(img.clone(), T)
    out = dict(coord=_np(coord), shape=np.asarray(shape), width=np.asarray(width),
               image=_np(img), selfadj=_np(out_img), kernel=np.asarray(T.value),
               kshape=np.asarray(T.shape, dtype=np.int32), ndim=np.int32(ndim))
    if d is not None:
        out["dcf"] = _np(d)
    np.savez_compressed(os.path.join(HERE, name + ".npz"), **out)
    print(f"{name}: kernel {np.asarray(T.value).shape} out {tuple(out_img.shape)}")


def lowrank_case(N, name, coord, shape, batch_shape, width, oversamp, weight=None, real_basis=False, seed=0):
    """Low-rank subspace NUFFT with a square basis (ncoeff = nframes, the only
    case the reference runs): forward with basis_adjoint (nframes, ncoeff),
    adjoint with basis (ncoeff, nframes)."""
    coord = torch.as_tensor(coord, dtype=torch.float32)
    plan = N.plan_nufft(coord, shape, width=width, oversamp=oversamp)
    ndim = coord.shape[-1]
    nframes = coord.shape[0]
    g = torch.Generator().manual_seed(seed)
    if real_basis:
        basis = torch.randn(nframes, nframes, generator=g)
    else:
        basis = torch.complex(torch.randn(nframes, nframes, generator=g), torch.randn(nframes, nframes, generator=g))
    basis_adj = basis.conj().t().contiguous()
    img_shape = list(batch_shape) + [nframes] + list(plan.shape)
    img = torch.complex(torch.randn(img_shape, generator=g), torch.randn(img_shape, generator=g))
    ksp_shape = list(batch_shape) + [nframes] + list(plan.interpolator.ishape)
    ksp = torch.complex(torch.randn(ksp_shape, generator=g), torch.randn(ksp_shape, generator=g))
    w = None if weight is None else torch.as_tensor(weight, dtype=torch.float32)
    y = N.apply_nufft(img.clone(), plan, basis_adjoint=basis_adj, weight=w)
    x = N.apply_nufft_adj(ksp.clone(), plan, basis=basis, weight=w)
    out = dict(coord=_np(coord), shape=np.asarray(shape), width=np.asarray(width),
               oversamp=np.asarray(oversamp, dtype=np.float64), image=_np(img), kspace=_np(ksp),
               basis=_np(basis), basis_adjoint=_np(basis_adj), fwd=_np(y), adj=_np(x), ndim=np.int32(ndim))
    if w is not None:
        out["weight"] = _np(w)
    np.savez_compressed(os.path.join(HERE, name + ".npz"), **out)
    print(f"{name}: fwd {tuple(y.shape)} adj {tuple(x.shape)}")


def lowrank_cases(N):
    # 2D, 4 frames of rotated radial spokes, complex basis, density weights
    c = np.stack([synth.radial_2d(6, 20, 16, angle_offset=0.41 * f) for f in range(4)])
    lowrank_case(N, "lowrank2d", c, 16, [2], 4, 1.25, weight=synth.ramp_dcf(c[0])[None].repeat(4, 0))
    # 3D, 3 frames, real basis
    c = np.stack([synth.kooshball_3d(20, 12, 8) * (1.0 - 0.1 * f) for f in range(3)]).astype(np.float32)
    lowrank_case(N, "lowrank3d", c, 8, [1], 4, 1.25, real_basis=True, seed=1)


def sparse_case(S, name, indexes, shape, batch_shape, weight=None, basis=False, seed=0):
    """Cartesian sparse FFT (src/deepmr/fft/sparse_fft.py): forward, adjoint,
    self-adjoint (Toeplitz counts; not with a basis) on seeded inputs."""
    idx = torch.as_tensor(indexes, dtype=torch.int16)
    mask = S.prepare_sampling(idx, shape)
    ndim = idx.shape[-1]
    nframes = idx.shape[0] if idx.ndim == 4 else 1
    sh = [shape] * ndim if np.isscalar(shape) else list(shape)
    g = torch.Generator().manual_seed(seed)
    b = ba = None
    if basis:
        b = torch.complex(torch.randn(nframes, nframes, generator=g), torch.randn(nframes, nframes, generator=g))
        ba = b.conj().t().contiguous()
    img_shape = list(batch_shape) + ([nframes] if nframes > 1 else []) + sh
    img = torch.complex(torch.randn(img_shape, generator=g), torch.randn(img_shape, generator=g))
    y = S.apply_sparse_fft(img.clone(), mask, basis_adjoint=ba,
                           weight=None if weight is None else torch.as_tensor(weight, dtype=torch.float32))
    ksp = torch.complex(torch.randn(tuple(y.shape), generator=g), torch.randn(tuple(y.shape), generator=g))
    x = S.apply_sparse_ifft(ksp.clone(), mask, basis=b,
                            weight=None if weight is None else torch.as_tensor(weight, dtype=torch.float32))
    out = dict(indexes=_np(idx), shape=np.asarray(shape), image=_np(img), kspace=_np(ksp), fwd=_np(y), adj=_np(x),
               ndim=np.int32(ndim))
    if weight is not None:
        out["weight"] = np.asarray(weight, np.float32)
    if basis:
        out["basis"] = _np(b)
        out["basis_adjoint"] = _np(ba)
    else:
        T = S.plan_toeplitz_fft(idx, shape)
        out["kernel"] = _np(T.value)
        out["selfadj"] = _np(S.apply_sparse_fft_selfadj(img.clone(), T))
    np.savez_compressed(os.path.join(HERE, name + ".npz"), **out)
    print(f"{name}: fwd {tuple(y.shape)} adj {tuple(x.shape)}")


def sparse_cases():
    S = sys.modules["deepmr.fft.sparse_fft"]
    rng = np.random.default_rng(7)
    # 2D, 3 frames, repeated indexes, per-sample weights
    idx = rng.integers(0, 12, size=(3, 5, 8, 2))
    idx[0, 0, :3] = idx[0, 0, 3]
    sparse_case(S, "sparse2d", idx, 12, [2], weight=rng.uniform(0.2, 1.0, (3, 5, 8)))
    # 2D anisotropic grid (10, 14), single frame
    idx = np.stack([rng.integers(0, 14, (6, 9)), rng.integers(0, 10, (6, 9))], -1)
    sparse_case(S, "sparse2d_aniso", idx, (10, 14), [3], seed=1)
    # 3D single frame
    idx = rng.integers(0, 8, size=(4, 10, 3))
    sparse_case(S, "sparse3d", idx, 8, [2], seed=2)
    # 2D, 3 frames, square complex subspace basis
    idx = rng.integers(0, 10, size=(3, 4, 6, 2))
    sparse_case(S, "sparse2d_lowrank", idx, 10, [2], basis=True, seed=3)


def main():
    N, _ = import_reference()
    if sys.argv[1:] == ["lowrank"]:
        lowrank_cases(N)
        return
    if sys.argv[1:] == ["cgsense"]:
        cgsense_case()
        return
    if sys.argv[1:] == ["sparse"]:
        sparse_cases()
        return
    if sys.argv[1:] == ["dcf"]:
        dcf_cases()
        return
    if sys.argv[1:] == ["calib"]:
        calib_cases()
        return

    # 2D golden-angle radial, width 3 / oversampling 2 (the 2D benchmark's kernel)
    c = synth.radial_2d(16, 32, 32)
    nufft_case(N, None, "radial2d_w3_os2", c, 32, [2], 3, 2.0, weight=synth.ramp_dcf(c))

    # 2D, library defaults width 4 / oversampling 1.25 (grid 30, not a power of 2)
    c = synth.radial_2d(20, 24, 24, angle_offset=0.1)
    nufft_case(N, None, "radial2d_w4_os125", c, 24, [3], 4, 1.25)

    # 2D with 3 frames, each with its own rotated trajectory (frames axis before space)
    c = np.stack([synth.radial_2d(4, 16, 16, angle_offset=0.37 * f) for f in range(3)])
    nufft_case(N, None, "frames2d", c, 16, [2], 4, 1.25)

    # 2D odd/anisotropic matrix (15, 20) and odd oversampled grid; real-valued inputs
    c = synth.radial_2d(12, 20, (15, 20), angle_offset=0.2)
    nufft_case(N, None, "aniso2d_real", c, (15, 20), [2], 3, 1.25,
               real_image=True, real_kspace=True)

    # 2D edge coordinates: exact -N/2, +N/2 (wraps), half-integers where k - W/2 is integral
    rng = np.random.default_rng(5)
    c = rng.uniform(-8, 8, size=(3, 10, 2)).astype(np.float32)
    c[0, 0] = [-8.0, -8.0]
    c[0, 1] = [8.0, 7.5]
    c[0, 2] = [0.5, -0.5]
    c[0, 3] = [1.5, 2.25]
    c[1, 4] = [-7.9999995, 7.9999995]
    nufft_case(N, None, "edges2d", c, 16, [1], 4, 1.25, weight=rng.uniform(0.1, 1, (3, 10)))

    # 1D
    c = np.sort(rng.uniform(-16, 16, size=(1, 40, 1)).astype(np.float32), axis=1)
    nufft_case(N, None, "line1d", c, 32, [2], 4, 1.25)

    # 3D golden-means kooshball, width 4 / oversampling 1.25 (the 3D benchmark's kernel)
    c = synth.kooshball_3d(40, 16, 12)
    nufft_case(N, None, "koosh3d_w4_os125", c, 12, [2], 4, 1.25, weight=synth.ramp_dcf(c))

    # 3D anisotropic matrix, per-axis widths and oversampling
    c = synth.kooshball_3d(30, 12, (8, 10, 12))
    nufft_case(N, None, "aniso3d", c, (8, 10, 12), [1], (3, 4, 5), (1.5, 1.25, 2.0))

    # Cartesian bypass: integer coordinates (every axis detected Cartesian, W=1)
    nodes = np.arange(6) - 3
    yy, xx = np.meshgrid(nodes, nodes, indexing="ij")
    c = np.stack([xx.ravel(), yy.ravel()], -1)[None].astype(np.float32)
    nufft_case(N, None, "cart2d", c, 6, [2], 4, 1.25)

    # Mixed: x Cartesian (integers), y non-Cartesian
    c = np.stack([np.repeat(np.arange(-4, 4), 5), rng.uniform(-4, 4, 40)], -1)[None].astype(np.float32)
    nufft_case(N, None, "mixed2d", c, 8, [2], 4, 1.25)

    # Toeplitz self-adjoint, 2D and 3D, with and without density weights, with frames
    c = synth.radial_2d(24, 32, 16)
    toeplitz_case(N, "toep2d", c, 16, [2], dcf=synth.ramp_dcf(c))
    c = synth.radial_2d(10, 16, 12, angle_offset=0.3)
    toeplitz_case(N, "toep2d_nodcf", c, 12, [1])
    c = np.stack([synth.radial_2d(6, 16, 10, angle_offset=0.5 * f) for f in range(2)])
    toeplitz_case(N, "toep2d_frames", c, 10, [2])
    c = synth.kooshball_3d(30, 16, 8)
    toeplitz_case(N, "toep3d", c, 8, [2], dcf=synth.ramp_dcf(c))

    lowrank_cases(N)
    sparse_cases()
    cgsense_case()
    calib_cases()
    dcf_cases()


if __name__ == "__main__":
    main()
