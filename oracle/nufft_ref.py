"""ORACLE — test infrastructure only, never part of the product path.

CPU restatement of the reference NUFFT pipeline (deepmr ``deepmr.fft``), used
to check the CUDA library. Only ``tests/``, ``__graft_entry__.smoke()`` and
``bench.py``'s CPU-baseline leg may use it.

The per-sample loops run in ``oracle/kernels.c`` (plain C, OpenMP); the plan
arithmetic, zero-padding, apodisation and FFTs are restated here with numpy /
torch-CPU operations chosen to reproduce the reference's float32/float64
promotion rules (numpy >= 2 scalar semantics). Each function cites the
reference routine it follows (paths relative to the reference project).

The restatement is pinned against outputs of the reference itself, generated
by ``tests/golden/make_golden.py`` and checked in ``tests/test_oracle_golden.py``.
"""

import ctypes
import itertools
import math
from dataclasses import dataclass

import numpy as np
import torch

from . import build as _build

_LIB = None


def lib():
    """Load (building first if needed) the oracle's C library."""
    global _LIB
    if _LIB is None:
        path = _build.build()
        L = ctypes.CDLL(path)
        f32p = ctypes.POINTER(ctypes.c_float)
        i32p = ctypes.POINTER(ctypes.c_int32)
        L.oracle_kb.restype = ctypes.c_double
        L.oracle_kb.argtypes = [ctypes.c_double, ctypes.c_double]
        L.oracle_prepare_interpolator.restype = None
        L.oracle_prepare_interpolator.argtypes = [
            f32p, ctypes.c_int64, ctypes.c_int, ctypes.c_double, ctypes.c_int,
            f32p, i32p,
        ]
        for name in ("oracle_interpolate", "oracle_gridding"):
            fn = getattr(L, name)
            fn.restype = None
            fn.argtypes = [
                ctypes.c_int, ctypes.c_int64, ctypes.c_int64, ctypes.c_int64,
                i32p, i32p, ctypes.c_void_p, ctypes.c_void_p,
                ctypes.POINTER(ctypes.c_void_p), ctypes.POINTER(ctypes.c_void_p),
            ]
        L.oracle_nudft.restype = None
        L.oracle_nudft.argtypes = [
            ctypes.c_int, ctypes.c_int64, ctypes.c_int64, i32p,
            ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p,
        ]
        _LIB = L
    return _LIB


def _ptr(a, ctype=ctypes.c_float):
    return a.ctypes.data_as(ctypes.POINTER(ctype))


def kaiser_bessel(x, beta):
    """KB kernel of src/deepmr/fft/_interp/plan.py:216-248 (double precision)."""
    return lib().oracle_kb(float(x), float(beta))


# --------------------------------------------------------------------------
# plan (src/deepmr/fft/nufft.py:27-132, src/deepmr/fft/_interp/plan.py:14-213)
# --------------------------------------------------------------------------
@dataclass
class OracleInterpolator:
    index: list  # per axis (z, y, x): int32 (F, npts, W)
    value: list  # per axis (z, y, x): float32 (F, npts, W)
    dshape: tuple  # oversampled grid (z, y, x)
    ishape: tuple  # (nviews, nsamples)
    scale: float
    ndim: int


@dataclass
class OraclePlan:
    ndim: int
    oversamp: tuple
    width: tuple
    beta: tuple
    os_shape: tuple
    shape: tuple
    interpolator: OracleInterpolator


def _axis_array(v, ndim, dtype):
    if np.isscalar(v):
        return np.asarray([v] * ndim, dtype=dtype)
    return np.asarray(v, dtype=dtype)


def cartesian_axes(coord, shape):
    """Per-axis Cartesian test of src/deepmr/fft/nufft.py:104-109.

    The reference multiplies coordinate axis ``ax`` (x, y, z order) by
    ``shape[ax]`` (z, y, x order) and tests closeness to an integer in float32
    with numpy.allclose; the list is then reversed into (z, y, x) order.
    """
    coord = np.asarray(coord, dtype=np.float32)
    ndim = coord.shape[-1]
    flags = []
    for ax in range(ndim):
        a = shape[ax] * coord[..., ax]  # int16 scalar * float32 -> float32
        flags.append(bool(np.allclose(a, np.round(a))))
    return np.asarray(flags[::-1])


def kernel_scaling(beta_xyz, width_xyz):
    """Sum of the separable kernel on its nodes, plan.py:190-213 (float64)."""
    axes = []
    for w, b in zip(width_xyz, beta_xyz):
        if w == 1:
            axes.append(np.array([1.0]))
            continue
        start = np.ceil(-w / 2)
        axes.append(np.array([kaiser_bessel((start + el) / (w / 2), b) for el in range(w)]))
    grids = np.meshgrid(*axes)
    return np.stack(grids, axis=0).prod(axis=0).sum()


def plan_interpolator(coord, os_shape_zyx, width_zyx, beta_zyx):
    """Interpolator tables of src/deepmr/fft/_interp/plan.py:14-143."""
    coord = torch.as_tensor(coord, dtype=torch.float32)
    ndim = coord.shape[-1]
    ishape = list(coord.shape[:-1])
    while len(ishape) < 3:
        ishape = [1] + ishape
    nframes = ishape[0]
    ishape = ishape[1:]
    npts = int(np.prod(ishape))
    shape_xyz = list(os_shape_zyx)[::-1]
    width_xyz = list(width_zyx)[::-1]
    beta_xyz = list(beta_zyx)[::-1]
    scale = kernel_scaling(beta_xyz, width_xyz)
    c = np.ascontiguousarray(coord.reshape(nframes * npts, ndim).numpy().T)
    index, value = [], []
    for a in range(ndim):
        w = int(width_xyz[a])
        ca = np.ascontiguousarray(c[a])
        if w == 1:
            # Cartesian axis: nearest node by truncation, weight 1 (plan.py:117-121)
            idx = torch.from_numpy(ca).to(torch.int32).numpy()[:, None].copy()
            val = np.ones((nframes * npts, 1), dtype=np.float32)
        else:
            val = np.zeros((nframes * npts, w), dtype=np.float32)
            idx = np.zeros((nframes * npts, w), dtype=np.int32)
            lib().oracle_prepare_interpolator(
                _ptr(ca), nframes * npts, w, float(beta_xyz[a]), int(shape_xyz[a]),
                _ptr(val), _ptr(idx, ctypes.c_int32),
            )
        index.append(idx.reshape(nframes, npts, w))
        value.append(val.reshape(nframes, npts, w))
    return OracleInterpolator(
        index[::-1], value[::-1], tuple(int(s) for s in os_shape_zyx),
        tuple(ishape), float(scale), ndim,
    )


def scale_coord(coord, shape_xyz, oversamp_xyz):
    """Coordinate rescale of src/deepmr/fft/nufft.py:411-420, in float32."""
    ndim = coord.shape[-1]
    out = coord.clone()
    for i in range(-ndim, 0):
        g = np.ceil(oversamp_xyz[i] * shape_xyz[i])  # float32
        out[..., i] *= g / shape_xyz[i]
        out[..., i] += g // 2
    return out


def plan_nufft(coord, shape, width=4, oversamp=1.25):
    """NUFFT plan of src/deepmr/fft/nufft.py:27-132 (CPU tables)."""
    coord = torch.as_tensor(coord).clone().cpu().to(torch.float32)
    ndim = coord.shape[-1]
    width = _axis_array(width, ndim, np.int16)
    oversamp = _axis_array(oversamp, ndim, np.float32)
    beta = math.pi * (((width / oversamp) * (oversamp - 0.5)) ** 2 - 0.8) ** 0.5
    if np.isscalar(shape):
        shape = np.asarray([shape] * ndim, dtype=np.int16)
    else:
        shape = np.asarray(shape, dtype=np.int16)[-ndim:]
    is_cart = cartesian_axes(coord.numpy(), shape)
    oversamp[is_cart] = 1.0
    width[is_cart] = 1
    os_shape = np.ceil(oversamp * shape).astype(np.int16)
    coord = scale_coord(coord, shape[::-1], oversamp[::-1])
    interp = plan_interpolator(coord, os_shape, width, beta)
    return OraclePlan(ndim, tuple(oversamp), tuple(width), tuple(beta),
                      tuple(os_shape), tuple(shape), interp)


# --------------------------------------------------------------------------
# helpers: resize (src/deepmr/_signal/resize.py:11-102), centered FFT
# (src/deepmr/fft/fft.py:9-167), apodisation (src/deepmr/fft/nufft.py:423-447)
# --------------------------------------------------------------------------
def resize(x, oshape):
    """Centered zero-pad / crop with offsets i//2 - o//2 (resize.py:80-97)."""
    oshape = list(oshape)
    ishape = list(x.shape)
    oshape = ishape[: len(ishape) - len(oshape)] + oshape
    if ishape == oshape:
        return x
    out = torch.zeros(oshape, dtype=x.dtype)
    islc, oslc = [], []
    for i, o in zip(ishape, oshape):
        si = max(i // 2 - o // 2, 0)
        so = max(o // 2 - i // 2, 0)
        n = min(i - si, o - so)
        islc.append(slice(si, si + n))
        oslc.append(slice(so, so + n))
    out[tuple(oslc)] = x[tuple(islc)]
    return out


def centered_fft(x, ndim, norm=None, inverse=False, centered=True):
    dims = tuple(range(-ndim, 0))
    op = torch.fft.ifftn if inverse else torch.fft.fftn
    if not centered:
        return op(x, dim=dims, norm=norm)
    return torch.fft.fftshift(op(torch.fft.ifftshift(x, dim=dims), dim=dims, norm=norm), dim=dims)


def apodize(x, ndim, oversamp, width, beta):
    """In-place KB apodisation, one axis at a time from the last (nufft.py:423-447)."""
    for n in range(1, ndim + 1):
        axis = -n
        if width[axis] == 1:
            continue
        i = x.shape[axis]
        os_i = np.ceil(oversamp[axis] * i)
        idx = torch.arange(i, dtype=torch.float32)
        ap = (beta[axis] ** 2 - (math.pi * width[axis] * (idx - i // 2) / os_i) ** 2) ** 0.5
        ap /= torch.sinh(ap)
        ap = ap / ap[int(i // 2)]
        ap = torch.nan_to_num(ap, nan=1.0)
        x *= ap.reshape([i] + [1] * (-axis - 1))
    return x


def _as_cfloat(x):
    x = torch.as_tensor(x)
    if x.dtype in (torch.float16, torch.float32, torch.float64):
        return x.to(torch.float32)
    return x.to(torch.complex64)


# --------------------------------------------------------------------------
# interpolation / gridding drivers (interp.py:14-120, grid.py:14-125)
# --------------------------------------------------------------------------
def _tables(interp):
    vals = [np.ascontiguousarray(v) for v in interp.value]
    idxs = [np.ascontiguousarray(i) for i in interp.index]
    vptr = (ctypes.c_void_p * 3)(*[v.ctypes.data for v in vals] + [0] * (3 - len(vals)))
    iptr = (ctypes.c_void_p * 3)(*[i.ctypes.data for i in idxs] + [0] * (3 - len(idxs)))
    width = np.asarray([v.shape[-1] for v in vals], dtype=np.int32)
    gshape = np.asarray(interp.dshape, dtype=np.int32)
    return vals, idxs, vptr, iptr, width, gshape


def interpolate(data_in, interp):
    """Grid -> samples, interp.py:14-120 (returns data_out / scale)."""
    data_in = _as_cfloat(data_in).to(torch.complex64)
    ndim = interp.ndim
    nframes = interp.index[0].shape[0]
    npts = int(np.prod(interp.ishape))
    batch_shape = data_in.shape[:-ndim] if nframes == 1 else data_in.shape[: -ndim - 1]
    batch = int(np.prod(batch_shape))
    x = data_in.reshape(batch, nframes, *interp.dshape).swapaxes(0, 1).contiguous().numpy()
    out = np.zeros((nframes, batch, npts), dtype=np.complex64)
    keep = _tables(interp)
    _, _, vptr, iptr, width, gshape = keep
    lib().oracle_interpolate(
        ndim, nframes, batch, npts, _ptr(gshape, ctypes.c_int32), _ptr(width, ctypes.c_int32),
        x.ctypes.data, out.ctypes.data, vptr, iptr,
    )
    out = torch.from_numpy(out)
    if nframes == 1:
        out = out[0].reshape(*batch_shape, *interp.ishape)
    else:
        out = out.swapaxes(0, 1).reshape(*batch_shape, nframes, *interp.ishape)
    return out / interp.scale


def gridding(data_in, interp):
    """Samples -> grid, grid.py:14-125 (returns data_out / scale)."""
    data_in = _as_cfloat(data_in).to(torch.complex64)
    ndim = interp.ndim
    nframes = interp.index[0].shape[0]
    npts = int(np.prod(interp.ishape))
    batch_shape = data_in.shape[:-2] if nframes == 1 else data_in.shape[:-3]
    batch = int(np.prod(batch_shape))
    x = data_in.reshape(batch, nframes, npts).swapaxes(0, 1).contiguous().numpy()
    out = np.zeros((nframes, batch, *interp.dshape), dtype=np.complex64)
    keep = _tables(interp)
    _, _, vptr, iptr, width, gshape = keep
    lib().oracle_gridding(
        ndim, nframes, batch, npts, _ptr(gshape, ctypes.c_int32), _ptr(width, ctypes.c_int32),
        out.ctypes.data, x.ctypes.data, vptr, iptr,
    )
    out = torch.from_numpy(out)
    if nframes == 1:
        out = out[0].reshape(*batch_shape, *interp.dshape)
    else:
        out = out.swapaxes(0, 1).reshape(*batch_shape, nframes, *interp.dshape)
    return out / interp.scale


def gridding_exact(data_in, interp):
    """`gridding` with every grid point summed in float64 (numpy bincount over
    the same tap tables), complex128 out. Not the reference's arithmetic: its
    sequential float32 sums lose the small late addends of grid points that
    collect many samples (the Toeplitz point-spread function of the full
    kooshball: 7.4e-5 relative L2 from this sum), so at full size a parallel
    implementation is checked against this exact sum instead."""
    data_in = _as_cfloat(data_in).to(torch.complex128)
    ndim = interp.ndim
    nframes = interp.index[0].shape[0]
    npts = int(np.prod(interp.ishape))
    batch_shape = data_in.shape[:-2] if nframes == 1 else data_in.shape[:-3]
    batch = int(np.prod(batch_shape))
    x = data_in.reshape(batch, nframes, npts).swapaxes(0, 1).contiguous().numpy()
    dshape = [int(d) for d in interp.dshape]
    size = int(np.prod(dshape))
    out = np.zeros((nframes, batch, size), dtype=np.complex128)
    for f in range(nframes):
        idx = [np.asarray(interp.index[a][f]).astype(np.int64) for a in range(ndim)]
        val = [np.asarray(interp.value[a][f]).astype(np.float64) for a in range(ndim)]
        for taps in itertools.product(*[range(v.shape[-1]) for v in val]):
            flat = np.zeros(npts, dtype=np.int64)
            w = np.ones(npts)
            for a, t in enumerate(taps):
                flat = flat * dshape[a] + idx[a][:, t]
                w = w * val[a][:, t]
            for b in range(batch):
                out[f, b] += np.bincount(flat, weights=w * x[f, b].real, minlength=size)
                if np.any(x[f, b].imag):
                    out[f, b] += 1j * np.bincount(flat, weights=w * x[f, b].imag, minlength=size)
    out = torch.from_numpy(out.reshape(nframes, batch, *dshape))
    if nframes == 1:
        out = out[0].reshape(*batch_shape, *dshape)
    else:
        out = out.swapaxes(0, 1).reshape(*batch_shape, nframes, *dshape)
    return out / interp.scale


# --------------------------------------------------------------------------
# NUFFT pipelines (src/deepmr/fft/nufft.py:450-669)
# --------------------------------------------------------------------------
def apply_nufft(image, plan, weight=None):
    """Forward NUFFT, nufft.py:450-528: apodize, pad, centered FFT, interpolate."""
    isnumpy = isinstance(image, np.ndarray)
    image = _as_cfloat(image).clone()
    ndim = plan.ndim
    apodize(image, ndim, plan.oversamp, plan.width, plan.beta)
    image = resize(image, list(image.shape[:-ndim]) + list(plan.os_shape))
    k = centered_fft(image, ndim, norm=None)
    k = interpolate(k, plan.interpolator)
    if weight is not None:
        k = torch.as_tensor(weight, dtype=torch.float32) * k
    return k.numpy() if isnumpy else k


def apply_nufft_adj(kspace, plan, weight=None, exact=False):
    """Adjoint NUFFT, nufft.py:531-606: grid, centered iFFT, crop, apodize
    (`exact`: the gridding sums in float64, `gridding_exact`, and the rest in
    complex128)."""
    isnumpy = isinstance(kspace, np.ndarray)
    kspace = _as_cfloat(kspace)
    ndim = plan.ndim
    if weight is not None:
        kspace = torch.as_tensor(weight, dtype=torch.float32) * kspace
    g = gridding_exact(kspace, plan.interpolator) if exact else gridding(kspace, plan.interpolator)
    img = centered_fft(g, ndim, norm=None, inverse=True)
    img = resize(img, list(img.shape[:-ndim]) + list(plan.shape))
    apodize(img, ndim, plan.oversamp, plan.width, plan.beta)
    return img.numpy() if isnumpy else img


def apply_nufft_lowrank(image, plan, basis_adjoint, weight=None):
    """Low-rank forward (src/deepmr/fft/_interp/interp.py:230-357): frame f is
    the NUFFT of sum_c basis_adjoint[f, c] image[..., c, :]. Restated through the
    linearity of apodisation, padding and FFT: combine, then transform."""
    ndim = plan.ndim
    ba = torch.as_tensor(basis_adjoint).to(torch.complex64)
    x = _as_cfloat(torch.as_tensor(image)).to(torch.complex64)
    xf = torch.einsum("fc,...cn->...fn", ba, x.reshape(*x.shape[: -ndim], -1)).reshape(
        *x.shape[: -ndim - 1], ba.shape[0], *x.shape[-ndim:])
    return apply_nufft(xf, plan, weight=weight)


def apply_nufft_adj_lowrank(kspace, plan, basis, weight=None):
    """Low-rank adjoint (src/deepmr/fft/_interp/grid.py:287-417): coefficient c
    is sum_f basis[c, f] times the adjoint NUFFT of frame f."""
    ndim = plan.ndim
    b = torch.as_tensor(basis).to(torch.complex64)
    xf = apply_nufft_adj(kspace, plan, weight=weight)
    return torch.einsum("cf,...fn->...cn", b, xf.reshape(*xf.shape[: -ndim], -1)).reshape(
        *xf.shape[: -ndim - 1], b.shape[0], *xf.shape[-ndim:])


def nufft(image, coord, shape=None, width=4, oversamp=1.25):
    """One-shot forward, src/deepmr/fft/__init__.py:145-218."""
    ndim = coord.shape[-1]
    if shape is None:
        shape = image.shape[-ndim:]
    return apply_nufft(image, plan_nufft(coord, shape, width, oversamp))


def nufft_adj(kspace, coord, shape, width=4, oversamp=1.25, exact=False):
    """One-shot adjoint, src/deepmr/fft/__init__.py:221-286."""
    return apply_nufft_adj(kspace, plan_nufft(coord, shape, width, oversamp), exact=exact)


@dataclass
class OracleGram:
    value: torch.Tensor
    shape: tuple
    ndim: int


def plan_toeplitz(coord, shape, dcf=None, width=4, exact=False):
    """Toeplitz kernel of src/deepmr/fft/toeplitz.py:15-157 (plain, no basis).
    `exact`: the point-spread function gridded with float64 sums
    (`gridding_exact`) and transformed in complex128, the kernel cast to
    complex64 at the end."""
    coord = torch.as_tensor(coord, dtype=torch.float32)
    ndim = coord.shape[-1]
    oversamp = np.asarray([2.0] * ndim)
    if np.isscalar(shape):
        shape = np.asarray([shape] * ndim, dtype=np.int16)
    else:
        shape = np.asarray(shape, dtype=np.int16)[-ndim:]
    if dcf is None:
        dcf = torch.ones(coord.shape[:-1], dtype=torch.float32)
    else:
        dcf = torch.as_tensor(dcf)
    delta = torch.ones(list(coord.shape[:-1]), dtype=torch.float32)
    is_cart = cartesian_axes(coord.numpy(), shape)
    oversamp[is_cart] = 1.0
    shape = np.ceil(oversamp * shape).astype(np.int16)
    # coord * float64 array promotes to float64; the plan casts back to float32
    psf = nufft_adj(dcf * delta, coord * torch.as_tensor(oversamp), shape, width=width, exact=exact)
    k = centered_fft(psf, ndim, norm="ortho")
    if k.shape[0] == 1:
        k = k[0]
    k = torch.fft.ifftshift(k, dim=list(range(-ndim, 0)))
    k /= torch.mean(abs(k[k != 0]))
    k = torch.nan_to_num(k)
    if exact:
        k = k.to(torch.complex64)
    return OracleGram(k, tuple(int(s) for s in shape), ndim)


def apply_selfadj(image, gram):
    """Toeplitz self-adjoint, nufft.py:609-669 with toeplitz.py:84-87 (plain)."""
    isnumpy = isinstance(image, np.ndarray)
    image = _as_cfloat(image)
    ndim = gram.ndim
    oshape = image.shape[-ndim:]
    x = resize(image, list(image.shape[:-ndim]) + list(gram.shape))
    k = centered_fft(x, ndim, norm="ortho", centered=False)
    k = gram.value * k
    x = centered_fft(k, ndim, norm="ortho", inverse=True, centered=False)
    x = resize(x, list(x.shape[:-ndim]) + list(oshape))
    return x.numpy() if isnumpy else x


# --------------------------------------------------------------------------
# exact operator (no reference counterpart): direct NUDFT in float64
# --------------------------------------------------------------------------
def nudft(image, coord, shape):
    """y[b,p] = sum_x img[b,x] exp(-2 pi i k.(x - N//2)/N), coord in grid units.

    image: (..., *shape) complex; coord: (M, ndim) (x, y, z order).
    Returns (..., M) complex128.
    """
    shape = [int(s) for s in shape]
    ndim = len(shape)
    img = np.ascontiguousarray(np.asarray(image, dtype=np.complex128))
    lead = img.shape[:-ndim]
    batch = int(np.prod(lead)) if lead else 1
    c = np.ascontiguousarray(np.asarray(coord, dtype=np.float64).reshape(-1, ndim))
    out = np.zeros((batch, c.shape[0]), dtype=np.complex128)
    sh = np.asarray(shape, dtype=np.int32)
    lib().oracle_nudft(ndim, batch, c.shape[0], _ptr(sh, ctypes.c_int32),
                       img.ctypes.data, c.ctypes.data, out.ctypes.data)
    return out.reshape(*lead, c.shape[0])


def rel_l2(a, b):
    """Relative L2 error ||a - b|| / ||b|| in float64."""
    a = np.asarray(a, dtype=np.complex128).ravel()
    b = np.asarray(b, dtype=np.complex128).ravel()
    nb = np.linalg.norm(b)
    return float(np.linalg.norm(a - b) / (nb if nb > 0 else 1.0))


# --------------------------------------------------------------------------
# float64 forward (finite-difference reference for the gradient tests): the
# reference's forward (nufft.py:450-528) with every step in float64; the
# oversampled spectrum is computed once and samples are evaluated on demand
# --------------------------------------------------------------------------
class Forward64:
    """y[..., p] = (1/scale) sum_taps prod KB * K[taps] in float64."""

    def __init__(self, image, coord, shape, width=4, oversamp=1.25):
        import itertools

        self._product = itertools.product
        coord = np.asarray(coord, dtype=np.float32)
        self.ndim = ndim = coord.shape[-1]
        self.plan = plan = plan_nufft(torch.as_tensor(coord), shape, width, oversamp)
        x = torch.as_tensor(np.asarray(image, dtype=np.complex128)).clone()
        for n in range(1, ndim + 1):
            axis = -n
            if plan.width[axis] == 1:
                continue
            i = x.shape[axis]
            os_i = math.ceil(float(plan.oversamp[axis]) * i)
            idx = torch.arange(i, dtype=torch.float64)
            b = float(plan.beta[axis])
            ap = (b**2 - (math.pi * int(plan.width[axis]) * (idx - i // 2) / os_i) ** 2) ** 0.5
            ap = ap / torch.sinh(ap)
            ap = torch.nan_to_num(ap / ap[i // 2], nan=1.0)
            x = x * ap.reshape([i] + [1] * (-axis - 1))
        os_shape = [int(s) for s in plan.os_shape]
        x = resize(x, list(x.shape[:-ndim]) + os_shape)
        self.K = centered_fft(x, ndim, norm=None).numpy()
        self.scale = plan.interpolator.scale
        self.width_xyz = [int(w) for w in plan.width][::-1]
        self.beta_xyz = [float(b) for b in plan.beta][::-1]
        self.G_xyz = os_shape[::-1]
        self.N_xyz = [int(s) for s in plan.shape][::-1]
        self.os_xyz = [float(o) for o in plan.oversamp][::-1]

    def rescaled(self, c):
        """Rescaled (grid-index) coordinates of one sample, float64."""
        out = []
        for a in range(self.ndim):
            g = math.ceil(self.os_xyz[a] * self.N_xyz[a])
            out.append(float(c[a]) * g / self.N_xyz[a] + g // 2)
        return out

    def sample(self, c):
        """y[..., one sample] at coordinates c (grid units, (x, y, z))."""
        taps, wts = [], []
        for a, k in enumerate(self.rescaled(c)):
            W = self.width_xyz[a]
            G = self.G_xyz[a]
            if W == 1:
                taps.append([int(k) % G])
                wts.append([1.0])
                continue
            x0 = math.ceil(k - W / 2)
            taps.append([(x0 + i) % G for i in range(W)])
            wts.append([kaiser_bessel(((x0 + i) - k) / (W / 2), self.beta_xyz[a]) for i in range(W)])
        acc = np.zeros(self.K.shape[:-self.ndim], dtype=np.complex128)
        for combo in self._product(*[range(len(t)) for t in taps]):
            w = 1.0
            index = []
            for a, i in enumerate(combo):
                w *= wts[a][i]
                index.append(taps[a][i])
            acc = acc + w * self.K[(...,) + tuple(index[::-1])]
        return acc / self.scale


# ---------------------------------------------------------------------------
# Cartesian sparse FFT (src/deepmr/fft/sparse_fft.py, src/deepmr/fft/_sparse/*)
# ---------------------------------------------------------------------------
def _sparse_index(indexes, ndim):
    idx = np.asarray(indexes).astype(np.int64)
    ish = list(idx.shape[:-1])
    while len(ish) < 3:
        ish = [1] + ish
    return idx.reshape(ish[0], -1, ndim), ish[0], tuple(ish[1:])


def _centred_fft(x, ndim, inverse=False):
    ax = tuple(range(-ndim, 0))
    x = np.fft.ifftshift(x, axes=ax)
    x = np.fft.ifftn(x, axes=ax) if inverse else np.fft.fftn(x, axes=ax)
    return np.fft.fftshift(x, axes=ax)


def sparse_fft(image, indexes, shape, basis_adjoint=None, weight=None):
    """Centred FFT (unnormalised) then sampling at integer indexes
    (sparse_fft.py:314-383, _sparse/dense2sparse.py); frames as the NUFFT."""
    ndim = np.asarray(indexes).shape[-1]
    idx, nframes, ishape = _sparse_index(indexes, ndim)
    x = np.asarray(image, dtype=np.complex128)
    if basis_adjoint is not None:
        x = np.einsum("fc,...cn->...fn", np.asarray(basis_adjoint), x.reshape(*x.shape[:-ndim], -1)).reshape(
            *x.shape[: -ndim - 1], nframes, *x.shape[-ndim:])
    X = _centred_fft(x, ndim)
    lead = X.shape[: -ndim - 1] if nframes > 1 else X.shape[:-ndim]
    X = X.reshape(-1, nframes, *X.shape[-ndim:])
    out = np.empty((X.shape[0], nframes, idx.shape[1]), np.complex128)
    for f in range(nframes):
        sel = tuple(idx[f, :, a] for a in range(ndim))[::-1]  # (z, y, x) order
        out[:, f] = X[(slice(None), f) + sel]
    if weight is not None:
        out = out * np.asarray(weight, np.float64).reshape(1, nframes, -1)
    shape_out = list(lead) + ([nframes] if nframes > 1 else []) + list(ishape)
    return out.reshape(shape_out).astype(np.complex64)


def sparse_ifft(kspace, indexes, shape, basis=None, weight=None):
    """Zero-fill (repeated indexes summed) then centred inverse FFT (1/N)
    (sparse_fft.py:386-450, _sparse/sparse2dense.py)."""
    ndim = np.asarray(indexes).shape[-1]
    idx, nframes, ishape = _sparse_index(indexes, ndim)
    sh = [int(shape)] * ndim if np.isscalar(shape) else [int(s) for s in shape]
    y = np.asarray(kspace, dtype=np.complex128)
    lead = y.shape[: -len(ishape) - 1] if nframes > 1 else y.shape[: -len(ishape)]
    y = y.reshape(-1, nframes, idx.shape[1])
    if weight is not None:
        y = y * np.asarray(weight, np.float64).reshape(1, nframes, -1)
    grid = np.zeros((y.shape[0], nframes, *sh), np.complex128)
    for f in range(nframes):
        sel = tuple(idx[f, :, a] for a in range(ndim))[::-1]
        for b in range(y.shape[0]):
            np.add.at(grid[b, f], sel, y[b, f])
    x = _centred_fft(grid, ndim, inverse=True)
    if basis is not None:
        x = np.einsum("cf,bfn->bcn", np.asarray(basis), x.reshape(x.shape[0], nframes, -1)).reshape(
            x.shape[0], -1, *sh)
        return x.reshape(list(lead) + [x.shape[1]] + sh).astype(np.complex64)
    return x.reshape(list(lead) + ([nframes] if nframes > 1 else []) + sh).astype(np.complex64)


def sparse_toeplitz_kernel(indexes, shape):
    """Sample counts per k-space point, ifftshifted and normalised (_sparse/toeplitz.py:15-113)."""
    ndim = np.asarray(indexes).shape[-1]
    idx, nframes, _ = _sparse_index(indexes, ndim)
    sh = [int(shape)] * ndim if np.isscalar(shape) else [int(s) for s in shape]
    k = np.zeros((nframes, *sh), np.float64)
    for f in range(nframes):
        np.add.at(k[f], tuple(idx[f, :, a] for a in range(ndim))[::-1], 1.0)
    k = np.fft.ifftshift(k, axes=tuple(range(-ndim, 0)))
    k = k if nframes > 1 else k[0]
    # normalised by the mean non-zero magnitude, NaN -> 0 (_sparse/toeplitz.py:107-111)
    nz = k[k != 0]
    return np.nan_to_num(k / (np.abs(nz).mean() if nz.size else np.nan))


def sparse_selfadj(image, kernel, ndim):
    """Uncentred orthonormal FFT, times the kernel, inverse (sparse_fft.py:453-503)."""
    ax = tuple(range(-ndim, 0))
    X = np.fft.fftn(np.asarray(image, np.complex128), axes=ax, norm="ortho")
    return np.fft.ifftn(X * np.asarray(kernel), axes=ax, norm="ortho").astype(np.complex64)
