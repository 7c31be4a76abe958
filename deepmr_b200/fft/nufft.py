"""NUFFT plan and application — drop-in for ``deepmr.fft.nufft``.

Same functions, argument meanings, layouts and scale conventions as the
reference module (src/deepmr/fft/nufft.py); the work runs in the sm_100a CUDA
library through its C ABI:

* ``plan_nufft``  -> Cartesian-axis test on the device, then a device-resident
  plan (rescaled coordinates sorted by spatial bin), nufft.py:27-132.
* ``apply_nufft`` -> one fused apodise/zero-pad/ifftshift kernel, cuFFT, and
  the bin-tiled interpolation kernel, nufft.py:212-245, 450-528.
* ``apply_nufft_adj`` -> bin-tiled gridding, cuFFT, one fused
  fftshift/crop/apodise kernel, nufft.py:289-322, 531-606.
* ``apply_nufft_selfadj`` -> Toeplitz pad/FFT/multiply/iFFT/crop,
  nufft.py:351-375, 609-669.

Computation always happens on a CUDA device. ``device="cpu"`` (the reference
default) keeps its meaning for the *caller*: results are returned on the
input's device, as the reference does (nufft.py:517-523); the plan computes
on the current CUDA device.
"""

__all__ = [
    "plan_nufft",
    "plan_toeplitz_nufft",
    "apply_nufft",
    "apply_nufft_adj",
    "apply_nufft_selfadj",
    "NUFFTPlan",
]

import ctypes
import math
import weakref
from dataclasses import dataclass

import numpy as np
import torch
import torch.autograd as autograd

from .. import _lib
from . import toeplitz as _toeplitz

# ---------------------------------------------------------------------------
# device plan
# ---------------------------------------------------------------------------


def compute_device(device):
    """CUDA device that does the work for a requested ``device``."""
    _lib.require_cuda()
    if device is None:
        return torch.device("cuda", torch.cuda.current_device())
    d = torch.device(device)
    if d.type == "cuda":
        return torch.device("cuda", d.index if d.index is not None else torch.cuda.current_device())
    return torch.device("cuda", torch.cuda.current_device())


def _destroy(handle):
    try:
        _lib.lib().dmr_plan_destroy(handle)
    except Exception:  # interpreter shutdown
        pass


class DevicePlan:
    """Device-resident interpolator: owns a ``dmr_plan`` of the CUDA library.

    Plays the role of the reference's ``Interpolator`` (src/deepmr/fft/_interp/
    plan.py:147-187): ``dshape`` is the oversampled grid (z, y, x), ``ishape``
    the per-frame sample shape (nviews, nsamples), ``scale`` the kernel-sum
    normalisation.
    """

    def __init__(self, coord, frame_offsets, ishape, ndim, shape, os_shape, width, beta,
                 oversamp, device, tile=None):
        self.ndim = int(ndim)
        self.dshape = tuple(int(s) for s in os_shape)
        self.ishape = tuple(int(s) for s in ishape) if ishape is not None else None
        self.frame_offsets = np.asarray(frame_offsets, dtype=np.int64)
        self.nframes = len(self.frame_offsets) - 1
        self.total = int(self.frame_offsets[-1])
        self.device = device
        self._params = (shape, os_shape, width, beta, oversamp, tile)
        self._coord = coord  # raw (total, ndim) float32 on `device`, kept for .to()
        self._build()

    def _build(self):
        shape, os_shape, width, beta, oversamp, tile = self._params
        L = _lib.lib()
        h = ctypes.c_void_p()
        foff = (ctypes.c_int64 * len(self.frame_offsets))(*self.frame_offsets.tolist())
        with torch.cuda.device(self.device):
            _lib.check(
                L.dmr_plan_create(
                    self.ndim,
                    _lib.i32_array(shape),
                    _lib.i32_array(os_shape),
                    _lib.i32_array(width),
                    _lib.f32_array(beta),
                    _lib.f32_array(oversamp),
                    _lib.ptr(self._coord),
                    foff,
                    self.nframes,
                    _lib.i32_array(tile) if tile is not None else None,
                    _lib.stream_ptr(self.device),
                    ctypes.byref(h),
                )
            )
        self.handle = h
        sc = ctypes.c_double()
        _lib.check(L.dmr_plan_scale(h, ctypes.byref(sc)))
        self.scale = float(sc.value)
        self._fin = weakref.finalize(self, _destroy, h)

    def to(self, device):
        dev = compute_device(device)
        if dev != self.device:
            self._fin()
            self.device = dev
            self._coord = self._coord.to(dev)
            self._build()
        return self

    def check_status(self, reset=True):
        """Raise ``DmrError`` (DMR_ERR_TIMEOUT) if a tensor-core gridding block of
        this plan's calls stopped on a bounded device wait since the last reset
        (the results of those calls are then partial). Synchronises the current
        stream of the plan's device; ``reset`` clears the status."""
        n = ctypes.c_int32()
        with torch.cuda.device(self.device):
            _lib.check(_lib.lib().dmr_plan_status(self.handle, ctypes.byref(n), int(bool(reset)),
                                                  _lib.stream_ptr(self.device)))

    def workspace(self, batch):
        n = ctypes.c_size_t()
        with torch.cuda.device(self.device):
            _lib.check(_lib.lib().dmr_nufft_workspace_bytes(self.handle, int(batch), ctypes.byref(n)))
        return torch.empty(int(n.value), dtype=torch.uint8, device=self.device)

    def workspace_lowrank(self, batch, ncoeff):
        n = ctypes.c_size_t()
        with torch.cuda.device(self.device):
            _lib.check(_lib.lib().dmr_nufft_lowrank_workspace_bytes(self.handle, int(batch), int(ncoeff),
                                                                    ctypes.byref(n)))
        return torch.empty(int(n.value), dtype=torch.uint8, device=self.device)


@dataclass
class NUFFTPlan:
    """NUFFT plan (fields of the reference's NUFFTPlan, nufft.py:379-404)."""

    ndim: int
    oversamp: tuple
    width: tuple
    beta: tuple
    os_shape: tuple
    shape: tuple
    interpolator: object
    device: str

    def to(self, device):
        """Dispatch to ``device`` (a CUDA device moves the plan; "cpu" keeps the
        current CUDA device for compute and only changes where results go)."""
        if device != self.device:
            self.interpolator.to(device)
            self.device = device
        return self


def _axis_param(v, ndim, dtype):
    if np.isscalar(v):
        return np.asarray([v] * ndim, dtype=dtype)
    return np.asarray(v, dtype=dtype)


def detect_cartesian(coord_dev, shape_zyx):
    """Per-axis Cartesian flags in (z, y, x) order (nufft.py:104-109), on the device."""
    ndim = coord_dev.shape[-1]
    flags = (ctypes.c_int32 * ndim)()
    with torch.cuda.device(coord_dev.device):
        _lib.check(
            _lib.lib().dmr_detect_cartesian(
                _lib.ptr(coord_dev), coord_dev.numel() // ndim, ndim,
                _lib.i32_array([int(s) for s in shape_zyx]), flags, _lib.stream_ptr(coord_dev.device),
            )
        )
    return np.asarray([bool(flags[a]) for a in range(ndim)][::-1])


def _frames(coord):
    """Frames, per-frame sample shape and CSR offsets of a coordinate tensor.

    (ncontrasts, nviews, nsamples, ndim); fewer dims get leading singletons
    (plan.py:66-77). A list/tuple of per-frame tensors gives frames of uneven
    length (an extension: samples then lie flat as (..., total)).
    """
    if isinstance(coord, (list, tuple)):
        parts = [torch.as_tensor(c, dtype=torch.float32) for c in coord]
        ndim = parts[0].shape[-1]
        lengths = [p.numel() // ndim for p in parts]
        offs = np.concatenate([[0], np.cumsum(lengths)]).astype(np.int64)
        flat = torch.cat([p.reshape(-1, ndim) for p in parts], 0)
        return flat, offs, None, ndim
    ishape = list(coord.shape[:-1])
    ndim = coord.shape[-1]
    while len(ishape) < 3:
        ishape = [1] + ishape
    nframes = ishape[0]
    ishape = ishape[1:]
    npts = int(np.prod(ishape))
    offs = (np.arange(nframes + 1, dtype=np.int64) * npts)
    return coord.reshape(-1, ndim), offs, tuple(ishape), ndim


def plan_nufft(coord, shape, width=4, oversamp=1.25, device="cpu", tile=None):
    """Precompute a NUFFT plan (reference: src/deepmr/fft/nufft.py:27-132).

    Parameters
    ----------
    coord : torch.Tensor | list
        K-space coordinates ``(ncontrasts, nviews, nsamples, ndim)`` in grid
        units ``(-shape/2, shape/2)``, axis order (x, y[, z]); fewer leading
        dims are singletons. A list of per-frame coordinate tensors gives frames
        of uneven length.
    shape : int | Iterable[int]
        Image size (z, y, x), scalar for isotropic.
    width : int | Iterable[int], optional
        Kaiser-Bessel kernel width. The default is ``4``.
    oversamp : float | Iterable[float], optional
        Grid oversampling. The default is ``1.25``.
    device : str, optional
        Device of the results for default calls; computation uses CUDA.
    tile : Iterable[int], optional
        Spatial bin size (z, y, x); ``None`` uses the tuned default.
    """
    dev = compute_device(device)
    if isinstance(coord, (list, tuple)):
        flat, offs, ishape, ndim = _frames(coord)
    else:
        coord = torch.as_tensor(coord).detach().clone().to(torch.float32)
        flat, offs, ishape, ndim = _frames(coord)
    flat = flat.to(dev, torch.float32).contiguous()

    width = _axis_param(width, ndim, np.int16)
    oversamp = _axis_param(oversamp, ndim, np.float32)
    # Kaiser-Bessel beta (nufft.py:98), float32 numpy arithmetic
    beta = math.pi * (((width / oversamp) * (oversamp - 0.5)) ** 2 - 0.8) ** 0.5
    if np.isscalar(shape):
        shape = np.asarray([shape] * ndim, dtype=np.int16)
    else:
        shape = np.asarray(shape, dtype=np.int16)[-ndim:]

    is_cart = detect_cartesian(flat, shape)
    oversamp[is_cart] = 1.0
    width[is_cart] = 1
    os_shape = np.ceil(oversamp * shape).astype(np.int16)
    if tile is None:
        from .. import autotune

        tile = autotune.lookup(ndim, int(width.max()), float(oversamp.max()))

    interp = DevicePlan(flat, offs, ishape, ndim, shape, os_shape, width, beta, oversamp, dev, tile)
    return NUFFTPlan(ndim, tuple(oversamp), tuple(width), tuple(beta), tuple(os_shape),
                     tuple(shape), interp, device)


def plan_toeplitz_nufft(coord, shape, basis=None, dcf=None, width=4, device="cpu"):
    """Toeplitz kernel for the self-adjoint NUFFT (reference: nufft.py:135-168)."""
    return _toeplitz.plan_toeplitz(coord, shape, basis, dcf, width, device)


# ---------------------------------------------------------------------------
# autograd wrappers (nufft.py:171-348): backward of each operator is the other
# ---------------------------------------------------------------------------
class ApplyNUFFT(autograd.Function):
    @staticmethod
    def forward(image, nufft_plan, basis_adjoint, weight, device, threadsperblock):
        return _apply_nufft(image, nufft_plan, basis_adjoint, weight, device, threadsperblock)

    @staticmethod
    def setup_context(ctx, inputs, output):
        _, nufft_plan, basis_adjoint, weight, device, threadsperblock = inputs
        ctx.set_materialize_grads(False)
        ctx.nufft_plan = nufft_plan
        ctx.basis_adjoint = basis_adjoint
        ctx.weight = weight
        ctx.device = device
        ctx.threadsperblock = threadsperblock

    @staticmethod
    def backward(ctx, kspace):
        basis = ctx.basis_adjoint.conj().t() if ctx.basis_adjoint is not None else None
        return (
            _apply_nufft_adj(kspace, ctx.nufft_plan, basis, ctx.weight, ctx.device, ctx.threadsperblock),
            None, None, None, None, None,
        )


class ApplyNUFFTAdjoint(autograd.Function):
    @staticmethod
    def forward(kspace, nufft_plan, basis, weight, device, threadsperblock):
        return _apply_nufft_adj(kspace, nufft_plan, basis, weight, device, threadsperblock)

    @staticmethod
    def setup_context(ctx, inputs, output):
        _, nufft_plan, basis, weight, device, threadsperblock = inputs
        ctx.set_materialize_grads(False)
        ctx.nufft_plan = nufft_plan
        ctx.basis = basis
        ctx.weight = weight
        ctx.device = device
        ctx.threadsperblock = threadsperblock

    @staticmethod
    def backward(ctx, image):
        basis_adjoint = ctx.basis.conj().t() if ctx.basis is not None else None
        return (
            _apply_nufft(image, ctx.nufft_plan, basis_adjoint, ctx.weight, ctx.device, ctx.threadsperblock),
            None, None, None, None, None,
        )


class ApplyNUFFTSelfAdjoint(autograd.Function):
    @staticmethod
    def forward(image, toeplitz_kern, device, threadsperblock):
        return _apply_nufft_selfadj(image, toeplitz_kern, device, threadsperblock)

    @staticmethod
    def setup_context(ctx, inputs, output):
        _, toeplitz_kern, device, threadsperblock = inputs
        ctx.set_materialize_grads(False)
        ctx.toeplitz_kern = toeplitz_kern
        ctx.device = device
        ctx.threadsperblock = threadsperblock

    @staticmethod
    def backward(ctx, image):
        return (_apply_nufft_selfadj(image, ctx.toeplitz_kern, ctx.device, ctx.threadsperblock),
                None, None, None)


def apply_nufft(image, nufft_plan, basis_adjoint=None, weight=None, device=None, threadsperblock=128):
    """Apply the NUFFT (reference: nufft.py:212-245).

    image ``(..., [ncontrasts,] *shape)`` -> kspace ``(..., [ncontrasts,] nviews, nsamples)``.
    ``threadsperblock`` is accepted for compatibility and ignored.
    """
    return ApplyNUFFT.apply(image, nufft_plan, basis_adjoint, weight, device, threadsperblock)


def apply_nufft_adj(kspace, nufft_plan, basis=None, weight=None, device=None, threadsperblock=128):
    """Apply the adjoint NUFFT (reference: nufft.py:289-322).

    kspace ``(..., [ncontrasts,] nviews, nsamples)`` -> image ``(..., [ncontrasts,] *shape)``.
    """
    return ApplyNUFFTAdjoint.apply(kspace, nufft_plan, basis, weight, device, threadsperblock)


def apply_nufft_selfadj(image, toeplitz_kern, device=None, threadsperblock=128):
    """Self-adjoint NUFFT through Toeplitz convolution (reference: nufft.py:351-375)."""
    return ApplyNUFFTSelfAdjoint.apply(image, toeplitz_kern, device, threadsperblock)


# ---------------------------------------------------------------------------
# implementations
# ---------------------------------------------------------------------------
def _to_origin(out, like):
    """Return ``out`` on the device of ``like``; pinned CPU inputs get pinned outputs
    (so the device-to-host copy runs at full PCIe speed)."""
    if like.device == out.device:
        return out
    if like.device.type == "cpu" and like.is_pinned():
        host = torch.empty(out.shape, dtype=out.dtype, pin_memory=True)
        host.copy_(out)
        return host
    return out.to(like.device)


def _as_cfloat(x):
    x = torch.as_tensor(x)
    if x.dtype in (torch.float16, torch.float32, torch.float64):
        return x.to(torch.float32)
    return x.to(torch.complex64)


# Gridding kernel of the adjoint: False (default) = shared-memory tiles flushed
# with global atomics; True = fixed-order owner tiles (bitwise reproducible).
DETERMINISTIC_GRIDDING = False

# Device status of the gridding (a bounded wait that ran out, DMR_ERR_TIMEOUT)
# is checked after every adjoint whose result returns to the host (that call
# synchronises anyway); True also checks after device-resident calls (one
# stream synchronisation each). DevicePlan.check_status checks on demand.
CHECK_STATUS = False


def set_status_check(on):
    """Check the gridding status after every adjoint call; returns the old setting."""
    global CHECK_STATUS
    old, CHECK_STATUS = CHECK_STATUS, bool(on)
    return old


def _basis_arg(basis, rows, cols, dev, name):
    """Subspace matrix as a contiguous complex64 device tensor of shape (rows, cols)
    (basis_adjoint: (nframes, ncoeff), indexed [frame, coeff] like the reference's
    kernels, interp.py:230-357; basis: (ncoeff, nframes), grid.py:287-417)."""
    b = torch.as_tensor(basis)
    b = b.to(torch.complex64) if b.is_complex() else b.to(torch.float32).to(torch.complex64)
    if b.dim() != 2 or (cols is not None and tuple(b.shape) != (rows, cols)) or (cols is None and b.shape[0] != rows):
        raise ValueError(f"{name} must have shape ({rows}, {cols if cols is not None else 'ncoeff'}), "
                         f"got {tuple(b.shape)}")
    return b.to(dev).contiguous()


def _sample_dims(interp):
    return len(interp.ishape) if interp.ishape is not None else 1


def _sample_shape(interp):
    return interp.ishape if interp.ishape is not None else (interp.total,)


def _kspace_shape(interp, batch_shape):
    """k-space layout: (..., [F,] nviews, nsamples), or (..., total) for uneven frames."""
    if interp.ishape is None:
        return list(batch_shape) + [interp.total]
    return list(batch_shape) + ([interp.nframes] if interp.nframes > 1 else []) + list(interp.ishape)


def _weight_arg(weight, batch_shape, interp, frames_shape, dev):
    """Returns (tensor, per_batch flag) for the C library's weight argument."""
    if weight is None:
        return None, 0
    w = torch.as_tensor(weight, dtype=torch.float32).to(dev)
    if w.numel() == interp.total:
        return w.contiguous(), 0
    return torch.broadcast_to(w, _kspace_shape(interp, batch_shape)).contiguous(), 1


# Pinned host inputs of at least this many bytes (input + output) run through a
# chunked pipeline: the copy in of one chunk of the batch, the compute of the
# previous chunk and the copy out of the one before overlap (H2D and D2H run on
# separate copy engines), instead of copy in -> compute -> copy out in series.
PIPELINE_MIN_BYTES = 64 << 20
PIPELINE_CHUNKS = 16
# batch items per chunk of a host-pipelined 3D adjoint, at least: atomic
# gridding of a few coils runs on the CUDA cores at a cost proportional to the
# coils; the deterministic tensor-core gridding costs about the same for 8
# coils as for 32
ADJOINT_MIN_CHUNK_3D = 2
ADJOINT_MIN_CHUNK_3D_DET = 8

_PIPE_STREAMS = {}


def _pipe_streams(dev):
    """(copy-in, compute, copy-out) streams of ``dev``, created once."""
    key = dev.index if dev.index is not None else torch.cuda.current_device()
    s = _PIPE_STREAMS.get(key)
    if s is None:
        with torch.cuda.device(key):
            s = (torch.cuda.Stream(), torch.cuda.Stream(), torch.cuda.Stream())
        _PIPE_STREAMS[key] = s
    return s


def _pipelinable(host, dev, batch, out_item_bytes):
    """True for a pinned, contiguous CPU input whose batch is worth chunking."""
    if dev.type != "cuda" or host.device.type != "cpu" or batch < 2:
        return False
    if not (host.is_contiguous() and host.is_pinned()):
        return False
    nbytes = host.numel() * host.element_size() + batch * out_item_bytes
    return nbytes >= PIPELINE_MIN_BYTES


def _pipeline_chunks(batch, min_chunk=1):
    """(number of chunks, batch items per chunk) of the host pipeline: up to
    PIPELINE_CHUNKS chunks of at least ``min_chunk`` items, equal but the last."""
    nch = max(1, min(PIPELINE_CHUNKS, batch // max(1, min_chunk)))
    cb = -(-batch // nch)
    return -(-batch // cb), cb


def _pipelined(x_h, out_h, batch, dev, run, ws_bytes, min_chunk=1):
    """Run ``run(x_dev, out_dev, b0, nb, ws, stream)`` over chunks of the
    flattened batch: ``x_h`` (batch, ...) and ``out_h`` (batch, ...) are pinned
    host tensors, device input/output buffers are double-buffered, and the
    compute stream runs the chunks in order with one workspace. Returns after
    every copy out has completed (``out_h`` is then valid on the host).
    Chunks hold at least ``min_chunk`` batch items."""
    nch, cb = _pipeline_chunks(batch, min_chunk)
    h2d, comp, d2h = _pipe_streams(dev)
    with torch.cuda.device(dev):
        cur = torch.cuda.current_stream(dev)
        xb = [torch.empty((cb,) + tuple(x_h.shape[1:]), dtype=x_h.dtype, device=dev) for _ in range(min(2, nch))]
        ob = [torch.empty((cb,) + tuple(out_h.shape[1:]), dtype=out_h.dtype, device=dev) for _ in range(min(2, nch))]
        ws = ws_bytes(cb)
        start = torch.cuda.Event()
        start.record(cur)
        for s in (h2d, comp, d2h):
            s.wait_event(start)
        ev_in = [torch.cuda.Event() for _ in range(nch)]
        ev_comp = [torch.cuda.Event() for _ in range(nch)]
        ev_out = [torch.cuda.Event() for _ in range(nch)]
        try:
            for i in range(nch):
                b0 = i * cb
                nb = min(cb, batch - b0)
                k = i % 2
                if i >= 2:
                    h2d.wait_event(ev_comp[i - 2])  # xb[k] is free once chunk i-2 is computed
                with torch.cuda.stream(h2d):
                    xb[k][:nb].copy_(x_h[b0:b0 + nb], non_blocking=True)
                ev_in[i].record(h2d)
                comp.wait_event(ev_in[i])
                if i >= 2:
                    comp.wait_event(ev_out[i - 2])  # ob[k] is free once chunk i-2 is copied out
                run(xb[k][:nb], ob[k][:nb], b0, nb, ws, ctypes.c_void_p(comp.cuda_stream))
                ev_comp[i].record(comp)
                d2h.wait_event(ev_comp[i])
                with torch.cuda.stream(d2h):
                    out_h[b0:b0 + nb].copy_(ob[k][:nb], non_blocking=True)
                ev_out[i].record(d2h)
        finally:
            for s in (h2d, comp, d2h):
                s.synchronize()
    return out_h


def _weight_chunk(w, wpb, b0, nb, batch):
    """Rows b0 .. b0+nb of per-batch weights (flattened batch); shared weights as they are."""
    if w is None or not wpb:
        return w
    per = w.numel() // batch
    return w.reshape(-1)[b0 * per:(b0 + nb) * per]


def _apply_nufft(image, nufft_plan, basis_adjoint, weight, device, threadsperblock):
    if basis_adjoint is not None:
        return _apply_nufft_lowrank(image, nufft_plan, basis_adjoint, weight, device)
    isnumpy = isinstance(image, np.ndarray)
    image = _as_cfloat(image)
    if device is not None:
        nufft_plan.to(device)
    interp = nufft_plan.interpolator
    dev = interp.device
    ndim = nufft_plan.ndim
    nframes = interp.nframes
    if nframes == 1:
        batch_shape = image.shape[:-ndim]
        frames_shape = ()
    else:
        batch_shape = image.shape[: -ndim - 1]
        frames_shape = (nframes,)
        if image.shape[-ndim - 1] != nframes:
            raise ValueError(f"expected {nframes} frames before the spatial axes, got {tuple(image.shape)}")
    if tuple(image.shape[-ndim:]) != tuple(int(s) for s in nufft_plan.shape):
        raise ValueError(f"image spatial shape {tuple(image.shape[-ndim:])} != plan shape {nufft_plan.shape}")
    batch = int(np.prod(batch_shape))
    kshape = _kspace_shape(interp, batch_shape)
    real = int(not image.is_complex())

    def run(xd, od, b0, nb, ws, stream):
        _lib.check(
            _lib.lib().dmr_nufft_forward(
                interp.handle, _lib.ptr(xd), real, _lib.ptr(od), nb,
                _lib.ptr(_weight_chunk(w, wpb, b0, nb, batch)), wpb, _lib.ptr(ws), ws.numel(), stream,
            )
        )

    if interp.total > 0 and _pipelinable(image, dev, batch, 8 * interp.total):
        w, wpb = _weight_arg(weight, batch_shape, interp, frames_shape, dev)
        out = torch.empty([batch] + kshape[len(batch_shape):], dtype=torch.complex64, pin_memory=True)
        _pipelined(image.reshape((batch,) + tuple(image.shape[len(batch_shape):])), out, batch, dev, run,
                   interp.workspace)
        return out.reshape(kshape)
    x = image.to(dev).contiguous()
    out = torch.empty(kshape, dtype=torch.complex64, device=dev)
    if batch > 0 and interp.total > 0:
        w, wpb = _weight_arg(weight, batch_shape, interp, frames_shape, dev)
        with torch.cuda.device(dev):
            run(x, out, 0, batch, interp.workspace(batch), _lib.stream_ptr(dev))
    out = _to_origin(out, image)
    return out.numpy(force=True) if isnumpy else out


def _apply_nufft_adj(kspace, nufft_plan, basis, weight, device, threadsperblock, deterministic=None):
    if basis is not None:
        return _apply_nufft_adj_lowrank(kspace, nufft_plan, basis, weight, device, deterministic)
    isnumpy = isinstance(kspace, np.ndarray)
    kspace = _as_cfloat(kspace)
    if device is not None:
        nufft_plan.to(device)
    interp = nufft_plan.interpolator
    dev = interp.device
    nframes = interp.nframes
    nsd = _sample_dims(interp)
    frames_shape = (nframes,) if nframes > 1 else ()
    if nframes == 1 or interp.ishape is None:
        batch_shape = kspace.shape[:-nsd]
    else:
        batch_shape = kspace.shape[: -nsd - 1]
    if list(kspace.shape) != _kspace_shape(interp, batch_shape):
        raise ValueError(f"kspace shape {tuple(kspace.shape)} does not match the plan samples {_sample_shape(interp)}")
    batch = int(np.prod(batch_shape))
    item = list(frames_shape) + [int(s) for s in nufft_plan.shape]
    real = int(not kspace.is_complex())
    det = int(DETERMINISTIC_GRIDDING if deterministic is None else deterministic)

    def run(yd, od, b0, nb, ws, stream):
        _lib.check(
            _lib.lib().dmr_nufft_adjoint(
                interp.handle, _lib.ptr(yd), real, _lib.ptr(od), nb,
                _lib.ptr(_weight_chunk(w, wpb, b0, nb, batch)), wpb, det, _lib.ptr(ws), ws.numel(), stream,
            )
        )

    min_chunk = (ADJOINT_MIN_CHUNK_3D_DET if det else ADJOINT_MIN_CHUNK_3D) if nufft_plan.ndim == 3 else 1
    if batch >= 2 * min_chunk and _pipelinable(kspace, dev, batch, 8 * int(np.prod(item))):
        w, wpb = _weight_arg(weight, batch_shape, interp, frames_shape, dev)
        out = torch.empty([batch] + item, dtype=torch.complex64, pin_memory=True)
        _pipelined(kspace.reshape((batch,) + tuple(kspace.shape[len(batch_shape):])), out, batch, dev, run,
                   interp.workspace, min_chunk)
        interp.check_status()
        return out.reshape(list(batch_shape) + item)
    y = kspace.to(dev).contiguous()
    out = torch.empty(list(batch_shape) + item, dtype=torch.complex64, device=dev)
    if batch > 0:
        w, wpb = _weight_arg(weight, batch_shape, interp, frames_shape, dev)
        with torch.cuda.device(dev):
            run(y, out, 0, batch, interp.workspace(batch), _lib.stream_ptr(dev))
    out = _to_origin(out, kspace)
    if batch > 0 and (CHECK_STATUS or out.device.type == "cpu"):
        interp.check_status()
    return out.numpy(force=True) if isnumpy else out


def _apply_nufft_lowrank(image, nufft_plan, basis_adjoint, weight, device):
    """Forward NUFFT of subspace coefficients: image (..., ncoeff, *shape) ->
    k-space (..., [nframes,] samples), frame f from sum_c basis_adjoint[f, c] image[c]."""
    isnumpy = isinstance(image, np.ndarray)
    image = _as_cfloat(image)
    if device is not None:
        nufft_plan.to(device)
    interp = nufft_plan.interpolator
    dev = interp.device
    ndim = nufft_plan.ndim
    nframes = interp.nframes
    x = image.to(dev)
    if tuple(x.shape[-ndim:]) != tuple(int(s) for s in nufft_plan.shape) or x.dim() < ndim + 1:
        raise ValueError(f"image {tuple(x.shape)} must be (..., ncoeff, *{tuple(nufft_plan.shape)})")
    ncoeff = int(x.shape[-ndim - 1])
    ba = _basis_arg(basis_adjoint, nframes, ncoeff, dev, "basis_adjoint")
    batch_shape = x.shape[: -ndim - 1]
    frames_shape = (nframes,) if nframes > 1 else ()
    batch = int(np.prod(batch_shape))
    x = x.contiguous()
    out = torch.empty(_kspace_shape(interp, batch_shape), dtype=torch.complex64, device=dev)
    if batch > 0 and interp.total > 0:
        w, wpb = _weight_arg(weight, batch_shape, interp, frames_shape, dev)
        ws = interp.workspace_lowrank(batch, ncoeff)
        with torch.cuda.device(dev):
            _lib.check(_lib.lib().dmr_nufft_forward_lowrank(
                interp.handle, _lib.ptr(x), int(not x.is_complex()), ncoeff, _lib.ptr(ba), _lib.ptr(out),
                batch, _lib.ptr(w), wpb, _lib.ptr(ws), ws.numel(), _lib.stream_ptr(dev)))
    out = _to_origin(out, image)
    return out.numpy(force=True) if isnumpy else out


def _apply_nufft_adj_lowrank(kspace, nufft_plan, basis, weight, device, deterministic=None):
    """Adjoint NUFFT onto subspace coefficients: k-space (..., [nframes,] samples)
    -> image (..., ncoeff, *shape), coefficient c from sum_f basis[c, f] A_f^H y_f."""
    isnumpy = isinstance(kspace, np.ndarray)
    kspace = _as_cfloat(kspace)
    if device is not None:
        nufft_plan.to(device)
    interp = nufft_plan.interpolator
    dev = interp.device
    nframes = interp.nframes
    y = kspace.to(dev)
    nsd = _sample_dims(interp)
    if nframes == 1 or interp.ishape is None:
        batch_shape = y.shape[:-nsd]
    else:
        batch_shape = y.shape[: -nsd - 1]
    if list(y.shape) != _kspace_shape(interp, batch_shape):
        raise ValueError(f"kspace shape {tuple(y.shape)} does not match the plan samples {_sample_shape(interp)}")
    b = torch.as_tensor(basis)
    if b.dim() != 2:
        raise ValueError(f"basis must have shape (ncoeff, {nframes}), got {tuple(b.shape)}")
    ncoeff = int(b.shape[0])
    bb = _basis_arg(b, ncoeff, nframes, dev, "basis")
    frames_shape = (nframes,) if nframes > 1 else ()
    batch = int(np.prod(batch_shape))
    y = y.contiguous()
    out = torch.empty(list(batch_shape) + [ncoeff] + [int(s) for s in nufft_plan.shape],
                      dtype=torch.complex64, device=dev)
    if batch > 0:
        w, wpb = _weight_arg(weight, batch_shape, interp, frames_shape, dev)
        ws = interp.workspace_lowrank(batch, ncoeff)
        det = int(DETERMINISTIC_GRIDDING if deterministic is None else deterministic)
        with torch.cuda.device(dev):
            _lib.check(_lib.lib().dmr_nufft_adjoint_lowrank(
                interp.handle, _lib.ptr(y), int(not y.is_complex()), ncoeff, _lib.ptr(bb), _lib.ptr(out), batch,
                _lib.ptr(w), wpb, det, _lib.ptr(ws), ws.numel(), _lib.stream_ptr(dev)))
    out = _to_origin(out, kspace)
    if batch > 0 and (CHECK_STATUS or out.device.type == "cpu"):
        interp.check_status()
    return out.numpy(force=True) if isnumpy else out


def _apply_nufft_selfadj(image, toeplitz_kern, device, threadsperblock):
    isnumpy = isinstance(image, np.ndarray)
    image = _as_cfloat(image)
    if device is not None:
        toeplitz_kern.to(device)
    out = _toeplitz.apply_toeplitz(image, toeplitz_kern)
    return out.numpy(force=True) if isnumpy else out


# ---------------------------------------------------------------------------
# differentiation w.r.t. the trajectory (no counterpart in the reference,
# whose plan is an opaque object and whose backward returns no coordinate
# gradient, nufft.py:188-209)
# ---------------------------------------------------------------------------
def traj_grad(nufft_plan, image, v, weight=None, post_scale=1.0):
    """g[..., a] = post_scale * sum_batch Re(conj(v) * d apply_nufft(image) / d coord[..., a]).

    Returns a float32 tensor shaped like the plan's coordinates
    ``(ncontrasts, nviews, nsamples, ndim)`` (flat ``(total, ndim)`` for
    uneven frames), in grid units.
    """
    interp = nufft_plan.interpolator
    dev = interp.device
    ndim = nufft_plan.ndim
    x = _as_cfloat(image).to(dev).contiguous()
    vv = torch.as_tensor(v).to(dev, torch.complex64).contiguous()
    nframes = interp.nframes
    batch_shape = x.shape[:-ndim] if nframes == 1 else x.shape[: -ndim - 1]
    frames_shape = () if nframes == 1 else (nframes,)
    batch = int(np.prod(batch_shape))
    out = torch.empty((interp.total, ndim), dtype=torch.float32, device=dev)
    w, wpb = _weight_arg(weight, batch_shape, interp, frames_shape, dev)
    ws = interp.workspace(batch)
    with torch.cuda.device(dev):
        _lib.check(_lib.lib().dmr_nufft_traj_grad(
            interp.handle, _lib.ptr(x), int(not x.is_complex()), _lib.ptr(vv), batch, _lib.ptr(w), wpb,
            float(post_scale), _lib.ptr(out), _lib.ptr(ws), ws.numel(), _lib.stream_ptr(dev)))
    return out


class NUFFTTraj(autograd.Function):
    """y = A(coord) x with gradients for the image (the reference's adjoint
    convention, nufft.py:188-209) and for the coordinates."""

    @staticmethod
    def forward(ctx, image, coord, shape, width, oversamp, device, weight):
        plan = plan_nufft(coord.detach(), shape, width, oversamp, device)
        ctx.plan, ctx.weight, ctx.coord_shape = plan, weight, coord.shape
        ctx.save_for_backward(image)
        return _apply_nufft(image.detach(), plan, None, weight, None, 128)

    @staticmethod
    def backward(ctx, g):
        (image,) = ctx.saved_tensors
        gx = gc = None
        if ctx.needs_input_grad[0]:
            gx = _apply_nufft_adj(g, ctx.plan, None, ctx.weight, None, 128).to(image.device)
        if ctx.needs_input_grad[1]:
            gc = traj_grad(ctx.plan, image.detach(), g, ctx.weight).reshape(ctx.coord_shape)
        return gx, gc, None, None, None, None, None


class NUFFTAdjTraj(autograd.Function):
    """x = A(coord)^H y (reference scale: exact adjoint / prod(os_shape)) with
    gradients for the k-space data and for the coordinates."""

    @staticmethod
    def forward(ctx, kspace, coord, shape, width, oversamp, device, weight):
        plan = plan_nufft(coord.detach(), shape, width, oversamp, device)
        ctx.plan, ctx.weight, ctx.coord_shape = plan, weight, coord.shape
        ctx.save_for_backward(kspace)
        return _apply_nufft_adj(kspace.detach(), plan, None, weight, None, 128)

    @staticmethod
    def backward(ctx, g):
        (kspace,) = ctx.saved_tensors
        gy = gc = None
        if ctx.needs_input_grad[0]:
            gy = _apply_nufft(g, ctx.plan, None, ctx.weight, None, 128).to(kspace.device)
        if ctx.needs_input_grad[1]:
            G = float(np.prod([int(s) for s in ctx.plan.os_shape]))
            gc = traj_grad(ctx.plan, g, kspace.detach(), ctx.weight, 1.0 / G).reshape(ctx.coord_shape)
        return gy, gc, None, None, None, None, None

