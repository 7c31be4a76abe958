"""CG-SENSE reconstruction on the device, and a continuous-batching server.

Reference: `recon_lstsq` with `toeplitz=True` (src/deepmr/recon/alg/classic_recon.py:25-243)
builds E = F * C and E^H E = C^H * NUFFTGramOp * C (src/deepmr/recon/alg/linop.py:108-148)
and runs `cg_solve` (src/deepmr/optim/cg.py:16-147) from x = 0 with AHy = E^H(dcf**0.5 * y).
Here:

* `cg_sense` computes AHy with this library's adjoint NUFFT (density weight
  dcf = dcf**0.5 twice, as the reference) and a coil combine, then runs CG
  with the fused SENSE + Toeplitz normal operator (`dmr_sense_normal`) and the
  device-resident CG of `dmr_cg_init` / `dmr_cg_step` (float64 inner products,
  no host synchronisation per iteration). The intensity rescaling of
  `recon_lstsq` (classic_recon.py:164) is left to the caller.
* `ReconServer` admits requests of different matrix sizes, coil counts and
  trajectories as device memory (an HBM budget) and request slots free up,
  keeps plans, Toeplitz kernels and coil maps resident across requests, and
  enqueues every admitted request's whole solve on its own CUDA stream, so up
  to `max_active` solves overlap on the GPU (continuous batching: requests
  that arrive while others run are admitted as slots and memory free up).
  Each request runs in a resident slot whose CG iteration is a captured CUDA
  graph (one launch per iteration). `run_sequential` is the plain per-call
  path: one request at a time, to completion, with eager launches. Requests
  carry host k-space (pinned), uploaded on the slot's stream; a result is
  copied back to pinned host memory before the request counts as done, so a
  latency runs from arrival to the result on the host. A cancelled request, a
  malformed one (coordinates, shapes) and one whose working set exceeds the
  whole HBM budget produce an error status instead of a result (`Admission`).

The CG reductions have a fixed order; with deterministic AHy gridding a
request's result does not depend on what else runs beside it (bitwise), with
atomic gridding (the server's default, faster) it agrees to float32 rounding.
"""

import ctypes
import importlib
import math
import time
from dataclasses import dataclass, field

import numpy as np
import torch

from . import _lib

# the package attribute deepmr_b200.fft.nufft is the one-shot function (as in
# the reference); take the submodule from the import system
_nufft = importlib.import_module("deepmr_b200.fft.nufft")


def _ws_bytes(ndim, kshape, batch, dev):
    n = ctypes.c_size_t()
    with torch.cuda.device(dev):
        _lib.check(_lib.lib().dmr_toeplitz_workspace_bytes(ndim, _lib.i32_array(kshape), int(batch),
                                                          ctypes.byref(n)))
    return int(n.value)


class SenseNormal:
    """AHA(x) = sum_c conj(S_c) T(S_c x) + lamda x (T: Toeplitz self-adjoint)."""

    def __init__(self, maps, gram, lamda=0.0):
        self.maps = maps.to(torch.complex64).contiguous()
        self.dev = self.maps.device
        self.ndim = gram.ndim
        self.kshape = [int(k) for k in gram.shape]
        self.ishape = [int(s) for s in self.maps.shape[-self.ndim:]]
        kv = gram.value
        if kv.dim() > self.ndim and int(np.prod(kv.shape[:-self.ndim])) != 1:
            raise ValueError("CG-SENSE takes a single-frame Toeplitz kernel")
        self.kernel = kv.reshape(self.kshape).to(self.dev, torch.complex64).contiguous()
        self.ncoils = int(self.maps.shape[0])
        self.lamda = float(lamda)
        self.ws_bytes = _ws_bytes(self.ndim, self.kshape, self.ncoils, self.dev)

    def workspace(self):
        """A private workspace (one per concurrent solve: the operator itself is read-only)."""
        return torch.empty(self.ws_bytes, dtype=torch.uint8, device=self.dev)

    def apply(self, x, out, ws, stream=None):
        st = _lib.stream_ptr(self.dev) if stream is None else ctypes.c_void_p(stream.cuda_stream)
        with torch.cuda.device(self.dev):
            _lib.check(_lib.lib().dmr_sense_normal(
                self.ndim, _lib.i32_array(self.kshape), _lib.i32_array(self.ishape), _lib.ptr(self.kernel),
                _lib.ptr(self.maps), self.ncoils, _lib.ptr(x), _lib.ptr(out), self.lamda, _lib.ptr(ws),
                ws.numel(), st))
        return out


class CGState:
    """Device vectors and scalars of one CG solve."""

    def __init__(self, ahy, normal):
        self.dev = ahy.device
        self.normal = normal
        self.ahy = ahy.contiguous()
        self.n = self.ahy.numel()
        self.x = torch.empty_like(self.ahy)
        self.r = torch.empty_like(self.ahy)
        self.p = torch.empty_like(self.ahy)
        self.q = torch.empty_like(self.ahy)
        self.ws = normal.workspace()
        nb = ctypes.c_size_t()
        _lib.check(_lib.lib().dmr_cg_state_bytes(ctypes.byref(nb)))
        self.state = torch.empty(int(nb.value), dtype=torch.uint8, device=self.dev)
        self.steps = 0

    def init(self, stream=None):
        st = _lib.stream_ptr(self.dev) if stream is None else ctypes.c_void_p(stream.cuda_stream)
        with torch.cuda.device(self.dev):
            _lib.check(_lib.lib().dmr_cg_init(_lib.ptr(self.ahy), _lib.ptr(self.x), _lib.ptr(self.r),
                                              _lib.ptr(self.p), self.n, _lib.ptr(self.state), st))

    def step(self, stream=None):
        st = _lib.stream_ptr(self.dev) if stream is None else ctypes.c_void_p(stream.cuda_stream)
        self.normal.apply(self.p, self.q, self.ws, stream)
        with torch.cuda.device(self.dev):
            _lib.check(_lib.lib().dmr_cg_step(_lib.ptr(self.x), _lib.ptr(self.r), _lib.ptr(self.p),
                                              _lib.ptr(self.q), self.n, _lib.ptr(self.state), st))
        self.steps += 1

    def residual(self, stream=None):
        st = _lib.stream_ptr(self.dev) if stream is None else ctypes.c_void_p(stream.cuda_stream)
        v = ctypes.c_double()
        _lib.check(_lib.lib().dmr_cg_residual(_lib.ptr(self.state), ctypes.byref(v), st))
        return v.value


def sense_adjoint(kspace, plan, maps, dcf=None, deterministic=True):
    """AHy = sum_c conj(S_c) nufft_adj(dcf * y_c) (E^H(dcf**0.5 y), classic_recon.py:153-156).

    With deterministic gridding AHy (and the whole reconstruction) is bitwise
    independent of concurrent work; atomic gridding is faster and agrees to
    float32 rounding.
    """
    img = _nufft._apply_nufft_adj(kspace, plan, None, dcf, None, 128, deterministic=deterministic)
    return (maps.conj() * img).sum(0)


def cg_sense(kspace, coord, shape, maps, dcf=None, niter=20, lamda=0.0, tol=0.0, width=4, gram_width=6,
             device="cuda", plan=None, gram=None):
    """CG-SENSE least-squares reconstruction (recon_lstsq with toeplitz=True, no rescaling).

    kspace (ncoils, [nviews,] nsamples) complex; coord (nviews, nsamples, ndim)
    grid units; maps (ncoils, *shape); dcf (nviews, nsamples) or None.
    Returns the image (*shape) complex64 on the device.
    """
    dev = _nufft.compute_device(device)
    maps = torch.as_tensor(maps).to(dev, torch.complex64)
    if plan is None:
        plan = _nufft.plan_nufft(coord, shape, width, 1.25, dev)
    if gram is None:
        gram = _nufft.plan_toeplitz_nufft(coord, shape, dcf=dcf, width=gram_width, device=dev)
    d = None if dcf is None else torch.as_tensor(dcf).to(dev, torch.float32)
    ahy = sense_adjoint(torch.as_tensor(kspace).to(dev, torch.complex64), plan, maps, d)
    cg = CGState(ahy, SenseNormal(maps, gram, lamda))
    cg.init()
    for _ in range(niter):
        cg.step()
        if tol > 0 and math.sqrt(max(cg.residual(), 0.0)) < tol:
            break
    return cg.x


# ---------------------------------------------------------------------------
# serving
# ---------------------------------------------------------------------------
@dataclass
class ReconRequest:
    rid: int
    kspace: torch.Tensor  # (ncoils, nviews, nsamples) complex64, host (pinned) or device
    traj_key: str  # identifies the trajectory (plans are cached by it)
    coord: object  # (nviews, nsamples, ndim) grid units
    shape: tuple
    maps_key: str  # identifies the coil maps (cached)
    maps: object  # (ncoils, *shape) complex64
    dcf: object = None
    niter: int = 20
    lamda: float = 0.0
    arrival: float = 0.0  # seconds after the start of the run
    cancelled: bool = False

    def cancel(self):
        """Withdraw the request: not admitted if still waiting; if already
        running, its result is dropped when it finishes (status "cancelled")."""
        self.cancelled = True


def _host_array(a):
    if isinstance(a, torch.Tensor):
        return a.detach().cpu().numpy()
    return np.asarray(a)


def working_set_bytes(req):
    """Device bytes one active request holds beside the resident caches: CG
    vectors, AHy, the adjoint's oversampled grids and the Toeplitz buffers."""
    ndim = len(req.shape)
    isize = int(np.prod(req.shape))
    ncoils = int(np.shape(req.kspace)[0]) if isinstance(req.kspace, np.ndarray) else int(req.kspace.shape[0])
    G = int(np.prod([math.ceil(1.25 * s) for s in req.shape]))
    K = int(np.prod([2 * s for s in req.shape]))
    return 8 * (6 * isize + 2 * ncoils * G + ncoils * isize + ncoils * K) + (1 << 20) * ndim


class Admission:
    """Host-side admission of `ReconServer` (no device work).

    FIFO over the requests that have arrived. The head request is rejected,
    with a status message, when it was cancelled, when it is malformed
    (non-finite or wrongly shaped coordinates; k-space, coil maps or density
    weights whose shape does not match the trajectory and image), or when its
    working set exceeds the whole HBM budget (it could never run). Otherwise it
    is admitted while a slot is free and its working set fits beside the active
    requests' (or nothing is active)."""

    def __init__(self, budget, max_active, request_bytes, known_trajectories=()):
        self.budget = int(budget)
        self.max_active = int(max_active)
        self.request_bytes = request_bytes
        self.known = known_trajectories  # trajectory keys already checked (planned)

    def validate(self, req):
        """None if `req` can run, else the reason it cannot."""
        if req.cancelled:
            return "cancelled"
        shape = tuple(int(n) for n in req.shape)
        ndim = len(shape)
        if ndim not in (1, 2, 3) or min(shape) < 1:
            return f"malformed request: image shape {shape}"
        if req.niter < 0:
            return f"malformed request: niter {req.niter}"
        if req.traj_key in self.known:
            kshape = None
        else:
            coord = _host_array(req.coord)
            if coord.ndim < 2 or coord.shape[-1] != ndim:
                return f"malformed coordinates: shape {tuple(coord.shape)} for a {ndim}D image"
            if not np.issubdtype(coord.dtype, np.number) or not np.isfinite(coord).all():
                return "malformed coordinates: non-finite values"
            kshape = tuple(coord.shape[:-1])
        ksp_shape = tuple(torch.as_tensor(req.kspace).shape) if not isinstance(req.kspace, np.ndarray) \
            else req.kspace.shape
        if len(ksp_shape) < 2:
            return f"malformed k-space: shape {ksp_shape}"
        if kshape is not None and tuple(ksp_shape[1:]) != kshape:
            return f"malformed k-space: shape {ksp_shape} for trajectory {kshape}"
        maps_shape = tuple(np.shape(req.maps)) if not isinstance(req.maps, torch.Tensor) else tuple(req.maps.shape)
        if maps_shape != (ksp_shape[0],) + shape:
            return f"malformed coil maps: shape {maps_shape} for {ksp_shape[0]} coils and image {shape}"
        if req.dcf is not None and kshape is not None and tuple(np.shape(req.dcf)) != kshape:
            return f"malformed density weights: shape {tuple(np.shape(req.dcf))} for trajectory {kshape}"
        nb = self.request_bytes(req)
        if nb > self.budget:
            return f"working set {nb} B exceeds the HBM budget {self.budget} B"
        return None

    def take(self, pending, now, realtime, nactive, used):
        """Next decision for the head of `pending` (sorted by arrival), which it
        pops: ("reject", req, reason) or ("admit", req, nbytes); None while the
        head has not arrived, no slot is free or its working set does not fit."""
        if not pending or (realtime and pending[0].arrival > now):
            return None
        req = pending[0]
        reason = self.validate(req)
        if reason is not None:
            pending.pop(0)
            return ("reject", req, reason)
        if nactive >= self.max_active:
            return None
        nb = self.request_bytes(req)
        if nactive and used + nb > self.budget:
            return None
        pending.pop(0)
        return ("admit", req, nb)


class _Slot:
    """Resident CG working set of one request at a time, with its stream and a
    CUDA graph of one CG iteration (normal operator + update) captured on it:
    an iteration is one graph launch instead of a dozen kernel launches."""

    def __init__(self, normal, dev, use_graph=True):
        self.stream = torch.cuda.Stream(dev)
        ishape = tuple(normal.ishape)
        # the result's landing buffer in pinned host memory, allocated once
        # (a pinned allocation while solves run can synchronise the device)
        self.host_out = torch.empty(ishape, dtype=torch.complex64, pin_memory=True)
        with torch.cuda.stream(self.stream):
            self.cg = CGState(torch.zeros(ishape, dtype=torch.complex64, device=dev), normal)
            # one eager iteration: cuFFT plans and every lazy setup exist before capture
            self.cg.init(self.stream)
            self.cg.step(self.stream)
        self.stream.synchronize()
        self.graph = None
        if use_graph:
            self.graph = torch.cuda.CUDAGraph()
            with torch.cuda.graph(self.graph, stream=self.stream):
                self.cg.step(self.stream)
            self.stream.synchronize()
        self.cg.steps = 0

    def start(self, ahy):
        """Load a request's AHy (on the slot's stream) and initialise CG."""
        self.cg.ahy.copy_(ahy)
        self.cg.init(self.stream)
        self.cg.steps = 0

    def step(self):
        if self.graph is not None:
            with torch.cuda.stream(self.stream):
                self.graph.replay()
            self.cg.steps += 1
        else:
            with torch.cuda.stream(self.stream):
                self.cg.step(self.stream)


@dataclass
class _Active:
    req: ReconRequest
    slot: _Slot
    nbytes: int
    done_event: object = None
    started: float = 0.0
    result: object = None


@dataclass
class ServeStats:
    latency: dict = field(default_factory=dict)  # rid -> seconds (arrival to result on the host)
    results: dict = field(default_factory=dict)  # rid -> image tensor (host)
    errors: dict = field(default_factory=dict)  # rid -> why the request produced no result
    wall: float = 0.0
    peak_active: int = 0
    peak_bytes: int = 0  # largest sum of active working sets

    def summary(self):
        lat = np.asarray(sorted(self.latency.values()))
        if lat.size == 0:
            return {}
        return {"requests": int(lat.size), "p50_ms": float(np.percentile(lat, 50) * 1e3),
                "p99_ms": float(np.percentile(lat, 99) * 1e3), "mean_ms": float(lat.mean() * 1e3),
                "throughput_rps": float(lat.size / self.wall) if self.wall > 0 else None,
                "wall_s": self.wall, "peak_active": self.peak_active, "errors": len(self.errors)}


class ReconServer:
    """Continuous-batching CG-SENSE server on one GPU (see module docstring).

    hbm_budget: bytes of device memory the active requests' working sets may
    use (resident plans/kernels/maps are accounted separately, in the caches).
    max_active: request slots.
    deterministic: grid AHy deterministically (results bitwise independent of
    the mix); otherwise with atomics (results agree to float32 rounding).
    """

    def __init__(self, device="cuda", hbm_budget=16 << 30, max_active=8, width=4, gram_width=6,
                 use_graphs=True, deterministic=False):
        self.dev = _nufft.compute_device(device)
        self.budget = int(hbm_budget)
        self.max_active = int(max_active)
        self.width, self.gram_width = width, gram_width
        self.use_graphs = bool(use_graphs)
        self.deterministic = bool(deterministic)
        self.plans = {}  # traj_key -> (plan, gram, dcf tensor)
        self.maps = {}  # maps_key -> tensor
        self.normals = {}  # (traj_key, maps_key, lamda) -> SenseNormal
        self.slots = {}  # normal key -> free _Slot list (resident working sets + graphs)

    # resident caches --------------------------------------------------------
    def _plan(self, req):
        if req.traj_key not in self.plans:
            plan = _nufft.plan_nufft(req.coord, req.shape, self.width, 1.25, self.dev)
            dcf = None if req.dcf is None else torch.as_tensor(req.dcf).to(self.dev, torch.float32)
            gram = _nufft.plan_toeplitz_nufft(req.coord, req.shape, dcf=dcf, width=self.gram_width,
                                              device=self.dev)
            self.plans[req.traj_key] = (plan, gram, dcf)
        return self.plans[req.traj_key]

    def _normal(self, req):
        key = (req.traj_key, req.maps_key, float(req.lamda))
        if key not in self.normals:
            if req.maps_key not in self.maps:
                self.maps[req.maps_key] = torch.as_tensor(req.maps).to(self.dev, torch.complex64).contiguous()
            _, gram, _ = self._plan(req)
            self.normals[key] = SenseNormal(self.maps[req.maps_key], gram, req.lamda)
        return self.normals[key]

    def request_bytes(self, req):
        """Working set of one active request (`working_set_bytes`)."""
        return working_set_bytes(req)

    def prepare(self, requests):
        """Build the resident plans, Toeplitz kernels, coil maps (and cuFFT
        plans), and the CG slots (with their captured iteration) the requests
        can use at once."""
        need = {}
        for r in requests:
            self._plan(r)
            key = self._key(r)
            need[key] = min(need.get(key, 0) + 1, self.max_active)
            free = self.slots.setdefault(key, [])
            while len(free) < need[key]:
                free.append(_Slot(self._normal(r), self.dev, self.use_graphs))

    @staticmethod
    def _key(req):
        return (req.traj_key, req.maps_key, float(req.lamda))

    def _take_slot(self, req):
        free = self.slots.setdefault(self._key(req), [])
        return free.pop() if free else _Slot(self._normal(req), self.dev, self.use_graphs)

    def _start(self, req, nbytes, now):
        # plans and maps first: a request they reject takes no slot
        plan, gram, dcf = self._plan(req)
        normal = self._normal(req)
        slot = self._take_slot(req)
        with torch.cuda.stream(slot.stream):
            # k-space upload (asynchronous from pinned host memory) on the slot's stream
            y = torch.as_tensor(req.kspace).to(self.dev, torch.complex64, non_blocking=True)
            slot.start(sense_adjoint(y, plan, normal.maps, dcf, self.deterministic))
        return _Active(req, slot, nbytes, started=now)

    def run(self, requests, realtime=True):
        """Serve `requests` (their `arrival` times are honoured when realtime).

        A request is admitted when it has arrived, a slot is free and its
        working set fits the HBM budget; admission enqueues its whole solve
        (AHy, CG init, one graph launch per iteration) on its slot's stream,
        so up to `max_active` solves run concurrently on the GPU while the
        host only admits and retires."""
        stats = ServeStats()
        pending = sorted(requests, key=lambda r: r.arrival)
        active, used = [], 0
        adm = Admission(self.budget, self.max_active, self.request_bytes, self.plans)
        t0 = time.perf_counter()
        while pending or active:
            now = time.perf_counter() - t0
            # admission (FIFO): arrived, a free slot, room in the HBM budget;
            # cancelled, malformed and over-budget requests get an error status
            while True:
                d = adm.take(pending, now, realtime, len(active), used)
                if d is None:
                    break
                kind, req, info = d
                if kind == "reject":
                    stats.errors[req.rid] = info
                    continue
                try:
                    a = self._start(req, info, now)
                except _lib.DmrError as e:
                    stats.errors[req.rid] = str(e)
                    continue
                for _ in range(req.niter):
                    a.slot.step()
                with torch.cuda.stream(a.slot.stream):
                    # the result leaves the slot for its pinned host buffer
                    a.slot.host_out.copy_(a.slot.cg.x, non_blocking=True)
                a.done_event = torch.cuda.Event()
                a.done_event.record(a.slot.stream)
                active.append(a)
                used += info
                stats.peak_bytes = max(stats.peak_bytes, used)
            stats.peak_active = max(stats.peak_active, len(active))
            # retire finished requests
            still = []
            for a in active:
                if a.done_event.query():
                    if a.req.cancelled:
                        stats.errors[a.req.rid] = "cancelled"
                    else:
                        # a host copy: the slot's buffer is reused by its next request
                        stats.results[a.req.rid] = a.slot.host_out.clone()
                        stats.latency[a.req.rid] = time.perf_counter() - t0 - a.req.arrival
                    self.slots[self._key(a.req)].append(a.slot)
                    used -= a.nbytes
                else:
                    still.append(a)
            if len(still) == len(active):
                # nothing finished: wait a little (for a completion or the next arrival)
                wait = 5e-5
                if pending and not active:
                    wait = max(0.0, min(pending[0].arrival - (time.perf_counter() - t0), 2e-3))
                time.sleep(wait)
            active = still
        torch.cuda.synchronize(self.dev)
        stats.wall = time.perf_counter() - t0
        return stats

    def run_sequential(self, requests, realtime=True):
        """Plain per-call path: one request at a time, to completion, on one stream."""
        stats = ServeStats()
        adm = Admission(self.budget, 1, self.request_bytes, self.plans)
        t0 = time.perf_counter()
        for req in sorted(requests, key=lambda r: r.arrival):
            now = time.perf_counter() - t0
            if realtime and req.arrival > now:
                time.sleep(req.arrival - now)
            reason = adm.validate(req)
            if reason is not None:
                stats.errors[req.rid] = reason
                continue
            try:
                plan, gram, dcf = self._plan(req)
                normal = self._normal(req)
            except _lib.DmrError as e:
                stats.errors[req.rid] = str(e)
                continue
            y = torch.as_tensor(req.kspace).to(self.dev, torch.complex64)
            cg = CGState(sense_adjoint(y, plan, normal.maps, dcf, self.deterministic), normal)
            cg.init()
            for _ in range(req.niter):
                cg.step()
            x = cg.x.cpu()
            stats.latency[req.rid] = time.perf_counter() - t0 - req.arrival
            stats.results[req.rid] = x
        stats.wall = time.perf_counter() - t0
        stats.peak_active = 1
        return stats


def synthetic_requests(n, rate_hz, seed=0, sizes=(128, 192, 256, 320), coils=(8, 16, 32), niter=20):
    """Seeded CG-SENSE serving workload: Poisson arrivals at `rate_hz`, matrix
    uniform over `sizes`, coils uniform over `coils`, radial or spiral
    trajectory, random-phase Gaussian-blob coil maps (sum |S|^2 = 1),
    k-space simulated from a seeded ellipse phantom plus noise."""
    from . import synth

    nf = _nufft

    rng = np.random.default_rng(seed)
    t = 0.0
    reqs = []
    cache = {}
    for i in range(n):
        t += rng.exponential(1.0 / rate_hz)
        N = int(rng.choice(sizes))
        C = int(rng.choice(coils))
        kind = "radial" if rng.random() < 0.5 else "spiral"
        tkey = f"{kind}{N}"
        if tkey not in cache:
            if kind == "radial":
                coord = synth.radial_2d(int(N * 1.0), 2 * N, N)
            else:
                nint = max(8, N // 8)
                coord = np.concatenate([synth.spiral_2d(4 * N, N, rotation=2 * np.pi * j / nint)
                                        for j in range(nint)], 0)
            cache[tkey] = (coord, synth.ramp_dcf(coord))
        coord, dcf = cache[tkey]
        mkey = f"maps{N}x{C}"
        if mkey not in cache:
            cache[mkey] = synth.coil_maps(C, (N, N), seed=N + C)
        maps = cache[mkey]
        pkey = f"ph{N}x{C}"
        if pkey not in cache:
            ph = torch.as_tensor(synth.ellipse_phantom(N, seed=N)).to(torch.complex64)
            cache[pkey] = torch.as_tensor(maps) * ph
        x = cache[pkey]
        plan = nf.plan_nufft(torch.as_tensor(coord), N, 4, 1.25, "cuda")
        y = nf.apply_nufft(x.cuda(), plan)
        y = y + 1e-2 * synth.complex_gaussian(tuple(y.shape), seed=1000 + i, device="cuda")
        # requests arrive with their k-space in pinned host memory
        reqs.append(ReconRequest(i, y.cpu().pin_memory(), tkey, coord, (N, N), mkey, maps, dcf, niter, 0.0, t))
    return reqs
