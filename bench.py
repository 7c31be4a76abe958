#!/usr/bin/env python
"""NUFFT benchmark on B200: 3D radial kooshball forward + adjoint.

Workload (one step, per GPU): 192^3 complex64 image, 32 coils, 50,000
golden-means spokes x 384 samples (19.2 M samples), Kaiser-Bessel width 4,
oversampling 1.25 (grid 240^3); one forward NUFFT of the 32-coil image and one
adjoint NUFFT (ramp density weights) of a 32-coil k-space. Synthetic seeded
inputs, resident in HBM for `value`; copied from pinned host memory through
the public API for `e2e`.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl reference]

`--impl reference` times the CPU restatement of the reference NUFFT (the
oracle: C loops + torch CPU FFTs, all host threads) on a bounded sample of the
same workload. Under torchrun (N > 1) each rank runs its own replica of the
workload (weak scaling, no data-path collective); timing is the max over ranks.
"""

import argparse
import datetime
import json
import math
import os
import subprocess
import sys
import tempfile
import time

import numpy as np
import torch

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

WORKLOAD = dict(N=192, coils=32, spokes=50000, samples=384, width=4, oversamp=1.25)
FALLBACK_HBM_GBS = 6650.0
METRIC = "NUFFT fwd+adj k-space samples/s (3D kooshball)"
# kernels that run the workload's interpolation / gridding (3D, width 4, 32 coils):
# tensor-core gridding (grid_tmem_kernel) unless DMR_NO_TC selects the cell-cube kernel
KERNELS = {"interp": "interp_cube_kernel",
           "grid": "grid_cube_kernel" if os.environ.get("DMR_NO_TC", "0") not in ("", "0") else "grid_tmem_kernel",
           "grid_det": "grid_tmem_kernel"}
UNIT = "samples/s"


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="b200", choices=["b200", "reference"])
    ap.add_argument("--small", action="store_true", help="reduced workload (profiling)")
    ap.add_argument("--medium", action="store_true", help="32-coil 128^3 workload (profiling)")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-extras", action="store_true", help="skip Toeplitz / per-kernel timing")
    return ap.parse_args()


def workload(args):
    w = dict(WORKLOAD)
    if args.small:
        w.update(N=128, coils=8, spokes=25000, samples=256)
    if getattr(args, "medium", False):
        w.update(N=128, coils=32, spokes=25000, samples=256)
    return w


def workload_name(w):
    return (f"3D radial kooshball {w['N']}^3, {w['coils']} coils, {w['spokes']} spokes x "
            f"{w['samples']} samples (golden means), KB width {w['width']}, oversampling "
            f"{w['oversamp']}: forward + adjoint NUFFT")


# ---------------------------------------------------------------------------
# distributed plumbing (one process per GPU, replicas)
# ---------------------------------------------------------------------------
def dist_init(args):
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if world > 1:
        import torch.distributed as dist

        backend = "nccl" if args.impl == "b200" else "gloo"
        if backend == "nccl":
            torch.cuda.set_device(local)
        dist.init_process_group(backend, timeout=datetime.timedelta(seconds=600))
    return world, rank, local


def barrier(world):
    if world > 1:
        import torch.distributed as dist

        dist.barrier()


def max_over_ranks(x, world, dev):
    if world == 1:
        return x
    import torch.distributed as dist

    t = torch.tensor([x], dtype=torch.float64, device=dev)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


# ---------------------------------------------------------------------------
# clocks during the timed region
# ---------------------------------------------------------------------------
class ClockSampler:
    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, dev):
        self.proc = None
        self.path = None
        try:
            uuid = str(torch.cuda.get_device_properties(dev).uuid)
            self.sel = ["-i", uuid if uuid.startswith("GPU-") else "GPU-" + uuid]
        except Exception:
            self.sel = []

    def start(self):
        fd, self.path = tempfile.mkstemp(suffix=".csv")
        os.close(fd)
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", *self.sel, f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits",
                 "-lms", "200", "-f", self.path],
                stdout=subprocess.DEVNULL, stderr=subprocess.DEVNULL)
        except Exception:
            self.proc = None

    def stop(self):
        if self.proc is None:
            return None
        time.sleep(0.25)
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        rows = []
        try:
            for line in open(self.path):
                parts = [p.strip() for p in line.split(",")]
                if len(parts) >= 9 and parts[1].replace(".", "").isdigit():
                    rows.append(parts)
        finally:
            os.unlink(self.path)
        if not rows:
            return None
        sm = [float(r[1]) for r in rows]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({n for r in rows for n, v in zip(names, r[5:9]) if v.lower() == "active"})
        return {"sm_mhz": float(np.median(sm)), "sm_max_mhz": float(max(float(r[2]) for r in rows)),
                "reasons": reasons, "samples": len(rows),
                "power_w_max": max((float(r[3]) for r in rows if r[3].replace(".", "").isdigit()), default=None)}


def measured_peak():
    path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    try:
        with open(path) as f:
            return float(json.load(f)["hbm_gbs"]), "measured"
    except Exception:
        return FALLBACK_HBM_GBS, "fallback"


def ncu_traffic(kernel, w):
    """DRAM bytes per launch of `kernel` for this workload from the committed ncu summary."""
    path = os.path.join(ROOT, "profiles", "dram_traffic.txt")
    if not os.path.exists(path):
        return None
    key = f"N={w['N']},coils={w['coils']},spokes={w['spokes']},samples={w['samples']}"
    for line in open(path):
        parts = line.split()
        if len(parts) >= 3 and parts[0] == kernel and parts[1] == key:
            return float(parts[2])
    return None


# ---------------------------------------------------------------------------
# CPU baseline: oracle restatement of the reference, all host threads
# ---------------------------------------------------------------------------
class CpuBaseline:
    """Times one forward + adjoint pair of the oracle on a bounded sample:
    the full trajectory with `coils` coils (default: one per host core, at most
    the workload's coil count)."""

    def __init__(self, w, coils=None):
        from oracle import nufft_ref as R
        from deepmr_b200 import synth

        self.R = R
        self.cores = os.cpu_count() or 1
        torch.set_num_threads(self.cores)
        c = torch.as_tensor(synth.kooshball_3d(w["spokes"], w["samples"], w["N"]))
        self.coils = coils or max(1, min(self.cores, w["coils"]))
        self.img = synth.complex_gaussian((self.coils,) + (w["N"],) * 3, seed=0)
        self.ksp = synth.complex_gaussian((self.coils,) + tuple(c.shape[:-1]), seed=1)
        self.dcf = synth.ramp_dcf(c.numpy())
        self.plan = R.plan_nufft(c, w["N"], w["width"], w["oversamp"])
        self.samples = self.coils * c.shape[0] * c.shape[1] * 2

    def run(self):
        t0 = time.perf_counter()
        self.R.apply_nufft(self.img, self.plan)
        self.R.apply_nufft_adj(self.ksp, self.plan, weight=self.dcf)
        return time.perf_counter() - t0

    def info(self, dt):
        return dict(value=self.samples / dt, unit=UNIT, cores=self.cores, kind="port",
                    sample=f"one forward + adjoint pair, full trajectory, {self.coils} coils "
                           f"(oracle: C loops with OpenMP + torch CPU FFT, {self.cores} threads)")


def parity_check(F, cb, plan, img, ksp, dcf, coils=(0, 1)):
    """Relative L2 error of the timed GPU path against the oracle at the full
    workload size, on two of its coils (coils are independent): forward,
    atomic (tensor-core) adjoint and deterministic adjoint."""
    R, sel = cb.R, list(coils)

    def rel(a, b):
        a = np.asarray(torch.as_tensor(a).cpu(), dtype=np.complex128).ravel()
        b = np.asarray(torch.as_tensor(b).cpu(), dtype=np.complex128).ravel()
        return float(np.linalg.norm(a - b) / np.linalg.norm(b))

    out = {"tol": 1e-5, "coils": sel, "reference": "oracle (CPU restatement of the reference), same inputs"}
    out["forward_rel_l2"] = rel(F.apply_nufft(img, plan)[sel], R.apply_nufft(img[sel].cpu(), cb.plan))
    x_ref = R.apply_nufft_adj(ksp[sel].cpu(), cb.plan, weight=dcf.cpu())
    for name, det in (("adjoint_atomic_rel_l2", False), ("adjoint_deterministic_rel_l2", True)):
        old = F.set_deterministic_gridding(det)
        try:
            x = F.apply_nufft_adj(ksp, plan, weight=dcf)[sel]
            plan.interpolator.check_status()
        finally:
            F.set_deterministic_gridding(old)
        out[name] = rel(x, x_ref)
    out["pass"] = all(v < out["tol"] for k, v in out.items() if k.endswith("_rel_l2"))
    return out


# ---------------------------------------------------------------------------
# B200 arm
# ---------------------------------------------------------------------------
def bench_config(w, args, world, deterministic=False):
    """`config` of the JSON line (the same for both arms)."""
    M = w["spokes"] * w["samples"]
    return {"workload": workload_name(w), "samples_per_step_per_gpu": 2 * w["coils"] * M,
            "grid": [math.ceil(w["oversamp"] * w["N"])] * 3,
            "gridding": "deterministic" if deterministic else "atomic",
            "l2": "inputs larger than L2 (image 1.8 GB, k-space 4.9 GB per GPU)"
            if not (args.small or args.medium) else "inputs larger than L2",
            "parallelism": f"replicas x{world} (one independent workload per GPU)"}


def alg_bytes(w, M):
    """Compulsory bytes of one interpolation / gridding launch (complex64 samples and
    grid, float32 coordinates, float32 density weight for gridding)."""
    G = math.ceil(w["oversamp"] * w["N"]) ** 3
    B = w["coils"]
    interp = 8 * B * G + 4 * 3 * M + 8 * B * M
    grid = interp + 4 * M
    return interp, grid


def run_b200(args):
    world, rank, local = dist_init(args)
    import deepmr_b200.fft as F
    from deepmr_b200 import _lib, synth

    dev = torch.device("cuda", local)
    torch.cuda.set_device(dev)
    w = workload(args)
    N, C = w["N"], w["coils"]
    coord = torch.as_tensor(synth.kooshball_3d(w["spokes"], w["samples"], N))
    M = coord.shape[0] * coord.shape[1]
    dcf = torch.as_tensor(synth.ramp_dcf(coord.numpy())).to(dev)
    plan = F.plan_nufft(coord, N, w["width"], w["oversamp"], device=dev)
    img = synth.complex_gaussian((C, N, N, N), seed=1 + rank, device=dev)
    ksp = synth.complex_gaussian((C,) + tuple(coord.shape[:-1]), seed=101 + rank, device=dev)

    def step():
        y = F.apply_nufft(img, plan)
        x = F.apply_nufft_adj(ksp, plan, weight=dcf)
        return y, x

    for _ in range(max(args.warmup, 3)):
        step()
    torch.cuda.synchronize()
    barrier(world)
    clocks = ClockSampler(dev)
    clocks.start()
    n0 = _lib.launch_count()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    torch.cuda.synchronize()
    e0.record()
    for _ in range(args.steps):
        step()
    e1.record()
    torch.cuda.synchronize()
    ms = e0.elapsed_time(e1)
    launches = (_lib.launch_count() - n0) // args.steps
    ck = clocks.stop()
    barrier(world)
    ms = max_over_ranks(ms, world, dev)
    samples_step = 2 * C * M
    value = world * samples_step * args.steps / (ms / 1e3)

    # end to end through the public API: pinned host buffers, copies in the timed region
    # (right after the device-resident timing, before the per-kernel timings and extras)
    e2e = None
    if not args.no_e2e:
        img_h = img.cpu().pin_memory()
        ksp_h = ksp.cpu().pin_memory()

        def estep():
            y = F.apply_nufft(img_h, plan)
            x = F.apply_nufft_adj(ksp_h, plan, weight=dcf)
            return y, x

        # two untimed calls so the pinned-host caching allocator holds both
        # generations of output buffers (a fresh pinned allocation is not a copy)
        y_h, x_h = estep()
        y_h, x_h = estep()
        torch.cuda.synchronize()
        barrier(world)
        ne = max(1, min(args.steps, 3))
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record()
        for _ in range(ne):
            y_h, x_h = estep()
        b.record()
        torch.cuda.synchronize()
        ems = max_over_ranks(a.elapsed_time(b), world, dev)
        e2e = {"value": world * samples_step * ne / (ems / 1e3), "unit": UNIT,
               "h2d_bytes_per_step": int(img_h.numel() * 8 + ksp_h.numel() * 8),
               "d2h_bytes_per_step": int(y_h.numel() * 8 + x_h.numel() * 8),
               "ms_per_step": ems / ne, "steps": ne}

    # per-kernel timing of the dominant kernels (same stream, CUDA events)
    interp_ms = grid_ms = None
    L = _lib.lib()
    st = _lib.stream_ptr(dev)
    ip = plan.interpolator
    gbuf = synth.complex_gaussian((C,) + tuple(ip.dshape), seed=7, device=dev)
    kout = torch.empty_like(ksp)

    def timed(fn, n):
        fn()
        torch.cuda.synchronize()
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record()
        for _ in range(n):
            fn()
        b.record()
        torch.cuda.synchronize()
        return a.elapsed_time(b) / n

    interp_ms = timed(lambda: _lib.check(L.dmr_interp(ip.handle, _lib.ptr(gbuf), _lib.ptr(kout), C, None, 0, st)), args.steps)
    grid_ms = timed(lambda: _lib.check(L.dmr_grid(ip.handle, _lib.ptr(ksp), 0, _lib.ptr(gbuf), C, _lib.ptr(dcf), 0,
                                                  int(F.deterministic_gridding()), st)), args.steps)
    det = 1 - int(F.deterministic_gridding())
    grid_other_ms = timed(lambda: _lib.check(L.dmr_grid(ip.handle, _lib.ptr(ksp), 0, _lib.ptr(gbuf), C, _lib.ptr(dcf),
                                                        0, det, st)), args.steps)
    fwd_ms = timed(lambda: F.apply_nufft(img, plan), args.steps)
    adj_ms = timed(lambda: F.apply_nufft_adj(ksp, plan, weight=dcf), args.steps)
    extras = {"forward_ms": fwd_ms, "adjoint_ms": adj_ms, "interp_kernel_ms": interp_ms,
              "grid_kernel_ms": grid_ms,
              ("grid_deterministic_ms" if det else "grid_atomic_ms"): grid_other_ms}
    if not args.no_extras:
        T = F.plan_toeplitz_nufft(coord, N, dcf=dcf, device=dev)
        extras["toeplitz_selfadj_ms"] = timed(lambda: F.apply_nufft_selfadj(img, T), max(3, args.steps // 2))
        del T
    del gbuf, kout
    torch.cuda.empty_cache()

    ib, gb = alg_bytes(w, M)
    gname, iname = KERNELS["grid_det" if F.deterministic_gridding() else "grid"], KERNELS["interp"]
    if grid_ms >= interp_ms:
        kname, kms, kbytes = gname, grid_ms, gb
    else:
        kname, kms, kbytes = iname, interp_ms, ib
    peak, peak_kind = measured_peak()
    achieved = kbytes / (kms / 1e3) / 1e9
    traffic = ncu_traffic(kname, w)
    roofline = {"bound": "hbm", "kernel": kname, "achieved": achieved, "peak": peak, "unit": "GB/s",
                "frac": achieved / peak, "traffic": traffic, "peak_source": peak_kind,
                "alg_bytes_per_launch": kbytes}

    # serving and the other configurations after the end-to-end leg: their
    # buffers stay out of the e2e timing
    serving = others = None
    if not args.no_extras and rank == 0:
        serving = run_serving(dev)
        others = run_other_configs(dev, max(3, args.steps // 2))

    cpu = parity = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        cb = CpuBaseline(w)
        cpu = cb.info(cb.run())
        parity = parity_check(F, cb, plan, img, ksp, dcf)

    if rank == 0:
        line = {
            "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
            "warmup": max(args.warmup, 3), "ms_per_step": ms / args.steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32 (complex64)",
            "data": "synthetic, seeded (golden-means kooshball, complex Gaussian image and k-space, ramp density weights)",
            "config": bench_config(w, args, world, F.deterministic_gridding()),
            "roofline": roofline, "cpu_baseline": cpu, "parity": parity, "e2e": e2e,
            "gpu_launches": int(launches),
            "clocks": ck, "extras": extras, "serving": serving, "other_configs": others,
        }
        print(json.dumps(line), flush=True)
    if world > 1:
        import torch.distributed as dist

        dist.destroy_process_group()


# ---------------------------------------------------------------------------
# the other configurations: 2D radial, batched uneven frames, differentiable DC
# ---------------------------------------------------------------------------
def _timed_events(fn, n, warm=3):
    for _ in range(warm):
        fn()
    torch.cuda.synchronize()
    a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    a.record()
    for _ in range(n):
        fn()
    b.record()
    torch.cuda.synchronize()
    return a.elapsed_time(b) / n


def nudft2d_fp64(img, coord, n):
    """Direct NUDFT y[b, p] = sum_x img[b, x] exp(-2 pi i k.(x - N//2) / N) in
    float64 on the GPU (coord in grid units, (x, y); image axes (y, x)),
    separable over the two axes, in chunks of samples."""
    dev = img.device
    x = img.to(torch.complex128)
    idx = torch.arange(n, device=dev, dtype=torch.float64) - n // 2
    c = torch.as_tensor(coord, device=dev, dtype=torch.float64).reshape(-1, 2)
    out = []
    for s in range(0, c.shape[0], 8192):
        cc = c[s:s + 8192]
        ex = torch.exp(-2j * math.pi * cc[:, 0:1] * idx[None, :] / n)  # (m, nx)
        ey = torch.exp(-2j * math.pi * cc[:, 1:2] * idx[None, :] / n)  # (m, ny)
        t = torch.einsum("byx,mx->bym", x, ex)
        out.append(torch.einsum("bym,my->bm", t, ey))
    return torch.cat(out, dim=1)


def run_other_configs(dev, steps):
    """Throughput of the other workload configurations with inputs resident in
    HBM (CUDA events, current stream), next to their plain or per-call forms."""
    import deepmr_b200.fft as F
    from deepmr_b200 import synth

    peak, _ = measured_peak()
    out = {}

    # 2D golden-angle radial: 128^2, 8 coils, 256 x 256 samples, width 3, oversampling 2
    N, C = 128, 8
    c = synth.radial_2d(256, 256, N)
    dcf = torch.as_tensor(synth.ramp_dcf(c)).to(dev)
    plan = F.plan_nufft(torch.as_tensor(c), N, 3, 2.0, device=dev)
    img = synth.complex_gaussian((C, N, N), seed=31, device=dev)
    ksp = synth.complex_gaussian((C,) + tuple(c.shape[:-1]), seed=32, device=dev)
    M = c.shape[0] * c.shape[1]
    eager = _timed_events(lambda: (F.apply_nufft(img, plan), F.apply_nufft_adj(ksp, plan, weight=dcf)), 10 * steps)
    op = F.CapturedNUFFT(plan, batch=C, weight=dcf.reshape(-1))
    # inputs resident in the operator's static buffers, as the eager calls' are in theirs
    op.x_in.copy_(img)
    op.y_in.copy_(ksp)
    graph = _timed_events(lambda: (op.forward(), op.adjoint()), 10 * steps)
    y = F.apply_nufft(img, plan)
    ref = nudft2d_fp64(img, c, N)
    yv = y.reshape(C, -1).to(torch.complex128)
    raw = float(torch.linalg.norm(yv - ref) / torch.linalg.norm(ref))
    scale = torch.vdot(yv.flatten(), ref.flatten()) / torch.vdot(yv.flatten(), yv.flatten())
    fitted = float(torch.linalg.norm(scale * yv - ref) / torch.linalg.norm(ref))
    out["radial2d_128_8coils"] = {
        "workload": "2D golden-angle radial 128^2, 8 coils, 256 spokes x 256 samples, KB width 3, "
                    "oversampling 2, ramp density weights: forward + adjoint",
        "samples_per_s": 2 * C * M / (eager / 1e3), "ms_per_pair": eager,
        "captured_graph": {"samples_per_s": 2 * C * M / (graph / 1e3), "ms_per_pair": graph},
        "nudft_fp64": {"rel_l2": raw, "rel_l2_after_global_scale_fit": fitted, "global_scale": abs(complex(scale)),
                       "note": "forward of all 8 coils at all 65,536 samples against a float64 direct NUDFT "
                               "on the GPU (the kernel's own approximation error at width 3, oversampling 2)"}}
    del plan, img, ksp, op, y, ref, yv
    torch.cuda.empty_cache()

    # batched uneven frames: 224^2, 16 coils, 500 spiral frames of U{800..1200} samples
    N, C, NF = 224, 16, 500
    rng = np.random.default_rng(3)
    coords = [synth.spiral_2d(int(L), N, rotation=f * synth.GOLDEN_ANGLE)[0]
              for f, L in enumerate(rng.integers(800, 1201, NF))]
    total = sum(x.shape[0] for x in coords)
    plan = F.plan_nufft(coords, N, 4, 1.25, device=dev)
    img = synth.complex_gaussian((C, NF, N, N), seed=41, device=dev)
    ksp = synth.complex_gaussian((C, total), seed=42, device=dev)
    batched = _timed_events(lambda: (F.apply_nufft(img, plan), F.apply_nufft_adj(ksp, plan)), steps)
    op = F.CapturedNUFFT(plan, batch=C)
    op.x_in.copy_(img.reshape(op.image_shape))
    op.y_in.copy_(ksp.reshape(op.kspace_shape))
    graph = _timed_events(lambda: (op.forward(), op.adjoint()), steps)
    del op
    torch.cuda.empty_cache()
    plans = [F.plan_nufft(torch.as_tensor(x), N, 4, 1.25, device=dev) for x in coords]
    offs = np.concatenate([[0], np.cumsum([x.shape[0] for x in coords])])
    kparts = [ksp[:, offs[f]:offs[f + 1]].reshape(C, 1, -1) for f in range(NF)]

    def per_frame():
        for f in range(NF):
            F.apply_nufft(img[:, f], plans[f])
            F.apply_nufft_adj(kparts[f], plans[f])

    plain = _timed_events(per_frame, max(1, steps // 2), warm=1)
    alg = 2 * (8 * C * NF * N * N + 4 * 2 * total + 8 * C * total)
    out["uneven_frames_224_16coils_500frames"] = {
        "workload": f"500 variable-density spiral frames of U{{800..1200}} samples ({total} in all), 224^2, "
                    "16 coils, KB width 4, oversampling 1.25: forward + adjoint of all frames",
        "batched": {"samples_per_s": 2 * C * total / (batched / 1e3), "ms_per_pair": batched,
                    "hbm_frac_of_measured": alg / (batched / 1e3) / 1e9 / peak},
        "batched_captured_graph": {"samples_per_s": 2 * C * total / (graph / 1e3), "ms_per_pair": graph},
        "per_frame_calls": {"samples_per_s": 2 * C * total / (plain / 1e3), "ms_per_pair": plain,
                            "note": "500 plans, one apply_nufft + apply_nufft_adj call per frame"},
        "alg_bytes_per_pair": alg}
    del plan, plans, img, ksp, kparts
    torch.cuda.empty_cache()

    # differentiable data consistency: 256^2, 12 coils, 402 x 512 radial, gradients of
    # ||A x - y||^2 with respect to the image and the trajectory
    N, C = 256, 12
    c = synth.radial_2d(402, 512, N)
    coord = torch.as_tensor(c).to(dev)
    x = synth.complex_gaussian((C, N, N), seed=51, device=dev)
    yobs = synth.complex_gaussian((C,) + tuple(c.shape[:-1]), seed=52, device=dev)
    M = c.shape[0] * c.shape[1]

    def dc_step():
        xx = x.clone().requires_grad_(True)
        cc = coord.clone().requires_grad_(True)
        r = F.nufft(xx, cc, width=4, oversamp=1.25, device=dev) - yobs
        loss = (r.real**2 + r.imag**2).sum()
        loss.backward()
        return xx.grad, cc.grad

    dc = _timed_events(dc_step, steps)
    out["dc_gradients_256_12coils"] = {
        "workload": "2D radial 256^2, 12 coils, 402 spokes x 512 samples, KB width 4, oversampling 1.25: "
                    "loss ||A x - y||^2 and its gradients w.r.t. the image and the trajectory (plan, forward, "
                    "adjoint, trajectory-gradient kernel)",
        "ms_per_step": dc, "samples_per_s": C * M / (dc / 1e3)}
    torch.cuda.empty_cache()
    return out


# ---------------------------------------------------------------------------
# serving: CG-SENSE requests, continuous batching vs the plain per-call path
# ---------------------------------------------------------------------------
def run_serving(dev, nreq=64, seed=0, max_active=4):
    """CG-SENSE serving workload (20 CG iterations, Toeplitz; matrix uniform over
    {128, 192, 256, 320}^2, coils over {8, 16, 32}, radial or spiral): all
    requests at once (burst), then Poisson arrivals at 80% of the plain path's
    burst throughput. Both paths run every request set once untimed first
    (plans, caching allocator, graphs). Requests carry their k-space in pinned
    host memory; latency = arrival to the result in host memory (upload,
    AHy, CG and download included)."""
    from deepmr_b200 import recon

    burst = recon.synthetic_requests(nreq, rate_hz=1e6, seed=seed)
    srv = recon.ReconServer(device=dev, max_active=max_active, hbm_budget=32 << 30)
    srv.prepare(burst)
    srv.run(burst, realtime=False)
    srv.run_sequential(burst, realtime=False)
    out = {"workload": f"{nreq} CG-SENSE requests, 20 iterations, Toeplitz normal operator, "
                       "matrix {128,192,256,320}^2, coils {8,16,32}, radial or spiral",
           "max_active": max_active}
    seq = srv.run_sequential(burst, realtime=False).summary()
    cont = srv.run(burst, realtime=False).summary()
    out["burst"] = {"plain": seq, "continuous": cont}
    rate = 0.8 * seq["throughput_rps"]
    pois = recon.synthetic_requests(nreq, rate_hz=rate, seed=seed + 1)
    srv.prepare(pois)
    srv.run(pois, realtime=False)
    srv.run_sequential(pois, realtime=False)
    out["poisson"] = {"rate_hz": rate, "plain": srv.run_sequential(pois).summary(),
                      "continuous": srv.run(pois).summary()}
    torch.cuda.synchronize(dev)
    return out


# ---------------------------------------------------------------------------
# reference arm: CPU restatement of the reference, host cores
# ---------------------------------------------------------------------------
def run_reference(args):
    """The reference's CPU algorithm (the oracle port: C loops with OpenMP over
    (frame, coil) for gridding and over samples for interpolation, torch CPU
    FFTs) on the host cores. Each step is one forward + adjoint pair over the
    full trajectory for as many coils as there are host threads (at most the
    workload's 32), so the per-(frame, coil) gridding keeps every core busy;
    time is linear in the coil count, and `value` is samples per second like
    the GPU arm's."""
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    w = workload(args)
    cores = os.cpu_count() or 1
    cb = CpuBaseline(w, max(1, min(cores, w["coils"])))
    coils = cb.coils
    for _ in range(max(args.warmup, 0)):
        cb.run()
    times = [cb.run() for _ in range(args.steps)]
    info = cb.info(sum(times) / len(times))
    samples = coils * w["spokes"] * w["samples"] * 2
    value = samples * len(times) / sum(times)
    info["value"] = value
    info["sample"] = (f"{coils} of {w['coils']} coils per step (one per host thread), full trajectory; "
                      + info["sample"])
    line = {
        "impl": "reference", "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 * sum(times) / len(times),
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32 (complex64)",
        "data": "synthetic, seeded (golden-means kooshball, complex Gaussian image and k-space, ramp density weights)",
        "config": bench_config(w, args, world),
        "cpu_baseline": info, "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0,
                                      "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


def main():
    args = parse()
    if args.impl == "reference":
        run_reference(args)
    else:
        run_b200(args)


if __name__ == "__main__":
    main()
