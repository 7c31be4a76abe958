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
# kernels the library launches for 3D, width 4, 32 coils (spread.cu dispatch)
# kernels that run the workload's interpolation / gridding (3D, width 4, 32 coils):
# tensor-core gridding unless DMR_NO_TC selects the cell-cube kernel
KERNELS = {"interp": "interp_cube_kernel",
           "grid": "grid_cube_kernel" if os.environ.get("DMR_NO_TC", "0") not in ("", "0") else "grid_tc_kernel",
           "grid_det": "grid_rt_kernel"}
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


# ---------------------------------------------------------------------------
# B200 arm
# ---------------------------------------------------------------------------
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

    # serving after the end-to-end leg: its request sets and slots stay out of the e2e timing
    serving = None
    if not args.no_extras and rank == 0:
        serving = run_serving(dev)

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        cb = CpuBaseline(w)
        cpu = cb.info(cb.run())

    if rank == 0:
        line = {
            "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
            "warmup": max(args.warmup, 3), "ms_per_step": ms / args.steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32 (complex64)",
            "data": "synthetic, seeded (golden-means kooshball, complex Gaussian image and k-space, ramp density weights)",
            "config": {"workload": workload_name(w), "samples_per_step_per_gpu": samples_step,
                       "grid": [math.ceil(w["oversamp"] * N)] * 3,
                       "gridding": "deterministic" if F.deterministic_gridding() else "atomic",
                       "l2": "inputs larger than L2 (image 1.8 GB, k-space 4.9 GB per GPU)"
                       if not args.small else "inputs larger than L2",
                       "parallelism": f"replicas x{world} (one independent workload per GPU)"},
            "roofline": roofline, "cpu_baseline": cpu, "e2e": e2e, "gpu_launches": int(launches),
            "clocks": ck, "extras": extras, "serving": serving,
        }
        print(json.dumps(line), flush=True)
    if world > 1:
        import torch.distributed as dist

        dist.destroy_process_group()


# ---------------------------------------------------------------------------
# serving: CG-SENSE requests, continuous batching vs the plain per-call path
# ---------------------------------------------------------------------------
def run_serving(dev, nreq=64, seed=0, max_active=4):
    """CG-SENSE serving workload (20 CG iterations, Toeplitz; matrix uniform over
    {128, 192, 256, 320}^2, coils over {8, 16, 32}, radial or spiral): all
    requests at once (burst), then Poisson arrivals at 80% of the plain path's
    burst throughput. Both paths run every request set once untimed first
    (plans, caching allocator, graphs). Latency = arrival to result on the host."""
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
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    w = workload(args)
    cores = os.cpu_count() or 1
    cb = CpuBaseline(w, max(1, min(cores, 8, w["coils"])))
    coils = cb.coils
    for _ in range(max(args.warmup, 0)):
        cb.run()
    times = [cb.run() for _ in range(args.steps)]
    info = cb.info(sum(times) / len(times))
    samples = coils * w["spokes"] * w["samples"] * 2
    value = samples * len(times) / sum(times)
    info["value"] = value
    line = {
        "impl": "reference", "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 * sum(times) / len(times),
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32 (complex64)",
        "data": "synthetic, seeded", "config": {"workload": workload_name(w),
                                                 "sample": f"{coils} of {w['coils']} coils per step"},
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
