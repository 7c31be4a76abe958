"""Autotuner for the spatial bin (shared-memory tile) size of NUFFT plans.

The best bin depends on the dimensionality, the kernel width and the grid
oversampling (they set the halo overhead and the shared-memory footprint of a
tile). `tune` times forward + adjoint NUFFTs on a representative synthetic
radial trajectory for each candidate bin and records the fastest in a JSON
table keyed by (ndim, width, oversampling); `plan_nufft(..., tile=None)`
consults the table and falls back to the library default when no entry
exists. Usage on a GPU:

    python -m deepmr_b200.autotune --ndim 3 --width 4 --oversamp 1.25
    python -m deepmr_b200.autotune --all
"""

import argparse
import json
import math
import os
import threading

import numpy as np
import torch

TABLE_PATH = os.path.join(os.path.dirname(os.path.abspath(__file__)), "tuning.json")

CANDIDATES = {
    1: [(64,), (128,), (256,), (512,)],
    2: [(8, 8), (16, 16), (16, 32), (32, 32)],
    3: [(4, 4, 4), (4, 4, 8), (4, 8, 8), (8, 8, 8)],
}

# representative workloads: (shape, coils, trajectory builder arguments)
WORKLOADS = {
    1: dict(n=4096, coils=8),
    2: dict(n=256, coils=16),
    3: dict(n=96, coils=16),
}

_lock = threading.Lock()
_table = None


def key(ndim, width, oversamp):
    return f"{int(ndim)}d-w{int(width)}-os{float(oversamp):g}"


def _load():
    global _table
    with _lock:
        if _table is None:
            try:
                with open(TABLE_PATH) as f:
                    _table = json.load(f)
            except (OSError, ValueError):
                _table = {}
    return _table


def lookup(ndim, width, oversamp):
    """Tuned bin (z, y, x order) for this configuration, or None."""
    entry = _load().get(key(ndim, width, oversamp))
    return tuple(entry["tile"]) if entry else None


def _trajectory(ndim, n):
    from . import synth

    if ndim == 1:
        rng = np.random.default_rng(0)
        return np.sort(rng.uniform(-n / 2, n / 2, (1, 1, 4 * n, 1)).astype(np.float32), axis=2)
    if ndim == 2:
        return synth.radial_2d(n, 2 * n, n)
    return synth.kooshball_3d(n * n // 4, 2 * n, n)


def _time(fn, repeats):
    fn()
    torch.cuda.synchronize()
    a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    a.record()
    for _ in range(repeats):
        fn()
    b.record()
    torch.cuda.synchronize()
    return a.elapsed_time(b) / repeats


def tune(ndim, width, oversamp, repeats=5, save=True, verbose=True, out=None):
    """Time each candidate bin and record the fastest; returns (tile, timings)."""
    import deepmr_b200.fft as F
    from . import synth

    w = WORKLOADS[ndim]
    n, coils = w["n"], w["coils"]
    coord = torch.as_tensor(_trajectory(ndim, n))
    img = synth.complex_gaussian((coils,) + (n,) * ndim, seed=0, device="cuda")
    timings = {}
    for tile in CANDIDATES[ndim]:
        plan = F.plan_nufft(coord, n, width, oversamp, device="cuda", tile=tile)
        ksp = F.apply_nufft(img, plan)
        ms = _time(lambda: (F.apply_nufft(img, plan), F.apply_nufft_adj(ksp, plan)), repeats)
        timings[str(tile)] = ms
        if verbose:
            print(f"{key(ndim, width, oversamp)} tile {tile}: {ms:.3f} ms", flush=True)
    best = min(CANDIDATES[ndim], key=lambda t: timings[str(t)])
    if save:
        table = _load()
        table[key(ndim, width, oversamp)] = {
            "tile": list(best), "ms": timings,
            "workload": f"{ndim}D n={n} coils={coils} radial, forward+adjoint",
            "device": torch.cuda.get_device_name(),
        }
        with open(out or TABLE_PATH, "w") as f:
            json.dump(table, f, indent=1, sort_keys=True)
    return best, timings


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--ndim", type=int)
    ap.add_argument("--width", type=int)
    ap.add_argument("--oversamp", type=float)
    ap.add_argument("--all", action="store_true", help="the benchmark configurations")
    ap.add_argument("--out", help="table path (default: the package table)")
    a = ap.parse_args()
    if a.all:
        for cfg in [(2, 3, 2.0), (2, 4, 1.25), (2, 6, 2.0), (3, 4, 1.25), (3, 6, 2.0), (1, 4, 1.25)]:
            tune(*cfg, out=a.out)
    else:
        tune(a.ndim, a.width, a.oversamp, out=a.out)


if __name__ == "__main__":
    main()
