"""Time the reference's own CPU NUFFT (Numba) against the oracle port on one
common case, to show what the port stands for in `bench.py --impl reference`.

Test infrastructure: it imports the reference project (read-only), so it runs
only where the reference is present; its location is ``DEEPMR_REFERENCE``
(the project root) or ``--reference PATH``::

    DEEPMR_REFERENCE=/path/to/deep-mr python oracle/time_reference.py

Case: reduced 3D kooshball, 192^3 image, 2 coils, 2000 golden-means spokes x
384 samples, Kaiser-Bessel width 4, oversampling 1.25, ramp density weights;
one forward + one adjoint per pair, after one untimed pair (Numba compiles
on the first call). The reference runs as shipped and with ``gc.collect``
replaced by a no-op (the reference calls it in every apply, nufft.py:526 and
604, and it dominates the CPU time); the port runs its C loops with OpenMP.
Both use every host thread. Prints one JSON line.
"""

import gc
import json
import os
import sys
import time

import numpy as np
import torch

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.join(ROOT, "tests", "golden"))

if "--reference" in sys.argv:
    i = sys.argv.index("--reference")
    os.environ["DEEPMR_REFERENCE"] = sys.argv[i + 1]
    del sys.argv[i:i + 2]

import make_golden  # noqa: E402  (reference import shims; needs DEEPMR_REFERENCE)

from deepmr_b200 import synth  # noqa: E402
from oracle import nufft_ref as R  # noqa: E402

N, SPOKES, SAMPLES, COILS, W, OS = 192, 2000, 384, 2, 4, 1.25


def _time_pairs(fwd, adj, img, ksp, dcf, reps):
    fwd(img)
    adj(ksp, dcf)
    tf, ta = [], []
    for _ in range(reps):
        t0 = time.perf_counter()
        fwd(img)
        t1 = time.perf_counter()
        adj(ksp, dcf)
        t2 = time.perf_counter()
        tf.append(t1 - t0)
        ta.append(t2 - t1)
    return float(np.median(tf)), float(np.median(ta))


def main(reps=3):
    torch.set_num_threads(os.cpu_count() or 1)
    coord = torch.as_tensor(synth.kooshball_3d(SPOKES, SAMPLES, N))
    dcf = torch.as_tensor(synth.ramp_dcf(coord.numpy()))
    img = synth.complex_gaussian((COILS, N, N, N), seed=0)
    ksp = synth.complex_gaussian((COILS, SPOKES, SAMPLES), seed=1)
    samples = COILS * SPOKES * SAMPLES

    Nref, _ = make_golden.import_reference()
    rplan = Nref.plan_nufft(coord, N, width=W, oversamp=OS)

    def rf(x):
        return Nref.apply_nufft(x, rplan)

    def ra(y, w):
        return Nref.apply_nufft_adj(y, rplan, weight=w)

    out = {"case": f"3D kooshball {N}^3, {COILS} coils, {SPOKES} spokes x {SAMPLES}, W {W}, os {OS}",
           "threads": os.cpu_count()}
    f, a = _time_pairs(rf, ra, img, ksp, dcf, reps)
    out["reference_as_shipped_ms"] = {"forward": 1e3 * f, "adjoint": 1e3 * a}
    collect = gc.collect
    gc.collect = lambda *args, **kwargs: 0
    try:
        f, a = _time_pairs(rf, ra, img, ksp, dcf, reps)
    finally:
        gc.collect = collect
    out["reference_gc_patched_ms"] = {"forward": 1e3 * f, "adjoint": 1e3 * a}
    out["reference_gc_patched_samples_per_s"] = 2 * samples / (f + a)

    oplan = R.plan_nufft(coord, N, W, OS)
    f, a = _time_pairs(lambda x: R.apply_nufft(x, oplan), lambda y, w: R.apply_nufft_adj(y, oplan, weight=w),
                       img, ksp, dcf, reps)
    out["port_ms"] = {"forward": 1e3 * f, "adjoint": 1e3 * a}
    out["port_samples_per_s"] = 2 * samples / (f + a)
    print(json.dumps(out))


if __name__ == "__main__":
    main()
