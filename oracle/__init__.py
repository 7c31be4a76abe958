"""ORACLE — test infrastructure only, never part of the product path.

A CPU restatement of the reference NUFFT (deepmr ``deepmr.fft``): plan
arithmetic and pipeline in ``nufft_ref.py``, per-sample loops in plain C
(``kernels.c``, built by ``build.py``), plus a float64 direct NUDFT.
It is pinned against golden vectors produced by running the reference itself
(``tests/golden/make_golden.py``). Only ``tests/``, ``__graft_entry__.smoke()``
and ``bench.py``'s CPU-baseline leg may import it, and only as the checker or
the timed CPU baseline.
"""
