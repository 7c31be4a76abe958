"""deepmr_b200 — B200-native (sm_100a) non-Cartesian NUFFT for deepmr.

``deepmr_b200.fft`` mirrors ``deepmr.fft``'s NUFFT API (plan_nufft, nufft,
nufft_adj, apply_*, Toeplitz self-adjoint) on hand-written CUDA kernels behind
the C ABI declared in ``include/deepmr_b200.h``. Its callers in the reference
are mirrored beside it: ``linops`` (NUFFT / SENSE operators, ``EncodingOp``),
``optim`` (``cg_solve``), ``calib`` (``find_acs``, ``espirit_cal``), ``dcf``
(Voronoi density compensation) and ``recon`` (device CG-SENSE and the
serving loop).
"""

from . import fft  # noqa: F401

__version__ = "0.1.0"
