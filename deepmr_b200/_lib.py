"""ctypes binding of the in-tree CUDA library ``lib/libdeepmr_b200.so``.

The library is required: if it is missing or cannot be loaded every entry
point raises (there is no CPU fallback). Build it with
``python -m deepmr_b200.build``.
"""

import ctypes
import os
import threading

import torch

_HERE = os.path.dirname(os.path.abspath(__file__))
# DMR_LIBRARY selects another build of the same library (same ABI)
LIB_PATH = os.environ.get("DMR_LIBRARY") or os.path.join(_HERE, "lib", "libdeepmr_b200.so")

ERRORS = {
    -1: "DMR_ERR_INVALID",
    -2: "DMR_ERR_CUDA",
    -3: "DMR_ERR_OOM",
    -4: "DMR_ERR_COORD",
    -5: "DMR_ERR_CUFFT",
    -6: "DMR_ERR_UNSUPPORTED",
    -7: "DMR_ERR_WORKSPACE",
    -8: "DMR_ERR_TIMEOUT",
}

# every symbol declared in include/deepmr_b200.h
SYMBOLS = (
    "dmr_version",
    "dmr_last_error",
    "dmr_launch_count",
    "dmr_tc_timeouts",
    "dmr_plan_status",
    "dmr_tc_test_stall",
    "dmr_fft3_fused",
    "dmr_tc_min_coils",
    "dmr_scratch_release",
    "dmr_det_scratch_limit",
    "dmr_detect_cartesian",
    "dmr_plan_create",
    "dmr_plan_destroy",
    "dmr_plan_scale",
    "dmr_plan_info",
    "dmr_interp",
    "dmr_grid",
    "dmr_nufft_workspace_bytes",
    "dmr_nufft_forward",
    "dmr_nufft_adjoint",
    "dmr_nufft_lowrank_workspace_bytes",
    "dmr_nufft_forward_lowrank",
    "dmr_nufft_adjoint_lowrank",
    "dmr_nufft_traj_grad",
    "dmr_toeplitz_workspace_bytes",
    "dmr_toeplitz_finalize",
    "dmr_toeplitz_apply",
    "dmr_sense_normal",
    "dmr_cg_state_bytes",
    "dmr_cg_init",
    "dmr_cg_step",
    "dmr_cg_residual",
    "dmr_toeplitz_normalize_noalloc",
)


class DmrError(RuntimeError):
    """Error returned by the CUDA library (carries the DMR_ERR_* code)."""

    def __init__(self, code, msg):
        super().__init__(f"{ERRORS.get(code, code)}: {msg}")
        self.code = code


_lock = threading.Lock()
_LIB = None

vp = ctypes.c_void_p
i32 = ctypes.c_int32
i64 = ctypes.c_int64
i32p = ctypes.POINTER(ctypes.c_int32)
i64p = ctypes.POINTER(ctypes.c_int64)
f32p = ctypes.POINTER(ctypes.c_float)
szp = ctypes.POINTER(ctypes.c_size_t)

_SIGS = {
    "dmr_version": (ctypes.c_int, []),
    "dmr_last_error": (ctypes.c_char_p, []),
    "dmr_launch_count": (i64, []),
    "dmr_tc_timeouts": (ctypes.c_int, [i64p, ctypes.c_int]),
    "dmr_plan_status": (ctypes.c_int, [vp, i32p, ctypes.c_int, vp]),
    "dmr_tc_test_stall": (ctypes.c_int, [ctypes.c_int]),
    "dmr_fft3_fused": (ctypes.c_int, [vp]),
    "dmr_tc_min_coils": (ctypes.c_int, [ctypes.c_int]),
    "dmr_scratch_release": (ctypes.c_int, [ctypes.c_int]),
    "dmr_det_scratch_limit": (ctypes.c_int64, [ctypes.c_int64]),
    "dmr_detect_cartesian": (ctypes.c_int, [vp, i64, ctypes.c_int, i32p, i32p, vp]),
    "dmr_plan_create": (
        ctypes.c_int,
        [ctypes.c_int, i32p, i32p, i32p, f32p, f32p, vp, i64p, i64, i32p, vp, ctypes.POINTER(vp)],
    ),
    "dmr_plan_destroy": (ctypes.c_int, [vp]),
    "dmr_plan_scale": (ctypes.c_int, [vp, ctypes.POINTER(ctypes.c_double)]),
    "dmr_plan_info": (ctypes.c_int, [vp, i64p, i64p, i32p]),
    "dmr_interp": (ctypes.c_int, [vp, vp, vp, i64, vp, ctypes.c_int, vp]),
    "dmr_grid": (ctypes.c_int, [vp, vp, ctypes.c_int, vp, i64, vp, ctypes.c_int, ctypes.c_int, vp]),
    "dmr_nufft_workspace_bytes": (ctypes.c_int, [vp, i64, szp]),
    "dmr_nufft_forward": (
        ctypes.c_int,
        [vp, vp, ctypes.c_int, vp, i64, vp, ctypes.c_int, vp, ctypes.c_size_t, vp],
    ),
    "dmr_nufft_adjoint": (
        ctypes.c_int,
        [vp, vp, ctypes.c_int, vp, i64, vp, ctypes.c_int, ctypes.c_int, vp, ctypes.c_size_t, vp],
    ),
    "dmr_nufft_lowrank_workspace_bytes": (ctypes.c_int, [vp, i64, i64, szp]),
    "dmr_nufft_forward_lowrank": (
        ctypes.c_int,
        [vp, vp, ctypes.c_int, i64, vp, vp, i64, vp, ctypes.c_int, vp, ctypes.c_size_t, vp],
    ),
    "dmr_nufft_adjoint_lowrank": (
        ctypes.c_int,
        [vp, vp, ctypes.c_int, i64, vp, vp, i64, vp, ctypes.c_int, ctypes.c_int, vp, ctypes.c_size_t, vp],
    ),
    "dmr_nufft_traj_grad": (
        ctypes.c_int,
        [vp, vp, ctypes.c_int, vp, i64, vp, ctypes.c_int, ctypes.c_double, vp, vp, ctypes.c_size_t, vp],
    ),
    "dmr_toeplitz_workspace_bytes": (ctypes.c_int, [ctypes.c_int, i32p, i64, szp]),
    "dmr_toeplitz_finalize": (
        ctypes.c_int,
        [ctypes.c_int, i32p, i64, vp, vp, vp, ctypes.c_size_t, vp],
    ),
    "dmr_toeplitz_apply": (
        ctypes.c_int,
        [ctypes.c_int, i32p, i32p, vp, i64, vp, ctypes.c_int, vp, i64, vp, ctypes.c_size_t, vp],
    ),
    "dmr_toeplitz_normalize_noalloc": (ctypes.c_int, [vp, i64, vp]),
    "dmr_sense_normal": (
        ctypes.c_int,
        [ctypes.c_int, i32p, i32p, vp, vp, i64, vp, vp, ctypes.c_float, vp, ctypes.c_size_t, vp],
    ),
    "dmr_cg_state_bytes": (ctypes.c_int, [szp]),
    "dmr_cg_init": (ctypes.c_int, [vp, vp, vp, vp, i64, vp, vp]),
    "dmr_cg_step": (ctypes.c_int, [vp, vp, vp, vp, i64, vp, vp]),
    "dmr_cg_residual": (ctypes.c_int, [vp, ctypes.POINTER(ctypes.c_double), vp]),
}


def lib():
    """Load the CUDA library (once). Raises if it is absent."""
    global _LIB
    if _LIB is not None:
        return _LIB
    with _lock:
        if _LIB is None:
            if not os.path.exists(LIB_PATH):
                raise RuntimeError(
                    f"deepmr_b200 CUDA library not found at {LIB_PATH}; "
                    "build it with `python -m deepmr_b200.build`"
                )
            L = ctypes.CDLL(LIB_PATH)
            for name, (res, args) in _SIGS.items():
                fn = getattr(L, name)
                fn.restype = res
                fn.argtypes = args
            _LIB = L
    return _LIB


def check(rc):
    if rc != 0:
        msg = lib().dmr_last_error().decode(errors="replace")
        raise DmrError(rc, msg)


def i32_array(values):
    arr = (ctypes.c_int32 * len(values))(*[int(v) for v in values])
    return arr


def f32_array(values):
    return (ctypes.c_float * len(values))(*[float(v) for v in values])


def ptr(t):
    """Device pointer of a tensor (None -> NULL)."""
    if t is None:
        return None
    return ctypes.c_void_p(t.data_ptr())


def stream_ptr(device):
    return ctypes.c_void_p(torch.cuda.current_stream(device).cuda_stream)


def launch_count():
    return int(lib().dmr_launch_count())


def require_cuda():
    if not torch.cuda.is_available():
        raise RuntimeError(
            "deepmr_b200 computes on a CUDA device (sm_100a); no CUDA device is available"
        )
