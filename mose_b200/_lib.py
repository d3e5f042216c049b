"""ctypes binding of libmose_gpu.so (include/mose_gpu.h).

Loading fails loudly when the library is missing: there is no CPU fallback.
"""
from __future__ import annotations

import ctypes as C
import os
from pathlib import Path

_HERE = Path(__file__).resolve().parent
# MOSE_GPU_LIB selects another build of the same library (e.g. a tuning variant)
LIB_PATH = Path(os.environ.get("MOSE_GPU_LIB", _HERE / "lib" / "libmose_gpu.so"))

ABI_VERSION = 2

OK = 0
ERR_INVALID, ERR_UNSUPPORTED, ERR_CUDA, ERR_INTERFACE_STATE, ERR_NAN_OR_NEG_P, ERR_METRICS, ERR_TIMEOUT, \
    ERR_NOT_READY = 1, 2, 3, 4, 5, 6, 7, 8

PRECISION_FP64_EXACT, PRECISION_FP64, PRECISION_MIXED = 0, 1, 2

class Config(C.Structure):
    """mose_gpu_config."""
    _fields_ = [("abi_version", C.c_int32), ("n_rk", C.c_int32), ("cfl", C.c_double),
                ("time_accurate", C.c_int32), ("ramp_iter", C.c_int32), ("limiter", C.c_int32),
                ("riemann", C.c_int32), ("integration", C.c_int32), ("precision", C.c_int32),
                ("ndir", C.c_int32), ("nsc", C.c_int32), ("gamma", C.c_double), ("rgas", C.c_double),
                ("device", C.c_int32), ("res_diter", C.c_int32)]


# Every exported symbol of include/mose_gpu.h, with its ctypes signature.
_D = C.c_void_p
_dp = C.POINTER(C.c_double)
_ip = C.POINTER(C.c_int32)
SIGNATURES = {
    "mose_gpu_default_config": (None, [C.POINTER(Config)]),
    "mose_gpu_create": (C.c_int, [C.POINTER(Config), C.POINTER(C.c_void_p)]),
    "mose_gpu_destroy": (None, [_D]),
    "mose_gpu_last_error": (C.c_char_p, [_D]),
    "mose_gpu_error_location": (C.c_int, [_D, _ip, _ip, _ip, _ip]),
    "mose_gpu_add_block": (C.c_int, [_D, C.c_int32, C.c_int32, C.c_int32, C.c_int32, _dp, _dp]),
    "mose_gpu_set_bcs": (C.c_int, [_D, _ip, _dp, C.c_int32]),
    "mose_gpu_setup": (C.c_int, [_D]),
    "mose_gpu_upload_prim": (C.c_int, [_D, C.c_int32, _dp]),
    "mose_gpu_download_prim": (C.c_int, [_D, C.c_int32, _dp]),
    "mose_gpu_upload_prim_old": (C.c_int, [_D, C.c_int32, _dp]),
    "mose_gpu_download_residual": (C.c_int, [_D, C.c_int32, _dp]),
    "mose_gpu_upload_residual": (C.c_int, [_D, C.c_int32, _dp]),
    "mose_gpu_download_dt": (C.c_int, [_D, C.c_int32, _dp]),
    "mose_gpu_upload_dt": (C.c_int, [_D, C.c_int32, _dp]),
    "mose_gpu_compute_dt": (C.c_int, [_D, C.c_double, C.c_int32, C.c_int32, _dp]),
    "mose_gpu_set_global_dt": (C.c_int, [_D, C.c_double]),
    "mose_gpu_copy_state": (C.c_int, [_D]),
    "mose_gpu_fill_ghosts": (C.c_int, [_D]),
    "mose_gpu_residual": (C.c_int, [_D]),
    "mose_gpu_rk_stage": (C.c_int, [_D, C.c_int32]),
    "mose_gpu_step": (C.c_int, [_D, _dp, _dp]),
    "mose_gpu_advance": (C.c_int, [_D, C.c_int32, _dp, _dp]),
    "mose_gpu_residual_norms": (C.c_int, [_D, _dp]),
    "mose_gpu_set_time": (C.c_int, [_D, C.c_double, C.c_int32]),
    "mose_gpu_get_time": (C.c_int, [_D, _dp, _ip]),
    "mose_gpu_synchronize": (C.c_int, [_D]),
    "mose_gpu_uniform_metrics": (C.c_int, [_D]),
    "mose_gpu_stream": (C.c_void_p, [_D]),
    "mose_gpu_residual_norms_noalloc": (C.c_int, [_D, _D, C.c_int32, C.c_int32, C.c_int32, _D, _D]),
    "mose_gpu_noalloc_last_error": (C.c_char_p, []),
    "mose_gpu_time_kernels": (C.c_int, [_D, C.c_int32, _dp, _ip]),
    "mose_gpu_launch_count": (C.c_int64, [_D]),
    "mose_gpu_download_metrics": (C.c_int, [_D, C.c_int32, _dp, _dp]),
    "mose_gpu_download_faces": (C.c_int, [_D, C.c_int32, C.c_int32, _dp, _dp]),
    "mose_gpu_check_fast_math": (C.c_int, [C.c_int64, C.c_uint64, _dp]),
    "mose_gpu_set_inflow_mach": (C.c_int, [_D, C.c_double]),
    "mose_gpu_set_riemann_minf": (C.c_int, [_D, C.c_double]),
    "mose_gpu_set_irs_beta": (C.c_int, [_D, C.c_double]),
    "mose_gpu_set_viscous": (C.c_int, [_D, C.c_int32, C.c_double, C.c_double, C.c_double]),
    "mose_gpu_set_sd_limiter": (C.c_int, [_D, C.c_int32]),
    "mose_gpu_add_series": (C.c_int, [_D, _dp, _dp, C.c_int32, C.c_int32, _ip]),
    "mose_gpu_set_tiling": (C.c_int, [_D, _ip]),
    "mose_gpu_get_tiling": (C.c_int, [_D, _ip]),
    "mose_gpu_autotune": (C.c_int, [_D, C.c_int32, _ip, _dp, _dp]),
    "mose_gpu_adjoint_forward": (C.c_int, [_D, C.c_int32, C.c_int32, C.c_int32, C.c_int32, _dp]),
    "mose_gpu_adjoint_backward": (C.c_int, [_D, _dp]),
    "mose_gpu_adjoint_step": (C.c_int, [_D, _dp]),
    "mose_gpu_upload_adjoint": (C.c_int, [_D, C.c_int32, _dp]),
    "mose_gpu_download_adjoint": (C.c_int, [_D, C.c_int32, _dp]),
}


_lib = None
_probe = None

# the measurement-only library (FP64 issue ceilings), not part of the ABI
PROBE_PATH = _HERE / "lib" / "libmose_probe.so"


def load_probe() -> C.CDLL:
    """Loads libmose_probe.so (bench and tests only); raises if not built."""
    global _probe
    if _probe is not None:
        return _probe
    if not PROBE_PATH.exists():
        raise RuntimeError(f"{PROBE_PATH} is missing: build it with `python -m mose_b200.build`")
    lib = C.CDLL(str(PROBE_PATH))
    lib.mose_probe_fp64_peak.restype = C.c_int
    lib.mose_probe_fp64_peak.argtypes = [C.c_int32, _dp]
    _probe = lib
    return lib


def load() -> C.CDLL:
    """Loads and types the library; raises if it was not built."""
    global _lib
    if _lib is not None:
        return _lib
    if not LIB_PATH.exists():
        raise RuntimeError(f"{LIB_PATH} is missing: build it with `python -m mose_b200.build` "
                           "(there is no CPU fallback for this path)")
    lib = C.CDLL(str(LIB_PATH))
    for name, (res, args) in SIGNATURES.items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    _lib = lib
    return lib
