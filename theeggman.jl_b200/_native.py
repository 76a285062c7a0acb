"""ctypes binding of libeggman_b200.so (the C ABI declared in include/eggman_b200.h).

The library is the only compute path: if it cannot be loaded, or finds no CUDA device, every
entry point raises.  There is no CPU fallback.
"""
from __future__ import annotations

import ctypes
import os
from functools import lru_cache

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libeggman_b200.so")

# status codes
EGG_OK = 0
EGG_ERR_ARGUMENT = 1
EGG_ERR_DIMENSION = 2
EGG_ERR_TOO_LARGE = 3
EGG_ERR_NO_PLAN = 4
EGG_ERR_CUDA = 5
EGG_ERR_TIMEOUT = 6
EGG_ERR_NO_DEVICE = 7
EGG_ERR_PLAN_INVALID = 8

# element types
EGG_F64, EGG_C128, EGG_F32, EGG_C64, EGG_I64 = 0, 1, 2, 3, 4
# precision modes (DP: all three; sieve: exact or fma)
PREC = {"exact": 0, "fma": 1, "mixed": 2}

DTYPE_OF = {
    np.dtype(np.float64): EGG_F64,
    np.dtype(np.complex128): EGG_C128,
    np.dtype(np.float32): EGG_F32,
    np.dtype(np.complex64): EGG_C64,
    np.dtype(np.int64): EGG_I64,
}

# Every symbol include/eggman_b200.h declares.
EXPORTS = (
    "egg_version", "egg_last_error", "egg_init", "egg_cache_bytes", "egg_cache_clear",
    "egg_dp_batch_bytes", "egg_dp_counts", "egg_plan_upload", "egg_plan_build", "egg_plan_info",
    "egg_plan_download", "egg_plan_release", "egg_dp_batch", "egg_dp_batch_device", "egg_sieve",
    "egg_sieve_device", "egg_sieve_batch", "egg_sieve_batch_device", "egg_sieve_device_noalloc", "egg_launch_count",
    "egg_dp_mix", "egg_dp_mix_device", "egg_dp_mix_tuning", "egg_dp_mix_set_tuning", "egg_sieve_reference_sum",
    "egg_sieve_repeated_batch", "egg_sieve_repeated_batch_device", "egg_selfcheck_division",
    "egg_dp_mix_set_engine", "egg_dp_mix_engine", "egg_selfcheck_barrier",
)


class ArgumentError(ValueError):
    """The reference's ArgumentError."""


class DimensionMismatch(ValueError):
    """The reference's DimensionMismatch."""


class DeviceError(RuntimeError):
    """A CUDA failure, a missing device, or a bounded device wait that ran out."""


class PlanError(RuntimeError):
    """No resident plan, or an uploaded plan failed the device-side structure check."""


_ERR_CLASS = {
    EGG_ERR_ARGUMENT: ArgumentError,
    EGG_ERR_DIMENSION: DimensionMismatch,
    EGG_ERR_TOO_LARGE: ArgumentError,   # the reference refuses oversized plans with ArgumentError
    EGG_ERR_NO_PLAN: PlanError,
    EGG_ERR_CUDA: DeviceError,
    EGG_ERR_TIMEOUT: DeviceError,
    EGG_ERR_NO_DEVICE: DeviceError,
    EGG_ERR_PLAN_INVALID: PlanError,
}


@lru_cache(maxsize=1)
def lib() -> ctypes.CDLL:
    """Load the library (raises OSError if it has not been built)."""
    if not os.path.exists(LIB_PATH):
        raise OSError(f"{LIB_PATH} is missing; build it with `python theeggman.jl_b200/build.py`")
    L = ctypes.CDLL(LIB_PATH)
    vp, i64, i32 = ctypes.c_void_p, ctypes.c_int64, ctypes.c_int
    p64 = ctypes.POINTER(ctypes.c_int64)
    L.egg_version.restype = ctypes.c_char_p
    L.egg_last_error.restype = ctypes.c_char_p
    L.egg_init.argtypes = [i32]
    L.egg_cache_bytes.restype = i64
    L.egg_launch_count.restype = i64
    L.egg_dp_batch_bytes.argtypes = [i32, i32, i64]
    L.egg_dp_batch_bytes.restype = i64
    L.egg_dp_counts.argtypes = [i32, p64, p64]
    L.egg_plan_upload.argtypes = [i32, i32, vp, vp, vp, i64, i64, i64]
    L.egg_plan_build.argtypes = [i32, i32]
    L.egg_plan_info.argtypes = [i32, i32, p64, p64, p64, p64]
    L.egg_plan_download.argtypes = [i32, i32, vp, vp, vp]
    L.egg_plan_release.argtypes = [i32, i32]
    L.egg_dp_batch.argtypes = [i32, i32, i32, i32, vp, i64, i64, vp]
    L.egg_dp_batch_device.argtypes = [i32, i32, i32, i32, vp, i64, vp, vp]
    L.egg_sieve.argtypes = [i32, i32, vp, i64, vp, i32, vp]
    L.egg_sieve_device.argtypes = [i32, i32, vp, i64, vp, i32, vp, vp]
    L.egg_sieve_batch.argtypes = [i32, i32, i64, i64, vp, vp, vp, vp, vp]
    L.egg_sieve_batch_device.argtypes = [i32, i32, i64, i64, vp, vp, vp, vp, vp, vp]
    L.egg_sieve_device_noalloc.argtypes = [i32, i32, vp, i64, vp, i32, vp, vp]
    L.egg_dp_mix.argtypes = [i32, i32, vp, i64, i64, vp, vp, vp]
    L.egg_dp_mix_device.argtypes = [i32, i32, vp, i64, i64, vp, vp, vp, vp]
    L.egg_dp_mix_tuning.argtypes = [i32, i32, i32, vp, vp]
    L.egg_dp_mix_set_tuning.argtypes = [i32, i32, i32, i32, i64]
    L.egg_sieve_reference_sum.argtypes = [i32, vp, i64, vp, i32, i64, vp]
    L.egg_sieve_repeated_batch.argtypes = [i32, i32, i64, i64, vp, i64, vp, i32, vp]
    L.egg_sieve_repeated_batch_device.argtypes = [i32, i32, i64, i64, vp, i64, vp, i32, vp, vp]
    L.egg_selfcheck_division.argtypes = [vp, vp, i64, vp, vp]
    L.egg_dp_mix_set_engine.argtypes = [i32]
    L.egg_selfcheck_barrier.argtypes = [i32, i64, vp]
    return L


def check(rc: int) -> None:
    if rc != EGG_OK:
        msg = lib().egg_last_error().decode(errors="replace")
        raise _ERR_CLASS.get(rc, DeviceError)(msg or f"eggman_b200 status {rc}")


def ptr(a: np.ndarray) -> int:
    return a.ctypes.data
