"""TheEggman.jl's hafnian hot paths on B200 (sm_100a).

The host side mirrors the reference's public API (``hafnian``, ``hafnian_repeated``, their batched
forms, ``reduction``, ``matched_reps``, the device-cache helpers).  All hafnians are computed by
``libeggman_b200.so`` -- hand-written CUDA for the subset DP and the Bjorklund/Glynn sieve -- behind
the C ABI in ``include/eggman_b200.h``.

The package directory's name is not a Python identifier; load it under the name
``theeggman_b200`` with ``importlib`` (``spec_from_file_location`` on this file with
``submodule_search_locations`` set to this directory).
"""
from ._native import ArgumentError, DeviceError, DimensionMismatch, PlanError, lib  # noqa: F401
from .hafnian import (  # noqa: F401
    B200Backend,
    download_plan,
    dp_batch_bytes,
    empty_gpu_cache,
    gpu_cache_bytes,
    hafnian,
    hafnian_repeated,
    hafnian_repeated_batch,
    hafnian_submatrices,
    reduction,
    sieve,
    upload_plan,
)
from .policy import DP_HARD_MAX, DP_MAX, UNROLL_MAX, matched_reps  # noqa: F401

__version__ = "0.1.0"
