"""The C ABI without a GPU: the library loads, exports every symbol include/eggman_b200.h declares,
answers its pure-host queries, and fails loudly (no CPU fallback) where no device exists."""
import ctypes
import os
import re

import numpy as np
import pytest

from conftest import ROOT


def declared_symbols():
    src = open(os.path.join(ROOT, "include", "eggman_b200.h")).read()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    return sorted(set(re.findall(r"\b(egg_\w+)\s*\(", src)))


def test_library_exports_every_declared_symbol(egg):
    from theeggman_b200 import _native

    L = _native.lib()
    decl = declared_symbols()
    assert len(decl) >= 15
    for name in decl:
        assert hasattr(L, name), name
    assert sorted(_native.EXPORTS) == decl


def test_version_and_counts(egg, orc):
    from theeggman_b200 import _native

    L = _native.lib()
    assert b"sm_100a" in L.egg_version()
    ns, nt = ctypes.c_int64(), ctypes.c_int64()
    for K in range(0, 65, 2):
        assert L.egg_dp_counts(K, ctypes.byref(ns), ctypes.byref(nt)) == 0
        assert (ns.value, nt.value) == orc.dp_counts(K)
    assert L.egg_dp_counts(66, ctypes.byref(ns), ctypes.byref(nt)) == _native.EGG_ERR_ARGUMENT
    assert L.egg_dp_batch_bytes(20, _native.EGG_C128, 3) == 3 * (10946 + 190) * 16
    assert L.egg_dp_batch_bytes(20, 99, 3) == -1


def _has_device():
    from theeggman_b200 import _native

    return _native.lib().egg_init(0) == 0


def test_fails_loudly_without_a_device(egg, W):
    from theeggman_b200 import _native

    if _has_device():
        pytest.skip("a CUDA device is present")
    L = _native.lib()
    assert L.egg_init(0) == _native.EGG_ERR_NO_DEVICE
    assert L.egg_last_error()
    with pytest.raises(egg.DeviceError):
        egg.hafnian(W.dense_real(20, 1), method="dp")
    with pytest.raises(egg.DeviceError):
        egg.hafnian(W.dense_real(20, 1), method="sieve")
    out = np.zeros(1)
    A = np.eye(2)
    reps = np.ones(1, np.int64)
    assert L.egg_sieve(0, 0, A.ctypes.data, 1, reps.ctypes.data, 0, out.ctypes.data) == _native.EGG_ERR_NO_DEVICE
