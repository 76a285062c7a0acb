"""egg_sieve_device_noalloc: the sieve for callers that cannot let the library allocate device
memory (their GPU memory belongs to another allocator, or they must not allocate once running).

The test hands the entry point its own device buffers for the matrix and the result, calls it twice
in a row (the fixed scratch keeps the previous call's contents, which must not leak into the next
result), and checks each result against the allocating entry point egg_sieve_device within the
sieve tests' tolerance.  It runs last so that a failure here cannot hide any other test, and it
passes on its own in a fresh process as well as after the rest.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def rel(a, b):
    return abs(complex(a) - complex(b)) / max(abs(complex(b)), 1e-300)


@pytest.mark.parametrize("cplx", [False, True])
@pytest.mark.parametrize("prec", [0, 1])
def test_noalloc_sieve_matches_allocating_entry_point(egg, W, cplx, prec):
    import torch

    from theeggman_b200 import _native as nat

    L = nat.lib()
    assert L.egg_init(0) == 0, L.egg_last_error()
    dev = torch.device("cuda", 0)
    stream = torch.cuda.Stream(dev)
    for N, glynn in ((16, False), (20, True), (24, False)):
        E = N // 2
        A = W.dense_complex(N, 300 + N, 0.5) if cplx else W.dense_real(N, 300 + N)
        x = np.array([2 * i for i in range(E)] + [2 * i + 1 for i in range(E)])
        Ax = A[np.ix_(x, x)]
        dA = torch.from_numpy(np.ascontiguousarray(Ax.T)).to(dev)  # column-major bytes
        reps = np.ones(E, dtype=np.int64)
        dtype = nat.EGG_C128 if cplx else nat.EGG_F64
        ref = torch.zeros(2, dtype=torch.float64, device=dev)
        got = torch.zeros(2, dtype=torch.float64, device=dev)
        torch.cuda.synchronize()
        assert L.egg_sieve_device(dtype, prec, dA.data_ptr(), E, reps.ctypes.data, int(glynn), ref.data_ptr(),
                                  stream.cuda_stream) == 0, L.egg_last_error()
        stream.synchronize()
        expect = complex(ref[0].item(), ref[1].item()) if cplx else ref[0].item()
        for call in range(2):
            got.fill_(float("nan"))
            torch.cuda.synchronize()
            rc = L.egg_sieve_device_noalloc(dtype, prec, dA.data_ptr(), E, reps.ctypes.data, int(glynn),
                                            got.data_ptr(), stream.cuda_stream)
            assert rc == 0, L.egg_last_error()
            stream.synchronize()
            val = complex(got[0].item(), got[1].item()) if cplx else got[0].item()
            assert rel(val, expect) <= 1e-15, (N, glynn, call, val, expect)


@pytest.mark.parametrize("prec", [0, 1])
def test_noalloc_at_32_edges_allocates_nothing(egg, W, prec):
    """The largest edge count the entry point accepts (E = 32, a 64 x 64 matrix), kept cheap with
    only five nonzero multiplicities (32 terms); the library's own device buffers must not grow."""
    import torch

    from theeggman_b200 import _native as nat

    L = nat.lib()
    assert L.egg_init(0) == 0, L.egg_last_error()
    dev = torch.device("cuda", 0)
    stream = torch.cuda.Stream(dev)
    E = 32
    A = W.dense_real(2 * E, 4321)
    dA = torch.from_numpy(np.ascontiguousarray(A.T)).to(dev)
    reps = np.zeros(E, dtype=np.int64)
    reps[[0, 5, 11, 20, 31]] = 1
    ref = torch.zeros(1, dtype=torch.float64, device=dev)
    got = torch.zeros(1, dtype=torch.float64, device=dev)
    torch.cuda.synchronize()
    assert L.egg_sieve_device(nat.EGG_F64, prec, dA.data_ptr(), E, reps.ctypes.data, 0, ref.data_ptr(),
                              stream.cuda_stream) == 0, L.egg_last_error()
    stream.synchronize()
    # One call first: the first call on a device looks up the fixed array's address.
    assert L.egg_sieve_device_noalloc(nat.EGG_F64, prec, dA.data_ptr(), E, reps.ctypes.data, 0, got.data_ptr(),
                                      stream.cuda_stream) == 0, L.egg_last_error()
    stream.synchronize()
    held = L.egg_cache_bytes()
    for call in range(2):
        got.fill_(float("nan"))
        torch.cuda.synchronize()
        rc = L.egg_sieve_device_noalloc(nat.EGG_F64, prec, dA.data_ptr(), E, reps.ctypes.data, 0, got.data_ptr(),
                                        stream.cuda_stream)
        assert rc == 0, L.egg_last_error()
        stream.synchronize()
        assert rel(got[0].item(), ref[0].item()) <= 1e-15, (call, got[0].item(), ref[0].item())
    assert L.egg_cache_bytes() == held


def test_noalloc_rejects_bad_arguments(egg):
    from theeggman_b200 import _native as nat

    L = nat.lib()
    out = np.zeros(1)
    reps = np.ones(40, dtype=np.int64)
    assert L.egg_sieve_device_noalloc(nat.EGG_F64, 0, None, 40, reps.ctypes.data, 0, out.ctypes.data, None) \
        == nat.EGG_ERR_TOO_LARGE
    assert L.egg_sieve_device_noalloc(7, 0, None, 2, reps.ctypes.data, 0, out.ctypes.data, None) == nat.EGG_ERR_ARGUMENT
