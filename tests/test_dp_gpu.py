"""Device subset DP through the C ABI, against the oracle.

EGG_PREC_EXACT must be bit-identical to the reference's CPU DP (src/dp.jl:344-363); EGG_PREC_FMA
within the reference GPU tolerance rtol=1e-12 (test/gpu.jl:12-24); Int64 inputs bit-exact in Int128.
Plans built on the device must equal the reference layout (src/dp.jl:223-304) entry for entry.
"""
import math

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def rel(a, b):
    return abs(complex(a) - complex(b)) / max(abs(complex(b)), 1e-300)


@pytest.fixture(scope="module")
def nat(egg):
    from theeggman_b200 import _native

    assert _native.lib().egg_init(0) == 0, "no CUDA device"
    return _native


def run_dp(egg, nat, P, K, dtype, prec="exact", max_batch=0, ib=None):
    """egg_dp_batch on a B x npairs instance-fastest P (the _haf_dp_backend contract)."""
    from theeggman_b200.hafnian import _dp_plan

    key = _dp_plan(K, ib)
    B = P.shape[0]
    Pf = np.asfortranarray(P)
    if dtype == nat.EGG_I64:
        out = np.zeros(2 * B, np.uint64)
    else:
        out = np.zeros(B, Pf.dtype)
    nat.check(nat.lib().egg_dp_batch(key[0], key[1], dtype, nat.PREC[prec], nat.ptr(Pf), B, max_batch, nat.ptr(out)))
    if dtype == nat.EGG_I64:
        vals = []
        for b in range(B):
            v = int(out[2 * b]) | (int(out[2 * b + 1]) << 64)
            vals.append(v - (1 << 128) if v >= (1 << 127) else v)
        return vals
    return out


def pairs_of(orc, A, K):
    return orc.gather_pairs(A, list(range(1, K + 1)), K)


@pytest.mark.parametrize("K", [2, 4, 6, 8, 10, 12, 16, 20, 24, 28])
def test_device_plan_equals_reference_layout(egg, nat, orc, K):
    for ib in ((4, 8) if K <= 24 else (4,)):
        from theeggman_b200.hafnian import _dp_plan

        _dp_plan(K, ib)
        st, tr, lv = egg.download_plan(K, ib)
        ref = orc.build_plan(K, ib)
        assert np.array_equal(st, ref.starts), (K, ib)
        assert np.array_equal(tr, ref.trans), (K, ib)
        assert np.array_equal(lv, ref.levels), (K, ib)


def test_uploaded_plan_is_validated(egg, nat, orc):
    egg.empty_gpu_cache()
    ref = orc.build_plan(12, 4)
    egg.upload_plan(12, 4, ref.starts, ref.trans, ref.levels)
    ref14 = orc.build_plan(14, 4)
    bad = ref14.trans.copy()
    bad[len(bad) // 2] = (np.int32(ref14.nstates + 5) << 9) | 1  # a child outside its level
    with pytest.raises(egg.PlanError):
        egg.upload_plan(14, 4, ref14.starts, bad, ref14.levels)
    bad = ref14.trans.copy()
    bad[7] = (bad[7] >> 9) << 9  # pair index 0
    with pytest.raises(egg.PlanError):
        egg.upload_plan(14, 4, ref14.starts, bad, ref14.levels)
    egg.empty_gpu_cache()


def _plan_device_bytes(nat, K, ib):
    import ctypes

    ns, nt, nl, db = (ctypes.c_int64() for _ in range(4))
    nat.check(nat.lib().egg_plan_info(K, ib, ctypes.byref(ns), ctypes.byref(nt), ctypes.byref(nl), ctypes.byref(db)))
    return db.value


def _reversed_plan(orc, K, ib):
    """The reference plan with each state's transitions in reverse order: still a valid plan (same
    children, same pairs), but summed in another order."""
    ref = orc.build_plan(K, ib)
    tr = ref.trans.copy()
    lv = ref.levels
    for L in range(1, len(lv) - 1):
        lo, hi = lv[L] - 1, lv[L + 1] - 1
        t0, t1 = ref.starts[lo] - 1, ref.starts[hi] - 1
        deg = (t1 - t0) // (hi - lo)
        tr[t0:t1] = tr[t0:t1].reshape(hi - lo, deg)[:, ::-1].ravel()
    return orc.Plan(K, ib, ref.nstates, ref.starts, tr, ref.levels)


@pytest.mark.parametrize("K", [14, 26])
def test_uploaded_plans_closed_form_or_explicit(egg, nat, orc, W, K):
    # The reference layout is recognised and evaluated without its array; any other valid plan
    # keeps its array and is summed in its own transition order.
    A = W.dense_real(K, 4400 + K)
    P = pairs_of(orc, A, K)[None, :]
    egg.empty_gpu_cache()
    ref = orc.build_plan(K, 4)
    egg.upload_plan(K, 4, ref.starts, ref.trans, ref.levels)
    assert _plan_device_bytes(nat, K, 4) == 0
    got = run_dp(egg, nat, P, K, nat.EGG_F64)[0]
    assert got == orc.haf_dp_pairs(P[0], ref, orc.F64)
    egg.empty_gpu_cache()
    rev = _reversed_plan(orc, K, 4)
    egg.upload_plan(K, 4, rev.starts, rev.trans, rev.levels)
    assert _plan_device_bytes(nat, K, 4) == rev.trans.nbytes
    got_rev = run_dp(egg, nat, P, K, nat.EGG_F64)[0]
    assert got_rev == orc.haf_dp_pairs(P[0], rev, orc.F64)
    assert rel(got_rev, got) < 1e-12
    egg.empty_gpu_cache()


@pytest.mark.parametrize("kind", ["f64", "c128", "f32", "c64"])
def test_exact_mode_bit_identical(egg, nat, orc, W, kind):
    dt = {"f64": np.float64, "c128": np.complex128, "f32": np.float32, "c64": np.complex64}[kind]
    code = {"f64": nat.EGG_F64, "c128": nat.EGG_C128, "f32": nat.EGG_F32, "c64": nat.EGG_C64}[kind]
    for K in (2, 4, 6, 8, 10, 12, 14, 16, 18, 20, 22, 24):
        Ps = []
        for b in range(3):
            A = (W.dense_complex(K, 7000 + 10 * K + b, 0.5) if kind[0] == "c" else W.dense_real(K, 7000 + 10 * K + b)).astype(dt)
            Ps.append(pairs_of(orc, A, K))
        P = np.stack(Ps)
        got = run_dp(egg, nat, P, K, code)
        plan = orc.build_plan(K, 4)
        for b in range(3):
            exp = orc.haf_dp_pairs(P[b], plan, {"f64": orc.F64, "c128": orc.C128, "f32": orc.F32, "c64": orc.C64}[kind])
            assert got[b] == exp, (K, b, got[b], exp)
        one = run_dp(egg, nat, P[:1], K, code)
        assert one[0] == got[0]


def test_exact_mode_n32_int32_and_int64_layouts(egg, nat, orc, W):
    K = 32
    A = W.dense_real(K, 3232)
    P = pairs_of(orc, A, K)[None, :]
    exp = orc.haf_dp_pairs(P[0], orc.build_plan(K, 4), orc.F64)
    assert run_dp(egg, nat, P, K, nat.EGG_F64)[0] == exp
    assert run_dp(egg, nat, P, K, nat.EGG_F64, ib=8)[0] == exp  # test/runtests.jl:269-281, v32 === v64


def test_fma_mode_within_gpu_tolerance(egg, nat, orc, W):
    for K in (14, 16, 20, 24):
        A = W.dense_complex(K, 101 + K, 0.5)
        P = pairs_of(orc, A, K)[None, :]
        exp = orc.haf_dp_pairs(P[0], orc.build_plan(K, 4), orc.C128)
        assert rel(run_dp(egg, nat, P, K, nat.EGG_C128, "fma")[0], exp) < 1e-12
        R = W.dense_real(K, 201 + K)
        P = pairs_of(orc, R, K)[None, :]
        exp = orc.haf_dp_pairs(P[0], orc.build_plan(K, 4), orc.F64)
        assert rel(run_dp(egg, nat, P, K, nat.EGG_F64, "fma")[0], exp) < 1e-12


def test_mixed_mode_error_stated(egg, nat, orc, W):
    """FP32 multiplies, FP64 accumulation: error stays near FP32 epsilon (cf. test/gpu.jl:58-69)."""
    for K in (12, 16, 20, 24):
        A = W.dense_complex(K, 301 + K, 0.5)
        P = pairs_of(orc, A, K)[None, :]
        exp = orc.haf_dp_pairs(P[0], orc.build_plan(K, 4), orc.C128)
        assert rel(run_dp(egg, nat, P, K, nat.EGG_C128, "mixed")[0], exp) < 1e-5


def test_int128_exact(egg, nat, orc, W):
    for K in (4, 8, 12, 16, 20, 24):
        G = W.er_graph(K, 0.5, 40 + K)
        P = pairs_of(orc, G, K)[None, :]
        assert run_dp(egg, nat, P.astype(np.int64), K, nat.EGG_I64)[0] == orc.dp_int128(G)
        J = np.ones((K, K), dtype=np.int64)
        Pj = pairs_of(orc, J, K)[None, :]
        assert run_dp(egg, nat, Pj, K, nat.EGG_I64)[0] == math.prod(range(1, K, 2))  # (K-1)!!


def test_chunking_and_determinism(egg, nat, orc, W):
    # test/gpu.jl:26-40, :88-94: batched == scalar, invariant to max_batch, reproducible
    K = 16
    P = np.stack([pairs_of(orc, W.dense_complex(K, 900 + b, 0.5), K) for b in range(7)])
    full = run_dp(egg, nat, P, K, nat.EGG_C128)
    for mb in (1, 2, 3, 100):
        assert np.array_equal(run_dp(egg, nat, P, K, nat.EGG_C128, max_batch=mb), full)
    for b in range(7):
        assert run_dp(egg, nat, P[b:b + 1], K, nat.EGG_C128)[0] == full[b]
    assert np.array_equal(run_dp(egg, nat, P, K, nat.EGG_C128), full)


@pytest.mark.parametrize("K,B", [(24, 5), (26, 2100)])
def test_level_kernel_batches(egg, nat, orc, W, K, B):
    # Degrees past the one-CTA kernel, with a small batch and with more instances than one block's
    # chunk of (state, instance) pairs: every instance equals its own single-instance evaluation,
    # and the first few equal the reference loop.
    rng = np.random.default_rng(K * 1000 + B)
    npairs = K * (K - 1) // 2
    P = rng.uniform(-1.0, 1.0, size=(B, npairs))
    got = run_dp(egg, nat, P, K, nat.EGG_F64)
    plan = orc.build_plan(K, 4)
    for b in sorted({0, 1, B // 2, B - 1}):
        assert got[b] == run_dp(egg, nat, P[b:b + 1], K, nat.EGG_F64)[0], b
        assert got[b] == orc.haf_dp_pairs(np.ascontiguousarray(P[b]), plan, orc.F64), b


def test_small_calls_repeated(egg, orc, W):
    """Many small single-instance calls of a few shapes, through the page-locked staging buffer:
    every call must read its own matrix and match the reference's DP bit for bit, in two element
    types, and again after the cache is cleared."""
    for N in (12, 20):
        for rep in range(2):
            for i in range(5):
                A = W.dense_real(N, 9000 + 10 * N + i)
                assert egg.hafnian(A, method="dp") == orc.haf_dp(A), (N, i)
                C = W.dense_complex(N, 9100 + 10 * N + i, 0.5)
                assert complex(egg.hafnian(C, method="dp")) == complex(orc.haf_dp(C)), (N, i)
            egg.empty_gpu_cache()


def test_cache_accounting(egg, nat, W):
    # test/gpu.jl:96-108
    egg.empty_gpu_cache()
    assert egg.gpu_cache_bytes() == 0
    A = W.dense_complex(16, 107, 0.5)
    egg.hafnian(A, backend=egg.B200Backend())
    used = egg.gpu_cache_bytes()
    assert used > 0
    egg.hafnian(A, backend=egg.B200Backend())
    assert egg.gpu_cache_bytes() == used
    egg.empty_gpu_cache()
    assert egg.gpu_cache_bytes() == 0


def test_no_plan_is_an_error(egg, nat):
    egg.empty_gpu_cache()
    out = np.zeros(1)
    P = np.zeros(6)
    assert nat.lib().egg_dp_batch(4, 4, nat.EGG_F64, 0, nat.ptr(P), 1, 0, nat.ptr(out)) == nat.EGG_ERR_NO_PLAN


@pytest.mark.parametrize("K", [36, 40])
def test_large_dp_properties(egg, nat, W, K):
    """Full-size (Int64 plan resident in HBM) checks that need no CPU evaluation:
    (K-1)!! for the all-ones graph in Int128, a single perfect matching's product in FP64, and the
    homogeneity haf(c A) = c^(K/2) haf(A)."""
    from theeggman_b200.hafnian import _gather_pairs_batch

    idx = np.arange(K)[None, :]
    J = np.ones((K, K), dtype=np.int64)
    P = _gather_pairs_batch(np.int64, J, idx, K)
    assert run_dp(egg, nat, P, K, nat.EGG_I64)[0] == math.prod(range(1, K, 2))
    a = 1.0 + W.uniform(K, K // 2)
    M = np.zeros((K, K))
    for i in range(K // 2):
        M[2 * i, 2 * i + 1] = M[2 * i + 1, 2 * i] = a[i]
    P = _gather_pairs_batch(np.float64, M, idx, K)
    got = run_dp(egg, nat, P, K, nat.EGG_F64)[0]
    exp = 1.0
    for v in a[::-1]:  # the recursion forms a1*(a2*(...*(an*1)))
        exp = v * exp
    assert got == exp
    A = W.dense_real(K, 4040, 0.0, 1.0)
    P1 = _gather_pairs_batch(np.float64, A, idx, K)
    P2 = _gather_pairs_batch(np.float64, 2.0 * A, idx, K)
    v1 = run_dp(egg, nat, P1, K, nat.EGG_F64)[0]
    v2 = run_dp(egg, nat, P2, K, nat.EGG_F64)[0]
    assert v2 == v1 * 2.0 ** (K // 2)  # scaling by 2 is exact
    egg.empty_gpu_cache()
