"""Host-side logic of the mirror (no GPU): strategy choice, matched_reps, validation and error
behaviour, checked against the reference's own regression expectations (test/runtests.jl:334-412,
:425-438, :520-587; test/gpu.jl:110-119, :149-154) and against the oracle's independent
restatement of the same policy."""
import numpy as np
import pytest


@pytest.fixture(scope="module")
def pol(egg):
    from theeggman_b200 import policy

    return policy


def test_method_selection(pol):
    # test/runtests.jl:334-344
    assert pol._choose_method(8, [1] * 4, 12)[0] == "unrolled"
    assert pol._choose_method(12, [1] * 6, 12)[0] == "unrolled"
    assert pol._choose_method(20, [1] * 10, 12)[0] == "dp"
    assert pol._choose_method(28, [1] * 14, 12)[0] == "dp"
    assert pol._choose_method(32, [1] * 16, 12)[0] == "dp"
    assert pol._choose_method(34, [1] * 17, 12)[0] == "sieve"
    assert pol._choose_method(28, pol.matched_reps([2] * 14)[1], 12)[0] == "sieve"
    assert pol._choose_method(16, pol.matched_reps([2] * 8)[1], 12)[0] == "dp"
    assert pol._choose_method(16, pol.matched_reps([2] * 8)[1], 12)[1] is True  # :117


def test_choice_thread_independent(pol):
    # test/runtests.jl:354-372
    for N in range(14, pol.DP_MAX + 1, 2):
        picks = [pol._choose_method_distinct(N, N // 2, nt)[0] for nt in (1, 2, 4, 8, 12, 32, 128, 1024)]
        assert all(p == picks[0] for p in picks) and picks[0] == "dp"
    for rpt in ([2] * 10, [2] * 14, [3] * 6, [4] * 6, [7, 7, 7, 7]):
        er = pol.matched_reps(rpt)[1]
        picks = [pol._choose_method(sum(rpt), er, nt)[0] for nt in (1, 12, 32, 128)]
        assert all(p == picks[0] for p in picks) and picks[0] == "sieve"


def test_backend_steering(pol):
    # test/runtests.jl:374-393 (the warning has no counterpart: the sieve runs on the device here)
    for nt in (1, 12, 32):
        for N in (16, 20, 28, pol.DP_MAX):
            assert pol._steer_backend(pol._choose_method_distinct(N, N // 2, nt)[0], "b", N, "auto") == "dp"
        for N in range(2, pol.UNROLL_MAX + 1, 2):
            assert pol._steer_backend(pol._choose_method_distinct(N, N // 2, nt)[0], "b", N, "auto") == "unrolled"
    assert pol._steer_backend("sieve", "b", 36, "auto") == "sieve"
    assert pol._steer_backend("sieve", None, 36, "auto") == "sieve"
    assert pol._steer_backend("unrolled", None, 8, "auto") == "unrolled"


def test_unrolled_crossover(pol):
    # test/runtests.jl:395-412
    def bestwork(er):
        return min(pol._sieve_variant_cost(er, sum(er), True)[0], pol._sieve_variant_cost(er, sum(er), False)[0])

    assert not pol._prefer_unrolled(12, bestwork(pol.matched_reps([6, 6])[1]))
    assert pol._prefer_unrolled(12, bestwork(pol.matched_reps([5, 5, 1, 1])[1]))
    for N in range(2, pol.UNROLL_MAX + 1, 2):
        assert pol._prefer_unrolled(N, bestwork([1] * (N // 2)))
    assert not pol._prefer_unrolled(pol.UNROLL_MAX + 2, 2**63 - 1)


def test_unrolled_muls_readme(pol):
    # README.md: "232 subsets, 1055 multiplies at N = 12"
    assert pol._unrolled_muls(12) == 1055


def test_dp_counts_and_limits(pol, orc):
    for K in range(0, 65, 2):
        assert pol._dp_counts(K) == orc.dp_counts(K)
    assert pol._dp_index_bytes(pol.DP_MAX) == 4 and pol._dp_index_bytes(pol.DP_MAX + 2) == 8
    for (nt, n, th) in ((10, 5, 12), (10**6, 3, 12), (10**6, 10**5, 12), (0, 1, 8)):
        c = pol._dp_level_chunks(nt, n, th)
        assert 1 <= c <= min(th, n)


def test_policy_matches_oracle(pol, orc, W):
    u = W.uniform(991, 4000)
    k = 0
    for trial in range(200):
        d = 2 + int(u[k] * 10); k += 1
        rpt = [int(u[k + i] * 5) for i in range(d)]
        k += d
        if sum(rpt) % 2:
            rpt[0] += 1
        x1, e1 = pol.matched_reps(rpt)
        x2, e2 = orc.matched_reps(rpt)
        assert (x1, e1) == (x2, e2), rpt
        if e1:
            for nt in (1, 12):
                assert pol._choose_method(sum(rpt), e1, nt) == orc.choose_method(sum(rpt), e1, nt)
                for g in (True, False):
                    assert pol._sieve_variant_cost(e1, sum(e1), g) == orc.sieve_variant_cost(e1, sum(e1), g)
    for N in range(2, 66, 2):
        for nt in (1, 12, 32):
            assert pol._choose_method_distinct(N, N // 2, nt) == orc.choose_method_distinct(N, N // 2, nt)


def test_check_method(pol, egg):
    with pytest.raises(egg.ArgumentError):
        pol._check_method("nonsense", 8)
    with pytest.raises(egg.ArgumentError):
        pol._check_method("unrolled", 14)
    pol._check_method("dp", pol.DP_HARD_MAX)
    with pytest.raises(egg.ArgumentError):
        pol._check_method("dp", pol.DP_HARD_MAX + 2)


def test_symmetry_tolerance(egg, W):
    # test/runtests.jl:520-542
    from theeggman_b200.hafnian import _check_symmetric

    for cplx in (False, True):
        A = W.dense_complex(6, 22, 0.5) if cplx else W.dense_real(6, 22)
        inside = A.copy()
        inside[1, 4] = A[4, 1] * (1 + np.sqrt(np.finfo(float).eps) / 8)
        _check_symmetric(inside)
        outside = A.copy()
        outside[1, 4] = A[4, 1] * (1 + 8 * np.sqrt(np.finfo(float).eps))
        with pytest.raises(egg.ArgumentError):
            _check_symmetric(outside)
    B = np.ones((4, 4))
    B[0, 1] = B[1, 0] = np.inf
    _check_symmetric(B)
    B[0, 1] = B[1, 0] = np.nan
    with pytest.raises(egg.ArgumentError):
        _check_symmetric(B)


def test_input_validation(egg, W):
    # test/runtests.jl:580-587, :346-351; test/gpu.jl:110-119 -- all raised before any device call
    A = W.dense_complex(4, 11, 0.5)
    with pytest.raises(egg.DimensionMismatch):
        egg.hafnian(np.random.default_rng(0).standard_normal((3, 4)))
    with pytest.raises(egg.ArgumentError):
        egg.hafnian(np.array([[1.0, 2.0], [3.0, 4.0]]))
    with pytest.raises(egg.DimensionMismatch):
        egg.hafnian_repeated(A, [1, 1, 1])
    with pytest.raises(egg.ArgumentError):
        egg.hafnian_repeated(A, [-1, 1, 1, 1])
    B16 = W.dense_complex(16, 16, 0.5)
    with pytest.raises(egg.ArgumentError):
        egg.hafnian(B16, method="unrolled")
    with pytest.raises(egg.ArgumentError):
        egg.hafnian(B16, method="nonsense")
    with pytest.raises(egg.ArgumentError):
        egg.hafnian(W.dense_complex(66, 17, 0.5), method="dp")
    A10 = W.dense_complex(10, 108, 0.5)
    with pytest.raises(egg.ArgumentError):
        egg.hafnian_repeated(A10, [[1] * 10, [1] * 9 + [0]])
    with pytest.raises(egg.ArgumentError):
        egg.hafnian_repeated(A10, [[1] * 10, [-1] + [1] * 9])
    with pytest.raises(egg.DimensionMismatch):
        egg.hafnian_repeated(A10, [[1] * 10, [1] * 9])
    with pytest.raises(egg.DimensionMismatch):
        egg.hafnian([A10, W.dense_complex(12, 1, 0.5)])
    bad = W.dense_complex(8, 23, 0.5)
    bad[0, 1] += 1
    with pytest.raises(egg.ArgumentError):
        egg.hafnian(bad)


def test_batch_symmetry_check_matches_per_matrix(egg, W):
    # A batch checks every matrix as hafnian(As[b]) would (src/hafnian.jl:1297-1300); the stacked
    # check raises the same error for the first offending matrix, as a list or as a 3-D array.
    from theeggman_b200.hafnian import _check_symmetric, _check_symmetric_stack

    mats = [W.dense_complex(8, 300 + b, 0.5) for b in range(6)]
    near = mats[1].copy()
    near[2, 5] = mats[1][5, 2] * (1 + np.sqrt(np.finfo(float).eps) / 8)  # inside the tolerance
    mats[1] = near
    _check_symmetric_stack(np.array(mats))
    bad3, bad4 = mats[3].copy(), mats[4].copy()
    bad3[6, 2] += 1
    bad4[0, 1] += 1
    mats[3], mats[4] = bad3, bad4
    with pytest.raises(egg.ArgumentError) as one:
        _check_symmetric(bad3)
    for batch in (mats, np.array(mats)):
        with pytest.raises(egg.ArgumentError) as got:
            egg.hafnian(batch)
        assert str(got.value) == str(one.value)
    nan = np.ones((3, 4, 4))
    nan[1, 2, 2] = np.nan  # the diagonal is not compared
    _check_symmetric_stack(nan)
    nan[2, 0, 3] = nan[2, 3, 0] = np.nan
    with pytest.raises(egg.ArgumentError):
        _check_symmetric_stack(nan)


def test_degenerate_sizes_need_no_device(egg, W):
    # N = 0 -> 1, odd -> 0, total 0 -> 1, odd total -> 0: no kernel is reached (src/hafnian.jl:1121-1122)
    assert egg.hafnian(np.zeros((0, 0))) == 1
    for N in (1, 3, 5, 7):
        assert egg.hafnian(W.dense_real(N, 2)) == 0
    A = W.dense_complex(4, 10, 0.5)
    assert egg.hafnian_repeated(A, [0, 0, 0, 0]) == 1
    assert egg.hafnian_repeated(A, [1, 0, 0, 0]) == 0


def test_dp_batch_bytes(egg, pol):
    # test/gpu.jl:149-154
    ns, _ = pol._dp_counts(20)
    assert egg.dp_batch_bytes(20, np.complex128, 1) == (ns + 190) * 16
    assert egg.dp_batch_bytes(20, np.complex64, 8) == 8 * (ns + 190) * 8


def test_permuted_distinct_is_permuted(egg, W):
    """The one-gather permutation of the distinct-row sieve equals _permuted(T, A, x) with
    x = [1, 3, ..., 2, 4, ...] (src/hafnian.jl:786-792, :1140-1145), entry for entry, for row- and
    column-major inputs that are not symmetric, and comes out column-major."""
    import importlib

    H = importlib.import_module("theeggman_b200.hafnian")
    for N in (2, 4, 20, 40):
        for dt in (np.float64, np.complex128, np.float32):
            A = np.asarray(W.dense_real(N, 5 + N), dtype=dt)
            A[0, 1] += 0.25
            want = H._permuted(np.dtype(dt), A, H._distinct_x(N // 2))
            for src in (A, np.asfortranarray(A)):
                got = H._permuted_distinct(np.dtype(dt), src)
                assert got.dtype == want.dtype and got.flags.f_contiguous
                assert np.array_equal(got, want)


def test_gather_pairs_one_is_pair_order(egg, W):
    """The single-matrix pair gather takes P[q] = A[i, j] for q = _pair_index(i, j, K) in the
    row-major upper triangle (src/unrolled.jl:60, src/dp.jl:452-477), for row- and column-major
    inputs that are not symmetric, in the requested element type."""
    import importlib

    H = importlib.import_module("theeggman_b200.hafnian")
    for K in (2, 4, 20, 33):
        A = np.asarray(W.dense_real(K, 70 + K))
        A[1, 0] += 0.5
        want = np.array([A[i, j] for i in range(K) for j in range(i + 1, K)])
        for src in (A, np.asfortranarray(A)):
            for T in (np.float64, np.complex128, np.float32):
                got = H._gather_pairs_one(np.dtype(T), src)
                assert got.shape == (1, K * (K - 1) // 2) and got.dtype == np.dtype(T)
                assert np.array_equal(got[0], want.astype(T))


def test_sieve_batch_pack_layout(egg, W):
    """The batched sieve's host packing: instance b's matrix column-major in the leading 2E_b block
    of slab[b], its multiplicities zero-padded, its variant as 0/1.  Checked against a plain
    element-by-element packing for one-size batches (whose stacking buffers are reused: two calls
    in a row with different matrices) and for mixed sizes, real and complex, with inputs that are
    not symmetric and of either memory order."""
    import importlib

    H = importlib.import_module("theeggman_b200.hafnian")
    rng = np.random.default_rng(11)

    def plain(CT, Axs, reps_list, glynns):
        B = len(Axs)
        Emax = max((len(r) for r in reps_list), default=0)
        lda = max(2 * Emax, 1)
        slab = np.zeros((B, lda, lda), CT)
        reps = np.zeros((B, max(Emax, 1)), np.int64)
        for b, (A, r) in enumerate(zip(Axs, reps_list)):
            m = 2 * len(r)
            for i in range(m):
                for j in range(m):
                    slab[b].reshape(-1)[i + j * lda] = A[i, j]  # column-major within the block
            reps[b, : len(r)] = r
        return slab, np.array([len(r) for r in reps_list], np.int64), reps, \
            np.array([1 if x else 0 for x in glynns], np.int32), Emax

    for CT in (np.float64, np.complex128):
        for sizes in ([3, 3, 3, 3], [3, 3, 3, 3], [1, 4, 2, 4, 0]):
            Axs, reps_list, glynns = [], [], []
            for k, E in enumerate(sizes):
                A = rng.standard_normal((2 * E, 2 * E)).astype(CT)
                if CT is np.complex128:
                    A = A + 1j * rng.standard_normal((2 * E, 2 * E))
                Axs.append(np.asfortranarray(A) if k % 2 else A)
                reps_list.append(list(rng.integers(1, 4, size=E)))
                glynns.append(bool(k % 2))
            got = H._sieve_batch_pack(CT, Axs, reps_list, glynns)
            want = plain(CT, Axs, reps_list, glynns)
            assert got[4] == want[4]
            for a, b in zip(got[:4], want[:4]):
                assert a.dtype == b.dtype and a.shape == b.shape and np.array_equal(a, b)


def test_gather_pairs_stack_equals_batch_gather(egg, W):
    """The all-rows pair gather of a (B, K, K) stack equals the general gather of
    _gather_pairs_batch (src/dp.jl:479-512) with every instance's rows in order, entry for entry,
    in the column-major layout (instance index fastest), for real, complex and integer inputs."""
    import importlib

    H = importlib.import_module("theeggman_b200.hafnian")
    rng = np.random.default_rng(5)
    for K in (2, 6, 20):
        for dt in (np.float64, np.complex128, np.int64):
            S = rng.integers(-9, 9, size=(7, K, K)).astype(dt)
            want = H._gather_pairs_batch(np.dtype(dt), S, np.tile(np.arange(K), (7, 1)), K)
            got = H._gather_pairs_stack(np.dtype(dt), S)
            assert got.dtype == want.dtype and got.flags.f_contiguous
            assert np.array_equal(got, want)


def test_repeated_batch_equal_patterns(egg, W, monkeypatch):
    """hafnian_repeated(A, rpts) evaluates each distinct pattern once and gives its value to every
    instance with that pattern, in order; distinct patterns keep the per-pattern strategy choice of
    the reference's loop (src/hafnian.jl:1355-1358).  The device calls are replaced by stand-ins
    whose value identifies the instance they were given, so the mapping is checked without a GPU."""
    import importlib

    H = importlib.import_module("theeggman_b200.hafnian")
    pol = importlib.import_module("theeggman_b200.policy")

    seen = []

    def fake_repeated(T, mats, stride, rpts, glynn, prec):
        # The device path of the sieve patterns: one shared matrix (stride 0), the raw patterns.
        assert stride == 0 and np.asarray(mats).ndim == 2
        seen.extend(tuple(r) for r in rpts)
        return np.array([float(np.sum(np.abs(mats))) * 1000 + 7 * sum(i * x for i, x in enumerate(r))
                         for r in rpts], dtype=T)

    def fake_dp(T, P, K, prec, max_batch, exact_int):
        seen.extend(range(np.asarray(P).shape[0]))
        return np.array([float(np.sum(np.abs(p))) for p in np.asarray(P)], dtype=T)

    monkeypatch.setattr(H, "_repeated_device", fake_repeated)
    monkeypatch.setattr(H, "_dp_device", fake_dp)
    A = W.dense_real(8, 17)
    pats = [[2, 2, 2, 2, 0, 0, 0, 0], [1, 1, 1, 1, 1, 1, 1, 1], [3, 1, 2, 0, 2, 0, 0, 0], [4, 4, 0, 0, 0, 0, 0, 0]]
    for method in ("auto", "sieve", "dp"):
        rpts = [pats[i] for i in (2, 0, 0, 3, 1, 2, 2, 0)]
        seen.clear()
        got = H.hafnian_repeated(A, rpts, method=method)
        assert len(seen) == len(pats)  # one evaluation per distinct pattern
        assert len(got) == len(rpts)
        for b, i in enumerate((2, 0, 0, 3, 1, 2, 2, 0)):
            want = H._hafnian_repeated_batch(A, [pats[i]], nthreads=None, glynn=None, method=method,
                                             check_symmetric=True, backend=None, max_batch=None, prec=None,
                                             exact=False)[0]
            assert got[b] == want, (method, b)
    assert pol.matched_reps([2, 2, 2, 2, 0, 0, 0, 0]) == tuple(map(list, H._pattern_choice((2, 2, 2, 2, 0, 0, 0, 0), 8)[:2]))


def test_scalar_sieve_marshalling(egg, W, monkeypatch):
    """A scalar sieve call hands the C ABI its matrix (column-major), its multiplicities (cached per
    pattern) and a result buffer (reused), and returns what the library writes there, in the
    input's type.  A stand-in for egg_sieve reads the arguments through their addresses and writes
    a value that depends on them, so the plumbing is checked without a GPU."""
    import ctypes
    import importlib

    H = importlib.import_module("theeggman_b200.hafnian")
    nat = importlib.import_module("theeggman_b200._native")

    class Stub:
        def egg_sieve(self, dtype, prec, ax, E, reps, glynn, out):
            r = np.ctypeslib.as_array((ctypes.c_int64 * max(E, 1)).from_address(reps))
            cplx = dtype == nat.EGG_C128
            n = 2 * E
            vals = np.ctypeslib.as_array((ctypes.c_double * (n * n * (2 if cplx else 1))).from_address(ax)) if E else []
            v = float(np.sum(r[:E]) * 1000 + np.sum(vals) + 7 * glynn)
            (ctypes.c_double * 2).from_address(out)[0] = v
            if cplx:
                (ctypes.c_double * 2).from_address(out)[1] = -v
            return 0

    monkeypatch.setattr(nat, "lib", lambda: Stub())
    for dt in (np.float64, np.complex128):
        for reps in ([1, 2, 3], [2, 2], [1, 2, 3]):
            E = len(reps)
            Ax = np.arange(4 * E * E, dtype=np.float64).reshape(2 * E, 2 * E).astype(dt)
            for glynn in (False, True):
                got = H._sieve_one(np.dtype(dt), Ax, reps, glynn)
                v = sum(reps) * 1000 + float(np.sum(Ax.view(np.float64))) + 7 * glynn
                want = complex(v, -v) if dt is np.complex128 else v
                assert type(got) is np.dtype(dt).type and got == want


def test_scalar_dp_marshalling(egg, W, monkeypatch):
    """A scalar DP call hands egg_dp_batch the pairs of _pair_index order with B = 1 and returns the
    value the library writes into the (reused) result buffer, in the input's type; exact integer
    calls read back a two's-complement Int128.  A stand-in for the library reads the pairs through
    their address, so the plumbing is checked without a GPU."""
    import ctypes
    import importlib

    H = importlib.import_module("theeggman_b200.hafnian")
    nat = importlib.import_module("theeggman_b200._native")
    monkeypatch.setattr(H, "_resident", set())

    class Stub:
        def egg_plan_build(self, K, ib):
            return 0

        def egg_dp_batch(self, K, ib, dtype, prec, P, B, max_batch, out):
            assert B == 1 and max_batch == 0
            npairs = K * (K - 1) // 2
            if dtype == nat.EGG_I64:
                p = np.ctypeslib.as_array((ctypes.c_int64 * npairs).from_address(P))
                v = -int(np.sum(p * np.arange(1, npairs + 1))) - (1 << 70)  # negative, beyond Int64
                u = v & ((1 << 128) - 1)
                o = (ctypes.c_uint64 * 2).from_address(out)
                o[0], o[1] = u & ((1 << 64) - 1), u >> 64
                return 0
            cplx = dtype == nat.EGG_C128
            p = np.ctypeslib.as_array((ctypes.c_double * (npairs * (2 if cplx else 1))).from_address(P))
            w = np.repeat(np.arange(1, npairs + 1), 2 if cplx else 1)
            o = (ctypes.c_double * 2).from_address(out)
            o[0] = float(np.sum(p * w)) + prec
            if cplx:
                o[1] = 1.0
            return 0

    monkeypatch.setattr(nat, "lib", lambda: Stub())
    A = np.arange(36, dtype=np.float64).reshape(6, 6)
    pairs = np.array([A[i, j] for i in range(6) for j in range(i + 1, 6)])
    w = np.arange(1, 16)
    for dt in (np.float64, np.complex128):
        got = egg.hafnian(A.astype(dt), method="dp", check_symmetric=False, prec="fma")
        want = float(np.sum(pairs * w)) + nat.PREC["fma"]
        assert type(got) is np.dtype(dt).type and got == (complex(want, 1.0) if dt is np.complex128 else want)
    got = egg.hafnian(A.astype(np.int64), method="dp", check_symmetric=False, exact=True)
    assert got == -int(np.sum(pairs.astype(np.int64) * w)) - (1 << 70)
