"""The oracle, pinned before it is trusted: against the reference's literal known answers, its
tabulated plan sizes, its plan invariants (test/runtests.jl:241-267), and 256-bit gold computed
independently of any kernel here (tests/golden/make_golden.py)."""
import numpy as np
import pytest

from conftest import dec, dec_matrix


def rel(a, b):
    a, b = complex(a), complex(b)
    return abs(a - b) / max(abs(b), 1e-300)


def test_known_answers(orc, golden):
    for case in golden["known_answers"]:
        A = dec_matrix(case["A"]) if case["A"] else np.zeros((0, 0))
        exp = dec(case["expect"])
        assert orc.hafnian(A) == exp, case["name"]
        if A.shape[0]:
            assert orc.hafnian(A, method="sieve") == exp
            assert orc.hafnian(A, method="sieve", glynn=True) == exp
            assert orc.brute_hafnian(A) == exp


def test_known_repeated(orc, golden):
    for case in golden["known_repeated"]:
        A = dec_matrix(case["A"])
        exp = dec(case["expect"])
        got = orc.hafnian_repeated(A, case["rpt"])
        assert rel(got, exp) <= 1e-15 or got == exp, case["name"]


def test_integer_exact_28(orc):
    A = np.array([[0, 1, 2, 3], [1, 0, 4, 5], [2, 4, 0, 6], [3, 5, 6, 0]], dtype=np.int64)
    assert orc.dp_int128(A) == 28


def test_dp_transition_table(orc, golden):
    for K, nt in golden["dp_transitions"].items():
        if K.startswith("_"):
            continue
        assert orc.dp_counts(int(K))[1] == nt


def test_dp_max_is_packing_limit(orc):
    # test/runtests.jl:222-239
    ns, _ = orc.dp_counts(32)
    assert 32 * 31 // 2 <= (1 << 9) - 1
    assert ns <= (2**31 - 1) >> 9
    ns2, _ = orc.dp_counts(34)
    assert (34 * 33 // 2).bit_length() + ns2.bit_length() > 31


@pytest.mark.parametrize("K", [4, 8, 12, 16])
@pytest.mark.parametrize("ib", [4, 8])
def test_plan_invariants(orc, K, ib):
    # test/runtests.jl:241-267
    p = orc.build_plan(K, ib)
    ns, nt = orc.dp_counts(K)
    bits = 9 if ib == 4 else 12
    assert p.nstates == ns and len(p.trans) == nt
    assert p.starts[0] == 1 and p.starts[-1] == nt + 1
    assert np.all(np.diff(p.starts) >= 0)
    for s in range(2, ns + 1):
        ch = p.trans[p.starts[s - 1] - 1: p.starts[s] - 1] >> bits
        assert np.all(ch < s)
    assert p.starts[1] == 1
    assert p.starts[ns] - p.starts[ns - 1] == K - 1
    pairs = p.trans & ((1 << bits) - 1)
    assert pairs.min() >= 1 and pairs.max() <= K * (K - 1) // 2


def test_plan_refusals(orc):
    # test/runtests.jl:295-297
    with pytest.raises(ValueError):
        orc.build_plan(66, 8)
    with pytest.raises(ValueError):
        orc.build_plan(34, 4)


def test_golden_random(orc, golden):
    """DP to machine precision; Glynn < 1e-12; inclusion-exclusion < 1e-9 and never better than
    Glynn... per draw the reference asserts ei >= eg only at N = 16..24, so that is checked there."""
    for case in golden["random"]:
        A = dec_matrix(case["A"])
        g = dec(case["gold"])
        N = case["N"]
        assert rel(orc.hafnian(A, method="dp"), g) < 1e-13, (N, case["kind"])
        assert rel(orc.hafnian(A, method="sieve", glynn=True), g) < 1e-12, (N, case["kind"])
        assert rel(orc.hafnian(A, method="sieve", glynn=False), g) < 1e-9, (N, case["kind"])
        if N <= 10:
            assert rel(orc.brute_hafnian(A), g) < 1e-13


def test_golden_repeated(orc, golden):
    for case in golden["repeated"]:
        A = dec_matrix(case["A"])
        g = dec(case["gold"])
        rpt = case["rpt"]
        for method in ("auto", "dp", "sieve"):
            got = orc.hafnian_repeated(A, rpt, method=method)
            assert rel(got, g) < 1e-10, (rpt, method)


def test_dp_threads_exact(orc, W):
    # test/runtests.jl:300-310: the DP is === across thread counts
    for N in (16, 20, 24):
        A = W.dense_complex(N, 18 + N, 0.5)
        ref = orc.haf_dp(A, nthreads=1)
        for nt in (2, 3, 7):
            assert orc.haf_dp(A, nthreads=nt) == ref


def test_int32_int64_layouts_identical(orc, W):
    # test/runtests.jl:269-281: v32 === v64
    for K in (8, 12, 16):
        A = W.dense_complex(K, 25 + K, 0.5)
        assert orc.haf_dp(A, idx_bytes=4) == orc.haf_dp(A, idx_bytes=8)


def test_matched_reps_invariants(orc):
    # test/runtests.jl:425-438
    for rpt in ([1, 1], [2, 2], [3, 1], [4, 1, 1], [2, 4], [5, 3], [1, 2, 3, 2], [0, 2, 2], [6, 2], [8]):
        x, er = orc.matched_reps(rpt)
        E = len(er)
        assert len(x) == 2 * E
        counts = [0] * len(rpt)
        for i in range(E):
            counts[x[i] - 1] += er[i]
            counts[x[E + i] - 1] += er[i]
        assert counts == list(rpt)


def test_hessenberg_reductions_agree(orc, W):
    # test/runtests.jl:160-191
    for m in (4, 8, 12, 20):
        z = W.normal(13 + m, 2 * m * m).reshape(2, m, m)
        M0 = z[0] + 1j * z[1]
        cg = orc.charpoly_check(M0, householder=False)
        ch = orc.charpoly_check(M0, householder=True)
        assert np.allclose(cg, ch, rtol=1e-9, atol=0) or np.linalg.norm(cg - ch) <= 1e-9 * np.linalg.norm(ch)
        mu = np.linalg.eigvals(M0)
        poly = np.array([1.0 + 0j])
        for zz in mu:
            poly = np.concatenate([poly, [0j]]) + np.concatenate([[0j], -zz * poly])
        n = m // 2
        assert np.linalg.norm(cg - poly[: n + 1]) <= 1e-8 * np.linalg.norm(poly[: n + 1])


def test_sieve_default_is_inclusion_exclusion(orc, W):
    # test/runtests.jl:108-119
    A = W.dense_complex(12, 26, 0.5)
    assert orc.hafnian(A, method="sieve") == orc.hafnian(A, method="sieve", glynn=False)
    assert orc.hafnian(A, method="sieve") != orc.hafnian(A, method="sieve", glynn=True)
    R = W.dense_complex(8, 27, 0.5)
    assert orc.choose_method(16, orc.matched_reps([2] * 8)[1], 12)[1]
    assert orc.hafnian_repeated(R, [2] * 8, method="sieve") == orc.hafnian_repeated(R, [2] * 8, method="sieve", glynn=True)


def test_sieve_sum_modes_agree(orc, W):
    """The double-double sum the device uses and the reference's plain sum differ only by the plain
    sum's rounding."""
    A = W.dense_real(16, 77)
    x = [2 * i + 1 for i in range(8)] + [2 * i + 2 for i in range(8)]
    Ax = orc.permuted(A, x)
    for glynn in (False, True):
        a = orc.calc_hafnian(Ax, [1] * 8, glynn, sum_mode=0)
        b = orc.calc_hafnian(Ax, [1] * 8, glynn, sum_mode=1)
        terms = orc.sieve_terms(Ax, [1] * 8, glynn, 0, 2 ** (7 if glynn else 8))
        bound = 2 * len(terms) * np.finfo(float).eps * np.sum(np.abs(terms))
        assert abs(a - b) <= bound
