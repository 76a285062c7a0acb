"""Device Bjorklund/Glynn sieve through the C ABI, against the oracle.

Each term is computed in the reference's order and rounding, and the terms are summed in
double-double, so the device result is compared with the oracle summing the same terms in
double-double (sum_mode 1): the bar is 1e-13 relative (the north-star sieve tolerance; in practice
the two agree to a few ulps).  Against the reference's own plain FP64 summation the difference is
bounded by that summation's rounding, and against 256-bit gold the reference's envelopes hold
(Glynn < 1e-12, inclusion-exclusion < 1e-9, test/runtests.jl:123-133).
"""
import numpy as np
import pytest

from conftest import dec, dec_matrix

pytestmark = pytest.mark.gpu


def rel(a, b):
    return abs(complex(a) - complex(b)) / max(abs(complex(b)), 1e-300)


def distinct_x(E):
    return [2 * i + 1 for i in range(E)] + [2 * i + 2 for i in range(E)]


@pytest.mark.parametrize("cplx", [False, True])
@pytest.mark.parametrize("glynn", [False, True])
def test_sieve_matches_oracle(egg, orc, W, cplx, glynn):
    for N in (2, 4, 6, 8, 10, 12, 14, 16, 18, 20, 22, 24):
        A = W.dense_complex(N, 60 + N, 0.5) if cplx else W.dense_real(N, 60 + N)
        E = N // 2
        Ax = orc.permuted(A, distinct_x(E))
        dd = orc.calc_hafnian(Ax, [1] * E, glynn, sum_mode=1)
        got = egg.sieve(Ax, [1] * E, glynn=glynn)
        assert rel(got, dd) <= 1e-13, (N, got, dd)
        plain = orc.calc_hafnian(Ax, [1] * E, glynn, sum_mode=0)
        steps = 2 ** (E - 1) if glynn else 2 ** E
        terms = orc.sieve_terms(Ax, [1] * E, glynn, 0, min(steps, 4096))
        if steps <= 4096:
            bound = 4 * steps * np.finfo(float).eps * np.sum(np.abs(terms)) * (0.5 ** (E - 1) if glynn else 1)
            assert abs(complex(got) - complex(plain)) <= bound + 1e-300


def test_sieve_golden_envelopes(egg, golden):
    for case in golden["random"]:
        A = dec_matrix(case["A"])
        g = dec(case["gold"])
        eg = rel(egg.hafnian(A, method="sieve", glynn=True), g)
        ei = rel(egg.hafnian(A, method="sieve", glynn=False), g)
        assert eg < 1e-12 and ei < 1e-9, (case["N"], case["kind"], eg, ei)


def test_repeated_rows_mixed_radix(egg, orc, golden):
    for case in golden["repeated"]:
        A = dec_matrix(case["A"])
        g = dec(case["gold"])
        rpt = case["rpt"]
        x, er = orc.matched_reps(rpt)
        Ax = orc.permuted(A, x)
        for glynn in (False, True):
            dd = orc.calc_hafnian(Ax, er, glynn, sum_mode=1)
            got = egg.sieve(Ax, er, glynn=glynn)
            assert rel(got, dd) <= 1e-13, (rpt, glynn)
            assert rel(got, g) < 1e-10, (rpt, glynn)
        assert rel(egg.hafnian_repeated(A, rpt, method="sieve"), g) < 1e-10


def test_edge_cases(egg, orc, W):
    A = W.dense_complex(4, 10, 0.5)
    assert egg.sieve(np.zeros((0, 0)), []) == 1
    assert egg.hafnian_repeated(A, [2, 0, 0, 0], method="sieve") == pytest.approx(A[0, 0], rel=1e-15)
    assert egg.hafnian(np.zeros((8, 8)), method="sieve") == 0
    assert egg.hafnian(np.zeros((8, 8)), method="sieve", glynn=True) == 0
    # large multiplicities and single-row patterns (test/runtests.jl:210-219)
    for rpt in ([7, 7, 7, 7], [12], [10, 2], [9, 3], [6, 2, 2, 2]):
        d = len(rpt)
        B = W.dense_complex(d, 99 + d, 0.5)
        x, er = orc.matched_reps(rpt)
        Bx = orc.permuted(B, x)
        for glynn in (False, True):
            assert rel(egg.sieve(Bx, er, glynn=glynn), orc.calc_hafnian(Bx, er, glynn, sum_mode=1)) <= 1e-13


def test_known_answers(egg, golden):
    for case in golden["known_answers"]:
        if not case["A"]:
            continue
        A = dec_matrix(case["A"])
        for glynn in (False, True):
            assert egg.hafnian(A, method="sieve", glynn=glynn) == dec(case["expect"])
    for case in golden["known_repeated"]:
        A = dec_matrix(case["A"])
        assert rel(egg.hafnian_repeated(A, case["rpt"], method="sieve"), dec(case["expect"])) <= 1e-15 or \
            egg.hafnian_repeated(A, case["rpt"], method="sieve") == dec(case["expect"])


def test_batch_equals_scalar(egg, orc, W):
    """One egg_sieve_batch call over instances of different edge counts and variants gives each
    instance's scalar result."""
    from theeggman_b200.hafnian import _sieve_device_batch

    mats, rpts = W.repeated_complex(12, d=10, total_max=24, seed=31)
    Axs, reps, gs = [], [], []
    for i, (A, r) in enumerate(zip(mats, rpts)):
        x, er = orc.matched_reps(r)
        Axs.append(orc.permuted(A, x))
        reps.append(er)
        gs.append(i % 2 == 0)
    vals = _sieve_device_batch(np.dtype(np.complex128), Axs, reps, gs)
    for Ax, er, g, v in zip(Axs, reps, gs, vals):
        assert rel(v, egg.sieve(Ax, er, glynn=g)) <= 1e-15
        assert rel(v, orc.calc_hafnian(Ax, er, g, sum_mode=1)) <= 1e-13


def test_config2_full_size_cross_check(egg, W):
    """N = 40 (E = 20, 2^20 inclusion-exclusion terms / 2^19 Glynn terms): the two variants agree,
    and both agree with the device DP (machine-precision, no cancellation) within the reference's
    envelopes."""
    A = W.dense_real(40, 2024, scale=1.0 / np.sqrt(40))
    ie = egg.hafnian(A, method="sieve", glynn=False)
    gl = egg.hafnian(A, method="sieve", glynn=True)
    dp = egg.hafnian(A, method="dp")
    assert rel(gl, dp) < 1e-12
    assert rel(ie, dp) < 1e-9
    egg.empty_gpu_cache()
