"""Pins the oracle's plan-free DP (orc_haf_dp_closed) to its stored-plan DP before the GPU parity
tests trust it at N = 36 and 40, where the stored plan (3.2 GB / 24 GB of transitions) is out of
reach.

The closed-form walk must list the same transitions as _build_dp_plan (src/dp.jl:223-304, restated
by orc_build_plan) entry for entry, and return the same bits as _haf_dp on the stored plan
(src/dp.jl:408-442) for every element type it supports, at any thread count.
"""
import numpy as np
import pytest


@pytest.mark.parametrize("K", [2, 4, 6, 8, 12, 16, 20, 24])
@pytest.mark.parametrize("idx_bytes", [4, 8])
def test_closed_form_lists_the_reference_plan(orc, K, idx_bytes):
    plan = orc.build_plan(K, idx_bytes)
    assert np.array_equal(orc.closed_trans(K, idx_bytes), plan.trans)


@pytest.mark.parametrize("K", [2, 4, 6, 10, 14, 18, 22, 26, 28])
def test_closed_form_values_are_bit_identical(orc, K):
    rng = np.random.default_rng(1000 + K)
    idx = list(range(1, K + 1))
    plan = orc.build_plan(K)
    A = rng.uniform(-1, 1, (K, K))
    A = A + A.T
    P = orc.gather_pairs(A, idx, K)
    ref = orc.haf_dp_pairs(P, plan, orc.F64, 4)
    for nt in (1, 3, 8):
        assert orc.haf_dp_closed(P, K, orc.F64, nt) == ref
    Z = rng.normal(size=(K, K)) + 1j * rng.normal(size=(K, K))
    Z = Z + Z.T
    Pz = orc.gather_pairs(Z, idx, K)
    assert orc.haf_dp_closed(Pz, K, orc.C128, 5) == orc.haf_dp_pairs(Pz, plan, orc.C128, 4)
    G = np.triu((rng.uniform(0, 1, (K, K)) < 0.5).astype(np.int64), 1)
    G = G + G.T
    Pg = orc.gather_pairs(G, idx, K)
    assert orc.haf_dp_closed(Pg, K, orc.I64, 7) == orc.haf_dp_pairs(Pg, plan, orc.I64, 4)


def test_closed_form_known_answers(orc):
    # haf(ones(K, K)) = (K-1)!! in exact Int128, including K = 36 where (K-1)!! > 2^63.
    for K in (8, 20, 36):
        P = np.ones(K * (K - 1) // 2, dtype=np.int64)
        want = 1
        for k in range(K - 1, 0, -2):
            want *= k
        assert orc.haf_dp_closed(P, K, orc.I64, 8) == want
    # The empty matrix has hafnian 1 (test/runtests.jl: hafnian(zeros(0, 0)) == 1).
    assert orc.haf_dp_closed(np.zeros(0), 0, orc.F64) == 1.0
