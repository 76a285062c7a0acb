"""Batches of hafnian_repeated(A_b, rpt_b) prepared on the device (egg_sieve_repeated_batch).

The device forms each instance's matched_reps (src/hafnian.jl:142-188), the sieve variant of the
reference's cost model (:855-884, :974-976) and the permuted matrix (:786-792).  The host path forms
the same three with the mirrored policy (policy.py) and hands them to egg_sieve_batch.  Both then
run the same kernels on the same matrices, so the results must be identical to the last bit, in
both arithmetic forms; the exact form is also checked against the oracle.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def rel(a, b):
    return abs(complex(a) - complex(b)) / max(abs(complex(b)), 1e-300)


def host_prepared(egg, orc, mats, rpts, T, prec, glynn=None):
    from theeggman_b200.hafnian import _sieve_device_batch

    Axs, ers, gs = [], [], []
    for A, r in zip(mats, rpts):
        x, er = orc.matched_reps(r)
        g = orc.choose_method(sum(r), er, 1)[1] if glynn is None else glynn
        Axs.append(orc.permuted(np.asarray(A, dtype=T), x))
        ers.append(list(er))
        gs.append(bool(g))
    return _sieve_device_batch(T, Axs, ers, gs, prec), Axs, ers, gs


@pytest.mark.parametrize("which", ["a", "b"])
@pytest.mark.parametrize("prec", ["exact", "fma"])
def test_device_preparation_equals_host_preparation(egg, orc, W, which, prec):
    if which == "a":
        mats, rpts = W.repeated_real(256, 14, 5)
        T = np.dtype(np.float64)
    else:
        mats, rpts = W.repeated_complex(32 if prec == "exact" else 128, 20, 48, 6)
        T = np.dtype(np.complex128)
    host, Axs, ers, gs = host_prepared(egg, orc, mats, rpts, T, prec)
    dev = egg.hafnian_repeated_batch(mats, rpts, prec=prec)
    assert np.array_equal(dev, host)
    if prec == "exact":
        for b in range(0, len(mats), max(1, len(mats) // 8)):
            dd = orc.calc_hafnian(Axs[b], ers[b], gs[b], nthreads=16, sum_mode=1)
            assert abs(complex(dev[b]) - complex(dd)) <= 1e-15 * abs(complex(dd)), b


def test_totals_variants_and_refusals(egg, orc, W):
    A = W.dense_real(6, 77)
    mats = [A] * 5
    rpts = [[0] * 6, [1, 0, 0, 0, 0, 0], [2, 2, 0, 1, 1, 0], [1, 1, 1, 1, 1, 1], [3, 1, 2, 0, 0, 2]]
    got = egg.hafnian_repeated_batch(mats, rpts)
    assert got[0] == 1.0 and got[1] == 0.0  # an empty pattern is 1, an odd total 0 (src/hafnian.jl:1201-1203)
    for b in (2, 3, 4):
        # A batch sums its terms in another fixed order than a single call: the same to 1e-15.
        assert rel(got[b], egg.hafnian_repeated(A, rpts[b], method="sieve")) <= 1e-15, b
    # A forced variant, both ways, as host preparation with that variant.
    for glynn in (False, True):
        host, *_ = host_prepared(egg, orc, mats[2:], rpts[2:], np.dtype(np.float64), None, glynn=glynn)
        assert np.array_equal(egg.hafnian_repeated_batch(mats[2:], rpts[2:], glynn=glynn), host), glynn
    # One matrix shared by every pattern: hafnian_repeated(A, rpts) sends its sieve patterns
    # through the same entry point with stride 0.
    pats = [[2, 2, 0, 1, 1, 0], [3, 1, 2, 0, 0, 0], [1, 1, 1, 1, 1, 1]]  # one total, as the reference requires
    shared = egg.hafnian_repeated(A, pats, method="sieve")
    for v, p in zip(shared, pats):
        assert rel(v, egg.hafnian_repeated(A, p, method="sieve")) <= 1e-15, p
    # 64 rows whose matching needs 33 edges: refused before any sieve runs.
    r33 = [1, 3, 3, 3, 3, 2, 2, 3, 1, 1, 3, 1, 3, 3, 1, 1, 3, 2, 1, 3, 1, 1, 1, 2, 1, 2, 1, 2, 1, 3, 1, 2, 2, 1, 1, 1,
           2, 3, 1, 3, 2, 3, 3, 2, 2, 3, 2, 2, 2, 1, 1, 2, 2, 2, 2, 1, 2, 1, 2, 3, 3, 1, 3, 2]
    assert len(orc.matched_reps(r33)[1]) == 33
    with pytest.raises(egg.ArgumentError):
        egg.hafnian_repeated_batch([W.dense_real(64, 5)], [r33])
    with pytest.raises(egg.ArgumentError):
        egg.hafnian_repeated_batch([A], [[-1, 1, 0, 0, 0, 0]])
