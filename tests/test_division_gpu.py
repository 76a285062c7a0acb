"""The reference-arithmetic sieve's division against correctly rounded division, bit for bit.

The reference divides each entry below the pivot by the pivot (`mult[i] = M[i, k-1] / x`,
src/hafnian.jl:235), an IEEE correctly rounded quotient.  The reference-arithmetic tiles form one
correctly rounded reciprocal per step and finish each quotient with Markstein's corrections, taking
the full division where an operand or the quotient leaves [2^-1000, 2^1000].  egg_selfcheck_division
runs that code on the device beside the device's own correctly rounded division; both must equal
numpy's IEEE quotient (NaN compared as NaN).
"""
import ctypes

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def run(egg, a, b):
    from theeggman_b200 import _native as N

    a = np.ascontiguousarray(a, dtype=np.float64)
    b = np.ascontiguousarray(b, dtype=np.float64)
    qs = np.empty_like(a)
    qr = np.empty_like(a)
    N.check(N.lib().egg_selfcheck_division(N.ptr(a), N.ptr(b), ctypes.c_int64(a.size), N.ptr(qs), N.ptr(qr)))
    return qs, qr


def assert_same(q, want, a, b, what):
    nan = np.isnan(want)
    assert np.array_equal(np.isnan(q), nan), what
    bad = np.flatnonzero(q[~nan].view(np.uint64) != want[~nan].view(np.uint64))
    if bad.size:
        i = np.flatnonzero(~nan)[bad[0]]
        raise AssertionError(f"{what}: {bad.size} mismatches; first a={a[i].hex()} b={b[i].hex()} "
                             f"got {q[i].hex()} want {want[i].hex()}")


def operands(seed):
    rng = np.random.default_rng(seed)
    parts = []
    n = 1 << 20
    # Random bit patterns: every exponent, subnormals, infinities and NaNs included.
    parts.append((rng.integers(0, 2**64, n, dtype=np.uint64).view(np.float64),
                  rng.integers(0, 2**64, n, dtype=np.uint64).view(np.float64)))
    # Log-uniform magnitudes across and beyond the range where the reciprocal is shared.
    def logu(k, lo, hi):
        return rng.choice([-1.0, 1.0], k) * np.ldexp(1.0 + rng.random(k), rng.integers(lo, hi, k))
    parts.append((logu(n, -1074, 1023), logu(n, -1074, 1023)))
    parts.append((logu(n, -1010, 1010), logu(n, -1010, 1010)))
    # The sieve's own operands: entries of U[-1,1]/sqrt(40) matrices and their updates.
    parts.append(((2 * rng.random(n) - 1) / np.sqrt(40.0), (2 * rng.random(n) - 1) / np.sqrt(40.0)))
    # Divisors and numerators next to the 2^-1000 and 2^1000 boundaries, and quotients next to 2^-1000.
    k = 1 << 16
    steps = rng.integers(-8, 9, k)
    edge_lo = np.nextafter(np.full(k, 2.0**-1000), np.where(steps < 0, 0.0, np.inf))
    edge_hi = np.nextafter(np.full(k, 2.0**1000), np.where(steps < 0, 0.0, np.inf))
    parts.append((logu(k, -4, 4), edge_lo * rng.choice([-1.0, 1.0], k)))
    parts.append((logu(k, -4, 4), edge_hi * rng.choice([-1.0, 1.0], k)))
    parts.append((edge_lo, logu(k, -4, 4)))
    parts.append((edge_hi, logu(k, -4, 4)))
    parts.append((logu(k, -1003, -996), logu(k, -4, 4)))
    # Quotients close to a rounding midpoint: b random, q with a 54th bit set, a = rn(b * q).
    m = 1 << 20
    bb = logu(m, -60, 60)
    q54 = np.ldexp(1.0 + (rng.integers(0, 2**52, m).astype(np.float64) + 0.5) / 2**52, rng.integers(-30, 30, m))
    parts.append((bb * q54, bb))
    # Exact quotients and signed specials.
    sp = np.array([0.0, -0.0, np.inf, -np.inf, np.nan, 1.0, -1.0, 5e-324, -5e-324, 2.0**-1022,
                   np.finfo(np.float64).max, 2.0**-1000, 2.0**1000, 3.0])
    A, B = np.meshgrid(sp, sp)
    parts.append((A.ravel(), B.ravel()))
    x = logu(k, -300, 300)
    parts.append((x, x))
    parts.append((x * 3.0, x))
    a = np.concatenate([p[0] for p in parts])
    b = np.concatenate([p[1] for p in parts])
    return a, b


def test_shared_reciprocal_division_is_correctly_rounded(egg):
    a, b = operands(20261204)
    qs, qr = run(egg, a, b)
    with np.errstate(all="ignore"):
        want = a / b
    assert_same(qr, want, a, b, "device correctly rounded division vs IEEE")
    assert_same(qs, want, a, b, "shared-reciprocal division vs IEEE")


def test_selfcheck_arguments(egg):
    from theeggman_b200 import _native as N

    z = np.zeros(1)
    assert N.lib().egg_selfcheck_division(N.ptr(z), N.ptr(z), ctypes.c_int64(0), N.ptr(z), N.ptr(z)) == N.EGG_OK
    with pytest.raises(egg.ArgumentError):
        N.check(N.lib().egg_selfcheck_division(N.ptr(z), N.ptr(z), ctypes.c_int64(-1), N.ptr(z), N.ptr(z)))
    with pytest.raises(egg.ArgumentError):
        N.check(N.lib().egg_selfcheck_division(None, N.ptr(z), ctypes.c_int64(1), N.ptr(z), N.ptr(z)))
