"""Algorithmic work of the two hot paths, the numerators of the roofline fractions.

Sieve (FP64 pipe).  Per term with m = 2 x (surviving edges) and n = N/2, counting a fused
multiply-add as 2 flops and a complex one as 8:
  * M build                 m^2 multiplies                        (src/hafnian.jl:583-593)
  * Hessenberg reduction    sum_{k=2}^{m-1} (m-k)(m-k+1) row-update FMAs
                            + sum_{k=2}^{m-1} (m-k) m column-update FMAs   (:239-255; m=40: 49,400)
  * La Budde charpoly       its multiply-adds, truncated to n+1 coefficients (:454-492)
  * series coefficient      sum_{t=1}^{n} min(t, m) multiply-adds, plus one scaling multiply each (:502-514)
summed over the terms' exact distribution of m (the convolution of _sieve_variant_cost, :855-884).

DP (HBM).  Per batch sharing one plan: ntrans x sizeof(I) plan bytes streamed once, plus per instance
2 x nstates state values (written once, read once) and npairs gathered pairs, each sizeof(T).
"""
from __future__ import annotations

from functools import lru_cache

from . import policy as pol


@lru_cache(maxsize=None)
def hess_fmas(m: int) -> int:
    return sum((m - k) * (m - k + 1) + (m - k) * m for k in range(2, m))


@lru_cache(maxsize=None)
def labudde_macs(m: int, n: int) -> int:
    c = 0
    for k in range(1, m + 1):
        c += min(k, n)
        for i in range(k - 1, max(1, k - n + 1) - 1, -1):
            d = k - i + 1
            c += 2 + max(0, min(n, d + i - 1) - d + 1)
    return c


@lru_cache(maxsize=None)
def series_macs(m: int, n: int) -> int:
    return sum(min(t, m) for t in range(1, n + 1))


@lru_cache(maxsize=None)
def term_flops(m: int, n: int, cplx: bool) -> int:
    if m == 0:
        return 0
    f = 2 * hess_fmas(m) + 2 * labudde_macs(m, n) + 3 * series_macs(m, n) + m * m
    return 4 * f if cplx else f


def surviving_distribution(edge_reps, glynn: bool) -> list[float]:
    """counts[c] = number of sieve terms that keep c edges (src/hafnian.jl:859-874)."""
    E = len(edge_reps)
    counts = [0.0] * (E + 1)
    counts[0] = 1.0
    for i in range(1, E + 1):
        r = int(edge_reps[i - 1])
        total = ((r + 2) // 2 if i == 1 else r + 1) if glynn else r + 1
        nzero = (1 if r % 2 == 0 else 0) if glynn else 1
        nkeep = total - nzero
        for c in range(i - 1, -1, -1):
            v = counts[c]
            counts[c] = v * nzero
            counts[c + 1] += v * nkeep
    return counts


def sieve_flops(edge_reps, glynn: bool, cplx: bool) -> float:
    n = int(sum(edge_reps))
    counts = surviving_distribution(edge_reps, glynn)
    return float(sum(counts[c] * term_flops(2 * c, n, cplx) for c in range(len(counts))))


def dp_bytes(K: int, B: int, value_bytes: int) -> int:
    """Algorithmic bytes of a DP that streams an explicit plan: the transition array once, every
    state written once and read once, and the pairs."""
    nstates, ntrans = pol._dp_counts(K)
    idx = pol._dp_index_bytes(K)
    return ntrans * idx + B * (2 * nstates + K * (K - 1) // 2) * value_bytes


def dp_bytes_closed(K: int, B: int, value_bytes: int) -> int:
    """Compulsory bytes of a DP on a closed-form plan (no transition array): every state written
    once and read once, and the pairs."""
    nstates, _ = pol._dp_counts(K)
    return B * (2 * nstates + K * (K - 1) // 2) * value_bytes


def dp_gather_bytes(K: int, B: int, value_bytes: int) -> int:
    """Bytes of the child-value loads, one per transition (served mostly from L2 and L1)."""
    _, ntrans = pol._dp_counts(K)
    return B * ntrans * value_bytes


# Nominal FP64 peak: 148 SMs x 64 FP64 FMA lanes x 2 flops x clock.  MEASURED_PEAKS.json carries no
# FP64 figure, so the sieve's fraction is stated against this nominal value at the measured max clock.
def fp64_nominal_tflops(sm_max_mhz: float, sms: int = 148) -> float:
    return sms * 64 * 2 * sm_max_mhz * 1e6 / 1e12
