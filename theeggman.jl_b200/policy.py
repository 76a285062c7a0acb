"""Strategy and sieve-variant choice, mirrored from the reference so that the same inputs are routed
to the same algorithm (and therefore give the same numbers) as TheEggman.jl.

Every function here is host-side integer/float bookkeeping; none of it touches the device.
Sources: src/hafnian.jl:626-647, :826-1011; src/dp.jl:96-124, :192-208, :370-388, :590-632;
src/unrolled.jl:52, :112-141.
"""
from __future__ import annotations

from functools import lru_cache
from math import comb

DP_MAX = 32            # src/dp.jl:96
DP_HARD_MAX = 64       # src/dp.jl:124
UNROLL_MAX = 12        # src/unrolled.jl:52
_DP_WEIGHT = 3         # src/dp.jl:590
_SIEVE_PARALLEL_CAP = 5  # src/hafnian.jl:968
_DP_PARALLEL_CAP = 4     # src/hafnian.jl:969
_DP_CHUNK_WORK = 2_000   # src/dp.jl:370
_INT_MAX = (1 << 63) - 1


def _pair_index(i: int, j: int, K: int) -> int:
    """Flat index of (i < j) in the row-major upper triangle, 1-based (src/unrolled.jl:60)."""
    return (i - 1) * K - (i * (i + 1)) // 2 + j


def _pair_bits(idx_bytes: int) -> int:
    """Bits of a packed transition that hold the pair index (src/dp.jl:170-171)."""
    return 9 if idx_bytes == 4 else 12


def _dp_index_bytes(K: int) -> int:
    """Int32 layout through DP_MAX, Int64 above (src/dp.jl:180)."""
    return 4 if K <= DP_MAX else 8


@lru_cache(maxsize=None)
def _dp_counts(K: int) -> tuple[int, int]:
    """(nstates, ntransitions) of the degree-K plan, closed form (src/dp.jl:192-208)."""
    nstates, ntrans = 1, 0
    for p in range(1, K + 1):
        lo, hi = p - 1, min(2 * (p - 1), K - 1)
        r = lo if lo % 2 == 0 else lo + 1
        while r <= hi:
            k = K - r - 1
            c = comb(K - p, k)
            nstates += c
            ntrans += c * k
            r += 2
    return nstates, ntrans


def _dp_level_chunks(ntrans: int, nstates: int, nthreads: int) -> int:
    """src/dp.jl:387-388."""
    return max(1, min(ntrans // _DP_CHUNK_WORK, min(nthreads, nstates)))


@lru_cache(maxsize=None)
def _unrolled_muls(K: int) -> int:
    """Multiplications of the degree-K unrolled kernel (src/unrolled.jl:112-141)."""
    if K < 2:
        return 0
    seen: set[int] = set()
    muls = 0
    stack = [(1 << K) - 1]
    while stack:
        mask = stack.pop()
        if mask in seen:
            continue
        seen.add(mask)
        low = mask & -mask
        rest = mask & ~low
        r = rest
        while r:
            bit = r & -r
            r &= ~bit
            sub = rest & ~bit
            if sub:
                muls += 1
                stack.append(sub)
    return muls


def _term_cost(E: int, n: int) -> int:
    """Rough multiply-add count of one sieve term (src/hafnian.jl:626)."""
    return (5 * (2 * E) ** 3) // 3 + 2 * E * n * n


def _clamp_work(x: float) -> int:
    """src/hafnian.jl:832 (Julia's round is half-to-even, as is Python's)."""
    return _INT_MAX if x >= 9.0e18 else int(round(x))


def _sieve_chunks(work: int, steps: int, nthreads: int) -> int:
    """src/hafnian.jl:646-647."""
    return 1 if work < 90_000 else min(nthreads, steps)


def _sieve_variant_cost(edge_reps, n: int, glynn: bool) -> tuple[int, int]:
    """Exact multiply-add and term counts of one sieve variant (src/hafnian.jl:855-884)."""
    E = len(edge_reps)
    if E == 0:
        return 0, 0
    counts = [0.0] * (E + 1)
    counts[0] = 1.0
    for i in range(1, E + 1):
        r = int(edge_reps[i - 1])
        total = ((r + 2) // 2 if i == 1 else r + 1) if glynn else r + 1
        nzero = (1 if r % 2 == 0 else 0) if glynn else 1
        nkeep = total - nzero
        for c in range(i - 1, -1, -1):
            v = counts[c]
            if v == 0.0:
                continue
            counts[c] = v * nzero
            counts[c + 1] += v * nkeep
    work = 0.0
    steps = 0.0
    for c in range(E + 1):
        if counts[c] == 0.0:
            continue
        steps += counts[c]
        work += counts[c] * _term_cost(c, n)
    return _clamp_work(work), _clamp_work(steps)


def _sieve_variant_cost_distinct(E: int, glynn: bool) -> tuple[int, int]:
    """Closed form for all-ones multiplicities (src/hafnian.jl:889-900)."""
    if E == 0:
        return 0, 0
    if glynn:
        steps = 2.0 ** (E - 1)
        return _clamp_work(steps * _term_cost(E, E)), _clamp_work(steps)
    work = 0.0
    for c in range(E + 1):
        work += comb(E, c) * float(_term_cost(c, E))
    return _clamp_work(work), _clamp_work(2.0 ** E)


def _sieve_speedup(nthreads: int, steps: int) -> int:
    return max(1, min(nthreads, steps, _SIEVE_PARALLEL_CAP))


def _dp_speedup(nthreads: int) -> int:
    return max(1, min(nthreads, _DP_PARALLEL_CAP))


def _prefer_unrolled(K: int, sieve_work: int) -> bool:
    """src/hafnian.jl:827-828."""
    return K <= UNROLL_MAX and _unrolled_muls(K) < sieve_work


def _prefer_dp(K: int, sieve_effective: int, nthreads: int) -> bool:
    """src/dp.jl:626-632."""
    if K > DP_MAX:
        return False
    _, ntrans = _dp_counts(K)
    return (ntrans // _dp_speedup(nthreads)) * _DP_WEIGHT < sieve_effective


def _decide(K, wg, sg, wi, si, E, n, nthreads) -> tuple[str, bool]:
    """src/hafnian.jl:974-983."""
    glynn = wg <= wi
    work, steps = (wg, sg) if glynn else (wi, si)
    parallel = _sieve_chunks(work, steps, nthreads) > 1
    effective = work // _sieve_speedup(nthreads, steps) if parallel else work
    if _prefer_unrolled(K, effective):
        return "unrolled", glynn
    if _prefer_dp(K, effective, nthreads if parallel else 1):
        return "dp", glynn
    return "sieve", glynn


def _choose_method(K: int, edge_reps, nthreads: int) -> tuple[str, bool]:
    """(method, glynn) for total degree K with sieve multiplicities edge_reps (:937-943)."""
    if len(edge_reps) == 0:
        return "sieve", False
    n = int(sum(edge_reps))
    wg, sg = _sieve_variant_cost(edge_reps, n, True)
    wi, si = _sieve_variant_cost(edge_reps, n, False)
    return _decide(K, wg, sg, wi, si, len(edge_reps), n, nthreads)


@lru_cache(maxsize=None)
def _choose_method_distinct(K: int, E: int, nthreads: int) -> tuple[str, bool]:
    """As _choose_method for all-ones multiplicities (:951-956)."""
    if E == 0:
        return "sieve", False
    wg, sg = _sieve_variant_cost_distinct(E, True)
    wi, si = _sieve_variant_cost_distinct(E, False)
    return _decide(K, wg, sg, wi, si, E, E, nthreads)


def _steer_backend(chosen: str, backend, K: int, method: str) -> str:
    """Reconcile the CPU cost model's choice with a device backend (src/hafnian.jl:999-1011).

    The reference warns when a backend is passed but the sieve is chosen, because its sieve has no
    device path and silently ran on the CPU.  Here both strategies run on the device, so the
    steering is kept (it decides which numbers come back) and the warning is not needed.
    """
    if backend is None:
        return chosen
    if chosen == "unrolled":
        return chosen
    if method == "auto" and K <= DP_MAX:
        return "dp"
    return chosen


def _check_method(method: str, K: int) -> None:
    """src/hafnian.jl:1058-1066."""
    from ._native import ArgumentError

    if method not in ("auto", "unrolled", "dp", "sieve"):
        raise ArgumentError(f"method must be :auto, :unrolled, :dp or :sieve, got :{method}")
    if method == "unrolled" and K > UNROLL_MAX:
        raise ArgumentError(f"method=:unrolled needs degree ≤ {UNROLL_MAX}, got {K}")
    if method == "dp" and K > DP_HARD_MAX:
        raise ArgumentError(f"method=:dp needs degree ≤ {DP_HARD_MAX}, got {K}")


def matched_reps(rpt) -> tuple[list[int], list[int]]:
    """Pair repeated rows into as few distinct edges as possible (src/hafnian.jl:142-188).

    Returns (x, edge_reps): x has length 2E with position i matched to i + E (1-based rows), and
    edge_reps[i] is the multiplicity of edge i.  Ties follow the reference's (count, row)
    descending order.
    """
    v = [(int(c), i + 1) for i, c in enumerate(rpt) if int(c) > 0]
    edges_a: list[int] = []
    edges_b: list[int] = []
    edge_reps: list[int] = []
    if not v:
        return edges_a, edge_reps
    v.sort(reverse=True)
    while len(v) > 1 or (len(v) == 1 and v[0][0] > 1):
        v.sort(reverse=True)
        reps1, x1 = v[0]
        if len(v) == 1 or reps1 > 2 * v[1][0]:
            edges_a.append(x1)
            edges_b.append(x1)
            edge_reps.append(reps1 // 2)
            if reps1 % 2 == 0:
                v.pop(0)
            else:
                v[0] = (1, x1)
        else:
            reps2, x2 = v[1]
            edges_a.append(x1)
            edges_b.append(x2)
            edge_reps.append(reps2)
            if reps1 > reps2:
                v[0] = (reps1 - reps2, x1)
                del v[1]
            else:
                del v[0:2]
    return edges_a + edges_b, edge_reps
