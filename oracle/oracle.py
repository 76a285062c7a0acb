"""CPU oracle for TheEggman.jl's subset DP and Bjorklund/Glynn sieve.

TEST INFRASTRUCTURE ONLY.  This module is the checker: only the tests, ``__graft_entry__.smoke()``
and the CPU-baseline leg of ``bench.py`` import it, and only to check or time the reference
algorithm.  The product library never calls it and has no CPU fallback.

The arithmetic lives in ``eggman_oracle.c`` (a line-by-line C restatement of ``src/dp.jl`` and
``src/hafnian.jl``, built with ``-ffp-contract=off`` so it rounds as Julia does).  This file adds:

* ctypes bindings for it;
* the reference's entry glue, ``hafnian`` / ``hafnian_repeated`` (src/hafnian.jl:1111-1147,
  :1194-1222), with the method and Glynn choice restated independently of the product's copy
  (src/hafnian.jl:826-1011, src/dp.jl:626-632, src/unrolled.jl:112-141), so that the product's
  policy mirror can be checked against it;
* 256-bit mpmath gold for small degrees (the reference uses ``Complex{BigFloat}`` at 256 bits,
  test/runtests.jl:123-133, :322-331).
"""
from __future__ import annotations

import ctypes
import os
import subprocess
from functools import lru_cache
from math import comb

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))


def _host_tag() -> str:
    """A short name for this host's CPU (model and feature flags): the oracle is compiled with
    -march=native, so a build made on one host must not be loaded on another."""
    import hashlib

    model, flags = "", ""
    try:
        with open("/proc/cpuinfo") as f:
            for line in f:
                if line.startswith("model name") and not model:
                    model = line.split(":", 1)[1].strip()
                elif line.startswith("flags") and not flags:
                    flags = line.split(":", 1)[1].strip()
                if model and flags:
                    break
    except OSError:
        pass
    return hashlib.sha1((model + "|" + flags).encode()).hexdigest()[:10]


_LIB_PATH = os.path.join(_HERE, "build", f"libeggoracle-{_host_tag()}.so")

F64, C128, F32, C64, I64, Q_F64, Q_C128 = 0, 1, 2, 3, 4, 5, 6

DP_MAX = 32          # src/dp.jl:96
DP_HARD_MAX = 64     # src/dp.jl:124
UNROLL_MAX = 12      # src/unrolled.jl:52
_DP_WEIGHT = 3       # src/dp.jl:590
_SIEVE_PARALLEL_CAP = 5  # src/hafnian.jl:968
_DP_PARALLEL_CAP = 4     # src/hafnian.jl:969


def build() -> str:
    """Compile the C oracle (idempotent)."""
    subprocess.run(["make", "-s", "-C", _HERE, "OUT=" + os.path.relpath(_LIB_PATH, _HERE)], check=True)
    return _LIB_PATH


@lru_cache(maxsize=1)
def lib() -> ctypes.CDLL:
    if not os.path.exists(_LIB_PATH):
        build()
    L = ctypes.CDLL(_LIB_PATH)
    vp, i64, i32 = ctypes.c_void_p, ctypes.c_int64, ctypes.c_int
    p64 = ctypes.POINTER(ctypes.c_int64)
    L.orc_dp_counts.argtypes = [i32, p64, p64]
    L.orc_build_plan.argtypes = [i32, i32, vp, vp, vp, p64]
    L.orc_haf_dp.argtypes = [i32, i32, vp, vp, vp, i64, i64, vp, i32, vp]
    L.orc_haf_dp_batch.argtypes = [i32, i32, vp, vp, vp, i64, i64, vp, i64, i64, i32, vp]
    L.orc_gather_pairs.argtypes = [i32, vp, i64, vp, i64, vp]
    L.orc_brute_hafnian.argtypes = [i32, vp, i64, vp]
    L.orc_matched_reps.argtypes = [vp, i64, vp, vp, p64]
    L.orc_sieve_variant_cost.argtypes = [vp, i32, i64, i32, p64, p64]
    L.orc_calc_hafnian.argtypes = [i32, vp, vp, i32, i32, i32, i32, vp]
    L.orc_sieve_terms.argtypes = [i32, vp, vp, i32, i32, i64, i64, vp]
    L.orc_charpoly_check.argtypes = [i32, vp, i32, vp]
    L.orc_max_threads.restype = i32
    L.orc_closed_trans.argtypes = [i32, i32, vp]
    L.orc_haf_dp_closed.argtypes = [i32, i32, vp, i32, vp]
    return L


def _ptr(a: np.ndarray) -> int:
    return a.ctypes.data


# ----------------------------------------------------------------------------------------------
# DP
# ----------------------------------------------------------------------------------------------

def pair_index(i: int, j: int, K: int) -> int:
    """_pair_index(i, j, K), src/unrolled.jl:60 (1-based, i < j)."""
    return (i - 1) * K - (i * (i + 1)) // 2 + j


def dp_counts(K: int) -> tuple[int, int]:
    """_dp_counts(K), src/dp.jl:192-208."""
    a, b = ctypes.c_int64(), ctypes.c_int64()
    lib().orc_dp_counts(K, ctypes.byref(a), ctypes.byref(b))
    return a.value, b.value


class Plan:
    """HafnianDPPlan{I} (src/dp.jl:150-156): 1-based starts/trans/levels arrays."""

    def __init__(self, K, idx_bytes, nstates, starts, trans, levels):
        self.K, self.idx_bytes, self.nstates = K, idx_bytes, nstates
        self.starts, self.trans, self.levels = starts, trans, levels


@lru_cache(maxsize=16)
def build_plan(K: int, idx_bytes: int = 0) -> Plan:
    """_build_dp_plan(K, I), src/dp.jl:223-304 (refusals raise ValueError)."""
    if idx_bytes == 0:
        idx_bytes = 4 if K <= DP_MAX else 8
    if K > DP_HARD_MAX:
        raise ValueError(f"degree {K} exceeds DP_HARD_MAX = {DP_HARD_MAX}")
    ns, nt = dp_counts(K)
    bits = 9 if idx_bytes == 4 else 12
    imax = 2**31 - 1 if idx_bytes == 4 else 2**63 - 1
    if K * (K - 1) // 2 > (1 << bits) - 1 or ns > (imax >> bits) or nt > imax:
        raise ValueError(f"degree {K} cannot be packed into a {8 * idx_bytes}-bit transition")
    dt = np.int32 if idx_bytes == 4 else np.int64
    starts = np.zeros(ns + 1, dtype=dt)
    trans = np.zeros(max(nt, 1), dtype=dt)
    levels = np.zeros(K // 2 + 3, dtype=dt)
    nl = ctypes.c_int64()
    rc = lib().orc_build_plan(K, idx_bytes, _ptr(starts), _ptr(trans), _ptr(levels), ctypes.byref(nl))
    if rc != 0:
        raise ValueError(f"degree {K} cannot be laid out in a {8 * idx_bytes}-bit plan (rc={rc})")
    return Plan(K, idx_bytes, ns, starts, trans[:nt], levels[: nl.value])


_NP_OF = {F64: np.float64, C128: np.complex128, F32: np.float32, C64: np.complex64, I64: np.int64}


def haf_dp_pairs(P: np.ndarray, plan: Plan, dtype: int, nthreads: int = 1):
    """_haf_dp's forward pass given gathered pairs P (src/dp.jl:408-442)."""
    out = np.zeros(2, dtype=np.float64) if dtype in (F64, F32, C64, C128) else None
    if dtype == F64:
        out = np.zeros(1, np.float64)
    elif dtype == C128:
        out = np.zeros(1, np.complex128)
    elif dtype == F32:
        out = np.zeros(1, np.float32)
    elif dtype == C64:
        out = np.zeros(1, np.complex64)
    else:
        out = np.zeros(4, np.uint64)  # up to 32 bytes (int128 / float128 / complex float128)
    src = {Q_F64: np.float64, Q_C128: np.complex128}.get(dtype, _NP_OF.get(dtype))
    P = np.ascontiguousarray(P, dtype=src)
    rc = lib().orc_haf_dp(dtype, plan.idx_bytes, _ptr(plan.starts), _ptr(plan.trans), _ptr(plan.levels),
                          len(plan.levels), plan.nstates, _ptr(P), nthreads, _ptr(out))
    if rc != 0:
        raise RuntimeError(f"orc_haf_dp failed rc={rc}")
    if dtype == I64:
        lo, hi = int(out[0]), int(out[1])
        v = lo | (hi << 64)
        return v - (1 << 128) if v >= (1 << 127) else v
    if dtype in (Q_F64, Q_C128):
        return out  # raw bytes; callers use quad_to_mpf
    return out[0]


def closed_trans(K: int, idx_bytes: int) -> np.ndarray:
    """The transitions of the degree-K plan as the closed-form walk lists them (orc_closed_trans),
    in the layout of build_plan's `trans`: the tests compare the two entry for entry."""
    ns, nt = dp_counts(K)
    out = np.zeros(max(nt, 1), dtype=np.int32 if idx_bytes == 4 else np.int64)
    if lib().orc_closed_trans(K, idx_bytes, _ptr(out)) != 0:
        raise ValueError(f"no closed-form plan for degree {K}")
    return out[:nt]


def haf_dp_closed(P: np.ndarray, K: int, dtype: int, nthreads: int = 1):
    """_haf_dp's forward pass (src/dp.jl:408-442) on the closed form of the degree-K plan, no stored
    transitions: the reference's states, transitions and per-state order, for degrees whose plan
    does not fit in host memory.  dtype F64, C128, I64 (Int128 states; returns a Python int) or
    Q_F64 (raw bytes)."""
    src = {F64: np.float64, C128: np.complex128, I64: np.int64, Q_F64: np.float64}[dtype]
    P = np.ascontiguousarray(P, dtype=src)
    out = np.zeros(4, np.uint64)
    rc = lib().orc_haf_dp_closed(dtype, K, _ptr(P), int(nthreads), _ptr(out))
    if rc != 0:
        raise RuntimeError(f"orc_haf_dp_closed failed rc={rc}")
    if dtype == F64:
        return out.view(np.float64)[0]
    if dtype == C128:
        return out.view(np.complex128)[0]
    if dtype == I64:
        v = int(out[0]) | (int(out[1]) << 64)
        return v - (1 << 128) if v >= (1 << 127) else v
    return out


def gather_pairs(A: np.ndarray, idx, K: int) -> np.ndarray:
    """_gather_pairs!(P, A, idx, K), src/dp.jl:452-462, with idx 1-based."""
    npairs = K * (K - 1) // 2
    P = np.empty(npairs, dtype=A.dtype)
    for i in range(1, K):
        for j in range(i + 1, K + 1):
            P[pair_index(i, j, K) - 1] = A[idx[i - 1] - 1, idx[j - 1] - 1]
    return P


def haf_dp(A: np.ndarray, idx=None, nthreads: int = 1, dtype: int | None = None, idx_bytes: int = 0):
    """_haf_dp(A, idx, plan; nthreads), src/dp.jl:408-442."""
    K = len(idx) if idx is not None else A.shape[0]
    idx = list(range(1, K + 1)) if idx is None else list(idx)
    if dtype is None:
        dtype = {np.dtype(np.float64): F64, np.dtype(np.complex128): C128, np.dtype(np.float32): F32,
                 np.dtype(np.complex64): C64, np.dtype(np.int64): I64}[A.dtype]
    if K == 0:
        return A.dtype.type(1)
    plan = build_plan(K, idx_bytes)
    return haf_dp_pairs(gather_pairs(A, idx, K), plan, dtype, nthreads)


def haf_dp_batch(P: np.ndarray, plan: Plan, dtype: int, nthreads: int = 1) -> np.ndarray:
    """Threaded batch loop (src/hafnian.jl:1226-1242) over a B x npairs instance-fastest P."""
    B, npairs = P.shape
    Pf = np.asfortranarray(P, dtype=_NP_OF[dtype])
    out = np.zeros(B, dtype=_NP_OF[dtype]) if dtype != I64 else np.zeros(2 * B, np.uint64)
    rc = lib().orc_haf_dp_batch(dtype, plan.idx_bytes, _ptr(plan.starts), _ptr(plan.trans), _ptr(plan.levels),
                                len(plan.levels), plan.nstates, _ptr(Pf), B, npairs, nthreads, _ptr(out))
    if rc != 0:
        raise RuntimeError("orc_haf_dp_batch failed")
    if dtype == I64:
        vals = []
        for b in range(B):
            v = int(out[2 * b]) | (int(out[2 * b + 1]) << 64)
            vals.append(v - (1 << 128) if v >= (1 << 127) else v)
        return vals
    return out


def quad_to_float(raw: np.ndarray, cplx: bool):
    """Decode __float128 bytes into Python floats via mpmath (exact)."""
    import mpmath

    def one(b: bytes):
        u = int.from_bytes(b, "little")
        sign = -1 if u >> 127 else 1
        ex = (u >> 112) & 0x7FFF
        frac = u & ((1 << 112) - 1)
        if ex == 0:
            return mpmath.mpf(sign * frac) * mpmath.mpf(2) ** (-16382 - 112)
        return sign * mpmath.mpf((1 << 112) | frac) * mpmath.mpf(2) ** (ex - 16383 - 112)

    b = raw.tobytes()
    with mpmath.workprec(256):
        if cplx:
            return mpmath.mpc(one(b[0:16]), one(b[16:32]))
        return one(b[0:16])


def dp_gold(A: np.ndarray):
    """DP in __float128 (113-bit) on the same plan: gold for the FP64 error envelopes."""
    cplx = np.iscomplexobj(A)
    v = haf_dp(A.astype(np.complex128 if cplx else np.float64), dtype=Q_C128 if cplx else Q_F64)
    return quad_to_float(v, cplx)


def dp_int128(A: np.ndarray) -> int:
    """Exact integer DP (Int64 entries, Int128 state values)."""
    return haf_dp(np.asarray(A, dtype=np.int64), dtype=I64)


def brute_hafnian(A: np.ndarray):
    """brute_hafnian(A), test/runtests.jl:11-25."""
    N = A.shape[0]
    cplx = np.iscomplexobj(A)
    Af = np.asfortranarray(A, dtype=np.complex128 if cplx else np.float64)
    out = np.zeros(1, np.complex128 if cplx else np.float64)
    rc = lib().orc_brute_hafnian(C128 if cplx else F64, _ptr(Af), N, _ptr(out))
    if rc != 0:
        raise ValueError("brute force is limited to N <= 20")
    return out[0]


# ----------------------------------------------------------------------------------------------
# Sieve
# ----------------------------------------------------------------------------------------------

def matched_reps(rpt) -> tuple[list[int], list[int]]:
    """matched_reps(rpt), src/hafnian.jl:142-188 (1-based rows in x)."""
    r = np.ascontiguousarray(rpt, dtype=np.int64)
    N = len(r)
    x = np.zeros(2 * N + 2, np.int64)
    er = np.zeros(N + 1, np.int64)
    E = ctypes.c_int64()
    lib().orc_matched_reps(_ptr(r), N, _ptr(x), _ptr(er), ctypes.byref(E))
    E = E.value
    return [int(v) for v in x[: 2 * E]], [int(v) for v in er[:E]]


def sieve_variant_cost(edge_reps, n: int, glynn: bool) -> tuple[int, int]:
    e = np.ascontiguousarray(edge_reps, dtype=np.int64)
    w, s = ctypes.c_int64(), ctypes.c_int64()
    lib().orc_sieve_variant_cost(_ptr(e), len(e), n, int(glynn), ctypes.byref(w), ctypes.byref(s))
    return w.value, s.value


def permuted(A: np.ndarray, x) -> np.ndarray:
    """_permuted(T, A, x), src/hafnian.jl:786-792."""
    xi = np.asarray(x, dtype=np.int64) - 1
    return np.ascontiguousarray(A[np.ix_(xi, xi)])


def calc_hafnian(Ax: np.ndarray, edge_reps, glynn: bool, nthreads: int = 1, sum_mode: int = 0):
    """_calc_hafnian(Ax, edge_reps; nthreads, glynn), src/hafnian.jl:684-738.

    sum_mode 0 is the reference's own FP64 summation; sum_mode 1 sums every term in double-double.
    """
    cplx = np.iscomplexobj(Ax)
    Af = np.asfortranarray(Ax, dtype=np.complex128 if cplx else np.float64)
    e = np.ascontiguousarray(edge_reps, dtype=np.int64)
    out = np.zeros(2, np.float64)
    rc = lib().orc_calc_hafnian(int(cplx), _ptr(Af), _ptr(e), len(e), int(glynn), nthreads, sum_mode, _ptr(out))
    if rc != 0:
        raise RuntimeError("orc_calc_hafnian failed")
    return complex(out[0], out[1]) if cplx else float(out[0])


def sieve_terms(Ax: np.ndarray, edge_reps, glynn: bool, j0: int, cnt: int) -> np.ndarray:
    """Values of sieve terms j0..j0+cnt-1 (_glynn_term!, src/hafnian.jl:528-602)."""
    cplx = np.iscomplexobj(Ax)
    Af = np.asfortranarray(Ax, dtype=np.complex128 if cplx else np.float64)
    e = np.ascontiguousarray(edge_reps, dtype=np.int64)
    out = np.zeros(2 * cnt, np.float64)
    lib().orc_sieve_terms(int(cplx), _ptr(Af), _ptr(e), len(e), int(glynn), j0, cnt, _ptr(out))
    o = out.reshape(cnt, 2)
    return o[:, 0] + 1j * o[:, 1] if cplx else o[:, 0].copy()


def charpoly_check(M: np.ndarray, householder: bool) -> np.ndarray:
    m = M.shape[0]
    Mf = np.asfortranarray(M, dtype=np.complex128)
    out = np.zeros(m // 2 + 1, np.complex128)
    lib().orc_charpoly_check(int(householder), _ptr(Mf), m, _ptr(out))
    return out


# ----------------------------------------------------------------------------------------------
# Policy restatement (independent of the product's copy)
# ----------------------------------------------------------------------------------------------

@lru_cache(maxsize=None)
def unrolled_muls(K: int) -> int:
    """_unrolled_cost(K), src/unrolled.jl:112-133."""
    if K < 2:
        return 0
    seen = set()
    muls = 0
    stack = [(1 << K) - 1]
    while stack:
        mask = stack.pop()
        if mask in seen:
            continue
        seen.add(mask)
        i = (mask & -mask).bit_length()
        rest = mask & ~(1 << (i - 1))
        r = rest
        while r:
            j = (r & -r).bit_length()
            r &= ~(1 << (j - 1))
            sub = rest & ~(1 << (j - 1))
            if sub:
                muls += 1
                stack.append(sub)
    return muls


def _clamp_work(x: float) -> int:
    return (1 << 63) - 1 if x >= 9.0e18 else round(x)


def _term_cost(E: int, n: int) -> int:
    return (5 * (2 * E) ** 3) // 3 + 2 * E * n * n


def sieve_variant_cost_distinct(E: int, glynn: bool) -> tuple[int, int]:
    """src/hafnian.jl:889-900."""
    if E == 0:
        return 0, 0
    if glynn:
        steps = 2.0 ** (E - 1)
        return _clamp_work(steps * _term_cost(E, E)), _clamp_work(steps)
    work = 0.0
    for c in range(E + 1):
        work += comb(E, c) * float(_term_cost(c, E))
    return _clamp_work(work), _clamp_work(2.0 ** E)


def sieve_chunks(work: int, steps: int, nthreads: int) -> int:
    return 1 if work < 90_000 else min(nthreads, steps)


def decide(K, wg, sg, wi, si, E, n, nthreads):
    """_decide, src/hafnian.jl:974-983."""
    glynn = wg <= wi
    work, steps = (wg, sg) if glynn else (wi, si)
    parallel = sieve_chunks(work, steps, nthreads) > 1
    eff = work // max(1, min(nthreads, steps, _SIEVE_PARALLEL_CAP)) if parallel else work
    if K <= UNROLL_MAX and unrolled_muls(K) < eff:
        return "unrolled", glynn
    nt = nthreads if parallel else 1
    if K <= DP_MAX:
        _, ntrans = dp_counts(K)
        if (ntrans // max(1, min(nt, _DP_PARALLEL_CAP))) * _DP_WEIGHT < eff:
            return "dp", glynn
    return "sieve", glynn


def choose_method(K, edge_reps, nthreads):
    if len(edge_reps) == 0:
        return "sieve", False
    n = sum(edge_reps)
    wg, sg = sieve_variant_cost(edge_reps, n, True)
    wi, si = sieve_variant_cost(edge_reps, n, False)
    return decide(K, wg, sg, wi, si, len(edge_reps), n, nthreads)


def choose_method_distinct(K, E, nthreads):
    if E == 0:
        return "sieve", False
    wg, sg = sieve_variant_cost_distinct(E, True)
    wi, si = sieve_variant_cost_distinct(E, False)
    return decide(K, wg, sg, wi, si, E, E, nthreads)


# ----------------------------------------------------------------------------------------------
# Entry glue (the reference's public API, CPU path)
# ----------------------------------------------------------------------------------------------

def hafnian(A: np.ndarray, method: str = "auto", glynn=None, nthreads: int = 1):
    """hafnian(A; method, glynn, nthreads), src/hafnian.jl:1111-1147 (CPU path, no backend).

    The unrolled kernel evaluates the same recursion in the same order as the DP (a left fold of
    S[p] * h_sub with the partner ascending), so it is served by the DP here.
    """
    A = np.asarray(A)
    if A.dtype.kind in "iub":
        A = A.astype(np.float64)
    N = A.shape[0]
    if N == 0:
        return A.dtype.type(1)
    if N % 2:
        return A.dtype.type(0)
    E = N // 2
    sel, sg = choose_method_distinct(N, E, nthreads)
    chosen = sel if method == "auto" else method
    use_glynn = sg if glynn is None else glynn
    if chosen in ("unrolled", "dp"):
        return haf_dp(A, None, nthreads)
    x = [0] * N
    for i in range(1, E + 1):
        x[i - 1] = 2 * i - 1
        x[E + i - 1] = 2 * i
    return calc_hafnian(permuted(A, x), [1] * E, use_glynn, nthreads)


def hafnian_repeated(A: np.ndarray, rpt, method: str = "auto", glynn=None, nthreads: int = 1):
    """hafnian_repeated(A, rpt; ...), src/hafnian.jl:1194-1222 (CPU path)."""
    A = np.asarray(A)
    if A.dtype.kind in "iub":
        A = A.astype(np.float64)
    total = int(sum(rpt))
    if total == 0:
        return A.dtype.type(1)
    if total % 2:
        return A.dtype.type(0)
    x, edge_reps = matched_reps(rpt)
    sel, sg = choose_method(total, edge_reps, nthreads)
    chosen = sel if method == "auto" else method
    use_glynn = sg if glynn is None else glynn
    if chosen != "sieve":
        idx = [i + 1 for i in range(len(rpt)) for _ in range(int(rpt[i]))]
        return haf_dp(A, idx, nthreads)
    return calc_hafnian(permuted(A, x), edge_reps, use_glynn, nthreads)


def max_threads() -> int:
    return int(lib().orc_max_threads())


# ----------------------------------------------------------------------------------------------
# 256-bit gold by the DP recursion (mpmath), for small degrees
# ----------------------------------------------------------------------------------------------

def mp_hafnian(A: np.ndarray, prec: int = 256):
    """Hafnian by the memoised recursion in mpmath at `prec` bits (gold for N <= ~24)."""
    import mpmath

    N = A.shape[0]
    if N % 2:
        return 0
    with mpmath.workprec(prec):
        if np.iscomplexobj(A):
            M = [[mpmath.mpc(complex(A[i, j])) for j in range(N)] for i in range(N)]
        else:
            M = [[mpmath.mpf(float(A[i, j])) for j in range(N)] for i in range(N)]
        memo = {0: mpmath.mpf(1)}

        def rec(mask):
            v = memo.get(mask)
            if v is not None:
                return v
            i = (mask & -mask).bit_length() - 1
            rest = mask & ~(1 << i)
            s = mpmath.mpf(0)
            r = rest
            while r:
                j = (r & -r).bit_length() - 1
                r &= r - 1
                s += M[i][j] * rec(rest & ~(1 << j))
            memo[mask] = s
            return s

        # iterative-friendly: evaluate by increasing popcount to bound recursion depth
        return rec((1 << N) - 1)
