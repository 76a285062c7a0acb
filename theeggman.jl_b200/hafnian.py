"""Public API: the reference's `hafnian` / `hafnian_repeated` surface, served by the B200 engine.

This mirrors src/hafnian.jl:1111-1374 (entry points, validation, strategy routing) and the device
hook of src/dp.jl:514-587.  Validation and routing are host logic; every hafnian is computed on the
GPU by libeggman_b200 (the subset DP or the sieve), never on the CPU.

Differences from the reference, all additive:
  * `:unrolled` (straight-line CPU code for degree <= 12, src/unrolled.jl) is served by the device
    DP, which evaluates the same recursion in the same order and so returns the same bits;
  * `prec` picks the rounding: "exact" = the reference CPU's, term by term, for both the DP and
    the sieve; "fma" = fused multiply-adds (the reference GPU kernel's DP rounding, and the
    register-resident sieve kernels); "mixed" = FP32 multiplies with FP64 accumulation in the
    DP.  The default (None) is "exact" for both: every sieve term in the reference's arithmetic
    (bit-identical to _glynn_term!), summed in double-double;
  * `exact=True` runs integer matrices in Int64/Int128 instead of promoting them to Float64.
"""
from __future__ import annotations

import os
from functools import lru_cache
import threading

import numpy as np

from . import _native as nat
from . import policy as pol
from ._native import ArgumentError, DimensionMismatch

_lock = threading.RLock()
_resident: set[tuple[int, int]] = set()


class B200Backend:
    """Marker for the device backend (the reference's `backend` keyword takes a KA backend)."""

    def __init__(self, device: int = 0):
        self.device = device

    def __repr__(self):
        return f"B200Backend({self.device})"


_NTHREADS = os.cpu_count() or 1


def _default_nthreads() -> int:
    return _NTHREADS


# ----------------------------------------------------------------------------------------------
# Plans and caches (src/dp.jl:306-329, :536-587)
# ----------------------------------------------------------------------------------------------

def _dp_plan(K: int, idx_bytes: int | None = None) -> tuple[int, int]:
    """Make the degree-K plan resident on the device (built there, cached for the session).

    Returns the cache key (K, idx_bytes).  Mirrors _dp_plan (src/dp.jl:325-329) and
    _device_plan (ext/TheEggmanKernelAbstractionsExt.jl:31-42) in one step.
    """
    ib = pol._dp_index_bytes(K) if idx_bytes is None else idx_bytes
    key = (K, ib)
    if key in _resident:
        return key
    with _lock:
        if key not in _resident:
            nat.check(nat.lib().egg_plan_build(K, ib))
            _resident.add(key)
    return key


def upload_plan(K: int, idx_bytes: int, starts: np.ndarray, trans: np.ndarray, levels: np.ndarray) -> None:
    """Upload a host-built plan in the reference layout (what the Julia shim does with the
    HafnianDPPlan it built; src/dp.jl:150-156)."""
    dt = np.int32 if idx_bytes == 4 else np.int64
    st = np.ascontiguousarray(starts, dtype=dt)
    tr = np.ascontiguousarray(trans, dtype=dt)
    lv = np.ascontiguousarray(levels, dtype=dt)
    with _lock:
        nat.check(nat.lib().egg_plan_upload(K, idx_bytes, nat.ptr(st), nat.ptr(tr) if tr.size else None,
                                            nat.ptr(lv), lv.size, st.size - 1, tr.size))
        _resident.add((K, idx_bytes))


def download_plan(K: int, idx_bytes: int) -> tuple[np.ndarray, np.ndarray, np.ndarray]:
    """Copy a resident plan back in the reference layout (starts, trans, levels)."""
    import ctypes

    ns, nt, nl, _ = (ctypes.c_int64() for _ in range(4))
    nat.check(nat.lib().egg_plan_info(K, idx_bytes, ctypes.byref(ns), ctypes.byref(nt), ctypes.byref(nl), None))
    dt = np.int32 if idx_bytes == 4 else np.int64
    starts = np.zeros(ns.value + 1, dt)
    trans = np.zeros(max(nt.value, 1), dt)
    levels = np.zeros(nl.value, dt)
    nat.check(nat.lib().egg_plan_download(K, idx_bytes, nat.ptr(starts), nat.ptr(trans), nat.ptr(levels)))
    return starts, trans[: nt.value], levels


def gpu_cache_bytes() -> int:
    """Device memory held by resident plans and work buffers (src/dp.jl:552-560)."""
    return int(nat.lib().egg_cache_bytes())


def empty_gpu_cache() -> None:
    """Drop every resident plan and work buffer (src/dp.jl:567-573)."""
    with _lock:
        nat.check(nat.lib().egg_cache_clear())
        _resident.clear()


def dp_batch_bytes(N: int, T, B: int) -> int:
    """B x (nstates + npairs) x sizeof(T) (src/dp.jl:584-587): an upper bound on the device memory
    one batch needs besides the plan."""
    nstates, _ = pol._dp_counts(N)
    return B * (nstates + N * (N - 1) // 2) * np.dtype(T).itemsize


# ----------------------------------------------------------------------------------------------
# Validation (src/hafnian.jl:744-809)
# ----------------------------------------------------------------------------------------------

def _haf_dtype(A: np.ndarray) -> np.dtype:
    """float(eltype(A)) (src/hafnian.jl:744): integers and bools promote to Float64."""
    return _haf_dtype_of(A.dtype)


def _haf_dtype_of(dt: np.dtype) -> np.dtype:
    if dt.kind in "iub":
        return np.dtype(np.float64)
    if dt in (np.float16,):
        return np.dtype(np.float32)
    if dt not in (np.float64, np.float32, np.complex128, np.complex64):
        raise ArgumentError(f"unsupported element type {dt}")
    return dt


def _checksquare(A: np.ndarray) -> int:
    if A.ndim != 2 or A.shape[0] != A.shape[1]:
        raise DimensionMismatch(f"matrix is not square: dimensions are {A.shape}")
    return A.shape[0]


def _check_symmetric(A: np.ndarray) -> None:
    """Symmetric to isapprox's default tolerance, squared (src/hafnian.jl:765-779); reports the
    first offending (i, j) in the reference's column-major order over the upper triangle."""
    n = A.shape[0]
    if n < 2:
        return
    X = np.asarray(A)
    kind = X.dtype.kind
    neq = X != X.T  # comparisons raise no floating-point warnings
    if not neq.any():
        return
    real_t = np.float32 if X.dtype in (np.float32, np.complex64) else np.float64
    tol = float(np.finfo(real_t).eps)
    with np.errstate(invalid="ignore", over="ignore"):
        if kind in "iub":
            Xf = X.astype(np.float64)
        else:
            Xf = X
        d = Xf - Xf.T
        ad = (d * np.conj(d)).real if np.iscomplexobj(d) else d * d
        ax = (Xf * np.conj(Xf)).real if np.iscomplexobj(Xf) else Xf * Xf
        ok = ad <= tol * np.maximum(ax, ax.T)
        bad = neq & ~ok
    bad = np.triu(bad, 1)
    if bad.any():
        jj, ii = np.nonzero(bad.T)  # column-major scan: j outer, i inner
        raise ArgumentError(f"matrix is not symmetric at ({ii[0] + 1}, {jj[0] + 1})")


def _check_symmetric_stack(S: np.ndarray) -> None:
    """_check_symmetric for each matrix of a (B, N, N) stack in order: one comparison of the stack
    with its transpose when every matrix is exactly symmetric (the usual case); otherwise the
    per-matrix check, which reports the first matrix that is not symmetric to tolerance."""
    if S.shape[1] < 2:
        return
    if not (S != S.transpose(0, 2, 1)).any():
        return
    for m in S:
        _check_symmetric(m)


# ----------------------------------------------------------------------------------------------
# Device calls
# ----------------------------------------------------------------------------------------------

@lru_cache(maxsize=None)
def _triu_pairs(K: int) -> tuple[np.ndarray, np.ndarray]:
    """(i, j) 0-based for q = 1..K(K-1)/2 in _pair_index order (row-major upper triangle).
    Cached per degree; the arrays are read-only."""
    iu, ju = np.triu_indices(K, 1)
    iu.setflags(write=False)
    ju.setflags(write=False)
    return iu, ju


@lru_cache(maxsize=None)
def _triu_flat(K: int) -> np.ndarray:
    """Row-major flat indices i * K + j of the pairs, in _pair_index order.  Cached; read-only."""
    iu, ju = _triu_pairs(K)
    f = iu * K + ju
    f.setflags(write=False)
    return f


def _gather_pairs_one(T: np.dtype, A: np.ndarray) -> np.ndarray:
    """The 1 x npairs P of a single K x K matrix (the rows taken in order), as one gather."""
    return A.ravel().take(_triu_flat(A.shape[0])).astype(T, copy=False).reshape(1, -1)


def _gather_pairs_stack(T: np.dtype, stack: np.ndarray) -> np.ndarray:
    """P[b, q] = A_b[i, j] for q = _pair_index(i, j, K) of a C-contiguous (B, K, K) stack, every row
    taken in order, column-major (instance index fastest): one gather of the pairs' rows of the
    transposed stack."""
    B, K = stack.shape[0], stack.shape[1]
    return stack.reshape(B, K * K).T[_triu_flat(K)].T.astype(T, copy=False)


def _gather_pairs_batch(T: np.dtype, mats: np.ndarray, idxs: np.ndarray, K: int) -> np.ndarray:
    """P[b, q] = A_b[idx_b[i], idx_b[j]] for q = _pair_index(i, j, K), instance index fastest
    (src/dp.jl:479-512).  mats is (B, N, N) or (N, N) shared; idxs is (B, K) 0-based."""
    iu, ju = _triu_pairs(K)
    ri = idxs[:, iu]
    ci = idxs[:, ju]
    if mats.ndim == 2:
        P = mats[ri, ci]
    else:
        P = mats[np.arange(mats.shape[0])[:, None], ri, ci]
    return np.asfortranarray(P.astype(T, copy=False))


def _dp_device(T: np.dtype, P: np.ndarray, K: int, prec: str, max_batch, exact_int: bool):
    """The B200 replacement of _haf_dp_backend(backend, P, plan; max_batch)
    (ext/TheEggmanKernelAbstractionsExt.jl:90-146)."""
    B = P.shape[0]
    key = _dp_plan(K)
    dtype = nat.EGG_I64 if exact_int else nat.DTYPE_OF[np.dtype(T)]
    P = np.asfortranarray(P)
    if exact_int:
        out = np.zeros(2 * B, np.uint64)
    else:
        out = np.zeros(B, T)
    if prec not in nat.PREC:
        raise ArgumentError(f"prec must be one of {tuple(nat.PREC)}")
    with _lock:
        nat.check(nat.lib().egg_dp_batch(key[0], key[1], dtype, nat.PREC[prec], nat.ptr(P), B,
                                         int(max_batch or 0), nat.ptr(out)))
    if exact_int:
        vals = []
        for b in range(B):
            v = int(out[2 * b]) | (int(out[2 * b + 1]) << 64)
            vals.append(v - (1 << 128) if v >= (1 << 127) else v)
        return vals
    return out


def _dp_one(T: np.dtype, P: np.ndarray, K: int, prec: str, exact_int: bool):
    """One hafnian through egg_dp_batch (B = 1), as _dp_device(...)[0], with its value read from a
    reused result buffer."""
    key = _dp_plan(K)
    dtype = nat.EGG_I64 if exact_int else nat.DTYPE_OF[np.dtype(T)]
    if prec not in nat.PREC:
        raise ArgumentError(f"prec must be one of {tuple(nat.PREC)}")
    P = np.ascontiguousarray(P)  # 1 x npairs: both memory orders at once
    with _lock:
        out, out_ptr = _one_out(np.dtype(np.uint64), 2) if exact_int else _one_out(np.dtype(T))
        nat.check(nat.lib().egg_dp_batch(key[0], key[1], dtype, nat.PREC[prec], nat.ptr(P), 1, 0, out_ptr))
        if exact_int:
            v = int(out[0]) | (int(out[1]) << 64)
            return v - (1 << 128) if v >= (1 << 127) else v
        return out[0]


def _dp_prec(prec) -> str:
    """DP rounding: the reference CPU's (exact) unless asked otherwise.  'reference' is 'exact':
    the DP's sum order is fixed by its plan, so its exact kernels already reproduce the reference
    bit for bit."""
    return "exact" if prec in (None, "reference") else prec


def _sieve_prec(prec) -> int:
    """Sieve kernel: the reference's term arithmetic for prec None (the default), 'exact' and
    'reference' (which also sums in the reference's order); the fused-multiply-add register tiles for
    'fma' and 'mixed' (the sieve has no mixed form)."""
    if prec not in (None, "exact", "fma", "mixed", "reference"):
        raise ArgumentError("prec must be one of None, 'exact', 'fma', 'mixed', 'reference'")
    return nat.PREC["fma"] if prec in ("fma", "mixed") else nat.PREC["exact"]


# The last equal-size batch shape's stacking buffers, reused (under _lock) so that a batch does not
# pay for fresh pages on every call.
_slab_bufs: dict = {}


def _sieve_batch_pack(CT, Axs: list, reps_list: list, glynns: list):
    """(slab, E, reps, glynn, Emax) of one egg_sieve_batch call: slab[b] holds instance b's matrix
    column-major in its leading 2E_b x 2E_b block, reps[b] its multiplicities (zero-padded).  For
    a batch of one size the slab is a reused buffer: call under _lock and use it before releasing."""
    B = len(Axs)
    lens = list(map(len, reps_list))
    E = np.array(lens, dtype=np.int64)
    Emax = max(lens) if B else 0
    g = np.array([1 if x else 0 for x in glynns], dtype=np.int32)
    if B and Emax and min(lens) == Emax:
        # Every instance the same size (a batch of one pattern): one stack, one transposing copy.
        m = 2 * Emax
        key = (B, m, np.dtype(CT))
        bufs = _slab_bufs.get(key)
        if bufs is None:
            _slab_bufs.clear()
            bufs = (np.empty((B, m, m), CT), np.empty((B, m, m), CT))
            _slab_bufs[key] = bufs
        np.stack(Axs, out=bufs[0])
        np.copyto(bufs[1], bufs[0].transpose(0, 2, 1))
        return bufs[1], E, np.array(reps_list, dtype=np.int64).reshape(B, Emax), g, Emax
    lda = max(2 * Emax, 1)
    slab = np.zeros((B, lda, lda), dtype=CT)  # per instance: column-major leading block
    for b, (Ax, r) in enumerate(zip(Axs, reps_list)):
        m = 2 * len(r)
        if m:
            slab[b, :m, :m] = np.asarray(Ax, dtype=CT).T  # store transposed so memory is column-major
    reps = np.zeros((B, max(Emax, 1)), dtype=np.int64)
    for b, r in enumerate(reps_list):
        reps[b, : len(r)] = r
    return slab, E, reps, g, Emax


def _sieve_device_batch(T: np.dtype, Axs: list[np.ndarray], reps_list: list[list[int]], glynns: list[bool],
                        prec=None) -> np.ndarray:
    """One egg_sieve_batch call over instances of possibly different edge counts."""
    B = len(Axs)
    cplx = np.dtype(T).kind == "c"
    CT = np.complex128 if cplx else np.float64
    if prec == "reference":
        # The reference's batch loop runs each instance with nthreads = 1, i.e. one chunk
        # (src/hafnian.jl:1297-1300, :1355-1358).
        return np.array([_sieve_reference(T, Ax, list(r), bool(gl), 1) for Ax, r, gl in zip(Axs, reps_list, glynns)],
                        dtype=T)
    out = np.zeros(B, CT)
    with _lock:
        slab, E, reps, g, Emax = _sieve_batch_pack(CT, Axs, reps_list, glynns)
        nat.check(nat.lib().egg_sieve_batch(nat.EGG_C128 if cplx else nat.EGG_F64, _sieve_prec(prec), B, Emax, nat.ptr(slab),
                                            nat.ptr(E), nat.ptr(reps), nat.ptr(g), nat.ptr(out)))
    return out.astype(T, copy=False)


def _sieve_one(T: np.dtype, Ax: np.ndarray, edge_reps: list[int], glynn: bool, prec=None, nthreads: int = 1):
    """The device sieve in place of _calc_hafnian(Ax, edge_reps; nthreads, glynn)
    (src/hafnian.jl:684-738).  The sieve runs in FP64 (complex: ComplexF64); the result is
    returned in T.  `nthreads` matters only for prec='reference'."""
    if prec == "reference":
        return _sieve_reference(T, Ax, edge_reps, glynn, nthreads)
    cplx = np.dtype(T).kind == "c"
    CT = np.complex128 if cplx else np.float64
    E = len(edge_reps)
    A = np.asfortranarray(np.asarray(Ax, dtype=CT))
    reps_ptr = _reps_array(tuple(edge_reps))[1]
    with _lock:
        out, out_ptr = _one_out(CT)
        nat.check(nat.lib().egg_sieve(nat.EGG_C128 if cplx else nat.EGG_F64, _sieve_prec(prec), nat.ptr(A) if E else None, E,
                                      reps_ptr, 1 if glynn else 0, out_ptr))
        v = out[0]
    return np.dtype(T).type(v)


@lru_cache(maxsize=256)
def _reps_array(reps: tuple):
    """(array, address) of a multiplicity pattern as the C ABI takes it (Int64; one zero for an
    empty pattern).  Cached per pattern; read-only."""
    a = np.array(reps if reps else (0,), dtype=np.int64)
    a.setflags(write=False)
    return a, a.ctypes.data


_one_outs: dict = {}


def _one_out(CT, n: int = 1):
    """(array, address) of the result buffer of a scalar call (n values of type CT), kept per kind
    and reused; use under _lock."""
    r = _one_outs.get((CT, n))
    if r is None:
        a = np.zeros(n, CT)
        r = _one_outs[(CT, n)] = (a, a.ctypes.data)
    return r


def _sieve_reference(T: np.dtype, Ax: np.ndarray, edge_reps: list[int], glynn: bool, nthreads: int):
    """_calc_hafnian(Ax, edge_reps; nthreads, glynn) to the last bit (src/hafnian.jl:684-738):
    every term in the reference's arithmetic, summed in the reference's chunks, nchunks =
    _sieve_chunks(work, steps, nthreads) (:646-647, :703-712), each chunk a plain FP64 sum from
    zero (:607-622), the chunk sums folded left to right (:729-732), Glynn's 2^-(n-1) last."""
    cplx = np.dtype(T).kind == "c"
    CT = np.complex128 if cplx else np.float64
    E = len(edge_reps)
    if E == 0:
        return np.dtype(T).type(1)
    work, steps = pol._sieve_variant_cost(edge_reps, int(sum(edge_reps)), glynn)
    nchunks = pol._sieve_chunks(work, steps, max(int(nthreads), 1))
    A = np.asfortranarray(np.asarray(Ax, dtype=CT))
    reps = np.ascontiguousarray(edge_reps, dtype=np.int64)
    out = np.zeros(1, CT)
    with _lock:
        nat.check(nat.lib().egg_sieve_reference_sum(nat.EGG_C128 if cplx else nat.EGG_F64, nat.ptr(A), E, nat.ptr(reps),
                                                    1 if glynn else 0, nchunks, nat.ptr(out)))
    return np.dtype(T).type(out[0])


def _permuted(T, A: np.ndarray, x: list[int]) -> np.ndarray:
    """Ax[a, b] = A[x[a], x[b]] (src/hafnian.jl:786-792)."""
    xi = np.asarray(x, dtype=np.int64) - 1
    return np.asarray(A)[np.ix_(xi, xi)].astype(T, copy=False)


@lru_cache(maxsize=None)
def _distinct_flat(N: int) -> np.ndarray:
    """Flat (row-major) indices into an N x N matrix such that A.ravel().take(f).reshape(N, N).T is
    _permuted(T, A, _distinct_x(N // 2)) in column-major layout: entry (a, b) of the transpose is
    A[x[b], x[a]].  Cached per degree; read-only."""
    xi = np.asarray(_distinct_x(N // 2), dtype=np.int64) - 1
    f = (xi[None, :] * N + xi[:, None]).ravel()
    f.setflags(write=False)
    return f


def _permuted_distinct(T, A: np.ndarray) -> np.ndarray:
    """_permuted(T, A, _distinct_x(N / 2)) as one gather, already in the column-major layout the
    sieve takes."""
    N = A.shape[0]
    return A.ravel().take(_distinct_flat(N)).reshape(N, N).T.astype(T, copy=False)


def _expanded_indices(rpt, total: int) -> np.ndarray:
    """Row i repeated rpt[i] times, 0-based (src/hafnian.jl:1014-1021)."""
    return np.repeat(np.arange(len(rpt), dtype=np.int64), np.asarray(rpt, dtype=np.int64))


def _distinct_x(E: int) -> list[int]:
    """Match vertex 2i-1 with 2i in the [first halves; second halves] layout (:1140-1145)."""
    return [2 * i + 1 for i in range(E)] + [2 * i + 2 for i in range(E)]


# ----------------------------------------------------------------------------------------------
# Entry points
# ----------------------------------------------------------------------------------------------

def _is_batch(A) -> bool:
    if isinstance(A, (list, tuple)):
        return True
    return isinstance(A, np.ndarray) and A.ndim == 3


def hafnian(A, *, nthreads: int | None = None, glynn: bool | None = None, method: str = "auto",
            check_symmetric: bool = True, backend=None, max_batch: int | None = None,
            prec: str | None = None, exact: bool = False):
    """Hafnian of the square symmetric matrix A (src/hafnian.jl:1111-1147), or of each matrix of a
    batch (a list, or a (B, N, N) array; src/hafnian.jl:1263-1301).

    `method` is "auto", "unrolled", "dp" or "sieve"; `glynn` forces the sieve variant; `backend`
    steers the automatic choice to the DP as the reference does.  The diagonal is ignored; odd N
    gives 0 and N = 0 gives 1.
    """
    if _is_batch(A):
        return _hafnian_batch(A, nthreads=nthreads, glynn=glynn, method=method, check_symmetric=check_symmetric,
                              backend=backend, max_batch=max_batch, prec=prec, exact=exact)
    A = np.asarray(A)
    N = _checksquare(A)
    exact_int = exact and A.dtype.kind in "iub"
    T = np.dtype(np.int64) if exact_int else _haf_dtype(A)
    nthreads = nthreads or _default_nthreads()
    if N == 0:
        return 1 if exact_int else T.type(1)
    if N % 2:
        return 0 if exact_int else T.type(0)
    pol._check_method(method, N)
    if check_symmetric:
        _check_symmetric(A)
    E = N // 2
    sel, sel_glynn = pol._choose_method_distinct(N, E, nthreads)
    chosen = pol._steer_backend(sel if method == "auto" else method, backend, N, method)
    use_glynn = sel_glynn if glynn is None else glynn
    if exact_int and chosen == "sieve":
        raise ArgumentError("exact integer hafnians run on the DP; pass method='dp'")
    if chosen in ("unrolled", "dp"):
        P = _gather_pairs_one(T, A)
        v = _dp_one(T, P, N, _dp_prec(prec), exact_int)
        return v if exact_int else T.type(v)
    return _sieve_one(T, _permuted_distinct(T, A), [1] * E, use_glynn, prec, nthreads)


def hafnian_repeated(A, rpt, *, nthreads: int | None = None, glynn: bool | None = None, method: str = "auto",
                     check_symmetric: bool = True, backend=None, max_batch: int | None = None,
                     prec: str | None = None, exact: bool = False):
    """Hafnian of A with row/column i repeated rpt[i] times, without forming that matrix
    (src/hafnian.jl:1194-1222); with a list of patterns, one hafnian per pattern
    (src/hafnian.jl:1317-1359).  The diagonal of A matters when some rpt[i] >= 2."""
    if len(rpt) and isinstance(rpt[0], (list, tuple, np.ndarray)):
        return _hafnian_repeated_batch(A, rpt, nthreads=nthreads, glynn=glynn, method=method,
                                       check_symmetric=check_symmetric, backend=backend, max_batch=max_batch,
                                       prec=prec, exact=exact)
    A = np.asarray(A)
    N = _checksquare(A)
    rpt = [int(r) for r in rpt]
    if len(rpt) != N:
        raise DimensionMismatch(f"rpt has length {len(rpt)}, expected {N}")
    if any(r < 0 for r in rpt):
        raise ArgumentError("rpt must contain non-negative integers")
    exact_int = exact and A.dtype.kind in "iub"
    T = np.dtype(np.int64) if exact_int else _haf_dtype(A)
    nthreads = nthreads or _default_nthreads()
    total = sum(rpt)
    if total == 0:
        return 1 if exact_int else T.type(1)
    if total % 2:
        return 0 if exact_int else T.type(0)
    pol._check_method(method, total)
    if check_symmetric:
        _check_symmetric(A)
    x, edge_reps = pol.matched_reps(rpt)
    sel, sel_glynn = pol._choose_method(total, edge_reps, nthreads)
    chosen = pol._steer_backend(sel if method == "auto" else method, backend, total, method)
    use_glynn = sel_glynn if glynn is None else glynn
    if chosen != "sieve":
        idx = _expanded_indices(rpt, total)
        P = _gather_pairs_batch(T, A, idx[None, :], total)
        v = _dp_device(T, P, total, _dp_prec(prec), None, exact_int)[0]
        return v if exact_int else T.type(v)
    if exact_int:
        raise ArgumentError("exact integer hafnians run on the DP; pass method='dp'")
    return _sieve_one(T, _permuted(T, A, x), edge_reps, use_glynn, prec, nthreads)


def _hafnian_batch(As, *, nthreads, glynn, method, check_symmetric, backend, max_batch, prec, exact):
    mats = [np.asarray(a) for a in As] if not isinstance(As, np.ndarray) else list(As)
    B = len(mats)
    if B == 0:
        return np.zeros(0, dtype=np.float64)
    dtypes = {m.dtype for m in mats}
    exact_int = exact and all(d.kind in "iub" for d in dtypes)
    T = np.dtype(np.int64) if exact_int else np.result_type(*[_haf_dtype_of(d) for d in dtypes])
    N = _checksquare(mats[0])
    stack = None
    if len({m.shape for m in mats}) > 1:
        for b, m in enumerate(mats):
            if _checksquare(m) != N:
                raise DimensionMismatch(f"matrix {b + 1} is {m.shape[0]}×{m.shape[1]}, expected {N}×{N}; a batch "
                                        "shares one strategy and one plan")
            if check_symmetric:
                _check_symmetric(m)
    else:
        stack = As if isinstance(As, np.ndarray) and As.ndim == 3 else np.array(mats)
        if check_symmetric:
            _check_symmetric_stack(stack)
    if N == 0:
        return [1] * B if exact_int else np.ones(B, T)
    if N % 2:
        return [0] * B if exact_int else np.zeros(B, T)
    pol._check_method(method, N)
    nthreads = nthreads or _default_nthreads()
    if backend is not None:
        chosen = pol._steer_backend(pol._choose_method_distinct(N, N // 2, nthreads)[0] if method == "auto" else method,
                                    backend, N, method)
    else:
        # Without a backend the reference loops over hafnian(As[b]; nthreads=1, ...) (:1297-1300);
        # every instance has the same size, so they all choose alike.
        chosen = pol._choose_method_distinct(N, N // 2, 1)[0] if method == "auto" else method
    if chosen in ("unrolled", "dp"):
        P = _gather_pairs_stack(T, np.ascontiguousarray(stack))
        return _dp_device(T, P, N, _dp_prec(prec), max_batch, exact_int)
    if exact_int:
        raise ArgumentError("exact integer hafnians run on the DP; pass method='dp'")
    sel_glynn = pol._choose_method_distinct(N, N // 2, 1 if backend is None else nthreads)[1]
    use_glynn = sel_glynn if glynn is None else glynn
    return _sieve_device_batch(T, [_permuted_distinct(T, m) for m in mats], [[1] * (N // 2)] * B, [use_glynn] * B,
                               prec)


@lru_cache(maxsize=4096)
def _pattern_choice(rp: tuple, total: int):
    """(x, edge_reps, method, glynn) of one multiplicity pattern: matched_reps (src/hafnian.jl:142-188)
    and the per-pattern choice of the reference's batch loop, _choose_method(total, edge_reps; nthreads
    = 1) (:1355-1358).  Both depend on the pattern alone, so they are cached."""
    x, er = pol.matched_reps(list(rp))
    sel, sg = pol._choose_method(total, er, 1)
    return tuple(x), tuple(er), sel, sg  # shared by every caller: immutable


def _hafnian_repeated_batch(A, rpts, *, nthreads, glynn, method, check_symmetric, backend, max_batch, prec, exact):
    A = np.asarray(A)
    B = len(rpts)
    exact_int = exact and A.dtype.kind in "iub"
    T = np.dtype(np.int64) if exact_int else _haf_dtype(A)
    if B == 0:
        return np.zeros(0, dtype=T)
    N = _checksquare(A)
    rpts = [[int(r) for r in rp] for rp in rpts]
    total = sum(rpts[0])
    for b, rp in enumerate(rpts):
        if len(rp) != N:
            raise DimensionMismatch(f"rpt {b + 1} has length {len(rp)}, expected {N}")
        if any(r < 0 for r in rp):
            raise ArgumentError(f"rpt {b + 1} contains a negative entry")
        if sum(rp) != total:
            raise ArgumentError(f"rpt {b + 1} sums to {sum(rp)}, but rpt 1 sums to {total}; a batch shares one plan, "
                                "so every pattern must have the same total")
    if check_symmetric:
        _check_symmetric(A)
    if total == 0:
        return [1] * B if exact_int else np.ones(B, T)
    if total % 2:
        return [0] * B if exact_int else np.zeros(B, T)
    pol._check_method(method, total)
    # Equal patterns over the one matrix are equal instances: each distinct pattern is evaluated
    # once (as its own scalar call would be) and its value given to every instance that has it.
    slot = {}
    order = [slot.setdefault(tuple(rp), len(slot)) for rp in rpts]
    if len(slot) < B:
        uniq = [list(k) for k in slot]
        vals = _hafnian_repeated_batch(A, uniq, nthreads=nthreads, glynn=glynn, method=method, check_symmetric=False,
                                       backend=backend, max_batch=max_batch, prec=prec, exact=exact)
        return [vals[i] for i in order] if exact_int else np.asarray(vals)[order]
    if backend is not None and method in ("auto", "dp") and total <= pol.DP_HARD_MAX:
        idxs = np.stack([_expanded_indices(rp, total) for rp in rpts])
        P = _gather_pairs_batch(T, A, idxs, total)
        return _dp_device(T, P, total, _dp_prec(prec), max_batch, exact_int)
    # Per-pattern choice, as the reference's loop over hafnian_repeated(A, rpts[b]; nthreads=1)
    # (:1355-1358), then one device call per strategy.
    out = [None] * B
    dp_idx, sv_idx, sv_ax, sv_reps, sv_g = [], [], [], [], []
    for b, rp in enumerate(rpts):
        x, er, sel, sg = _pattern_choice(tuple(rp), total)
        chosen = sel if method == "auto" else method
        if chosen != "sieve":
            dp_idx.append(b)
        else:
            sv_idx.append(b)
            if prec == "reference":  # the other forms permute on the device
                sv_ax.append(_permuted(T, A, x))
                sv_reps.append(er)
                sv_g.append(sg if glynn is None else glynn)
    if dp_idx:
        idxs = np.stack([_expanded_indices(rpts[b], total) for b in dp_idx])
        vals = _dp_device(T, _gather_pairs_batch(T, A, idxs, total), total, _dp_prec(prec), max_batch, exact_int)
        for k, b in enumerate(dp_idx):
            out[b] = vals[k]
    if sv_idx:
        if exact_int:
            raise ArgumentError("exact integer hafnians run on the DP; pass method='dp'")
        if prec == "reference":
            vals = _sieve_device_batch(T, sv_ax, sv_reps, sv_g, prec)
        else:
            # One call on the shared matrix: the device forms each pattern's matching, variant and
            # permuted matrix itself.
            vals = _repeated_device(T, np.asarray(A), 0, [rpts[b] for b in sv_idx], glynn, prec)
        for k, b in enumerate(sv_idx):
            out[b] = vals[k]
    return out if exact_int else np.array(out, dtype=T)


def _repeated_device(T: np.dtype, mats: np.ndarray, stride: int, rpts, glynn, prec) -> np.ndarray:
    """egg_sieve_repeated_batch over B patterns: mats is one d x d matrix (stride 0) or a B x d x d
    stack (stride d * d); the device forms each instance's matching, variant and permuted matrix."""
    cplx = np.dtype(T).kind == "c"
    CT = np.complex128 if cplx else np.float64
    R = np.ascontiguousarray(rpts, dtype=np.int64)
    B, d = R.shape
    # Column-major per matrix: store each transposed (the matrices are symmetric, but be exact).
    M = np.ascontiguousarray(np.swapaxes(np.asarray(mats, dtype=CT), -1, -2))
    out = np.zeros(B, CT)
    g = -1 if glynn is None else (1 if glynn else 0)
    with _lock:
        nat.check(nat.lib().egg_sieve_repeated_batch(nat.EGG_C128 if cplx else nat.EGG_F64, _sieve_prec(prec), B, d,
                                                     nat.ptr(M), stride, nat.ptr(R), g, nat.ptr(out)))
    return out.astype(T, copy=False)


def hafnian_repeated_batch(As, rpts, *, glynn: bool | None = None, check_symmetric: bool = True,
                           prec: str | None = None) -> np.ndarray:
    """hafnian_repeated(As[b], rpts[b]; method=:sieve) for every b, in one device call.

    Each instance has its own d x d matrix and multiplicity vector (the reference's
    hafnian_repeated(A, rpts) shares one matrix and runs its batch as a CPU loop,
    src/hafnian.jl:1317-1359).  The device forms every instance's matched_reps, the sieve variant
    of the reference's cost model (unless `glynn` forces one) and its permuted matrix, then runs
    the batched sieve.  A zero total gives 1 and an odd total 0.  prec as for the sieve."""
    S = np.asarray(As)
    if S.ndim != 3 or S.shape[1] != S.shape[2]:
        raise DimensionMismatch(f"expected B square matrices of one size, got an array of shape {S.shape}")
    B, d = S.shape[0], S.shape[1]
    R = np.asarray(rpts)
    if R.shape != (B, d):
        raise DimensionMismatch(f"{B} matrices of size {d} need {B} multiplicity vectors of length {d}, got {R.shape}")
    if B == 0:
        return np.zeros(0)
    R = np.ascontiguousarray(R, dtype=np.int64)
    if (R < 0).any():
        b = int(np.nonzero((R < 0).any(axis=1))[0][0])
        raise ArgumentError(f"rpt {b + 1} contains a negative entry")
    T = _haf_dtype_of(S.dtype)
    if check_symmetric and d >= 2:
        # One comparison for the whole stack; only matrices that differ from their transpose get
        # the reference's tolerance test (and its error message).
        with np.errstate(invalid="ignore"):
            diff = (S != S.transpose(0, 2, 1)).reshape(B, -1).any(axis=1)
        for b in np.nonzero(diff)[0]:
            _check_symmetric(S[b])
    if prec == "reference":
        vals = []
        for A, rp in zip(S, R.tolist()):
            x, er, _, sg = _pattern_choice(tuple(rp), sum(rp))
            tot = sum(rp)
            if tot == 0:
                vals.append(T.type(1))
            elif tot % 2:
                vals.append(T.type(0))
            else:
                vals.append(_sieve_reference(T, _permuted(T, A, list(x)), list(er), sg if glynn is None else glynn, 1))
        return np.array(vals, dtype=T)
    return _repeated_device(T, S, d * d, R, glynn, prec)


def _mix_layout(rows_list) -> tuple[np.ndarray, np.ndarray]:
    """(offsets[B + 1] int64, concatenated rows int32) of a list of 0-based row-index sequences."""
    sizes = np.fromiter((len(r) for r in rows_list), dtype=np.int64, count=len(rows_list))
    offsets = np.zeros(len(rows_list) + 1, dtype=np.int64)
    np.cumsum(sizes, out=offsets[1:])
    flat = (np.concatenate([np.asarray(r, dtype=np.int64) for r in rows_list]) if offsets[-1]
            else np.zeros(0, dtype=np.int64))
    return offsets, np.ascontiguousarray(flat, dtype=np.int32)


def hafnian_submatrices(A, rows_list, *, check_symmetric: bool = True, prec: str | None = None,
                        exact: bool = False):
    """Hafnians of the principal submatrices A[r, r] of one parent, one per 0-based row-index
    sequence r in `rows_list`, in one device call whatever the mix of sizes.

    Each result equals ``hafnian(A[np.ix_(r, r)], method="dp", prec=prec)`` (repeated indices act
    as repeated rows, as in hafnian_repeated); odd sizes give 0 and empty ones 1.  Float64,
    ComplexF64 or, with ``exact=True``, integer parents (Int128 results as Python ints).  The
    reference has no counterpart: its batch form takes one size per call
    (src/hafnian.jl:1263-1301).
    """
    A = np.asarray(A)
    n = _checksquare(A)
    if check_symmetric:
        _check_symmetric(A)
    exact_int = exact and A.dtype.kind in "iub"
    if exact_int:
        T, code = np.dtype(np.int64), nat.EGG_I64
    else:
        T = _haf_dtype(A)
        T = np.dtype(np.complex128) if T.kind == "c" else np.dtype(np.float64)
        code = nat.DTYPE_OF[T]
    B = len(rows_list)
    if B == 0:
        return [] if exact_int else np.zeros(0, dtype=T)
    offsets, flat = _mix_layout(rows_list)
    Af = np.asfortranarray(A.astype(T, copy=False))
    out = np.zeros(2 * B, np.uint64) if exact_int else np.zeros(B, T)
    prec_name = _dp_prec(prec)
    if prec_name not in nat.PREC:
        raise ArgumentError(f"prec must be one of {tuple(nat.PREC)}")
    with _lock:
        nat.check(nat.lib().egg_dp_mix(code, nat.PREC[prec_name], nat.ptr(Af), n, B, nat.ptr(offsets),
                                       nat.ptr(flat) if len(flat) else None, nat.ptr(out)))
    if exact_int:
        vals = []
        for b in range(B):
            v = int(out[2 * b]) | (int(out[2 * b + 1]) << 64)
            vals.append(v - (1 << 128) if v >= (1 << 127) else v)
        return vals
    return out


def reduction(A, rpt) -> np.ndarray:
    """A with row/column i repeated rpt[i] times (src/hafnian.jl:1369-1374)."""
    A = np.asarray(A)
    if _checksquare(A) != len(rpt):
        raise DimensionMismatch("rpt must have one entry per row of A")
    idx = _expanded_indices(rpt, int(sum(rpt)))
    return A[np.ix_(idx, idx)]


def sieve(Ax, edge_reps, *, glynn: bool = False, prec: str | None = None, nthreads: int | None = None):
    """The device sieve on a pre-permuted matrix: _calc_hafnian(Ax, edge_reps; nthreads, glynn)
    (src/hafnian.jl:684), the seam the reference has no device hook for.  prec='exact' evaluates
    every term in the reference's rounding and sums them in double-double (the default);
    prec='reference' also sums them in the reference's order for `nthreads` threads, so the result
    is the reference's to the last bit; prec='fma' uses the fused-multiply-add register tiles."""
    Ax = np.asarray(Ax)
    T = _haf_dtype(Ax)
    return _sieve_one(T, Ax, list(edge_reps), glynn, prec, nthreads or _default_nthreads())
