"""Generate tests/golden/golden.json: the fixtures the oracle and the device path are pinned to.

TheEggman.jl is pure Julia and Julia is not available here, so the reference cannot be run to
produce vectors.  The fixtures are therefore:

  1. The literal known answers in the reference's own tests and docstrings
     (test/runtests.jl:52-56, :465-468; src/hafnian.jl:1104-1105, :1183-1190).
  2. The closed-form plan sizes the reference tabulates (src/dp.jl:34-37 / README.md, the
     "DP transitions" row; src/dp.jl:73-78 plan sizes are derived from these).
  3. Seeded random symmetric matrices (SplitMix64, theeggman.jl_b200/workloads.py) with their
     hafnians computed independently of every kernel in this repository: by enumerating perfect
     matchings (test/runtests.jl:11-25's definition) for N <= 10, and by the memoised subset
     recursion for 12 <= N <= 20 -- both in 256-bit mpmath arithmetic, the precision the reference
     uses for its gold values (test/runtests.jl:123-133).
  4. Repeated-row cases: hafnian_repeated(A, rpt) gold via the expanded matrix
     (reduction, src/hafnian.jl:1369-1374) at 256 bits.
  5. N = 24 matrices drawn from the N = 40 sieve workloads' distributions (real U[-1, 1]/sqrt(N),
     complex parts N(0, 1/(2N))), gold by the memoised recursion at 256 bits.

Numbers are stored as hex floats (complex as [re, im]) so they round-trip exactly.
Run:  python tests/golden/make_golden.py
"""
from __future__ import annotations

import importlib.util
import json
import os
import sys

import mpmath
import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))


def _workloads():
    spec = importlib.util.spec_from_file_location("egg_workloads", os.path.join(ROOT, "theeggman.jl_b200", "workloads.py"))
    m = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(m)
    return m


def enc(x):
    if isinstance(x, (complex, np.complexfloating)):
        return [float(x.real).hex(), float(x.imag).hex()]
    return float(x).hex()


def enc_mp(v):
    if isinstance(v, mpmath.mpc):
        return [float(v.real).hex(), float(v.imag).hex()]
    return float(v).hex()


def enc_matrix(A):
    return [[enc(v) for v in row] for row in A]


def brute_mp(A):
    """Sum over all perfect matchings, pairing the first remaining index (test/runtests.jl:11-25)."""
    N = A.shape[0]
    M = [[mpmath.mpmathify(complex(A[i, j]) if np.iscomplexobj(A) else float(A[i, j])) for j in range(N)] for i in range(N)]

    def rec(rem):
        if not rem:
            return mpmath.mpf(1)
        i = rem[0]
        s = mpmath.mpf(0)
        for t in range(1, len(rem)):
            s += M[i][rem[t]] * rec(rem[1:t] + rem[t + 1:])
        return s

    return rec(list(range(N))) if N % 2 == 0 else mpmath.mpf(0)


def memo_mp(A):
    """haf(S) = sum_{t in S, t != min S} A[min S, t] haf(S \\ {min S, t}) (src/dp.jl:6-8)."""
    N = A.shape[0]
    M = [[mpmath.mpmathify(complex(A[i, j]) if np.iscomplexobj(A) else float(A[i, j])) for j in range(N)] for i in range(N)]
    memo = {0: mpmath.mpf(1)}
    full = (1 << N) - 1
    # bottom-up by popcount so no deep recursion
    order = sorted(range(1 << N), key=lambda m: bin(m).count("1")) if N <= 14 else None
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
    del order
    return rec(full) if N % 2 == 0 else mpmath.mpf(0)


def main():
    mpmath.mp.prec = 256
    W = _workloads()
    out = {"_doc": "generated by tests/golden/make_golden.py; see its docstring"}

    out["known_answers"] = [
        {"name": "empty", "A": [], "expect": enc(1.0), "src": "test/runtests.jl:52"},
        {"name": "2x2", "A": enc_matrix(np.array([[0.0, 1.0], [1.0, 0.0]])), "expect": enc(1.0),
         "src": "test/runtests.jl:53"},
        {"name": "4x4 integer", "A": enc_matrix(np.array([[0, 1, 2, 3], [1, 0, 4, 5], [2, 4, 0, 6], [3, 5, 6, 0]], float)),
         "expect": enc(28.0), "src": "test/runtests.jl:55-56; src/hafnian.jl:1104-1105"},
    ]
    out["known_repeated"] = [
        {"name": "doctest 11", "A": enc_matrix(np.array([[1.0, 2.0], [2.0, 3.0]])), "rpt": [2, 2], "expect": enc(11.0),
         "src": "src/hafnian.jl:1183-1190"},
    ]
    # hafnian_repeated(A, [2,0,0,0]) == A[1,1], all-zero rpt gives 1, odd total gives 0
    A4 = W.dense_complex(4, 10, 0.5)
    out["known_repeated"] += [
        {"name": "rpt [2,0,0,0] is A[1,1]", "A": enc_matrix(A4), "rpt": [2, 0, 0, 0], "expect": enc(A4[0, 0]),
         "src": "test/runtests.jl:468"},
        {"name": "rpt all zero", "A": enc_matrix(A4), "rpt": [0, 0, 0, 0], "expect": enc(1.0), "src": "test/runtests.jl:465"},
        {"name": "rpt odd total", "A": enc_matrix(A4), "rpt": [1, 0, 0, 0], "expect": enc(0.0), "src": "test/runtests.jl:466"},
    ]
    out["dp_transitions"] = {"12": 1076, "16": 10226, "20": 89665, "24": 748776, "28": 6052062, "32": 47786401,
                             "_src": "src/dp.jl:34-37, README.md (DP transitions row)"}

    cases = []
    for N in (2, 4, 6, 8, 10):
        for kind in ("real", "complex"):
            seed = 100 + N * 10 + (kind == "complex")
            A = W.dense_real(N, seed) if kind == "real" else W.dense_complex(N, seed, 0.5)
            cases.append({"N": N, "kind": kind, "seed": seed, "A": enc_matrix(A), "gold": enc_mp(brute_mp(A)),
                          "how": "matching enumeration, 256-bit"})
    for N in (12, 14, 16, 18, 20):
        for kind in ("real", "complex"):
            seed = 100 + N * 10 + (kind == "complex")
            A = W.dense_real(N, seed) if kind == "real" else W.dense_complex(N, seed, 0.5)
            cases.append({"N": N, "kind": kind, "seed": seed, "A": enc_matrix(A), "gold": enc_mp(memo_mp(A)),
                          "how": "memoised subset recursion, 256-bit"})
    out["random"] = cases

    # The distributions of the N = 40 sieve workloads, at N = 24 where 256-bit gold is cheap (the
    # error check of the N = 40 sieve configuration, at the N of the reference's own envelope
    # test, test/runtests.jl:123-133): real U[-1, 1]/sqrt(N), complex parts N(0, 1/(2N)).
    c2 = []
    for i in range(4):
        for kind in ("real", "complex"):
            N = 24
            seed = 2400 + 10 * i + (kind == "complex")
            A = W.dense_real(N, seed, scale=1.0 / np.sqrt(N)) if kind == "real" else W.dense_complex(N, seed, 1.0 / (2 * N))
            c2.append({"N": N, "kind": kind, "seed": seed, "A": enc_matrix(A), "gold": enc_mp(memo_mp(A)),
                       "how": "memoised subset recursion, 256-bit"})
    out["config2_n24"] = c2

    rep = []
    for i, rpt in enumerate(([2, 2, 2], [1, 2, 3, 2], [6, 6], [3, 3, 3, 3], [8, 4], [5, 5, 1, 1], [4, 1, 1], [0, 2, 2],
                             [2, 2, 2, 1, 1, 0], [3, 3, 2, 0, 0, 0], [1, 1, 1, 1, 1, 1], [4, 4, 4, 4], [2] * 7)):
        d = len(rpt)
        A = W.dense_complex(d, 500 + i, 0.5)
        idx = np.repeat(np.arange(d), rpt)
        Ar = A[np.ix_(idx, idx)]
        g = memo_mp(Ar)
        rep.append({"rpt": rpt, "A": enc_matrix(A), "gold": enc_mp(g), "how": "subset recursion on reduction(A, rpt)"})
    out["repeated"] = rep

    with open(os.path.join(HERE, "golden.json"), "w") as f:
        json.dump(out, f, indent=1)
    print("wrote", os.path.join(HERE, "golden.json"))


if __name__ == "__main__":
    sys.setrecursionlimit(10000)
    main()
