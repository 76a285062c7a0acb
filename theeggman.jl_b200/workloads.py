"""Seeded synthetic inputs for the hafnian workloads (there is no public dataset: the reference's own
benchmarks draw random symmetric matrices, benchmark/competitors/hafnian_bench.jl:144-159).

The generator is SplitMix64 (a counter-based 64-bit mixer), vectorised in numpy, so that every
input is reproducible bit-for-bit from its seed on any machine.  Workloads:

  * ``dense_real(N, seed, lo, hi)`` / ``dense_complex(N, seed, sigma2)``: symmetric matrices with
    iid upper triangles (mirrored);
  * ``er_graph(N, p, seed)``: 0/1 adjacency of an Erdos-Renyi graph;
  * ``gbs_mix(...)``: many index subsets of one 64x64 complex A = U diag(tanh r) U^T with U Haar;
  * ``repeated_real(...)`` / ``repeated_complex(...)``: batches of small B with repetition patterns.
"""
from __future__ import annotations

import numpy as np

_M64 = np.uint64(0xFFFFFFFFFFFFFFFF)


def splitmix64(seed: int, n: int) -> np.ndarray:
    """n consecutive SplitMix64 outputs for stream `seed` (state starts at seed)."""
    with np.errstate(over="ignore"):
        k = np.arange(1, n + 1, dtype=np.uint64)
        z = (np.uint64(seed & 0xFFFFFFFFFFFFFFFF) + k * np.uint64(0x9E3779B97F4A7C15)) & _M64
        z = (z ^ (z >> np.uint64(30))) * np.uint64(0xBF58476D1CE4E5B9)
        z = (z ^ (z >> np.uint64(27))) * np.uint64(0x94D049BB133111EB)
        z = z ^ (z >> np.uint64(31))
    return z


def uniform(seed: int, n: int) -> np.ndarray:
    """n doubles in [0, 1) from the top 53 bits."""
    return (splitmix64(seed, n) >> np.uint64(11)).astype(np.float64) * (1.0 / (1 << 53))


def normal(seed: int, n: int) -> np.ndarray:
    """n standard normals by Box-Muller on pairs of uniforms."""
    m = (n + 1) // 2
    u = uniform(seed, 2 * m)
    u1 = 1.0 - u[0::2]  # (0, 1]
    u2 = u[1::2]
    r = np.sqrt(-2.0 * np.log(u1))
    z = np.concatenate([r * np.cos(2 * np.pi * u2), r * np.sin(2 * np.pi * u2)])
    return z[:n]


def _sym_from_upper(vals: np.ndarray, N: int) -> np.ndarray:
    A = np.zeros((N, N), dtype=vals.dtype)
    iu = np.triu_indices(N)
    A[iu] = vals[: len(iu[0])]
    return A + np.triu(A, 1).T


def dense_real(N: int, seed: int, lo: float = -1.0, hi: float = 1.0, scale: float = 1.0) -> np.ndarray:
    """Symmetric N x N, upper triangle (with diagonal) iid U[lo, hi] * scale."""
    v = (lo + (hi - lo) * uniform(seed, N * (N + 1) // 2)) * scale
    return _sym_from_upper(v, N)


def dense_complex(N: int, seed: int, sigma2: float) -> np.ndarray:
    """Symmetric N x N complex, real and imaginary parts iid N(0, sigma2)."""
    k = N * (N + 1) // 2
    z = normal(seed, 2 * k) * np.sqrt(sigma2)
    return _sym_from_upper(z[:k] + 1j * z[k:], N)


def er_graph(N: int, p: float, seed: int) -> np.ndarray:
    """0/1 Int64 adjacency of G(N, p) (zero diagonal)."""
    v = (uniform(seed, N * (N + 1) // 2) < p).astype(np.int64)
    A = _sym_from_upper(v, N)
    np.fill_diagonal(A, 0)
    return A


def haar_unitary(n: int, seed: int) -> np.ndarray:
    """Haar-random n x n unitary: QR of a complex Ginibre matrix with the R-diagonal phase fix."""
    z = normal(seed, 2 * n * n).reshape(2, n, n)
    G = (z[0] + 1j * z[1]) / np.sqrt(2.0)
    Q, R = np.linalg.qr(G)
    d = np.diag(R)
    return Q * (d / np.abs(d))[None, :]


def gbs_parent(n: int = 64, seed: int = 4) -> np.ndarray:
    """A = U diag(tanh r) U^T, U Haar, r_i ~ U[0, 1] (complex symmetric)."""
    U = haar_unitary(n, seed)
    r = uniform(seed + 1, n)
    return (U * np.tanh(r)[None, :]) @ U.T


def gbs_mix(B: int = 4096, n: int = 64, degrees=range(8, 33, 2), seed: int = 4):
    """B instances: even degree N uniform over `degrees`, N distinct rows of the parent without
    replacement.  Returns (A, list of 0-based index arrays)."""
    A = gbs_parent(n, seed)
    degs = np.array(list(degrees), dtype=np.int64)
    u = uniform(seed + 2, B)
    Ns = degs[np.minimum((u * len(degs)).astype(np.int64), len(degs) - 1)]
    idxs = []
    for b in range(B):
        keys = uniform(seed + 1000 + b, n)
        idxs.append(np.sort(np.argsort(keys, kind="stable")[: Ns[b]]))
    return A, idxs


def repeated_real(B: int = 1024, d: int = 14, seed: int = 5):
    """B symmetric d x d real matrices with entries U[-1, 1] and rpt = fill(2, d)."""
    mats = [dense_real(d, seed * 1_000_003 + b) for b in range(B)]
    return mats, [[2] * d for _ in range(B)]


def repeated_complex(B: int = 1024, d: int = 20, total_max: int = 48, seed: int = 6):
    """B symmetric d x d complex matrices with N(0, 1/(2d)) parts... specifically N(0, 1/40) at
    d = 20, and rpt_i iid uniform in {1, 2, 3, 4}; patterns over `total_max` (or odd) are trimmed
    by decrementing positive entries chosen by the stream until the total is <= total_max and
    even."""
    mats, rpts = [], []
    for b in range(B):
        s = seed * 1_000_003 + b
        mats.append(dense_complex(d, s, 1.0 / (2 * d)))
        u = uniform(s + 7, d + 256)
        rpt = (1 + np.minimum((u[:d] * 4).astype(np.int64), 3)).tolist()
        k = d
        while sum(rpt) > total_max or sum(rpt) % 2:
            pos = [i for i, r in enumerate(rpt) if r > 0]
            i = pos[int(u[k % len(u)] * len(pos)) % len(pos)]
            rpt[i] -= 1
            k += 1
        rpts.append(rpt)
    return mats, rpts
