"""Parity at the benchmarked configurations, on the benchmarked inputs, against the oracle.

Each test draws the same seeded matrices `bench.py` times and checks the device against the CPU
restatement of the reference (oracle/), at full size:

  * configuration 1, N = 20 real: the DP bit for bit; the sieve in its three forms;
  * configuration 2, N = 40 real (U[-1,1]/sqrt N) and complex (parts N(0, 1/2N)), inclusion-exclusion
    (the reference's choice for distinct rows) and Glynn:
      - prec="exact": every term in the reference's arithmetic, summed in double-double; equal to
        the oracle's double-double sum of its terms within 1e-15 (src/hafnian.jl:528-602);
      - prec="reference": the reference's own summation, 16 chunks (_sieve_sum with nthreads = 16,
        src/hafnian.jl:684-738): bit-identical (==) to the oracle's plain sum;
      - prec="fma" (register tiles, fused multiply-adds): within 4 N eps kappa of the oracle,
        kappa = sum|terms| / |result|, the cancellation of the alternating sum;
    and N = 24 draws of the same distributions against 256-bit gold;
  * configuration 3, N = 36 and 40, U[0,1] in FP64 and an Erdos-Renyi graph in Int128: bit for bit
    against the oracle's plan-free walk of the reference DP (the stored plan is 24 GB at N = 40);
  * configuration 4, the 4096-instance mix: 5 instances of every degree bit for bit against the
    oracle DP;
  * configuration 5, both 1024-instance batches of hafnian_repeated: 64 instances each against the
    oracle's sieve.
"""
import numpy as np
import pytest

from conftest import dec, dec_matrix

pytestmark = pytest.mark.gpu

EPS = np.finfo(float).eps


def rel(a, b):
    return abs(complex(a) - complex(b)) / max(abs(complex(b)), 1e-300)


def distinct_x(E):
    return [2 * i + 1 for i in range(E)] + [2 * i + 2 for i in range(E)]


def sieve_steps(reps, glynn):
    steps = 1
    for i, r in enumerate(reps):
        steps *= (r + 2) // 2 if (glynn and i == 0) else r + 1
    return steps


def kappa(orc, Ax, reps, glynn, ref):
    """sum |terms| / |result|: by how much the alternating sum magnifies one term's rounding."""
    n = sum(reps)
    terms = orc.sieve_terms(Ax, reps, glynn, 0, sieve_steps(reps, glynn))
    scale = 0.5 ** (n - 1) if glynn else 1.0
    return float(np.sum(np.abs(terms)) * scale / max(abs(complex(ref)), 1e-300))


def check_sieve_forms(egg, orc, Ax, reps, glynn, N, nthreads=16):
    """The three sieve forms of one instance against the oracle; returns the relative errors."""
    dd = orc.calc_hafnian(Ax, reps, glynn, nthreads=16, sum_mode=1)
    plain = orc.calc_hafnian(Ax, reps, glynn, nthreads=nthreads, sum_mode=0)
    ex = egg.sieve(Ax, reps, glynn=glynn, prec="exact")
    assert rel(ex, dd) <= 1e-15, ("exact", ex, dd)
    rf = egg.sieve(Ax, reps, glynn=glynn, prec="reference", nthreads=nthreads)
    assert complex(rf) == complex(plain), ("reference", rf, plain)
    fm = egg.sieve(Ax, reps, glynn=glynn, prec="fma")
    k = kappa(orc, Ax, reps, glynn, dd)
    assert rel(fm, dd) <= 4 * N * EPS * k + 1e-15, ("fma", fm, dd, k)
    return {"exact": rel(ex, plain), "fma": rel(fm, plain), "kappa": k}


# ---- configuration 1 ------------------------------------------------------------------------------

def test_config1_n20(egg, orc, W):
    A = W.dense_real(20, 2020)
    assert egg.hafnian(A, method="dp") == orc.haf_dp(A)
    Ax = orc.permuted(A, distinct_x(10))
    for glynn in (False, True):
        check_sieve_forms(egg, orc, Ax, [1] * 10, glynn, 20)
    # The public API's sieve (the cost model picks inclusion-exclusion for distinct rows).
    got = egg.hafnian(A, method="sieve", prec="reference", nthreads=16)
    assert got == orc.calc_hafnian(Ax, [1] * 10, False, nthreads=16, sum_mode=0)


# ---- configuration 2 ------------------------------------------------------------------------------

@pytest.mark.parametrize("cplx", [False, True])
@pytest.mark.parametrize("glynn", [False, True])
def test_config2_sieve_n40(egg, orc, W, cplx, glynn):
    N, E = 40, 20
    A = W.dense_complex(N, 2025, 1.0 / (2 * N)) if cplx else W.dense_real(N, 2024, scale=1.0 / np.sqrt(N))
    Ax = orc.permuted(A, distinct_x(E))
    errs = check_sieve_forms(egg, orc, Ax, [1] * E, glynn, N)
    # Through the public API from the unpermuted matrix, with its symmetry check.
    got = egg.hafnian(A, method="sieve", glynn=glynn, prec="reference", nthreads=16)
    assert complex(got) == complex(orc.calc_hafnian(Ax, [1] * E, glynn, nthreads=16, sum_mode=0))
    print(f"config2 cplx={cplx} glynn={glynn}: {errs}")


def test_config2_gold_n24(egg, orc, golden):
    """N = 24 draws of the configuration-2 distributions against 256-bit gold.  Real U[-1,1]/sqrt N
    hafnians can nearly cancel (kappa up to 7e6 here), so the bar is the rounding bound 4 N eps kappa
    of any FP64 evaluation of the terms; the DP keeps the reference's 1e-13 envelope."""
    for case in golden["config2_n24"]:
        A = dec_matrix(case["A"])
        gold = dec(case["gold"])
        N = A.shape[0]
        E = N // 2
        Ax = orc.permuted(A, distinct_x(E))
        assert rel(egg.hafnian(A, method="dp"), gold) < 1e-13, case["seed"]
        for glynn in (False, True):
            k = kappa(orc, Ax, [1] * E, glynn, gold)
            for prec in ("exact", "fma"):
                v = egg.hafnian(A, method="sieve", glynn=glynn, prec=prec)
                assert rel(v, gold) <= 4 * N * EPS * k, (case["seed"], glynn, prec, rel(v, gold), k)


# ---- configuration 3 ------------------------------------------------------------------------------

@pytest.mark.parametrize("N", [36, 40])
def test_config3_fp64(egg, orc, W, N):
    A = W.dense_real(N, 3636 if N == 36 else 4040, 0.0, 1.0)
    P = orc.gather_pairs(A, list(range(1, N + 1)), N)
    want = orc.haf_dp_closed(P, N, orc.F64, orc.max_threads())
    assert egg.hafnian(A, method="dp", prec="exact") == want


@pytest.mark.parametrize("N", [36, 40])
def test_config3_int128(egg, orc, W, N):
    G = W.er_graph(N, 0.5, 4041 if N == 40 else 3637)
    P = orc.gather_pairs(G, list(range(1, N + 1)), N)
    want = orc.haf_dp_closed(P, N, orc.I64, orc.max_threads())
    assert egg.hafnian(G, method="dp", exact=True) == want


# ---- configuration 4 ------------------------------------------------------------------------------

def test_config4_full_mix(egg, orc, W):
    A, idxs = W.gbs_mix(4096, 64, range(8, 33, 2), 4)
    got = egg.hafnian_submatrices(A, idxs, prec="exact")
    assert len(got) == 4096
    by_deg = {}
    for b, r in enumerate(idxs):
        by_deg.setdefault(len(r), []).append(b)
    assert sorted(by_deg) == list(range(8, 33, 2))
    checked = 0
    for K, bs in sorted(by_deg.items()):
        for b in bs[:5]:
            r = [int(i) + 1 for i in idxs[b]]
            want = orc.haf_dp_closed(orc.gather_pairs(A, r, K), K, orc.C128, 8)
            assert got[b] == want, (K, b, got[b], want)
            checked += 1
    assert checked >= 64


# ---- configuration 5 ------------------------------------------------------------------------------

def _repeated_batch(orc, W, which):
    if which == "a":
        mats, rpts = W.repeated_real(1024, 14, 5)
    else:
        mats, rpts = W.repeated_complex(1024, 20, 48, 6)
    inst = []
    for A, r in zip(mats, rpts):
        x, er = orc.matched_reps(r)
        g = orc.choose_method(sum(r), er, 1)[1]
        inst.append((orc.permuted(A, x), list(er), bool(g), sum(r)))
    return inst


@pytest.mark.parametrize("which", ["a", "b"])
def test_config5_batches(egg, orc, W, which):
    from theeggman_b200.hafnian import _sieve_device_batch

    inst = _repeated_batch(orc, W, which)
    T = np.dtype(np.float64 if which == "a" else np.complex128)
    Axs, ers, gs = [i[0] for i in inst], [i[1] for i in inst], [i[2] for i in inst]
    fma = _sieve_device_batch(T, Axs, ers, gs, "fma")
    nex = 1024 if which == "a" else 64
    ex = _sieve_device_batch(T, Axs[:nex], ers[:nex], gs[:nex], "exact")
    for b in range(0, 1024, 16):  # 64 instances
        Ax, er, g, N = inst[b]
        dd = orc.calc_hafnian(Ax, er, g, nthreads=16, sum_mode=1)
        if b < nex:
            assert rel(ex[b], dd) <= 1e-15, (b, ex[b], dd)
        k = kappa(orc, Ax, er, g, dd)
        assert rel(fma[b], dd) <= 4 * N * EPS * k + 1e-15, (b, fma[b], dd, k)
    # The reference's own batch loop sums each instance in one chunk (nthreads = 1).
    ref = _sieve_device_batch(T, Axs[:8], ers[:8], gs[:8], "reference")
    for b in range(8):
        Ax, er, g, _ = inst[b]
        assert complex(ref[b]) == complex(orc.calc_hafnian(Ax, er, g, nthreads=1, sum_mode=0)), b
