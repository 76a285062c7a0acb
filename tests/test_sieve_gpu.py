"""Device Bjorklund/Glynn sieve through the C ABI, against the oracle.

prec="exact": every term is computed in the reference's order and rounding, and the terms are summed
in double-double, so the device result is compared with the oracle summing the same terms in
double-double (sum_mode 1): the bar is 1e-15 relative (in practice they are equal).  Against the
reference's own plain FP64 summation the difference is bounded by that summation's rounding.

prec="fma" (the register-resident fused-multiply-add kernels): each term differs from the reference's by its
own rounding (fused multiply-adds, a Newton reciprocal, another pivot among near-equal candidates),
and the sieve's alternating sum magnifies that by kappa = sum|terms| / |result|.  The bar is the
rounding-error bound 4 N eps kappa (+1e-15), with kappa computed from the oracle's terms.

Against 256-bit gold both modes stay inside the reference's own envelopes (Glynn < 1e-12,
inclusion-exclusion < 1e-9, test/runtests.jl:123-133).
"""
import numpy as np
import pytest

from conftest import dec, dec_matrix

pytestmark = pytest.mark.gpu

EPS = np.finfo(float).eps


def kappa(orc, Ax, reps, glynn, ref):
    """sum |terms| / |result| for the sieve of (Ax, reps): the cancellation factor."""
    n = sum(reps)
    steps = 1
    for i, r in enumerate(reps):
        steps *= (r + 2) // 2 if (glynn and i == 0) else r + 1
    terms = orc.sieve_terms(Ax, reps, glynn, 0, steps)
    scale = 0.5 ** (n - 1) if glynn else 1.0
    return float(np.sum(np.abs(terms)) * scale / max(abs(complex(ref)), 1e-300))


def rel(a, b):
    return abs(complex(a) - complex(b)) / max(abs(complex(b)), 1e-300)


def distinct_x(E):
    return [2 * i + 1 for i in range(E)] + [2 * i + 2 for i in range(E)]


@pytest.mark.parametrize("cplx", [False, True])
@pytest.mark.parametrize("glynn", [False, True])
def test_sieve_matches_oracle(egg, orc, W, cplx, glynn):
    for N in (2, 4, 6, 8, 10, 12, 14, 16, 18, 20, 22, 24):
        A = W.dense_complex(N, 60 + N, 0.5) if cplx else W.dense_real(N, 60 + N)
        E = N // 2
        Ax = orc.permuted(A, distinct_x(E))
        dd = orc.calc_hafnian(Ax, [1] * E, glynn, sum_mode=1)
        got = egg.sieve(Ax, [1] * E, glynn=glynn, prec="exact")
        assert rel(got, dd) <= 1e-15, (N, got, dd)
        fast = egg.sieve(Ax, [1] * E, glynn=glynn, prec="fma")
        assert rel(fast, dd) <= 4 * N * EPS * kappa(orc, Ax, [1] * E, glynn, dd) + 1e-15, (N, fast, dd)
        plain = orc.calc_hafnian(Ax, [1] * E, glynn, sum_mode=0)
        steps = 2 ** (E - 1) if glynn else 2 ** E
        terms = orc.sieve_terms(Ax, [1] * E, glynn, 0, min(steps, 4096))
        if steps <= 4096:
            bound = 4 * steps * np.finfo(float).eps * np.sum(np.abs(terms)) * (0.5 ** (E - 1) if glynn else 1)
            assert abs(complex(got) - complex(plain)) <= bound + 1e-300


@pytest.mark.parametrize("prec", ["exact", "fma"])
def test_sieve_golden_envelopes(egg, golden, prec):
    for case in golden["random"]:
        A = dec_matrix(case["A"])
        g = dec(case["gold"])
        eg = rel(egg.hafnian(A, method="sieve", glynn=True, prec=prec), g)
        ei = rel(egg.hafnian(A, method="sieve", glynn=False, prec=prec), g)
        assert eg < 1e-12 and ei < 1e-9, (case["N"], case["kind"], eg, ei)


def test_repeated_rows_mixed_radix(egg, orc, golden):
    for case in golden["repeated"]:
        A = dec_matrix(case["A"])
        g = dec(case["gold"])
        rpt = case["rpt"]
        x, er = orc.matched_reps(rpt)
        Ax = orc.permuted(A, x)
        for glynn in (False, True):
            dd = orc.calc_hafnian(Ax, er, glynn, sum_mode=1)
            got = egg.sieve(Ax, er, glynn=glynn, prec="exact")
            assert rel(got, dd) <= 1e-15, (rpt, glynn)
            assert rel(got, g) < 1e-10, (rpt, glynn)
            fast = egg.sieve(Ax, er, glynn=glynn, prec="fma")
            assert rel(fast, dd) <= 4 * 2 * len(er) * EPS * kappa(orc, Ax, er, glynn, dd) + 1e-15, (rpt, glynn)
            assert rel(fast, g) < 1e-10, (rpt, glynn)
        assert rel(egg.hafnian_repeated(A, rpt, method="sieve"), g) < 1e-10


def test_edge_cases(egg, orc, W):
    A = W.dense_complex(4, 10, 0.5)
    assert egg.sieve(np.zeros((0, 0)), []) == 1
    assert egg.hafnian_repeated(A, [2, 0, 0, 0], method="sieve") == pytest.approx(A[0, 0], rel=1e-15)
    assert egg.hafnian(np.zeros((8, 8)), method="sieve") == 0
    assert egg.hafnian(np.zeros((8, 8)), method="sieve", glynn=True) == 0
    # large multiplicities and single-row patterns (test/runtests.jl:210-219)
    for rpt in ([7, 7, 7, 7], [12], [10, 2], [9, 3], [6, 2, 2, 2]):
        d = len(rpt)
        B = W.dense_complex(d, 99 + d, 0.5)
        x, er = orc.matched_reps(rpt)
        Bx = orc.permuted(B, x)
        for glynn in (False, True):
            dd = orc.calc_hafnian(Bx, er, glynn, sum_mode=1)
            assert rel(egg.sieve(Bx, er, glynn=glynn, prec="exact"), dd) <= 1e-15
            bound = 4 * 2 * len(er) * EPS * kappa(orc, Bx, er, glynn, dd) + 1e-15
            assert rel(egg.sieve(Bx, er, glynn=glynn), dd) <= bound


@pytest.mark.parametrize("prec", ["exact", "fma"])
def test_known_answers(egg, golden, prec):
    for case in golden["known_answers"]:
        if not case["A"]:
            continue
        A = dec_matrix(case["A"])
        for glynn in (False, True):
            assert egg.hafnian(A, method="sieve", glynn=glynn, prec=prec) == dec(case["expect"])
    for case in golden["known_repeated"]:
        A = dec_matrix(case["A"])
        assert rel(egg.hafnian_repeated(A, case["rpt"], method="sieve"), dec(case["expect"])) <= 1e-15 or \
            egg.hafnian_repeated(A, case["rpt"], method="sieve") == dec(case["expect"])


@pytest.mark.parametrize("prec", ["exact", "fma"])
def test_batch_equals_scalar(egg, orc, W, prec):
    """One egg_sieve_batch call over instances of different edge counts and variants gives each
    instance's scalar result."""
    from theeggman_b200.hafnian import _sieve_device_batch

    mats, rpts = W.repeated_complex(12, d=10, total_max=24, seed=31)
    Axs, reps, gs = [], [], []
    for i, (A, r) in enumerate(zip(mats, rpts)):
        x, er = orc.matched_reps(r)
        Axs.append(orc.permuted(A, x))
        reps.append(er)
        gs.append(i % 2 == 0)
    vals = _sieve_device_batch(np.dtype(np.complex128), Axs, reps, gs, prec)
    for Ax, er, g, v in zip(Axs, reps, gs, vals):
        assert rel(v, egg.sieve(Ax, er, glynn=g, prec=prec)) <= 1e-15
        dd = orc.calc_hafnian(Ax, er, g, sum_mode=1)
        tol = 1e-15 if prec == "exact" else 4 * 2 * len(er) * EPS * kappa(orc, Ax, er, g, dd) + 1e-15
        assert rel(v, dd) <= tol


@pytest.mark.parametrize("cplx", [False, True])
def test_batch_mixes_subset_and_odometer_instances(egg, orc, W, cplx):
    """One batch holding distinct-row inclusion-exclusion instances (dealt as edge subsets) beside
    Glynn and repeated-row instances (walked on the odometer), of different edge counts: every
    level kernel takes each instance its own way, and each result is the scalar call's."""
    from theeggman_b200.hafnian import _sieve_device_batch

    T = np.dtype(np.complex128 if cplx else np.float64)
    Axs, reps, gs = [], [], []
    for i, N in enumerate((8, 14, 20, 12, 16, 18)):
        A = W.dense_complex(N, 500 + i, 0.5) if cplx else W.dense_real(N, 500 + i)
        E = N // 2
        Axs.append(orc.permuted(A, distinct_x(E)))
        reps.append([1] * E)
        gs.append(i % 3 == 1)  # two Glynn instances among the distinct-row ones
    mats, rpts = (W.repeated_complex(4, d=10, total_max=22, seed=41) if cplx else W.repeated_real(4, 9, seed=41))
    for A, r in zip(mats, rpts):
        x, er = orc.matched_reps(r)
        Axs.append(orc.permuted(A, x))
        reps.append(er)
        gs.append(len(Axs) % 2 == 0)
    vals = _sieve_device_batch(T, Axs, reps, gs, "fma")
    for Ax, er, g, v in zip(Axs, reps, gs, vals):
        dd = orc.calc_hafnian(Ax, er, g, sum_mode=1)
        tol = 4 * 2 * sum(er) * EPS * kappa(orc, Ax, er, g, dd) + 1e-15
        assert rel(v, dd) <= tol, (er, g, v, dd)
        assert rel(v, egg.sieve(Ax, er, glynn=g, prec="fma")) <= 1e-15


@pytest.mark.parametrize("cplx", [False, True])
def test_batch_sharing_multiplicity_patterns(egg, orc, W, cplx):
    """A batch whose repeated-row instances share multiplicity patterns (several matrices with one
    rpt, under each variant) takes their terms from one list per pattern and level; beside them a
    pattern held by one instance only, and a distinct-row instance.  Each result is the scalar
    call's, and within 4 N eps kappa of the oracle's double-double sum."""
    from theeggman_b200.hafnian import _sieve_device_batch

    T = np.dtype(np.complex128 if cplx else np.float64)
    Axs, reps, gs = [], [], []
    for i, rpt in enumerate([[2] * 8] * 6 + [[1, 3, 2, 2, 4]] * 4 + [[3, 1, 2, 2]]):
        d = len(rpt)
        A = W.dense_complex(d, 900 + i, 0.5) if cplx else W.dense_real(d, 900 + i)
        x, er = orc.matched_reps(rpt)
        Axs.append(orc.permuted(A, x))
        reps.append(er)
        gs.append(i % 2 == 1)
    A = W.dense_complex(14, 990, 0.5) if cplx else W.dense_real(14, 990)
    Axs.append(orc.permuted(A, distinct_x(7)))
    reps.append([1] * 7)
    gs.append(False)
    vals = _sieve_device_batch(T, Axs, reps, gs, "fma")
    for Ax, er, g, v in zip(Axs, reps, gs, vals):
        dd = orc.calc_hafnian(Ax, er, g, sum_mode=1)
        tol = 4 * 2 * sum(er) * EPS * kappa(orc, Ax, er, g, dd) + 1e-15
        assert rel(v, dd) <= tol, (er, g, v, dd)
        assert rel(v, egg.sieve(Ax, er, glynn=g, prec="fma")) <= 1e-14


@pytest.mark.parametrize("glynn", [False, True])
def test_two_rows_per_lane_tiles(egg, orc, W, glynn):
    """Real terms with 32 < m <= 48 run on tiles of two rows per lane (La Budde's table by two
    diagonals per lane): N = 34 puts every Glynn term, and the largest inclusion-exclusion terms,
    there.  Bar as for the other register-tile results: 4 N eps kappa against the oracle's
    double-double sum of the reference's terms."""
    N, E = 34, 17
    A = W.dense_real(N, 3434, scale=1.0 / np.sqrt(N))
    Ax = orc.permuted(A, distinct_x(E))
    dd = orc.calc_hafnian(Ax, [1] * E, glynn, nthreads=8, sum_mode=1)
    got = egg.sieve(Ax, [1] * E, glynn=glynn, prec="fma")
    assert rel(got, dd) <= 4 * N * EPS * kappa(orc, Ax, [1] * E, glynn, dd) + 1e-15, (got, dd)


def test_device_entry_point_orders_with_the_caller_stream(egg, W):
    """egg_sieve_device forks its latency-bound launches (small levels, and the exact kernel's share
    of terms too large for the register tiles) onto the library's side streams, and joins them back
    before the reduction.  So a matrix written on the caller's stream just before the call, and a
    copy of the result queued just after it, with no synchronisation in between, must give the host
    entry point's result to the bit."""
    import torch

    from theeggman_b200 import _native as nat

    L = nat.lib()
    dev = torch.device("cuda", 0)
    stream = torch.cuda.Stream(dev)
    for N, cplx in ((20, False), (40, False), (36, True)):
        E = N // 2
        A = W.dense_complex(N, 600 + N, 0.5) if cplx else W.dense_real(N, 600 + N, scale=1.0 / np.sqrt(N))
        Ax = A[np.ix_(np.array(distinct_x(E)) - 1, np.array(distinct_x(E)) - 1)]
        host = egg.sieve(Ax, [1] * E, prec="fma")
        src = torch.from_numpy(np.ascontiguousarray(Ax.T)).to(dev)  # column-major bytes
        dA = torch.zeros_like(src)
        out = torch.full((2,), float("nan"), dtype=torch.float64, device=dev)
        reps = np.ones(E, dtype=np.int64)
        torch.cuda.synchronize()
        with torch.cuda.stream(stream):
            dA.copy_(src)  # queued on the caller's stream, not yet done when the sieve is queued
            rc = L.egg_sieve_device(nat.EGG_C128 if cplx else nat.EGG_F64, 1, dA.data_ptr(), E, reps.ctypes.data, 0,
                                    out.data_ptr(), stream.cuda_stream)
            got = out.clone()  # queued right after
        stream.synchronize()
        assert rc == 0, L.egg_last_error()
        val = complex(got[0].item(), got[1].item()) if cplx else got[0].item()
        assert val == (complex(host) if cplx else float(host)), (N, val, host)


def test_config2_full_size_cross_check(egg, W):
    """N = 40 (E = 20, 2^20 inclusion-exclusion terms / 2^19 Glynn terms), both kernels: Glynn agrees
    with the device DP (machine precision, no cancellation) within the metric's 1e-10 (the
    reference's tighter 1e-12 envelope is quoted at N <= 24; here Glynn lands at ~3e-12-1e-11)."""
    A = W.dense_real(40, 2024, scale=1.0 / np.sqrt(40))
    dp = egg.hafnian(A, method="dp")
    for prec in ("exact", "fma"):
        ie = egg.hafnian(A, method="sieve", glynn=False, prec=prec)
        gl = egg.hafnian(A, method="sieve", glynn=True, prec=prec)
        assert rel(gl, dp) < 1e-10, prec
        # kappa ~ 2.9e8 for this matrix's inclusion-exclusion sum (sum|terms| / |hafnian|), so any
        # FP64 evaluation lands ~1e-9 away; the reference's own CPU result differs from the DP by 5e-10.
        assert rel(ie, dp) < 1e-8, prec
    egg.empty_gpu_cache()


# ---- prec="reference": the reference's summation order -----------------------------------------
# Every term in the reference's arithmetic (the exact kernel), summed as _sieve_sum does for the
# given thread count: nchunks = _sieve_chunks(work, steps, nthreads) chunks of the term range, each a
# plain FP64 sum from zero, the chunk sums folded left to right (src/hafnian.jl:607-622, :714-738).
# The bar is equality with the oracle's sum_mode 0, which restates that summation.

@pytest.mark.parametrize("cplx", [False, True])
@pytest.mark.parametrize("glynn", [False, True])
def test_reference_order_bit_identical(egg, orc, W, cplx, glynn):
    multi = False
    for N in (2, 8, 14, 20, 24, 30):
        A = W.dense_complex(N, 300 + N, 0.5) if cplx else W.dense_real(N, 300 + N)
        E = N // 2
        Ax = orc.permuted(A, distinct_x(E))
        work, steps = orc.sieve_variant_cost([1] * E, E, glynn)
        for k in (1, 3, 12, 64):
            multi |= orc.sieve_chunks(work, steps, k) > 1
            want = orc.calc_hafnian(Ax, [1] * E, glynn, nthreads=k, sum_mode=0)
            got = egg.sieve(Ax, [1] * E, glynn=glynn, prec="reference", nthreads=k)
            assert complex(got) == complex(want), (N, k, got, want)
    assert multi  # the sizes above reach the threaded (several-chunk) summation


@pytest.mark.parametrize("cplx", [False, True])
def test_reference_order_pivot_edge_cases(egg, orc, cplx):
    """Matrices of small integers (entries -2..2, a third of them zero): the Hessenberg pivots meet
    exact ties of magnitude (the first row of largest |entry| wins, src/hafnian.jl:212-221) and zero
    columns (the step is skipped, :231-232) at every size, on the register tiles (m <= 32) and the
    shared-memory kernel (m > 32, N = 34); the reference order must still be matched to the bit.
    Then a NaN and an infinity among the entries: the result is NaN exactly when the reference's
    is, and otherwise equal."""
    rng = np.random.default_rng(4242 + cplx)

    def draw(N):
        v = rng.choice([-2, -1, 0, 0, 1, 2], size=(N, N)).astype(float)
        if cplx:
            v = v + 1j * rng.choice([-1, 0, 0, 1], size=(N, N))
        return np.triu(v) + np.triu(v, 1).T

    for N in (6, 12, 20, 26, 34):
        for _ in range(2):
            A = draw(N)
            E = N // 2
            Ax = orc.permuted(A, distinct_x(E))
            for glynn in (False, True):
                want = orc.calc_hafnian(Ax, [1] * E, glynn, nthreads=1, sum_mode=0)
                got = egg.sieve(Ax, [1] * E, glynn=glynn, prec="reference", nthreads=1)
                assert complex(got) == complex(want), (N, glynn, got, want)
    for bad in (float("nan"), float("inf")):
        A = draw(12)
        A[3, 7] = A[7, 3] = bad
        Ax = orc.permuted(A, distinct_x(6))
        for glynn in (False, True):
            want = complex(orc.calc_hafnian(Ax, [1] * 6, glynn, nthreads=1, sum_mode=0))
            got = complex(egg.sieve(Ax, [1] * 6, glynn=glynn, prec="reference", nthreads=1))
            assert np.isnan(got) == np.isnan(want), (bad, glynn, got, want)
            if not np.isnan(want):
                assert got == want, (bad, glynn, got, want)


@pytest.mark.parametrize("cplx", [False, True])
def test_reference_order_repeated_rows(egg, orc, W, cplx):
    """hafnian_repeated's mixed-radix odometer, both variants, through the public entry point."""
    A = W.dense_complex(10, 91, 0.5) if cplx else W.dense_real(10, 91)
    for rpt in ([2, 3, 1, 0, 2, 2, 1, 3, 1, 1], [4, 4, 2, 2, 2, 2, 0, 0, 1, 1], [2] * 10):
        x, er = orc.matched_reps(rpt)
        Ax = orc.permuted(A, x)
        for glynn in (False, True):
            for k in (1, 7, 32):
                want = orc.calc_hafnian(Ax, er, glynn, nthreads=k, sum_mode=0)
                got = egg.hafnian_repeated(A, rpt, method="sieve", glynn=glynn, prec="reference", nthreads=k)
                assert complex(got) == complex(want), (rpt, glynn, k, got, want)


def test_reference_order_public_api(egg, orc, W):
    """hafnian(A; method, nthreads) end to end, the method choice included, and the batch form
    (each instance with one thread, as the reference's batch loop runs them)."""
    for N in (16, 22, 26):
        A = W.dense_real(N, 700 + N)
        for k in (1, 8, 12):
            for method in ("auto", "sieve"):
                want = orc.hafnian(A, method=method, nthreads=k)
                got = egg.hafnian(A, method=method, prec="reference", nthreads=k)
                assert complex(got) == complex(want), (N, k, method)
    mats = [W.dense_real(18, 800 + b) for b in range(3)]
    got = egg.hafnian(mats, method="sieve", prec="reference")
    want = [orc.hafnian(m, method="sieve", nthreads=1) for m in mats]
    assert [complex(g) for g in got] == [complex(w) for w in want]
    assert egg.sieve(np.zeros((0, 0)), [], prec="reference") == 1.0
