"""The public mirror on the device, following the reference's own testsets
(test/runtests.jl:50-220, :440-469, :544-578; test/gpu.jl:12-94)."""
import numpy as np
import pytest

from conftest import dec, dec_matrix

pytestmark = pytest.mark.gpu


def rel(a, b):
    return abs(complex(a) - complex(b)) / max(abs(complex(b)), 1e-300)


def test_closed_forms(egg, W):
    # test/runtests.jl:51-66
    assert egg.hafnian(np.zeros((0, 0))) == 1
    assert egg.hafnian(np.array([[0.0, 1.0], [1.0, 0.0]])) == 1.0
    A = np.array([[0, 1, 2, 3], [1, 0, 4, 5], [2, 4, 0, 6], [3, 5, 6, 0]])
    assert egg.hafnian(A) == 28.0
    assert egg.hafnian(A, exact=True) == 28
    B = W.dense_complex(8, 1, 0.5)
    C = B.copy()
    np.fill_diagonal(C, 3 * np.diag(B) + 7)
    assert egg.hafnian(B) == egg.hafnian(C)


def test_vs_golden_and_oracle(egg, orc, golden):
    # test/runtests.jl:75-83 against 256-bit gold; the DP path is bit-identical to the oracle
    for case in golden["random"]:
        A = dec_matrix(case["A"])
        g = dec(case["gold"])
        got = egg.hafnian(A, method="dp")
        assert got == orc.hafnian(A, method="dp"), case["N"]
        assert rel(got, g) < 1e-13
        assert rel(egg.hafnian(A), g) < 1e-9  # default strategy (DP or sieve by the cost model)


def test_element_types(egg, W):
    # test/runtests.jl:85-97
    A = W.dense_real(8, 4)
    assert isinstance(egg.hafnian(A), np.float64)
    assert isinstance(egg.hafnian(A.astype(np.complex128)), np.complex128)
    assert isinstance(egg.hafnian(A.astype(np.float32)), np.float32)
    assert isinstance(egg.hafnian(A.astype(np.complex64)), np.complex64)
    I8 = np.round(10 * A).astype(np.int64)
    assert rel(egg.hafnian(I8), egg.hafnian(I8.astype(float))) == 0


def test_strategies_agree(egg, W):
    # test/runtests.jl:193-220
    for N in range(2, 13, 2):
        A = W.dense_complex(N, 14 + N, 0.5)
        g = egg.hafnian(A, method="sieve", glynn=True)
        assert rel(egg.hafnian(A, method="unrolled"), g) < 1e-10
        assert rel(egg.hafnian(A, method="dp"), g) < 1e-10
    for N in (14, 16, 18):
        A = W.dense_complex(N, 114 + N, 0.5)
        assert rel(egg.hafnian(A, method="dp"), egg.hafnian(A, method="sieve", glynn=True)) < 1e-9
    for i, rpt in enumerate(([2, 2, 2], [1, 2, 3, 2], [2] * 6, [6, 6], [3, 3, 3, 3], [8, 4], [5, 5, 1, 1], [10, 2],
                             [12], [4, 4], [9, 3], [6, 2, 2, 2])):
        A = W.dense_complex(len(rpt), 300 + i, 0.5)
        s = egg.hafnian_repeated(A, rpt, method="sieve")
        assert rel(egg.hafnian_repeated(A, rpt, method="unrolled"), s) < 1e-10
        assert rel(egg.hafnian_repeated(A, rpt, method="dp"), s) < 1e-10
        assert rel(egg.hafnian_repeated(A, rpt), egg.hafnian(egg.reduction(A, rpt), method="dp")) < 1e-10


def test_repeated_consistency(egg, W):
    # test/runtests.jl:449-469
    A = W.dense_complex(6, 9, 0.5)
    assert rel(egg.hafnian_repeated(A, [1] * 6), egg.hafnian(A)) < 1e-12
    for rpt in ([2, 2, 2, 1, 1, 0], [3, 3, 2, 0, 0, 0]):
        assert rel(egg.hafnian_repeated(A, rpt), egg.hafnian(egg.reduction(A, rpt))) < 1e-10
    C = A.copy()
    C[0, 0] += 5
    assert rel(egg.hafnian_repeated(A, [2, 2, 1, 1, 0, 0]), egg.hafnian_repeated(C, [2, 2, 1, 1, 0, 0])) > 1e-8


def test_views_and_check_symmetric(egg, W):
    # test/runtests.jl:471-491, :544-563
    F = W.dense_complex(2 * 12 + 4, 19, 0.5)
    A = np.ascontiguousarray(F[:12, :12])
    base = egg.hafnian(A)
    for V in (F[:12, :12], F[2:14, 2:14], F[0:24:2, 0:24:2]):
        assert rel(egg.hafnian(V), egg.hafnian(np.array(V))) == 0
    assert egg.hafnian(A, check_symmetric=False) == base
    bad = W.dense_complex(8, 23, 0.5)
    bad[0, 1] += 1
    upper = bad.copy()
    iu = np.triu_indices(8, 1)
    upper[(iu[1], iu[0])] = upper[iu]
    assert egg.hafnian(bad, check_symmetric=False) == egg.hafnian(upper)


def test_batched_matches_scalar(egg, W):
    # test/gpu.jl:26-40
    be = egg.B200Backend()
    As = [W.dense_complex(16, 102 + b, 0.5) for b in range(7)]
    scalar = [egg.hafnian(A, backend=be) for A in As]
    assert np.array_equal(egg.hafnian(As, backend=be), scalar)
    for mb in (1, 2, 3, 100):
        assert np.array_equal(egg.hafnian(As, backend=be, max_batch=mb), scalar)
    assert np.array_equal(egg.hafnian(As[:1], backend=be), scalar[:1])
    assert len(egg.hafnian([], backend=be)) == 0


def test_batched_repeated_matches_scalar(egg, W):
    # test/gpu.jl:42-56
    be = egg.B200Backend()
    A = W.dense_complex(16, 103, 0.5)
    rpts = [[2, 2, 2, 1, 1, 0, 0, 0, 1, 1, 2, 2, 1, 1, 0, 0], [1] * 16, [4, 4, 4, 4] + [0] * 12]
    scalar = [egg.hafnian_repeated(A, r, backend=be, method="dp") for r in rpts]
    assert np.array_equal(egg.hafnian_repeated(A, rpts, backend=be), scalar)
    assert np.array_equal(egg.hafnian_repeated(A, rpts, backend=be, max_batch=2), scalar)
    # without a backend each pattern picks its own strategy (the loop of :1355-1358)
    loop = [egg.hafnian_repeated(A, r, nthreads=1) for r in rpts]
    assert np.allclose(egg.hafnian_repeated(A, rpts), loop, rtol=1e-12, atol=0)


def test_complex64_path(egg, W):
    # test/gpu.jl:58-69
    be = egg.B200Backend()
    for N in (12, 16, 20):
        A = W.dense_complex(N, 104 + N, 0.5)
        v32 = egg.hafnian(A.astype(np.complex64), backend=be)
        v64 = egg.hafnian(A, backend=be)
        assert isinstance(v32, np.complex64)
        assert rel(v32, v64) < 1e-5


def test_integer_exact_er_graph(egg, orc, W):
    for N in (16, 20, 24):
        G = W.er_graph(N, 0.5, N)
        assert egg.hafnian(G, exact=True, method="dp") == orc.dp_int128(G)


def test_determinism(egg, W):
    # test/gpu.jl:88-94
    be = egg.B200Backend()
    A = W.dense_complex(18, 106, 0.5)
    assert egg.hafnian(A, backend=be) == egg.hafnian(A, backend=be)
    As = [W.dense_complex(18, 206 + b, 0.5) for b in range(4)]
    assert np.array_equal(egg.hafnian(As, backend=be), egg.hafnian(As, backend=be))
