"""Mixed-degree batches (egg_dp_mix, hafnian_submatrices) against per-instance DP calls and the
oracle: every result must equal hafnian(A[r, r]; method=:dp) of the same precision mode."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def nat(egg):
    from theeggman_b200 import _native

    assert _native.lib().egg_init(0) == 0, "no CUDA device"
    return _native


@pytest.fixture
def level_engine(nat):
    """Runs a test on the per-level engine (launch per level, graph replay), then restores the default."""
    L = nat.lib()
    prev = L.egg_dp_mix_engine()
    nat.check(L.egg_dp_mix_set_engine(0))
    yield
    nat.check(L.egg_dp_mix_set_engine(prev))


def _sub(A, r):
    r = np.asarray(r, dtype=np.int64)
    return A[np.ix_(r, r)]


def _mix(W, B, n, sizes, seed):
    rng = np.random.default_rng(seed)
    return [rng.choice(n, size=int(rng.choice(sizes)), replace=False) for _ in range(B)]


@pytest.mark.parametrize("cplx", [False, True])
def test_mix_equals_single_calls(egg, W, orc, cplx):
    n = 40
    A = W.gbs_parent(n, 11) if cplx else W.dense_real(n, 12)
    rows = _mix(W, 60, n, [0, 1, 2, 3, 4, 6, 8, 11, 12, 16, 20, 22, 24, 26], 5)
    got = egg.hafnian_submatrices(A, rows, check_symmetric=False)
    for b, r in enumerate(rows):
        k = len(r)
        if k == 0:
            assert got[b] == 1
        elif k % 2:
            assert got[b] == 0
        else:
            assert got[b] == egg.hafnian(_sub(A, r), method="dp", check_symmetric=False), (b, k)
    # the oracle on a few instances (bit-identical in the exact mode)
    plan_cache = {}
    for b, r in enumerate(rows[:12]):
        k = len(r)
        if k < 2 or k % 2:
            continue
        plan = plan_cache.setdefault(k, orc.build_plan(k, 4))
        P = orc.gather_pairs(np.asarray(A), [int(i) + 1 for i in r], k)
        assert got[b] == orc.haf_dp_pairs(P, plan, orc.C128 if cplx else orc.F64), (b, k)


def test_mix_repeated_rows_and_modes(egg, W):
    n = 24
    A = W.gbs_parent(n, 21)
    rows = [[0, 0, 1, 2], [3, 3, 3, 3, 5, 6], list(range(20)), [7, 8], [1, 2, 3, 4, 5, 6, 7, 8, 9, 10]]
    got = egg.hafnian_submatrices(A, rows, check_symmetric=False)
    for b, r in enumerate(rows):
        assert got[b] == egg.hafnian(_sub(A, r), method="dp", check_symmetric=False)
    fma = egg.hafnian_submatrices(A, rows, check_symmetric=False, prec="fma")
    mixed = egg.hafnian_submatrices(A, rows, check_symmetric=False, prec="mixed")
    for b in range(len(rows)):
        assert abs(fma[b] - got[b]) <= 1e-12 * abs(got[b])
        assert abs(mixed[b] - got[b]) <= 1e-5 * abs(got[b])


def test_mix_integer_parent_exact(egg, W, orc):
    n = 30
    G = W.er_graph(n, 0.5, 31)
    rows = _mix(W, 25, n, [2, 4, 10, 16, 20], 9)
    got = egg.hafnian_submatrices(G, rows, exact=True, check_symmetric=False)
    for b, r in enumerate(rows):
        assert got[b] == orc.dp_int128(_sub(G, r)), b


def test_mix_gbs_shape(egg, W):
    # The configuration-4 generator at a reduced count: degrees 8..32, distinct rows of the
    # 64 x 64 parent; every result equals its single call.
    A, idxs = W.gbs_mix(96, 64, range(8, 33, 2), 4)
    got = egg.hafnian_submatrices(A, idxs, check_symmetric=False)
    for b in range(0, 96, 7):
        assert got[b] == egg.hafnian(_sub(A, idxs[b]), method="dp", check_symmetric=False), b
    again = egg.hafnian_submatrices(A, idxs, check_symmetric=False)
    assert np.array_equal(got, again)


def test_mix_refusals(egg, W):
    A = W.dense_real(10, 3)
    with pytest.raises(egg.ArgumentError):
        egg.hafnian_submatrices(A, [[0, 1], [2, 10]], check_symmetric=False)
    with pytest.raises(egg.ArgumentError):
        egg.hafnian_submatrices(A, [[0, -1]], check_symmetric=False)
    assert len(egg.hafnian_submatrices(A, [], check_symmetric=False)) == 0


@pytest.mark.parametrize("prec", ["exact", "fma", "mixed"])
def test_mix_evaluations_agree(egg, nat, W, prec, level_engine):
    # Degrees past the whole-instance kernel, pinned to each evaluation in turn: batched groups of
    # several sizes and grouped single instances must give the same bits.
    import ctypes

    n = 40
    A = W.gbs_parent(n, 41)
    rng = np.random.default_rng(77)
    rows = [rng.choice(n, size=k, replace=False) for k in [24, 26, 24, 28, 26, 24, 26, 28, 24, 30, 26, 28, 24]]
    L = nat.lib()
    results = []
    for batched, group in [(1, 64), (1, 2), (0, 1), (0, 3), (0, 16)]:
        for K in (24, 26, 28, 30):
            nat.check(L.egg_dp_mix_set_tuning(K, nat.EGG_C128, nat.PREC[prec], batched, group))
        results.append(egg.hafnian_submatrices(A, rows, check_symmetric=False, prec=prec))
        b, g = ctypes.c_int(), ctypes.c_int64()
        nat.check(L.egg_dp_mix_tuning(26, nat.EGG_C128, nat.PREC[prec], ctypes.byref(b), ctypes.byref(g)))
        assert (b.value, g.value) == (batched, group)
    for r in results[1:]:
        assert np.array_equal(r, results[0])
    if prec == "exact":
        for b, r in enumerate(rows):
            assert results[0][b] == egg.hafnian(_sub(A, r), method="dp", check_symmetric=False)


def test_mix_graph_replay(egg, nat, W, level_engine):
    # The second call of a shape records a graph and later calls replay it: results must not
    # change, including when the row sets change but the degree counts do not.
    A = W.gbs_parent(48, 51)
    rng = np.random.default_rng(3)
    sizes = [8, 10, 24, 26, 24, 12, 26, 9, 0, 28]
    rows1 = [rng.choice(48, size=k, replace=False) for k in sizes]
    rows2 = [rng.choice(48, size=k, replace=False) for k in sizes]
    L = nat.lib()
    first = egg.hafnian_submatrices(A, rows1, check_symmetric=False)
    n0 = L.egg_launch_count()
    second = egg.hafnian_submatrices(A, rows1, check_symmetric=False)
    n1 = L.egg_launch_count()
    third = egg.hafnian_submatrices(A, rows1, check_symmetric=False)
    n2 = L.egg_launch_count()
    other = egg.hafnian_submatrices(A, rows2, check_symmetric=False)
    assert np.array_equal(first, second) and np.array_equal(first, third)
    assert n2 - n1 == n1 - n0 > 0  # a replay counts the kernels it runs
    for b, r in enumerate(rows2):
        exp = egg.hafnian(_sub(A, r), method="dp", check_symmetric=False) if len(r) else 1
        assert other[b] == exp, b


def test_tuner_choice_persists_across_processes(tmp_path):
    """The tuner writes its per-degree choice to the tuning file, and a later process on the same
    GPU model starts from it without timing again (egg_dp_mix_tuning answers before any batch)."""
    import json
    import os
    import subprocess
    import sys

    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    script = f"""
import ctypes, json, sys
sys.path.insert(0, {root!r}); sys.path.insert(0, {os.path.join(root, 'tests')!r})
from conftest import load_package
egg = load_package()
from theeggman_b200 import workloads as W, _native as nat
L = nat.lib()
assert L.egg_dp_mix_set_engine(0) == 0  # the per-level engine is the one that tunes
if sys.argv[1] == "tune":
    A, idxs = W.gbs_mix(8, 64, [24], 4)
    egg.hafnian_submatrices(A, idxs)
b, g = ctypes.c_int(), ctypes.c_int64()
rc = L.egg_dp_mix_tuning(24, 1, 0, ctypes.byref(b), ctypes.byref(g))
print(json.dumps([rc, b.value, g.value]))
"""
    path = tmp_path / "tuning" / "mix_tuning.json"
    env = dict(os.environ, EGG_TUNE_CACHE=str(path))
    runs = []
    for mode in ("tune", "read"):
        r = subprocess.run([sys.executable, "-c", script, mode], env=env, capture_output=True, text=True, timeout=300)
        assert r.returncode == 0, r.stderr[-2000:]
        runs.append(json.loads(r.stdout.strip().splitlines()[-1]))
        if mode == "tune":
            text = path.read_text()
            assert '"K": 24' in text and '"dtype": 1' in text, text
    assert runs[0][0] == 0 and runs[1] == runs[0], runs


def _engine_results(egg, nat, engine, fn):
    L = nat.lib()
    prev = L.egg_dp_mix_engine()
    nat.check(L.egg_dp_mix_set_engine(engine))
    try:
        n0 = L.egg_launch_count()
        out = fn()
        return out, L.egg_launch_count() - n0
    finally:
        nat.check(L.egg_dp_mix_set_engine(prev))


@pytest.mark.parametrize("dtype,prec", [("f64", "exact"), ("f64", "fma"), ("f64", "mixed"), ("c128", "exact"),
                                        ("c128", "fma"), ("c128", "mixed"), ("int", "exact")])
def test_persistent_engine_equals_level_engine(egg, nat, W, dtype, prec):
    """One cooperative launch per call (egg_mix_persist.cu) gives the per-level engine's bits, for
    every element type and precision mode, on a mix of every degree 0..32 with odd sizes, empty row
    sets and repeated rows."""
    n = 48
    if dtype == "int":
        A = W.er_graph(n, 0.5, 61)
    elif dtype == "c128":
        A = W.gbs_parent(n, 62)
    else:
        A = W.dense_real(n, 63)
    rng = np.random.default_rng(64)
    sizes = list(range(0, 33)) * 3
    rows = [rng.choice(n, size=k, replace=False) for k in sizes]
    rows += [[0, 0, 1, 1], [5, 5, 5, 5, 7, 9]]
    kw = dict(check_symmetric=False)
    if dtype == "int":
        kw["exact"] = True
    else:
        kw["prec"] = prec
    lev, nl = _engine_results(egg, nat, 0, lambda: egg.hafnian_submatrices(A, rows, **kw))
    per, npers = _engine_results(egg, nat, 1, lambda: egg.hafnian_submatrices(A, rows, **kw))
    assert np.array_equal(per, lev)
    assert npers == 1 and nl > 1, (npers, nl)
    if dtype != "int" and prec == "exact":
        for b in range(0, len(rows), 9):
            r = rows[b]
            exp = egg.hafnian(_sub(A, r), method="dp", check_symmetric=False) if len(r) else 1
            assert per[b] == exp, b


def test_persistent_engine_waves(egg, nat, W):
    """A mix whose level buffers exceed the persistent launch's budget runs in waves of instances
    (600 instances of degree 32 in Float64: two waves): same bits as the per-level engine."""
    A = W.dense_real(40, 71)
    rng = np.random.default_rng(72)
    rows = [rng.choice(40, size=32, replace=False) for _ in range(600)]
    rows += [rng.choice(40, size=k, replace=False) for k in (30, 28, 8, 2, 0, 31)]
    lev, _ = _engine_results(egg, nat, 0, lambda: egg.hafnian_submatrices(A, rows, check_symmetric=False))
    per, npers = _engine_results(egg, nat, 1, lambda: egg.hafnian_submatrices(A, rows, check_symmetric=False))
    assert npers == 1
    assert np.array_equal(per, lev)
    # Only odd and empty row sets: no degree bin, the launch only scatters.
    rows = [[1], [], [2, 3, 4], []]
    per, npers = _engine_results(egg, nat, 1, lambda: egg.hafnian_submatrices(A, rows, check_symmetric=False))
    assert npers == 1 and list(per) == [0.0, 1.0, 0.0, 1.0]


def test_persistent_engine_device_entry(egg, nat, W):
    """egg_dp_mix_device on the persistent engine equals the host entry; the engine switch refuses
    other values."""
    import torch

    A = W.gbs_parent(40, 81)
    rng = np.random.default_rng(82)
    rows = [rng.choice(40, size=k, replace=False) for k in (24, 26, 8, 0, 3, 28)]
    host = egg.hafnian_submatrices(A, rows, check_symmetric=False)
    offs = np.zeros(len(rows) + 1, dtype=np.int64)
    offs[1:] = np.cumsum([len(r) for r in rows])
    flat = np.concatenate([np.asarray(r, dtype=np.int32) for r in rows])
    dev = torch.device("cuda", 0)
    dA = torch.from_numpy(np.asfortranarray(A).ravel(order="F").view(np.float64).copy()).to(dev)
    drows = torch.from_numpy(flat).to(dev)
    dout = torch.empty(2 * len(rows), dtype=torch.float64, device=dev)
    L = nat.lib()
    st = torch.cuda.Stream(dev)  # a stream of the caller's (the legacy default stream would be handle 0)
    st.wait_stream(torch.cuda.current_stream(dev))
    nat.check(L.egg_dp_mix_device(nat.EGG_C128, 0, dA.data_ptr(), 40, len(rows), nat.ptr(offs), drows.data_ptr(),
                                  dout.data_ptr(), st.cuda_stream))
    st.synchronize()
    got = dout.cpu().numpy().view(np.complex128)
    assert np.array_equal(got, host)
    with pytest.raises(egg.ArgumentError):
        nat.check(L.egg_dp_mix_set_engine(2))


def test_barrier_bounded_wait(egg, nat):
    """The persistent launch's grid barrier: with every block present it passes; made to expect one
    block more than the grid has, each wait runs out after its limit, the launch still ends, the
    call reports EGG_ERR_TIMEOUT, and the device stays usable."""
    import ctypes

    L = nat.lib()
    passes = ctypes.c_int64(0)
    nat.check(L.egg_selfcheck_barrier(0, 200_000_000, ctypes.byref(passes)))
    assert passes.value > 0 and passes.value % 3 == 0
    rc = L.egg_selfcheck_barrier(1, 20_000_000, ctypes.byref(passes))
    assert rc == nat.EGG_ERR_TIMEOUT, rc
    assert b"ran out" in L.egg_last_error()
    with pytest.raises(egg.ArgumentError):
        nat.check(L.egg_selfcheck_barrier(0, 10, None))
    A = np.array([[0.0, 2.0], [2.0, 0.0]])
    assert egg.hafnian_submatrices(A, [[0, 1]], check_symmetric=False)[0] == 2.0
