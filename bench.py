"""Benchmark: hafnians/s on B200 for TheEggman.jl's hot paths.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference] [--workload NAME]

The default workload is the N = 40 sieve of configuration 2(a): one real symmetric 40 x 40 matrix
with entries U[-1, 1]/sqrt(40), hafnian(A; method = :sieve), which the reference runs as
inclusion-exclusion (2^20 terms; its cost model's choice for distinct rows), every term in the
reference's arithmetic (the API default).  A step is one full hafnian.  The default run then times
every other configuration of the metric in the same process (the `per_config` list).  Under torchrun every rank computes its own matrix (seed + rank): the sieve instances are
independent, so N GPUs run N replicas with no data-path collective ("scaling": "weak"); the only
collectives are the timing barrier and the max-over-ranks reduction.

Reported:
  value      hafnians/s over all ranks, inputs resident in HBM, device time (CUDA events on the
             launching stream, max over ranks), L2 flushed between steps (256 MiB write outside
             the timed events);
  e2e        the same metric through the public API (host matrix in, host value out: the
             host->device copy of the matrix and the device->host read of the result are inside
             the timed region);
  roofline   the dominant kernel's algorithmic FP64 flop rate against the FP64 peak;
  cpu_baseline  the oracle's restatement of the reference algorithm on this host's cores.
"""
from __future__ import annotations

import argparse
import importlib.util
import json
import os
import statistics
import subprocess
import sys
import tempfile
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
METRIC = "hafnians/s at N=20/32/40 + batched mix, 1 B200, rel err ≤1e-10 vs plain FP64"


def load_package():
    if "theeggman_b200" in sys.modules:
        return sys.modules["theeggman_b200"]
    d = os.path.join(ROOT, "theeggman.jl_b200")
    spec = importlib.util.spec_from_file_location("theeggman_b200", os.path.join(d, "__init__.py"),
                                                  submodule_search_locations=[d])
    mod = importlib.util.module_from_spec(spec)
    sys.modules["theeggman_b200"] = mod
    spec.loader.exec_module(mod)
    return mod


def measured_peaks() -> dict:
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            return json.load(f)
    except OSError:
        return {}


def rel_err(a, b) -> float:
    """|a - b| / |b| (complex-aware; integers exactly)."""
    if isinstance(a, int) and isinstance(b, int):
        return 0.0 if a == b else abs(a - b) / max(abs(b), 1)
    a, b = complex(a), complex(b)
    if a == b:
        return 0.0
    return abs(a - b) / max(abs(b), 1e-300)


# The committed ncu summary (kernel and workload) whose DRAM traffic figure belongs to a workload.
PROFILE_OF = {"sieve40": "sieve_level_kernel_exact_sieve40.md", "sieve40f": "sieve_level_kernel_sieve40.md",
              "sieve40c": "sieve_level_kernel_exact_sieve40c.md",
              "sieve40cf": "sieve_level_kernel_sieve40c.md", "sieve40gf": "sieve_level_kernel_sieve40g.md",
              "rep14f": "sieve_level_kernel_rep14.md", "dp40": "dpc_fixed_kernel_dp40.md",
              "dp20": "dpc_cluster_kernel_dp20.md", "mix4096": "dpc_fixed_kernel_mix4096.md"}


def profile_traffic(name: str):
    """DRAM bytes per launch from a committed ncu summary (a line `dram_bytes_per_launch: X`)."""
    p = os.path.join(ROOT, "profiles", name)
    try:
        for line in open(p):
            if line.startswith("dram_bytes_per_launch:"):
                return float(line.split(":", 1)[1].strip())
    except OSError:
        pass
    return None


# ------------------------------------------------------------------------------------------------
# Workloads
# ------------------------------------------------------------------------------------------------

class SieveWorkload:
    """One N x N sieve hafnian per step (configuration 2: N = 40, real or complex; configuration 1's
    sieve run: N = 20 real U[-1,1])."""

    kind = "sieve"

    def __init__(self, egg, W, N: int, cplx: bool, glynn, seed: int, config: str = "2", prec: str = "exact"):
        from theeggman_b200 import policy as pol
        from theeggman_b200 import roofline as R

        self.egg, self.N, self.cplx = egg, N, cplx
        self.forced_glynn = glynn is not None
        E = N // 2
        self.E = E
        if config == "1":
            self.A = W.dense_real(N, seed)
        else:
            self.A = (W.dense_complex(N, seed, 1.0 / (2 * N)) if cplx else W.dense_real(N, seed, scale=1.0 / np.sqrt(N)))
        sel_glynn = pol._choose_method_distinct(N, E, os.cpu_count() or 1)[1]
        self.glynn = sel_glynn if glynn is None else glynn
        x = [2 * i + 1 for i in range(E)] + [2 * i + 2 for i in range(E)]
        xi = np.array(x) - 1
        self.Ax = np.asfortranarray(self.A[np.ix_(xi, xi)])
        self.reps = np.ones(E, dtype=np.int64)
        self.flops = R.sieve_flops([1] * E, self.glynn, cplx)
        self.dtype = 1 if cplx else 0
        # "exact": every term in the reference's arithmetic (the API default); "fma": the register
        # tiles with fused multiply-adds.
        self.prec_name = prec
        self.prec = {"exact": 0, "fma": 1}[prec]
        self.hafnians_per_step = 1
        self.dtype_name = "c128" if cplx else "f64"
        label = ("config1: N=20 Float64 U[-1,1]" if config == "1" else
                 f"config2{'b' if cplx else 'a'}: N={N} {'ComplexF64 N(0,1/(2N)) parts' if cplx else 'Float64 U[-1,1]/sqrt(N)'}")
        self.name = (f"{label}, "
                     f"hafnian(A; method=:sieve) = {'Glynn' if self.glynn else 'inclusion-exclusion'}, "
                     f"{2 ** (E - 1) if self.glynn else 2 ** E} terms")

    def setup_device(self, torch, dev):
        ct = torch.complex128 if self.cplx else torch.float64
        self.dAx = torch.from_numpy(np.ascontiguousarray(self.Ax.T)).to(dev, ct)  # column-major bytes
        self.dout = torch.zeros(1, dtype=ct, device=dev)

    def step_device(self, stream_ptr):
        L = self.egg.lib()
        rc = L.egg_sieve_device(self.dtype, self.prec, self.dAx.data_ptr(), self.E, self.reps.ctypes.data,
                                int(self.glynn), self.dout.data_ptr(), stream_ptr)
        if rc:
            raise RuntimeError(L.egg_last_error().decode())

    def step_e2e(self):
        # The public call with its defaults (symmetry check included); the variant is left to the
        # cost model unless the workload forces one, and prec is passed only when not the default.
        kw = {"glynn": self.glynn} if self.forced_glynn else {}
        if self.prec_name != "exact":
            kw["prec"] = self.prec_name
        return self.egg.hafnian(self.A, method="sieve", **kw)

    def device_result(self):
        v = self.dout.cpu().numpy()[0]
        return [complex(v) if self.cplx else float(v)]

    def check(self, O, dev_vals, e2e_val):
        """The timed result against the oracle: the reference's own plain FP64 summation (all host
        threads, the reference's default) and the double-double sum of the reference's terms."""
        plain = O.calc_hafnian(self.Ax, [1] * self.E, self.glynn, nthreads=O.max_threads(), sum_mode=0)
        dd = O.calc_hafnian(self.Ax, [1] * self.E, self.glynn, nthreads=O.max_threads(), sum_mode=1)
        got = dev_vals[0]
        return {"vs_reference_plain_fp64": rel_err(got, plain), "vs_reference_terms_dd": rel_err(got, dd),
                "e2e_vs_device": rel_err(e2e_val, got), "bar": 1e-10,
                "reference": "oracle calc_hafnian (src/hafnian.jl:684-738), plain FP64 sum with "
                             f"nthreads={O.max_threads()}, and the double-double sum of the same terms"}


    @property
    def h2d_bytes(self):
        return self.Ax.nbytes + 8 * self.E + 64

    @property
    def d2h_bytes(self):
        return 16 if self.cplx else 8

    def roofline(self, ms, peaks):
        from theeggman_b200 import roofline as R

        sm_max = float(peaks.get("sm_max_mhz", 1965.0))
        peak = R.fp64_nominal_tflops(sm_max)
        achieved = self.flops / (ms / 1e3) / 1e12
        roof = {"bound": "fp64", "achieved": achieved, "peak": peak, "unit": "TFLOP/s", "frac": achieved / peak,
                "peak_source": f"nominal FP64: 148 SMs x 64 FMA/clk x 2 x {sm_max:.0f} MHz (no FP64 figure in "
                               "MEASURED_PEAKS.json)",
                "work": f"{self.flops:.4e} algorithmic flops per hafnian"}
        if getattr(self, "prec_name", "fma") == "exact":
            # The reference rounds every product and every sum, so each algorithmic FMA issues as a
            # multiply and an add: the form's own ceiling is half the nominal rate.
            roof["separate_rounding_peak"] = peak / 2
            roof["frac_of_separate_rounding_peak"] = achieved / (peak / 2)
        return roof

    def cpu_sample(self, nthreads):
        from oracle import oracle as O

        O.calc_hafnian(self.Ax, [1] * self.E, self.glynn, nthreads=nthreads)  # warm the thread pool
        t = time.perf_counter()
        O.calc_hafnian(self.Ax, [1] * self.E, self.glynn, nthreads=nthreads)
        return 1.0 / (time.perf_counter() - t), "one full hafnian of the same workload (every sieve term), all host threads"


class DPWorkload:
    """B hafnians of degree N per step through the subset DP (configurations 1 and 3)."""

    kind = "dp"

    def __init__(self, egg, W, N: int, B: int, kind: str, prec: str, seed: int):
        from theeggman_b200.hafnian import _gather_pairs_batch

        self.egg, self.N, self.B, self.prec_name = egg, N, B, prec
        self.code = {"f64": 0, "c128": 1, "i64": 4}[kind]
        self.prec = {"exact": 0, "fma": 1, "mixed": 2}[prec]
        T = {"f64": np.float64, "c128": np.complex128, "i64": np.int64}[kind]
        self.T = np.dtype(T)
        if kind == "i64":
            self.mats = [W.er_graph(N, 0.5, seed + b) for b in range(B)]
        elif kind == "c128":
            self.mats = [W.dense_complex(N, seed + b, 1.0 / (2 * N)) for b in range(B)]
        elif N >= 36:
            self.mats = [W.dense_real(N, seed + b, 0.0, 1.0) for b in range(B)]
        else:
            self.mats = [W.dense_real(N, seed + b) for b in range(B)]
        self.P = _gather_pairs_batch(T, np.stack(self.mats), np.tile(np.arange(N), (B, 1)), N)
        self.hafnians_per_step = B
        self.dtype_name = {"f64": "f64", "c128": "c128", "i64": "int64->int128"}[kind]
        dist = {"f64": "Float64 U[0,1]" if N >= 36 else "Float64 U[-1,1]", "c128": "ComplexF64 N(0,1/(2N)) parts",
                "i64": "0/1 Erdos-Renyi p=0.5 adjacency, Int128"}[kind]
        self.name = f"DP N={N} B={B} {dist}, prec={prec}"
        self.vbytes = {"f64": 8, "c128": 16, "i64": 8}[kind]
        if prec == "mixed":
            self.vbytes //= 2  # states and pairs are stored in FP32

    def setup_device(self, torch, dev):
        from theeggman_b200.hafnian import _dp_plan

        self.key = _dp_plan(self.N)
        tdt = {np.dtype(np.float64): torch.float64, np.dtype(np.complex128): torch.complex128,
               np.dtype(np.int64): torch.int64}[self.T]
        self.dP = torch.from_numpy(np.ascontiguousarray(self.P.T)).to(dev, tdt)
        self.dout = torch.zeros(2 * self.B, dtype=torch.float64, device=dev)

    def step_device(self, stream_ptr):
        L = self.egg.lib()
        rc = L.egg_dp_batch_device(self.key[0], self.key[1], self.code, self.prec, self.dP.data_ptr(), self.B,
                                   self.dout.data_ptr(), stream_ptr)
        if rc:
            raise RuntimeError(L.egg_last_error().decode())

    def step_e2e(self):
        kw = {"exact": True} if self.code == 4 else {}
        if self.prec_name != "exact":
            kw["prec"] = self.prec_name
        if self.B == 1:
            return self.egg.hafnian(self.mats[0], method="dp", **kw)
        return self.egg.hafnian(self.mats, method="dp", backend=self.egg.B200Backend(), **kw)

    def device_result(self):
        raw = self.dout.cpu().numpy()
        if self.code == 4:  # Int128, little-endian pairs of 64-bit words
            u = raw.view(np.uint64)
            vals = []
            for b in range(self.B):
                v = int(u[2 * b]) | (int(u[2 * b + 1]) << 64)
                vals.append(v - (1 << 128) if v >= (1 << 127) else v)
            return vals
        if self.code == 1:
            return list(raw.view(np.complex128)[: self.B])
        return list(raw[: self.B])

    def check(self, O, dev_vals, e2e_val):
        """The timed results against the oracle's restatement of the reference DP (plan-free walk of
        the same states and order above N = 28), in FP64 (Int128 for integer graphs).  The mixed
        form is compared with the FP64 value."""
        nb = min(self.B, 4)
        dt = {0: O.F64, 1: O.C128, 4: O.I64}[self.code]
        worst = 0.0
        for b in range(nb):
            P = O.gather_pairs(self.mats[b], list(range(1, self.N + 1)), self.N)
            want = O.haf_dp_closed(P, self.N, dt, O.max_threads())
            worst = max(worst, rel_err(dev_vals[b], want))
        e2e0 = e2e_val if self.B == 1 else e2e_val[0]
        return {"max_vs_reference_fp64": worst, "instances_checked": nb, "e2e_vs_device": rel_err(e2e0, dev_vals[0]),
                "bar": 1e-10 if self.prec_name == "mixed" else 0.0,
                "reference": "oracle DP (src/dp.jl:344-442) in the reference's order and rounding"
                             + (", Int128" if self.code == 4 else "")}

    @property
    def h2d_bytes(self):
        return sum(m.nbytes for m in self.mats)

    @property
    def d2h_bytes(self):
        return self.B * (16 if self.code in (1, 4) else 8)

    def roofline(self, ms, peaks):
        return dp_roofline([(self.N, self.B)], self.vbytes, ms, peaks)

    def cpu_sample(self, nthreads):
        from oracle import oracle as O
        from theeggman_b200 import policy as pol

        if self.N > 32:
            # A CPU plan at this degree is gigabytes (24 GB of transitions at N = 40): time the
            # reference loop on the N = 32 plan and scale by the transition counts.
            Ns = 32
            A = self.mats[0][:Ns, :Ns].astype(np.float64 if self.code != 4 else np.int64)
            dt = O.F64 if self.code != 4 else O.I64
            plan = O.build_plan(Ns, 4)
            P = O.gather_pairs(A, list(range(1, Ns + 1)), Ns)
            O.haf_dp_pairs(P, plan, dt, nthreads)
            t = time.perf_counter()
            O.haf_dp_pairs(P, plan, dt, nthreads)
            dtm = time.perf_counter() - t
            scale = pol._dp_counts(self.N)[1] / pol._dp_counts(Ns)[1]
            return 1.0 / (dtm * scale), (f"the reference DP loop on the N={Ns} plan ({dtm * 1e3:.1f} ms), scaled by "
                                         f"the transition count to N={self.N} (x{scale:.1f})")
        plan = O.build_plan(self.N, 4)
        nb = min(self.B, 64)
        dt = {0: O.F64, 1: O.C128, 4: O.I64}[self.code]
        Psub = np.asfortranarray(self.P[:nb])
        O.haf_dp_batch(Psub, plan, dt, nthreads)
        t = time.perf_counter()
        O.haf_dp_batch(Psub, plan, dt, nthreads)
        return nb / (time.perf_counter() - t), f"{nb} instances through the reference's batch loop, all host threads"


def dp_roofline(bins, vbytes, ms, peaks):
    """HBM roofline of closed-form DP levels over (degree, instances) bins: compulsory bytes (each
    state written once and read once, plus the pairs; no transition array exists to stream), with
    the child-load bytes beside them."""
    from theeggman_b200 import roofline as R

    byts = sum(R.dp_bytes_closed(K, B, vbytes) for K, B in bins)
    gath = sum(R.dp_gather_bytes(K, B, vbytes) for K, B in bins)
    peak = float(peaks.get("hbm_gbs", 6650.0))
    achieved = byts / (ms / 1e3) / 1e9
    return {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak,
            "peak_source": "MEASURED_PEAKS.json hbm_gbs" if "hbm_gbs" in peaks else "fallback 6650 GB/s",
            "work": f"{byts:.4e} compulsory bytes per step (every state written once and read once, plus the pairs; "
                    "closed-form plan, so no transition array is read)",
            "child_load_bytes_per_step": gath, "child_load_GBps": gath / (ms / 1e3) / 1e9}


class MixWorkload:
    """Configuration 4: B hafnians of principal submatrices of one 64 x 64 complex GBS parent, each
    of an even degree uniform in {8, ..., 32} with distinct rows, all in one call per step
    (egg_dp_mix_device; `seq` instead makes one single-instance DP call per hafnian, the
    one-at-a-time GPU path the batched form is compared with)."""

    kind = "dp"

    def __init__(self, egg, W, B: int, prec: str, seq: bool, seed: int, engine: int = 0):
        from theeggman_b200.hafnian import _mix_layout

        self.egg, self.B, self.prec_name, self.seq, self.engine = egg, B, prec, seq, engine
        self.prec = {"exact": 0, "fma": 1, "mixed": 2}[prec]
        self.A, self.idxs = W.gbs_mix(B, 64, range(8, 33, 2), seed)
        self.offsets, self.flat = _mix_layout(self.idxs)
        self.hafnians_per_step = B
        self.dtype_name = "c128"
        self.vbytes = 8 if prec == "mixed" else 16
        degs = np.bincount([len(r) for r in self.idxs], minlength=65)
        self.bins = [(K, int(degs[K])) for K in range(2, 65, 2) if degs[K]]
        self.name = (f"config4: {B} hafnians of A[r, r], A = U diag(tanh r) U^T 64x64 complex (U Haar), |r| even "
                     f"uniform in 8..32, distinct rows; prec={prec}; "
                     + ("one single-instance DP call per hafnian" if seq else
                        "one egg_dp_mix call per step, " + ("one cooperative launch" if engine == 1 else
                                                            "per-level launches replayed as a CUDA graph")))

    def setup_device(self, torch, dev):
        from theeggman_b200.hafnian import _dp_plan, _gather_pairs_batch

        self.dA = torch.from_numpy(np.ascontiguousarray(self.A.T)).to(dev, torch.complex128)
        self.drows = torch.from_numpy(self.flat.astype(np.int32)).to(dev)
        self.dout = torch.zeros(self.B, dtype=torch.complex128, device=dev)
        if self.seq:
            self.keys = {K: _dp_plan(K) for K, _ in self.bins}
            self.dPs = [torch.from_numpy(np.ascontiguousarray(
                _gather_pairs_batch(np.dtype(np.complex128), self.A, np.asarray(r)[None, :], len(r))[0])).to(dev)
                for r in self.idxs]

    def step_device(self, stream_ptr):
        L = self.egg.lib()
        if self.seq:
            for b, r in enumerate(self.idxs):
                K = len(r)
                key = self.keys[K]
                rc = L.egg_dp_batch_device(key[0], key[1], 1, self.prec, self.dPs[b].data_ptr(), 1,
                                           self.dout.data_ptr() + 16 * b, stream_ptr)
                if rc:
                    raise RuntimeError(L.egg_last_error().decode())
            return
        L.egg_dp_mix_set_engine(self.engine)
        rc = L.egg_dp_mix_device(1, self.prec, self.dA.data_ptr(), 64, self.B, self.offsets.ctypes.data,
                                 self.drows.data_ptr(), self.dout.data_ptr(), stream_ptr)
        if rc:
            raise RuntimeError(L.egg_last_error().decode())

    def step_e2e(self):
        kw = {} if self.prec_name == "exact" else {"prec": self.prec_name}
        if self.seq:
            return [self.egg.hafnian(self.A[np.ix_(r, r)], method="dp", **kw) for r in self.idxs]
        self.egg.lib().egg_dp_mix_set_engine(self.engine)
        return self.egg.hafnian_submatrices(self.A, self.idxs, **kw)

    def device_result(self):
        return list(self.dout.cpu().numpy())

    def check(self, O, dev_vals, e2e_val):
        """Two instances of every degree against the oracle DP (FP64, the reference's order); the
        mixed form against the oracle too, so its figure is its own error."""
        worst, n = 0.0, 0
        seen = {}
        for b, r in enumerate(self.idxs):
            K = len(r)
            if seen.get(K, 0) >= 2:
                continue
            seen[K] = seen.get(K, 0) + 1
            want = O.haf_dp_closed(O.gather_pairs(self.A, [int(i) + 1 for i in r], K), K, O.C128, O.max_threads())
            worst = max(worst, rel_err(dev_vals[b], want))
            n += 1
        e2e_worst = max(rel_err(a, b) for a, b in zip(e2e_val, dev_vals))
        out = {"max_vs_reference_fp64": worst, "instances_checked": n, "e2e_vs_device": e2e_worst,
               "bar": 1e-10 if self.prec_name != "exact" else 0.0,
               "reference": "oracle DP (src/dp.jl:344-442), ComplexF64 in the reference's order"}
        if self.prec_name != "exact" and not self.seq:
            # Every result's own error: against the FP64 path in the reference's rounding (itself
            # bit-identical to the oracle on the instances above).
            ref = self.egg.hafnian_submatrices(self.A, self.idxs, prec="exact")
            errs = np.array([rel_err(a, b) for a, b in zip(dev_vals, ref)])
            out["every_result_vs_fp64"] = {"max": float(errs.max()), "median": float(np.median(errs)),
                                           "p99": float(np.quantile(errs, 0.99)), "count": int(len(errs))}
        return out

    @property
    def h2d_bytes(self):
        if self.seq:  # each call copies its instance's pairs
            return sum(16 * len(r) * (len(r) - 1) // 2 for r in self.idxs)
        return self.A.nbytes + self.flat.nbytes + self.offsets.nbytes + 4 * self.B  # parent, rows, bounds, order

    @property
    def d2h_bytes(self):
        return 16 * self.B

    def roofline(self, ms, peaks):
        return dp_roofline(self.bins, self.vbytes, ms, peaks)

    def extra_config(self):
        """The per-degree evaluation the library's tuner chose (degrees <= 22 run whole-instance)."""
        import ctypes

        if self.seq:
            return {}
        if self.engine == 1:
            return {"engine": "one cooperative launch per call: gather, every degree's levels in lockstep, scatter"}
        L = self.egg.lib()
        tiles = {}
        for K, _ in self.bins:
            b, g = ctypes.c_int(), ctypes.c_int64()
            if K > 22 and L.egg_dp_mix_tuning(K, 1, self.prec, ctypes.byref(b), ctypes.byref(g)) == 0:
                tiles[str(K)] = f"{'batched' if b.value else 'grouped'} x{g.value}"
        return {"tuned_tiles": tiles}

    def cpu_sample(self, nthreads):
        from oracle import oracle as O

        # The reference loop over the mix, timed on up to 4 instances per degree and scaled by the
        # degree counts.
        total = 0.0
        for K, cnt in self.bins:
            rs = [r for r in self.idxs if len(r) == K][:4]
            plan = O.build_plan(K, 4)
            P = O.gather_pairs(self.A, [int(i) + 1 for i in rs[0]], K)
            O.haf_dp_pairs(P, plan, O.C128, nthreads)
            t = time.perf_counter()
            for r in rs:
                O.haf_dp_pairs(O.gather_pairs(self.A, [int(i) + 1 for i in r], K), plan, O.C128, nthreads)
            total += (time.perf_counter() - t) / len(rs) * cnt
        return self.B / total, ("the reference DP on up to 4 instances per degree, scaled by the degree counts "
                                f"({len(self.bins)} degrees), all host threads")


class RepeatedWorkload:
    """B hafnian_repeated sieves per step (configuration 5)."""

    kind = "sieve"

    def __init__(self, egg, W, which: str, B: int, seed: int, prec: str = "exact"):
        from theeggman_b200 import roofline as R
        from theeggman_b200 import policy as pol

        self.egg = egg
        self.prec_name = prec
        self.prec = {"exact": 0, "fma": 1}[prec]
        if which == "a":
            mats, rpts = W.repeated_real(B, 14, seed)
            self.cplx = False
        else:
            mats, rpts = W.repeated_complex(B, 20, 48, seed)
            self.cplx = True
        self.mats, self.rpts = mats, rpts
        self.inst = []
        flops = 0.0
        for A, r in zip(mats, rpts):
            x, er = pol.matched_reps(r)
            xi = np.array(x) - 1
            g = pol._choose_method(sum(r), er, 1)[1]
            self.inst.append((np.ascontiguousarray(A[np.ix_(xi, xi)]), er, g))
            flops += R.sieve_flops(er, g, self.cplx)
        self.flops = flops
        self.B = B
        self.hafnians_per_step = B
        self.dtype_name = "c128" if self.cplx else "f64"
        self.name = (f"config5{which}: {B} x hafnian_repeated(B, rpt), "
                     + ("14x14 Float64 U[-1,1], rpt=fill(2,14)" if which == "a" else
                        "20x20 ComplexF64 N(0,1/40) parts, rpt iid U{1..4} trimmed to total <= 48 and even")
                     + ", mixed-radix sieve, variant by the cost model")

    def setup_device(self, torch, dev):
        # The raw inputs stay resident: each instance's d x d matrix and its multiplicities.  The
        # device forms every instance's matching, variant and permuted matrix in each step.
        CT = np.complex128 if self.cplx else np.float64
        self.stack = np.ascontiguousarray(np.stack([np.asarray(A, dtype=CT).T for A in self.mats]))
        self.R = np.ascontiguousarray(self.rpts, dtype=np.int64)
        self.d = self.stack.shape[1]
        self.dstack = torch.from_numpy(self.stack).to(dev)
        self.drpts = torch.from_numpy(self.R).to(dev)
        self.dout = torch.zeros(2 * self.B, dtype=torch.float64, device=dev)

    def step_device(self, stream_ptr):
        L = self.egg.lib()
        rc = L.egg_sieve_repeated_batch_device(1 if self.cplx else 0, self.prec, self.B, self.d, self.dstack.data_ptr(),
                                               self.d * self.d, self.drpts.data_ptr(), -1, self.dout.data_ptr(),
                                               stream_ptr)
        if rc:
            raise RuntimeError(L.egg_last_error().decode())

    def step_e2e(self):
        kw = {} if self.prec_name == "exact" else {"prec": self.prec_name}
        return self.egg.hafnian_repeated_batch(self.mats, self.rpts, **kw)

    @property
    def h2d_bytes(self):
        return int(self.stack.nbytes + self.R.nbytes)

    @property
    def d2h_bytes(self):
        return self.B * (16 if self.cplx else 8)

    roofline = SieveWorkload.roofline

    def cpu_sample(self, nthreads):
        from oracle import oracle as O

        nb = min(self.B, 64)
        t = time.perf_counter()
        for Ax, er, g in self.inst[:nb]:
            O.calc_hafnian(Ax, er, g, nthreads=nthreads)
        return nb / (time.perf_counter() - t), f"{nb} instances, each with the reference's sieve threading"

    def device_result(self):
        raw = self.dout.cpu().numpy()
        return list(raw.view(np.complex128)[: self.B]) if self.cplx else list(raw[: self.B])

    def check(self, O, dev_vals, e2e_val):
        """16 instances against the oracle's sieve of the same terms (double-double sum), with the
        reference's plain-sum figure beside it."""
        worst_dd, worst_plain = 0.0, 0.0
        for b in range(0, self.B, max(1, self.B // 16)):
            Ax, er, g = self.inst[b]
            dd = O.calc_hafnian(Ax, er, g, nthreads=O.max_threads(), sum_mode=1)
            plain = O.calc_hafnian(Ax, er, g, nthreads=1, sum_mode=0)
            worst_dd = max(worst_dd, rel_err(dev_vals[b], dd))
            worst_plain = max(worst_plain, rel_err(dev_vals[b], plain))
        e2e_worst = max(rel_err(a, b) for a, b in zip(e2e_val, dev_vals))
        return {"max_vs_reference_terms_dd": worst_dd, "max_vs_reference_plain_fp64": worst_plain,
                "instances_checked": 16, "e2e_vs_device": e2e_worst, "bar": 1e-10,
                "reference": "oracle calc_hafnian (src/hafnian.jl:684-738) per instance"}


def make_workload(name: str, egg, W, rank: int):
    # Sieve workloads run the reference's arithmetic (the API default) unless their name ends in
    # "f": the fused-multiply-add register tiles.
    if name == "sieve40":
        return SieveWorkload(egg, W, 40, False, None, 2024 + rank)
    if name == "sieve40f":
        return SieveWorkload(egg, W, 40, False, None, 2024 + rank, prec="fma")
    if name == "sieve40c":
        return SieveWorkload(egg, W, 40, True, None, 2025 + rank)
    if name == "sieve40cf":
        return SieveWorkload(egg, W, 40, True, None, 2025 + rank, prec="fma")
    if name == "sieve40g":
        return SieveWorkload(egg, W, 40, False, True, 2024 + rank)
    if name == "sieve40gf":
        return SieveWorkload(egg, W, 40, False, True, 2024 + rank, prec="fma")
    if name == "sieve20":
        return SieveWorkload(egg, W, 20, False, None, 2020 + rank, config="1")
    if name == "sieve20f":
        return SieveWorkload(egg, W, 20, False, None, 2020 + rank, config="1", prec="fma")
    if name == "dp20":
        return DPWorkload(egg, W, 20, 1, "f64", "exact", 2020 + rank)
    if name == "dp32":
        return DPWorkload(egg, W, 32, 1, "f64", "exact", 3232 + rank)
    if name == "dp36":
        return DPWorkload(egg, W, 36, 1, "f64", "exact", 3636 + rank)
    if name == "dp40":
        return DPWorkload(egg, W, 40, 1, "f64", "exact", 4040 + rank)
    if name == "dp40mixed":
        return DPWorkload(egg, W, 40, 1, "f64", "mixed", 4040 + rank)
    if name == "dp40int":
        return DPWorkload(egg, W, 40, 1, "i64", "exact", 4041 + rank)
    if name == "dp20x1024":
        return DPWorkload(egg, W, 20, 1024, "c128", "exact", 7000 + rank)
    if name == "mix4096":
        return MixWorkload(egg, W, 4096, "exact", False, 4 + 100 * rank)
    if name == "mix4096fma":
        return MixWorkload(egg, W, 4096, "fma", False, 4 + 100 * rank)
    if name == "mix4096mixed":
        return MixWorkload(egg, W, 4096, "mixed", False, 4 + 100 * rank)
    if name == "mix4096one":
        return MixWorkload(egg, W, 4096, "exact", False, 4 + 100 * rank, engine=1)
    if name == "mix4096seq":
        return MixWorkload(egg, W, 4096, "exact", True, 4 + 100 * rank)
    if name == "rep14":
        return RepeatedWorkload(egg, W, "a", 1024, 5 + 100 * rank)
    if name == "rep14f":
        return RepeatedWorkload(egg, W, "a", 1024, 5 + 100 * rank, prec="fma")
    if name == "rep20c":
        return RepeatedWorkload(egg, W, "b", 1024, 6 + 100 * rank)
    if name == "rep20cf":
        return RepeatedWorkload(egg, W, "b", 1024, 6 + 100 * rank, prec="fma")
    raise SystemExit(f"unknown workload {name}")


# ------------------------------------------------------------------------------------------------
# Clocks
# ------------------------------------------------------------------------------------------------

class ClockSampler:
    FIELDS = ("index,pci.bus_id,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, bus_id: str | None):
        self.bus = (bus_id or "").lower()
        self.f = tempfile.NamedTemporaryFile("w+", suffix=".csv", delete=False)
        try:
            self.p = subprocess.Popen(["nvidia-smi", f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits",
                                       "-lms", "200"], stdout=self.f, stderr=subprocess.DEVNULL)
        except OSError:
            self.p = None

    def stop(self) -> dict:
        if self.p is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.p.terminate()
        try:
            self.p.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.p.kill()
        self.f.flush()
        rows = []
        for line in open(self.f.name):
            parts = [s.strip() for s in line.split(",")]
            if len(parts) < 10:
                continue
            if self.bus and not parts[1].lower().endswith(self.bus[-12:]):
                continue
            rows.append(parts)
        os.unlink(self.f.name)
        if not rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["no samples"]}
        sm = [float(r[2]) for r in rows if r[2].replace(".", "").isdigit()]
        reasons = set()
        names = ("hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap")
        for r in rows:
            for nm, v in zip(names, r[6:10]):
                if v.strip().lower() == "active":
                    reasons.add(nm)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": float(rows[0][3]),
                "reasons": sorted(reasons), "samples": len(rows)}


# ------------------------------------------------------------------------------------------------
# Arms
# ------------------------------------------------------------------------------------------------

def dist_env():
    return int(os.environ.get("RANK", 0)), int(os.environ.get("WORLD_SIZE", 1)), int(os.environ.get("LOCAL_RANK", 0))


def run_reference(args):
    """The reference's algorithm on this host's CPU cores: the oracle's restatement of
    src/dp.jl / src/hafnian.jl with the reference's threading policy.  Julia is not installed, so
    the Julia package itself cannot run; the oracle is the closest executable form of it."""
    rank, world, _ = dist_env()
    if rank != 0:
        return
    sys.path.insert(0, ROOT)
    egg = load_package()
    from oracle import oracle as O
    from theeggman_b200 import workloads as W

    O.build()
    wl = make_workload(args.workload or "sieve40", egg, W, 0)
    cores = O.max_threads()
    for _ in range(args.warmup):
        wl.cpu_sample(cores)
    rates = []
    sample = ""
    for _ in range(args.steps):
        r, sample = wl.cpu_sample(cores)
        rates.append(r)
    value = statistics.median(rates)
    print(json.dumps({
        "impl": "reference", "metric": METRIC, "value": value, "unit": "hafnians/s", "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 * wl.hafnians_per_step / value,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": wl.dtype_name,
        "data": "synthetic (seeded SplitMix64)", "config": {"workload": wl.name, "host": "CPU"},
        "cpu_baseline": {"value": value, "unit": "hafnians/s", "cores": cores, "kind": "port",
                         "sample": f"median of {args.steps} samples: {sample}"},
        "e2e": {"value": value, "unit": "hafnians/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }))


# The rest of the metric, timed in the default run after the headline: every configuration of the
# metric with its own value, e2e, roofline, CPU baseline and error against the oracle.  (name,
# timed steps at most): the heavy end-to-end forms take fewer steps so that the whole default run
# stays within a few minutes.
PER_CONFIG = [("dp20", 20), ("sieve20", 20), ("sieve20f", 20), ("dp32", 10), ("sieve40", 10), ("sieve40f", 10),
              ("sieve40c", 3), ("sieve40cf", 5), ("sieve40gf", 5), ("dp36", 5), ("dp40", 5), ("dp40mixed", 5),
              ("dp40int", 5), ("dp20x1024", 10), ("mix4096", 10), ("mix4096one", 10), ("mix4096fma", 10), ("mix4096mixed", 10), ("mix4096seq", 3),
              ("rep14", 10), ("rep14f", 10), ("rep20c", 3), ("rep20cf", 3)]
PER_CONFIG_BUDGET_S = 300.0


class Device:
    """The timing context of one rank: its device, a dedicated stream and the L2 flush buffer."""

    def __init__(self, torch, local):
        self.torch = torch
        self.dev = torch.device("cuda", local)
        torch.cuda.set_device(self.dev)
        # A dedicated stream: the legacy default stream's handle is NULL, which the C ABI reads as
        # "use the library's own stream", and events on one stream do not time work on another.
        self.stream = torch.cuda.Stream(self.dev)
        self.sp = self.stream.cuda_stream
        self.flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device=self.dev)

    def bus_id(self):
        props = self.torch.cuda.get_device_properties(self.dev)
        bus = getattr(props, "pci_bus_id", None)
        if bus is None:
            try:
                bus = "%02x:%02x" % (props.pci_bus_id, props.pci_device_id)
            except AttributeError:
                bus = None
        return str(bus) if bus is not None and not isinstance(bus, int) else None


def measure(wl, D, L, steps, warmup, world, clocks=None):
    """Time `steps` device steps (inputs resident, L2 flushed between steps outside the events),
    then `steps` end-to-end public-API calls; max over ranks.  Returns the figures and the last
    results of both."""
    import torch
    import torch.distributed as dist

    for _ in range(warmup):
        wl.step_device(D.sp)
    torch.cuda.synchronize(D.dev)
    if clocks is not None:
        time.sleep(0.3)
    if world > 1:
        dist.barrier()
    torch.cuda.synchronize(D.dev)
    launches0 = L.egg_launch_count()
    evs = []
    for _ in range(steps):
        with torch.cuda.stream(D.stream):
            D.flush.fill_(1.0)
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record(D.stream)
        wl.step_device(D.sp)
        e1.record(D.stream)
        evs.append((e0, e1))
    torch.cuda.synchronize(D.dev)
    launches = L.egg_launch_count() - launches0  # the library's own kernel launches, counted by it
    if world > 1:
        dist.barrier()
    clk = clocks.stop() if clocks is not None else None
    ms = sum(a.elapsed_time(b) for a, b in evs)
    t = torch.tensor([ms], dtype=torch.float64, device=D.dev)
    if world > 1:
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
    ms_max = float(t.item())
    dev_vals = wl.device_result()

    # End to end through the public API, host arrays in and out.
    e2e_val = None
    for _ in range(max(1, min(warmup, 3))):
        e2e_val = wl.step_e2e()
    if world > 1:
        dist.barrier()
    t0 = time.perf_counter()
    for _ in range(steps):
        e2e_val = wl.step_e2e()
    e2e_s = time.perf_counter() - t0
    te = torch.tensor([e2e_s], dtype=torch.float64, device=D.dev)
    if world > 1:
        dist.all_reduce(te, op=dist.ReduceOp.MAX)
    return {"ms": ms_max, "value": world * steps * wl.hafnians_per_step / (ms_max / 1e3),
            "e2e": world * steps * wl.hafnians_per_step / float(te.item()), "launches": launches, "clocks": clk,
            "dev_vals": dev_vals, "e2e_val": e2e_val}


def cpu_leg(wl, args):
    """Rank 0 at N = 1 only: the oracle as the CPU baseline (the reference's algorithm on the host's
    cores) and as the checker of the timed results."""
    from oracle import oracle as O

    O.build()
    cores = O.max_threads()
    rate, sample = wl.cpu_sample(cores)
    return O, {"value": rate, "unit": "hafnians/s", "cores": cores, "kind": "port", "sample": sample}


def form_of(wl) -> str:
    """The arithmetic form a workload times."""
    p = getattr(wl, "prec_name", "fma")
    if wl.kind == "sieve":
        return {"fma": "prec=fma: register-tile terms with fused multiply-adds, double-double sum",
                "exact": "prec=exact: every term in the reference's arithmetic, double-double sum"}[p]
    return {"exact": "prec=exact: the reference's per-state order and rounding",
            "fma": "prec=fma: fused multiply-adds",
            "mixed": "prec=mixed: FP32 products, FP64 sums"}[p]


def line_for(wl, name, m, steps, warmup, world, peaks, cpu, err):
    roof = wl.roofline(m["ms"] / steps, peaks)
    roof["traffic"] = profile_traffic(PROFILE_OF.get(name, ""))
    return {
        "workload_key": name, "value": m["value"], "unit": "hafnians/s", "steps": steps, "warmup": warmup,
        "ms_per_step": m["ms"] / steps, "dtype": wl.dtype_name,
        "config": {"workload": wl.name, "form": form_of(wl),
                   **(wl.extra_config() if hasattr(wl, "extra_config") else {})},
        "e2e": {"value": m["e2e"], "unit": "hafnians/s", "h2d_bytes_per_step": wl.h2d_bytes,
                "d2h_bytes_per_step": wl.d2h_bytes, "path": "the public API from host memory, default arguments"},
        "roofline": roof, "cpu_baseline": cpu, "rel_err": err, "gpu_launches": m["launches"],
    }


def run_ours(args):
    import torch
    import torch.distributed as dist

    rank, world, local = dist_env()
    D = Device(torch, local)
    if world > 1:
        from datetime import timedelta

        dist.init_process_group("nccl", timeout=timedelta(seconds=120), device_id=D.dev)
    sys.path.insert(0, ROOT)
    egg = load_package()
    from theeggman_b200 import workloads as W

    L = egg.lib()
    if L.egg_init(local) != 0:
        raise SystemExit(L.egg_last_error().decode())
    headline = args.workload or "sieve40"
    wl = make_workload(headline, egg, W, rank)
    wl.setup_device(torch, D.dev)
    torch.cuda.synchronize(D.dev)
    clocks = ClockSampler(D.bus_id())
    m = measure(wl, D, L, args.steps, args.warmup, world, clocks)

    peaks = measured_peaks()
    solo = rank == 0 and world == 1 and not args.no_cpu_baseline
    cpu, err = None, None
    if solo:
        O, cpu = cpu_leg(wl, args)
        err = wl.check(O, m["dev_vals"], m["e2e_val"])
    if rank == 0:
        line = line_for(wl, headline, m, args.steps, args.warmup, world, peaks, cpu, err)
        line.pop("workload_key")
        line = {"metric": METRIC, **{k: line[k] for k in ("value", "unit")}, "n_gpus": world, "steps": args.steps,
                "warmup": args.warmup, "ms_per_step": line["ms_per_step"], "higher_is_better": True,
                "scaling": "weak", "vs_baseline": None, "dtype": line["dtype"], "data": "synthetic (seeded SplitMix64)",
                "config": {**line["config"], "l2": "flushed between steps (256 MiB write outside the timed events)",
                           "parallelism": f"replicas x{world}" if world > 1 else "single GPU"},
                "e2e": line["e2e"], "roofline": line["roofline"], "cpu_baseline": cpu, "rel_err": err,
                "clocks": m["clocks"], "gpu_launches": m["launches"]}
    # The other configurations of the metric, in the same process (single GPU, default run only).
    if args.workload is None and world == 1 and not args.no_per_config:
        per = []
        t_start = time.perf_counter()
        pclocks = ClockSampler(D.bus_id())
        for name, cap in PER_CONFIG:
            if time.perf_counter() - t_start > PER_CONFIG_BUDGET_S:
                per.append({"workload_key": name, "skipped": "per-configuration time budget spent"})
                continue
            w2 = make_workload(name, egg, W, rank)
            w2.setup_device(torch, D.dev)
            torch.cuda.synchronize(D.dev)
            st = min(args.steps, cap)
            m2 = measure(w2, D, L, st, max(args.warmup, 3), world)
            cpu2, err2 = None, None
            if solo:
                O, cpu2 = cpu_leg(w2, args)
                err2 = w2.check(O, m2["dev_vals"], m2["e2e_val"])
            per.append(line_for(w2, name, m2, st, max(args.warmup, 3), world, peaks, cpu2, err2))
            del w2
            torch.cuda.empty_cache()
        line["per_config"] = per
        line["per_config_clocks"] = pclocks.stop()
    if rank == 0:
        print(json.dumps(line, default=float))
    if world > 1:
        dist.barrier()
        dist.destroy_process_group()


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--workload", default=None,
                    help="time one workload (default: the N = 40 sieve headline plus every configuration of the metric)")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-per-config", action="store_true", help="time the headline only")
    args = ap.parse_args()
    if args.impl == "reference":
        run_reference(args)
    else:
        run_ours(args)


if __name__ == "__main__":
    main()
