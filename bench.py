"""Benchmark: hafnians/s on B200 for TheEggman.jl's hot paths.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference] [--workload NAME]

The default workload is the N = 40 sieve of configuration 2(a): one real symmetric 40 x 40 matrix
with entries U[-1, 1]/sqrt(40), hafnian(A; method = :sieve), which the reference runs as
inclusion-exclusion (2^20 terms; its cost model's choice for distinct rows).  A step is one full
hafnian.  Under torchrun every rank computes its own matrix (seed + rank): the sieve instances are
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
    """One N x N sieve hafnian per step (configuration 2: N = 40, real or complex)."""

    def __init__(self, egg, W, N: int, cplx: bool, glynn, seed: int):
        from theeggman_b200 import policy as pol
        from theeggman_b200 import roofline as R

        self.egg, self.N, self.cplx = egg, N, cplx
        E = N // 2
        self.E = E
        self.A = (W.dense_complex(N, seed, 1.0 / (2 * N)) if cplx else W.dense_real(N, seed, scale=1.0 / np.sqrt(N)))
        sel_glynn = pol._choose_method_distinct(N, E, os.cpu_count() or 1)[1]
        self.glynn = sel_glynn if glynn is None else glynn
        x = [2 * i + 1 for i in range(E)] + [2 * i + 2 for i in range(E)]
        xi = np.array(x) - 1
        self.Ax = np.asfortranarray(self.A[np.ix_(xi, xi)])
        self.reps = np.ones(E, dtype=np.int64)
        self.flops = R.sieve_flops([1] * E, self.glynn, cplx)
        self.dtype = 1 if cplx else 0
        self.prec = 1  # EGG_PREC_FMA: the register-resident kernels (the API default for the sieve)
        self.name = (f"config2{'b' if cplx else 'a'}: N={N} {'ComplexF64 N(0,1/(2N)) parts' if cplx else 'Float64 U[-1,1]/sqrt(N)'}, "
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
        return self.egg.hafnian(self.A, method="sieve", glynn=self.glynn, check_symmetric=False, prec="fma")

    launches_per_step = 2  # sieve kernel + fixed-order reduction kernel
    kernel = "sieve"

    @property
    def h2d_bytes(self):
        return self.Ax.nbytes + 8 * self.E + 64

    @property
    def d2h_bytes(self):
        return 16 if self.cplx else 8

    def cpu_time(self, nthreads: int):
        from oracle import oracle as O

        t = time.perf_counter()
        O.calc_hafnian(self.Ax, [1] * self.E, self.glynn, nthreads=nthreads)
        return time.perf_counter() - t


def make_workload(name: str, egg, W, rank: int):
    if name == "sieve40":
        return SieveWorkload(egg, W, 40, False, None, 2024 + rank)
    if name == "sieve40c":
        return SieveWorkload(egg, W, 40, True, None, 2025 + rank)
    if name == "sieve40g":
        return SieveWorkload(egg, W, 40, False, True, 2024 + rank)
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
    src/hafnian.jl's sieve with its own threading policy (Julia is not installed, so the Julia
    package itself cannot run; the oracle is the closest executable form of it)."""
    rank, world, _ = dist_env()
    if rank != 0:
        return
    sys.path.insert(0, ROOT)
    egg = load_package()
    from oracle import oracle as O
    from theeggman_b200 import workloads as W

    O.build()
    wl = make_workload(args.workload, egg, W, 0)
    cores = O.max_threads()
    for _ in range(args.warmup):
        wl.cpu_time(cores)
    times = [wl.cpu_time(cores) for _ in range(args.steps)]
    total = sum(times)
    value = args.steps / total
    print(json.dumps({
        "impl": "reference", "metric": METRIC, "value": value, "unit": "hafnians/s", "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 * total / args.steps,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": {"workload": wl.name, "host": "CPU"},
        "cpu_baseline": {"value": value, "unit": "hafnians/s", "cores": cores, "kind": "port",
                         "sample": f"{args.steps} full hafnians (every sieve term), all host threads"},
        "e2e": {"value": value, "unit": "hafnians/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }))


def run_ours(args):
    import torch
    import torch.distributed as dist

    rank, world, local = dist_env()
    dev = torch.device("cuda", local)
    torch.cuda.set_device(dev)
    if world > 1:
        from datetime import timedelta

        dist.init_process_group("nccl", timeout=timedelta(seconds=120), device_id=dev)
    sys.path.insert(0, ROOT)
    egg = load_package()
    from theeggman_b200 import workloads as W

    L = egg.lib()
    if L.egg_init(local) != 0:
        raise SystemExit(L.egg_last_error().decode())
    wl = make_workload(args.workload, egg, W, rank)
    wl.setup_device(torch, dev)
    torch.cuda.synchronize(dev)
    # A dedicated stream: the legacy default stream's handle is NULL, which the C ABI reads as
    # "use the library's own stream", and events on one stream do not time work on another.
    stream = torch.cuda.Stream(dev)
    sp = stream.cuda_stream
    flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device=dev)

    for _ in range(args.warmup):
        wl.step_device(sp)
    torch.cuda.synchronize(dev)

    props = torch.cuda.get_device_properties(dev)
    bus = getattr(props, "pci_bus_id", None)
    if bus is None:
        try:
            bus = "%02x:%02x" % (props.pci_bus_id, props.pci_device_id)
        except AttributeError:
            bus = None
    clocks = ClockSampler(str(bus) if bus is not None and not isinstance(bus, int) else None)
    time.sleep(0.3)
    if world > 1:
        dist.barrier()
    torch.cuda.synchronize(dev)
    evs = []
    for _ in range(args.steps):
        with torch.cuda.stream(stream):
            flush.fill_(1.0)
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        wl.step_device(sp)
        e1.record(stream)
        evs.append((e0, e1))
    torch.cuda.synchronize(dev)
    if world > 1:
        dist.barrier()
    clk = clocks.stop()
    ms = sum(a.elapsed_time(b) for a, b in evs)
    t = torch.tensor([ms], dtype=torch.float64, device=dev)
    if world > 1:
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
    ms_max = float(t.item())
    value = world * args.steps / (ms_max / 1e3)

    # End to end through the public API, host arrays in and out.
    for _ in range(max(1, args.warmup // 2)):
        wl.step_e2e()
    if world > 1:
        dist.barrier()
    t0 = time.perf_counter()
    for _ in range(args.steps):
        wl.step_e2e()
    e2e_s = time.perf_counter() - t0
    te = torch.tensor([e2e_s], dtype=torch.float64, device=dev)
    if world > 1:
        dist.all_reduce(te, op=dist.ReduceOp.MAX)
    e2e_value = world * args.steps / float(te.item())

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        from oracle import oracle as O

        O.build()
        cores = O.max_threads()
        wl.cpu_time(cores)  # warm the thread pool
        ct = wl.cpu_time(cores)
        cpu = {"value": 1.0 / ct, "unit": "hafnians/s", "cores": cores, "kind": "port",
               "sample": "one full hafnian of the same workload (every sieve term), all host threads"}

    peaks = measured_peaks()
    sm_max = float(peaks.get("sm_max_mhz", 1965.0))
    from theeggman_b200 import roofline as R

    peak = R.fp64_nominal_tflops(sm_max)
    achieved = wl.flops / (ms_max / args.steps / 1e3) / 1e12
    traffic = profile_traffic(f"{wl.kernel}_{args.workload}.txt")
    if rank == 0:
        line = {
            "metric": METRIC, "value": value, "unit": "hafnians/s", "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": ms_max / args.steps, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f64", "data": "synthetic (seeded SplitMix64)",
            "config": {"workload": wl.name, "l2": "flushed between steps (256 MiB write outside the timed events)",
                       "parallelism": f"replicas x{world}" if world > 1 else "single GPU"},
            "e2e": {"value": e2e_value, "unit": "hafnians/s", "h2d_bytes_per_step": wl.h2d_bytes,
                    "d2h_bytes_per_step": wl.d2h_bytes, "path": "hafnian(A; method=:sieve) from host memory"},
            "roofline": {"bound": "fp64", "achieved": achieved, "peak": peak, "unit": "TFLOP/s",
                         "frac": achieved / peak, "traffic": traffic,
                         "peak_source": f"nominal FP64: 148 SMs x 64 FMA/clk x 2 x {sm_max:.0f} MHz (no FP64 figure "
                                        "in MEASURED_PEAKS.json)",
                         "work": f"{wl.flops:.4e} algorithmic flops per hafnian"},
            "cpu_baseline": cpu, "clocks": clk, "gpu_launches": wl.launches_per_step * args.steps,
        }
        print(json.dumps(line))
    if world > 1:
        dist.barrier()
        dist.destroy_process_group()


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--workload", default="sieve40")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    args = ap.parse_args()
    if args.impl == "reference":
        run_reference(args)
    else:
        run_ours(args)


if __name__ == "__main__":
    main()
