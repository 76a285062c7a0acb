"""Per-device state of the library, checked on the CPU.

The library keeps its device-resident tables per GPU (csrc/egg_perdevice.h): the closed-form
binomial table that the DP and the sieve read, and the fixed scratch of the entry point that
allocates nothing.  A process holding two GPUs must never hand device 0's address to a kernel on
device 1.  With one GPU per run, the bookkeeping is exercised here by a small C++ driver that calls
it with device indices directly.
"""
import os
import shutil
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


@pytest.mark.skipif(shutil.which("g++") is None, reason="needs g++")
def test_per_device_values_are_set_up_per_device(tmp_path):
    exe = tmp_path / "perdevice_check"
    subprocess.run(["g++", "-std=c++17", "-O1", "-pthread", "-I", os.path.join(ROOT, "theeggman.jl_b200", "csrc"),
                    os.path.join(ROOT, "tests", "perdevice_check.cpp"), "-o", str(exe)], check=True)
    r = subprocess.run([str(exe)], capture_output=True, text=True)
    assert r.returncode == 0 and r.stdout.strip().endswith("ok"), r.stdout + r.stderr


@pytest.mark.skipif(shutil.which("g++") is None, reason="needs g++")
def test_tuner_file_round_trip(tmp_path):
    """The mixed-degree tuner's choices survive the process: the file format
    (csrc/egg_tunecache.h) written, merged per (device, SMs, degree, type, mode) and read back."""
    exe = tmp_path / "tunecache_check"
    subprocess.run(["g++", "-std=c++17", "-O1", "-I", os.path.join(ROOT, "theeggman.jl_b200", "csrc"),
                    os.path.join(ROOT, "tests", "tunecache_check.cpp"), "-o", str(exe)], check=True)
    r = subprocess.run([str(exe), str(tmp_path)], capture_output=True, text=True)
    assert r.returncode == 0 and r.stdout.strip().endswith("ok"), r.stdout + r.stderr
