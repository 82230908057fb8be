"""The header-only C++ adapters (include/yannq_gpu/yannq_gpu.hpp): a RunRBM-style
driver in the reference example's call pattern compiles against them (CPU), and
on a GPU it runs, the energy goes down towards the exact ground energy."""
import os
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
SRC = os.path.join(ROOT, "tests", "cpp", "rbm_tfi_driver.cpp")
LIBDIR = os.path.join(ROOT, "yannq_b200")


def _build(tmp_path):
    exe = str(tmp_path / "rbm_tfi_driver")
    cmd = ["g++", "-std=c++17", "-O2", "-Wall", "-Wextra", "-I", os.path.join(ROOT, "include"), SRC, "-o", exe,
           "-L", LIBDIR, "-lyannq_b200", f"-Wl,-rpath,{LIBDIR}"]
    out = subprocess.run(cmd, capture_output=True, text=True)
    assert out.returncode == 0, out.stderr
    return exe


def test_adapters_compile(tmp_path):
    _build(tmp_path)


@pytest.mark.gpu
def test_adapter_driver_runs(tmp_path, orc):
    exe = _build(tmp_path)
    out = subprocess.run([exe, "40"], capture_output=True, text=True, timeout=600)
    assert out.returncode == 0, out.stdout[-2000:] + out.stderr[-2000:]
    last = [l for l in out.stdout.splitlines() if l.startswith("OK")][0].split()
    e_first, e_last = float(last[1]), float(last[2])
    e0 = orc.ed_ground(orc.Ham.tfi(10, -1.0, -1.0)) / 10
    assert e_last < e_first
    assert e_last >= e0 - 1e-3
