"""The header-only C++ adapters (include/yannq_gpu/yannq_gpu.hpp): RunRBM-style
drivers in the reference example's call pattern compile against them (CPU), and
on a GPU they run and the energy goes down towards the exact ground energy: the
TFI chain with local moves, the J1J2 chain with exchange moves (which also
constructs the XXX, XYZNNN and KitaevHex adapters), and the AmplitudePhase
example's RunAmplitudePhaseExact loop."""
import os
import subprocess

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
LIBDIR = os.path.join(ROOT, "yannq_b200")


def _build(tmp_path, name="rbm_tfi_driver"):
    exe = str(tmp_path / name)
    src = os.path.join(ROOT, "tests", "cpp", name + ".cpp")
    cmd = ["g++", "-std=c++17", "-O2", "-Wall", "-Wextra", "-I", os.path.join(ROOT, "include"), src, "-o", exe,
           "-L", LIBDIR, "-lyannq_b200", f"-Wl,-rpath,{LIBDIR}"]
    out = subprocess.run(cmd, capture_output=True, text=True)
    assert out.returncode == 0, out.stderr
    return exe


@pytest.mark.parametrize("name", ["rbm_tfi_driver", "j1j2_driver", "amplitude_phase_driver", "run_rbm_reference_shape"])
def test_adapters_compile(tmp_path, name):
    _build(tmp_path, name)


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


@pytest.mark.gpu
def test_j1j2_driver_runs(tmp_path, orc):
    exe = _build(tmp_path, "j1j2_driver")
    run_dir = tmp_path / "run"
    run_dir.mkdir()
    out = subprocess.run([exe, "40"], capture_output=True, text=True, timeout=600, cwd=run_dir)
    assert out.returncode == 0, out.stdout[-2000:] + out.stderr[-2000:]
    # RunRBM.hpp:155-164 checkpoints at ll % saveWfPer == 0
    assert sorted(p.name for p in run_dir.iterdir()) == ["w0000.dat", "w0020.dat", "w0040.dat"]
    n, m, bias, p = orc.rbm_unarchive((run_dir / "w0020.dat").read_bytes(), 1)
    assert (n, m, bias) == (12, 12, True) and np.all(np.isfinite(p))
    assert "RESUME 168" in out.stdout
    terms = {l.split()[1]: (int(l.split()[2]), int(l.split()[3])) for l in out.stdout.splitlines()
             if l.startswith("TERMS")}
    assert terms == {"XXX": (10, 10), "XYZNNN": (10, 20), "KitaevHex": (16, 32), "KitaevHexAniso": (16, 32),
                     "J1J2": (12, 24)}
    assert "HAMSWEEP 64" in out.stdout
    last = [l for l in out.stdout.splitlines() if l.startswith("OK")][0].split()
    e_first, e_last = float(last[1]), float(last[2])
    e0 = orc.ed_ground(orc.Ham.j1j2(12, 1.0, 0.2, True), 1, 6) / 12
    assert e_last < e_first
    assert e_last >= e0 - 1e-3


@pytest.mark.gpu
def test_amplitude_phase_driver_runs(tmp_path, orc):
    exe = _build(tmp_path, "amplitude_phase_driver")
    out = subprocess.run([exe, "60"], capture_output=True, text=True, timeout=600)
    assert out.returncode == 0, out.stdout[-2000:] + out.stderr[-2000:]
    g = [l for l in out.stdout.splitlines() if l.startswith("GETTERS")][0].split()
    assert int(g[1]) == (12 * 12) ** 2 and int(g[2]) == 144 + 30 + 120 + 40 + 24
    last = [l for l in out.stdout.splitlines() if l.startswith("OK")][0].split()
    e_first, e_last = float(last[1]), float(last[2])
    e0 = orc.ed_ground(orc.Ham.j1j2(12, 1.0, 0.2, True), 1, 6) / 12
    assert e_last < e_first
    assert e_last >= e0 - 1e-9


@pytest.mark.gpu
def test_reference_shaped_run_with_randomizer(tmp_path, orc):
    """RunRBM::run(sampler, callback, randomizer, std::move(ham), nSweeps, nDiscard)
    as Examples/RBMTFI.cpp calls it: the host randomizer is called once per chain
    per epoch (nTmp x K chains, epochs 0..maxIter), and the energy goes down
    towards the ground state."""
    exe = _build(tmp_path, "run_rbm_reference_shape")
    out = subprocess.run([exe, "30"], capture_output=True, text=True, timeout=600)
    assert out.returncode == 0, out.stdout[-2000:] + out.stderr[-2000:]
    calls = int([l for l in out.stdout.splitlines() if l.startswith("RANDOMIZER")][0].split()[1])
    assert calls == 31 * 2 * 16
    last = [l for l in out.stdout.splitlines() if l.startswith("OK")][0].split()
    e_first, e_last = float(last[1]), float(last[2])
    e0 = orc.ed_ground(orc.Ham.tfi(10, -1.0, -1.0)) / 10
    assert e_last < e_first
    assert e_last >= e0 - 1e-3
