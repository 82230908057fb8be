"""The small plain configuration end to end on the device, FP64 (the reference's
Examples/RBMTFI.cpp:20-88 call pattern and Runners/RunRBMExact.hpp:29-82):
TFI chain N = 16, periodic, J = -1, h = -1, RBM alpha = 2 (M = 32, P = 560),
complex128 parameters N(0, 0.01^2), 16 chains re-randomised every epoch, 64
thermalisation + 64 recorded sweeps (1024 samples), S-form LLT with shift 1e-3,
SGD 0.01, 200 epochs.

* Sampled run: every epoch's energy against the oracle's restated runner
  (tests/golden/config_a_trajectory.json, made by make_config_a_trajectory.py):
  the same Philox streams give the same samples as long as no Metropolis
  decision differs, so the energies agree to 1e-9 relative epoch by epoch while
  both runs hold the same samples (checked for the first 50 epochs), and the
  mean over the last 50 epochs agrees within Monte Carlo error.
* Exact-summation run (RunRBMExact, SRMatExact over all 2^16 states): 200
  epochs of yq_exact_iteration; the first epochs track the oracle loop (orc.exact
  + LLT + SGD) to 1e-10, and at the final parameters E and energyGrad agree with
  orc.exact to 1e-11.
* Both runs end above the exact ground energy (Lanczos) and within 0.5 % of it.
"""
import json
import os

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

HERE = os.path.dirname(os.path.abspath(__file__))


@pytest.fixture(scope="module")
def traj():
    with open(os.path.join(HERE, "golden", "config_a_trajectory.json")) as f:
        return json.load(f)


@pytest.fixture(scope="module")
def ctx():
    from yannq_b200 import api

    c = api.Context(0)
    yield c
    c.close()


def test_config_a_sampled_run_matches_oracle_runner(ctx, orc, traj):
    from yannq_b200 import api

    n, m = traj["n"], traj["m"]
    q = api.RBM(ctx, n, m, True, api.C128)
    q.init_random(traj["seed"], 0.01)
    assert np.max(np.abs(q.get_params() - orc.init_params(n, m, traj["seed"], 0.01))) == 0.0
    H = api.Hamiltonian.tfi(ctx, n, -1.0, -1.0)
    S = api.Sampler(q, traj["chains"])
    sr = api.SR(q, H, S, api.SR_AUTO, api.PREC_FP64)
    es = []
    for ll in range(traj["epochs"]):
        r = sr.iteration(traj["n_sweeps"], traj["n_discard"], traj["seed"], ll, traj["shift"], traj["lr"],
                         reinit=True)
        es.append(r.energy)
    es, ref = np.array(es) / n, np.array(traj["energies"]) / n
    np.testing.assert_allclose(es[:50], ref[:50], rtol=1e-9, atol=0)
    tail, rtail = es[-50:], ref[-50:]
    sem = np.hypot(tail.std(ddof=1), rtail.std(ddof=1)) / np.sqrt(50)
    assert abs(tail.mean() - rtail.mean()) <= 4 * sem + 1e-12, (tail.mean(), rtail.mean(), sem)
    e0 = traj["ed_energy"] / n
    assert es[-50:].mean() > e0 and abs(es[-50:].mean() - e0) < 5e-3 * abs(e0)
    assert es[-50:].mean() < es[0]
    for x in (sr, S, H, q):
        x.close()


def test_exact_iteration_tracks_oracle_loop(ctx, orc):
    """RunRBMExact epochs (constructExact, LLT of corrMat + lambda, SGD) against the
    oracle's SRMatExact restatement and LLT, N = 10 (2^10 states)."""
    from yannq_b200 import api

    n, m, shift, lr = 10, 20, 1e-3, 0.05
    q = api.RBM(ctx, n, m, True, api.C128)
    p = orc.init_params(n, m, 5, 0.05)
    q.set_params(p)
    H = api.Hamiltonian.tfi(ctx, n, -1.0, -1.0)
    h = orc.Ham.tfi(n, -1.0, -1.0)
    for _ in range(3):
        e, var, nv = api.exact_iteration(q, H, shift, lr)
        ref = orc.exact(h, m, p)
        st, v = orc.cholesky_solve(ref["S"] + shift * np.eye(len(p)), ref["grad"])
        assert st == 0
        p = p - lr * v
        assert e == pytest.approx(ref["energy"], rel=1e-11)
        assert var == pytest.approx(ref["energy_var"], rel=1e-8, abs=1e-12)
        assert nv == pytest.approx(np.linalg.norm(v), rel=1e-9)
        assert np.max(np.abs(q.get_params() - p)) <= 1e-10 * np.max(np.abs(p))
    for x in (H, q):
        x.close()


def test_config_a_exact_summation_run(ctx, orc, traj):
    from yannq_b200 import api

    n, m = traj["n"], traj["m"]
    q = api.RBM(ctx, n, m, True, api.C128)
    q.init_random(traj["seed"], 0.01)
    H = api.Hamiltonian.tfi(ctx, n, -1.0, -1.0)
    es = [api.exact_iteration(q, H, traj["shift"], traj["lr"])[0] / n for _ in range(traj["epochs"])]
    e0 = traj["ed_energy"] / n
    assert es[-1] < es[0]
    assert es[-1] > e0 and abs(es[-1] - e0) < 5e-3 * abs(e0)
    h = orc.Ham.tfi(n, -1.0, -1.0)
    p = q.get_params()
    ref = orc.exact(h, m, p, with_S=False)
    got = api.exact(q, H, with_S=False)
    assert got["energy"] == pytest.approx(ref["energy"], rel=1e-11)
    assert np.max(np.abs(got["grad"] - ref["grad"])) <= 1e-11 * max(1.0, np.max(np.abs(ref["grad"])))
    for x in (H, q):
        x.close()
