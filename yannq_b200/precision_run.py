"""Precision run of the 12 x 12 TFI RBM alpha = 2 workload: the mixed path against
the FP64 path over many iterations.

    python -m yannq_b200.precision_run --iters 300 --every 50 > precision.json

Both paths start from the same FP64 parameters (N(0, 0.01^2) from the seed) and
use the same Philox seeds per iteration (1024 persistent chains, 64
thermalisation sweeps, then 8 decorrelation + 8 recorded sweeps per iteration,
T-form SR with shift 1e-3, SGD 0.01).  Reported:

* the energy per site of every iteration of both runs, and the means and
  standard errors over the last quarter of the iterations (the runs sample
  independently once a Metropolis decision differs, so they agree within
  Monte Carlo error, not draw for draw);
* every `--every` iterations, on one and the same sample set drawn by the mixed
  machine: the energy per site, the force F and the SR update v of the mixed
  SR step against an FP64 SR step on the same samples and parameters (FP64
  machine, FP64 O, DMMA Gram, FP64 Cholesky).
"""
import argparse
import json
import os
import sys

import numpy as np

sys.path.insert(0, os.path.dirname(os.path.dirname(os.path.abspath(__file__))))

LX, LY, ALPHA, J, H = 12, 12, 2, -1.0, -3.0
CHAINS, SWEEPS, DISCARD, THERM, SHIFT, LR, SEED = 1024, 8, 8, 64, 1e-3, 0.01, 20261203


def _problem(api, ctx, prec, seed):
    n = LX * LY
    q = api.RBM(ctx, n, ALPHA * n, True, api.C64 if prec == "mixed" else api.C128)
    q.init_random(seed, 0.01)
    H_ = api.Hamiltonian.tfi2d(ctx, LX, LY, J, H)
    S = api.Sampler(q, CHAINS, api.MOVE_LOCAL)
    sr = api.SR(q, H_, S, api.SR_T, api.PREC_MIXED if prec == "mixed" else api.PREC_FP64)
    return q, H_, S, sr


def _same_samples(api, ctx, qm, Sm, srm):
    """SR of the mixed machine's current samples, mixed vs FP64, same parameters."""
    n = LX * LY
    sig, th = Sm.get_samples()
    srm.construct()
    vm, _, _ = srm.solve(SHIFT, api.SOLVE_LLT)
    em, _ = srm.energy()
    P = qm.dim
    Fm = srm.get(2, P)
    qf = api.RBM(ctx, n, ALPHA * n, True, api.C128)
    qf.set_params(qm.get_params())
    Hf = api.Hamiltonian.tfi2d(ctx, LX, LY, J, H)
    Sf = api.Sampler(qf, CHAINS, api.MOVE_LOCAL)
    Sf.put_samples(sig, qf.theta(sig))
    srf = api.SR(qf, Hf, Sf, api.SR_T, api.PREC_FP64)
    srf.construct()
    vf, _, _ = srf.solve(SHIFT, api.SOLVE_LLT)
    ef, _ = srf.energy()
    out = {"E_per_site_mixed": em / n, "E_per_site_fp64": ef / n, "dE_per_site": abs(em - ef) / n,
           "v_rel_err": float(np.linalg.norm(vm - vf) / np.linalg.norm(vf))}
    Ff = srf.get(2, P)
    out["F_rel_err"] = float(np.linalg.norm(Fm - Ff) / np.linalg.norm(Ff))
    for x in (srf, Sf, Hf, qf):
        x.close()
    return out


def steady(api, a):
    """Steady-state comparison at a converged parameter set.

    An FP64 run of `--pre` iterations from the initial parameters gives p*; then for
    each of `--pairs` seeds a mixed run and an FP64 run start from p* with the same
    Philox seed (64 thermalisation sweeps, then the bench's 8 + 8 sweeps per
    iteration) for `--iters` iterations, and the mean energy per site over the last
    `--iters - --burn` iterations is taken per run.  The pair differences (mixed -
    FP64) are independent across seeds, so their mean and standard error resolve a
    systematic difference below the Monte Carlo noise of a single pair."""
    ctx = api.Context(0)
    n = LX * LY
    q, H_, S, sr = _problem(api, ctx, "fp64", SEED)
    pre = []
    for it in range(a.pre):
        r = sr.iteration(SWEEPS, THERM + DISCARD if it == 0 else DISCARD, SEED, it, SHIFT, LR, reinit=it == 0)
        pre.append(r.energy / n)
    pstar = q.get_params()
    for x in (sr, S, H_, q):
        x.close()
    if a.save_params:
        np.save(a.save_params, pstar.astype(np.complex64))
    pairs = []
    for k in range(a.pairs):
        seed = a.seed + 1000 * k
        tails = {}
        for prec in ("mixed", "fp64"):
            q, H_, S, sr = _problem(api, ctx, prec, SEED)
            q.set_params(pstar)
            ir = 2 if prec == "mixed" else 0
            e = []
            for it in range(a.iters):
                r = sr.iteration(SWEEPS, THERM + DISCARD if it == 0 else DISCARD, seed, it, SHIFT, LR,
                                 reinit=it == 0, ir_steps=ir)
                e.append(r.energy / n)
            tail = np.array(e[a.burn:])
            tails[prec] = float(tail.mean())
            for x in (sr, S, H_, q):
                x.close()
        pairs.append({"seed": seed, "mixed": tails["mixed"], "fp64": tails["fp64"],
                      "diff": tails["mixed"] - tails["fp64"]})
    ctx.close()
    d = np.array([p["diff"] for p in pairs])
    mx = np.array([p["mixed"] for p in pairs])
    fp = np.array([p["fp64"] for p in pairs])
    out = {"workload": "tfi2d_12x12_rbm_alpha2", "mode": "steady", "pre_iterations": a.pre,
           "pre_energy_per_site_last10": float(np.mean(pre[-10:])), "iterations_per_run": a.iters,
           "burn_in": a.burn, "pairs": pairs,
           "mean_diff_per_site": float(d.mean()),
           "sem_diff_per_site": float(d.std(ddof=1) / np.sqrt(len(d))) if len(d) > 1 else None,
           "mixed_mean": float(mx.mean()), "mixed_sem": float(mx.std(ddof=1) / np.sqrt(len(mx))) if len(mx) > 1 else None,
           "fp64_mean": float(fp.mean()), "fp64_sem": float(fp.std(ddof=1) / np.sqrt(len(fp))) if len(fp) > 1 else None}
    print(json.dumps(out))


def main():
    from yannq_b200 import api

    ap = argparse.ArgumentParser()
    ap.add_argument("--iters", type=int, default=300)
    ap.add_argument("--every", type=int, default=50)
    ap.add_argument("--seed", type=int, default=SEED, help="parameter and Philox seed of both runs")
    ap.add_argument("--steady", action="store_true", help="seed pairs at a converged parameter set (see steady())")
    ap.add_argument("--pre", type=int, default=300, help="--steady: FP64 iterations that reach p*")
    ap.add_argument("--pairs", type=int, default=36, help="--steady: seed pairs")
    ap.add_argument("--burn", type=int, default=25, help="--steady: iterations left out of each run's mean")
    ap.add_argument("--save-params", default="", help="--steady: write p* (complex64 .npy) here")
    a = ap.parse_args()
    if a.steady:
        steady(api, a)
        return
    ctx = api.Context(0)
    n = LX * LY
    runs = {}
    checks = []
    for prec in ("mixed", "fp64"):
        q, H_, S, sr = _problem(api, ctx, prec, a.seed)
        ir = 2 if prec == "mixed" else 0
        e = []
        for it in range(a.iters):
            first = it == 0
            r = sr.iteration(SWEEPS, THERM + DISCARD if first else DISCARD, a.seed, it, SHIFT, LR, reinit=first,
                             ir_steps=ir)
            e.append(r.energy / n)
            if prec == "mixed" and a.every and (it + 1) % a.every == 0:
                S.sample(SWEEPS, DISCARD, a.seed + 1, 1_000_000 + it, False)
                checks.append(dict(iteration=it + 1, **_same_samples(api, ctx, q, S, sr)))
        tail = np.array(e[-max(1, a.iters // 4):])
        runs[prec] = {"E_per_site": e, "tail_mean": float(tail.mean()),
                      "tail_sem": float(tail.std(ddof=1) / np.sqrt(len(tail))) if len(tail) > 1 else 0.0}
        for x in (sr, S, H_, q):
            x.close()
    ctx.close()
    d = abs(runs["mixed"]["tail_mean"] - runs["fp64"]["tail_mean"])
    sem = float(np.hypot(runs["mixed"]["tail_sem"], runs["fp64"]["tail_sem"]))
    print(json.dumps({"workload": "tfi2d_12x12_rbm_alpha2", "seed": a.seed, "iterations": a.iters, "runs": runs,
                      "tail_dE_per_site": d, "tail_combined_sem": sem, "same_sample_checks": checks}))


if __name__ == "__main__":
    main()
