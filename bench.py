#!/usr/bin/env python
"""VMC iterations/s of one variational Monte Carlo step (sample -> E_loc -> O ->
SR solve -> SGD update) on one B200, mixed precision vs plain FP64.

Workload (the precision configuration): 2D transverse-field Ising model on a
periodic 12 x 12 lattice (N = 144), H = -sum ZZ - 3 sum X, RBM alpha = 2
(M = 288, P = 41,904), parameters N(0, 0.01^2) from the seed; 1024 persistent
Metropolis chains of single-spin flips, 64 thermalisation sweeps before timing,
then per iteration 8 decorrelation + 8 recorded sweeps -> 8192 samples; SR in
the sample-space form T = O~ O~^H / Ns + 1e-3 I (Ns < P), Cholesky, SGD lr 0.01.

  mixed: complex64 sampling / E_loc / O, BF16x3 tcgen05 Gram with FP32
         accumulation, panel Cholesky (FP64 tile panels, BF16x3 tcgen05 trailing
         updates) as the preconditioner of three CG iterations with FP64
         residuals, FP64 means.
  fp64:  complex128 end to end, FP64 DMMA (tensor-core m8n8k4) Gram, FP64 tile
         Cholesky.

--impl reference times the CPU restatement of the reference path (OpenMP
oracle + numpy BLAS/LAPACK for the dense algebra) on a bounded sample of the
same workload per step and extrapolates each piece to one iteration (the line
says so field by field); --impl reference --cpu-full-iteration times one whole
iteration beside that estimate.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import threading
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

W = dict(workload="tfi2d_12x12_rbm_alpha2", lx=12, ly=12, J=-1.0, h=-3.0, alpha=2, chains=1024, n_sweeps=8,
         n_discard=8, therm=64, shift=1e-3, lr=0.01, seed=20261203, init_sd=0.01)
METRIC = "VMC iters/s (sample+E_loc+O+SR) mixed vs FP64 plain, same B200, equal E err"


def _peaks():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            return json.load(f), "measured"
    except OSError:
        return {"hbm_gbs": 6650.0, "bf16_tflops": 1590.0, "bf16_tflops_sustained": 1400.0}, "fallback"


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled every 200 ms while timing."""

    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,clocks_event_reasons.hw_slowdown,"
         "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
         "clocks_event_reasons.sw_power_cap")

    def __init__(self, device):
        self.device, self.rows, self.proc = device, [], None

    def start(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", f"--id={self.device}", f"--query-gpu={self.Q}",
                                          "--format=csv,noheader,nounits", "-lms", "200"], stdout=subprocess.PIPE,
                                         stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except OSError:
            self.proc = None

    def _read(self):
        for line in self.proc.stdout:
            self.rows.append([x.strip() for x in line.split(",")])

    def stop(self):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()
        sm = [float(r[1]) for r in self.rows if len(r) > 2 and r[1].replace(".", "").isdigit()]
        mx = [float(r[2]) for r in self.rows if len(r) > 2 and r[2].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[i] for r in self.rows if len(r) >= 9 for i in range(4) if r[5 + i] == "Active"})
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": reasons, "samples": len(self.rows)}


def _dist():
    ws = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    lrank = int(os.environ.get("LOCAL_RANK", "0"))
    pg = None
    if ws > 1:
        import datetime

        import torch.distributed as dist

        dist.init_process_group("gloo", timeout=datetime.timedelta(seconds=600))
        pg = dist
    return ws, rank, lrank, pg


def _barrier(pg):
    if pg:
        pg.barrier()


def _max(pg, x):
    if not pg:
        return x
    import torch

    t = torch.tensor([x], dtype=torch.float64)
    pg.all_reduce(t, op=pg.ReduceOp.MAX)
    return float(t.item())


def _build_problem(api, ctx, precision):
    n = W["lx"] * W["ly"]
    m = W["alpha"] * n
    dtype = api.C64 if precision == "mixed" else api.C128
    q = api.RBM(ctx, n, m, True, dtype)
    q.init_random(W["seed"], W["init_sd"])
    H = api.Hamiltonian.tfi2d(ctx, W["lx"], W["ly"], W["J"], W["h"])
    S = api.Sampler(q, W["chains"], api.MOVE_LOCAL)
    sr = api.SR(q, H, S, api.SR_T, api.PREC_MIXED if precision == "mixed" else api.PREC_FP64)
    return q, H, S, sr


def _run_precision(api, ctx, precision, steps, warmup, pg, device, with_e2e):
    import numpy as np

    q, H, S, sr = _build_problem(api, ctx, precision)
    ir = 2 if precision == "mixed" else 0
    epoch = 0

    def it(reinit, n_discard):
        nonlocal epoch
        r = sr.iteration(W["n_sweeps"], n_discard, W["seed"], epoch, W["shift"], W["lr"], reinit=reinit, ir_steps=ir)
        epoch += 1
        return r

    it(True, W["therm"])  # thermalisation of the persistent chains (untimed)
    for _ in range(max(0, warmup - 1)):
        it(False, W["n_discard"])
    ctx.synchronize()
    _barrier(pg)
    clocks = ClockSampler(device)
    clocks.start()
    l0 = api.launch_count()
    stage_sum = {k: 0.0 for k in api.STAGES}
    energies = []
    t0 = time.perf_counter()
    for _ in range(steps):
        r = it(False, W["n_discard"])
        energies.append(r.energy)
        for k in stage_sum:
            stage_sum[k] += ctx.stage_ms(k)
    ctx.synchronize()
    wall = time.perf_counter() - t0
    launches = (api.launch_count() - l0) // max(1, steps)
    clk = clocks.stop()
    _barrier(pg)
    dev_ms = _max(pg, stage_sum["total"]) / steps
    out = dict(ms_per_step=dev_ms, wall_ms_per_step=1e3 * wall / steps, stages_ms={k: v / steps for k, v in
                                                                                     stage_sum.items()},
               energy_per_site=float(np.mean(energies)) / (W["lx"] * W["ly"]), launches=launches, clocks=clk,
               accept_rate=r.accept_rate, P=q.dim, Ns=W["chains"] * W["n_sweeps"])
    if with_e2e:
        # end to end through the public API: parameters from pinned host memory in,
        # updated parameters and the energy back, every step
        pin = api.PinnedArray((q.dim,), np.complex128)
        q.get_params(pin.array)
        ctx.synchronize()
        t0 = time.perf_counter()
        for _ in range(steps):
            q.set_params(pin.array)
            it(False, W["n_discard"])
            q.get_params(pin.array)
        ctx.synchronize()
        e2e_ms = 1e3 * (time.perf_counter() - t0) / steps
        out["e2e_ms"] = _max(pg, e2e_ms)
        out["h2d_bytes"] = q.dim * 16
        out["d2h_bytes"] = q.dim * 16 + 8 * 8 + W["chains"] * 8
        pin.free()
    out["chains_per_cta"] = S.chains_per_cta()  # the sampler autotuner's choice
    for x in (sr, S, H, q):
        x.close()
    return out


def _cpu_iteration_pieces(orc, rep, cores, full):
    """One iteration of the reference path on the host cores -- the oracle's
    restated SamplerMT / Energy / constructDelta (C++, OpenMP over chains and
    samples) and numpy BLAS/LAPACK for T = O~ O~^H / Ns, its Cholesky and the two
    triangular solves, v = O~^H y -- either whole (full=True) or as a bounded
    sample whose pieces are scaled to the whole iteration.  Returns {piece:
    {"timed": what ran, "s": measured seconds, "scale": factor to one iteration}}."""
    import numpy as np
    import scipy.linalg as sla

    n = W["lx"] * W["ly"]
    m = W["alpha"] * n
    Ns = W["chains"] * W["n_sweeps"]
    ham = orc.Ham.tfi2d(W["lx"], W["ly"], W["J"], W["h"])
    p = orc.init_params(n, m, W["seed"], W["init_sd"])
    # the sample keeps every host thread busy for about eight chains each, and the
    # zgemm block large enough to run near the full product's efficiency
    ch = W["chains"] if full else min(W["chains"], max(64, 8 * cores))
    no = Ns if full else 2048
    nb = Ns if full else 2048
    nc = Ns if full else 4096
    out = {}
    t = time.perf_counter()
    s, th, _, _ = orc.sample(n, m, p, ch, seed=W["seed"], epoch=rep, n_sweeps=W["n_sweeps"],
                             n_discard=W["n_discard"], nthreads=cores)
    out["sample"] = {"timed": f"{ch} chains x {W['n_discard'] + W['n_sweeps']} sweeps",
                     "s": time.perf_counter() - t, "scale": W["chains"] / ch}
    t = time.perf_counter()
    e = orc.eloc(ham, m, p, s, th, nthreads=cores)
    out["eloc"] = {"timed": f"{len(s)} samples", "s": time.perf_counter() - t, "scale": Ns / len(s)}
    rows = np.resize(np.arange(len(s)), no)  # sample rows reused when the sample has fewer than `no`
    t = time.perf_counter()
    O = orc.logderiv_rows(n, m, p, s[rows], th[rows], nthreads=cores)
    Oc = O - O.mean(axis=0)
    out["O"] = {"timed": f"{no} logDeriv rows + centring", "s": time.perf_counter() - t, "scale": Ns / no}
    del O
    A = Oc[:nb] if nb <= no else np.resize(Oc, (nb, Oc.shape[1]))
    t = time.perf_counter()
    T = A @ A.conj().T / Ns
    out["T"] = {"timed": f"{nb} x {nb} block of T (zgemm, K = {A.shape[1]})", "s": time.perf_counter() - t,
                "scale": (Ns / nb) ** 2}
    if full:
        G = T
        G[np.diag_indices(Ns)] += W["shift"]
        y0 = (e - e.mean()) / Ns
    else:
        X = np.random.default_rng(0).normal(size=(nc, nc)) + 1j * np.random.default_rng(1).normal(size=(nc, nc))
        G = X @ X.conj().T / nc + np.eye(nc)
        y0 = np.ones(nc, np.complex128)
    t = time.perf_counter()
    L = np.linalg.cholesky(G)
    out["cholesky"] = {"timed": f"{nc} x {nc} Cholesky", "s": time.perf_counter() - t, "scale": (Ns / nc) ** 3}
    t = time.perf_counter()
    y = sla.solve_triangular(L, y0, lower=True)
    y = sla.solve_triangular(L, y, lower=True, trans="C")
    out["solve"] = {"timed": f"two {nc} x {nc} triangular solves", "s": time.perf_counter() - t,
                    "scale": (Ns / nc) ** 2}
    t = time.perf_counter()
    v = A.conj().T @ (y[:nb] if nb <= len(y) else np.resize(y, nb))
    out["update"] = {"timed": f"O~^H y over {nb} rows", "s": time.perf_counter() - t, "scale": Ns / nb}
    del T, G, L, Oc, A, v
    return out


def _cpu_estimate(pieces):
    return sum(x["s"] * x["scale"] for x in pieces.values())


def cpu_sample(steps=1, warmup=0):
    """Reference CPU path on the host cores: every step times the bounded sample of
    one iteration (_cpu_iteration_pieces) and scales each piece to the whole
    iteration.  Returns (estimated iterations/s, cores, description, measured
    seconds per step, the last step's pieces)."""
    from oracle import pyoracle as orc

    orc.build()
    cores = os.cpu_count() or 1
    est, wall = [], []
    pieces = None
    for rep in range(warmup + steps):
        t = time.perf_counter()
        pieces = _cpu_iteration_pieces(orc, rep, cores, full=False)
        if rep >= warmup:
            wall.append(time.perf_counter() - t)
            est.append(_cpu_estimate(pieces))
    sample = ("each step times a bounded sample of one Ns = 8192 iteration and scales every piece to it: " +
              "; ".join(f"{k}: {v['timed']} x {v['scale']:.4g}" for k, v in pieces.items()) +
              " (OpenMP oracle restatement + numpy BLAS/LAPACK; the whole-iteration estimate is checked against one "
              "fully measured iteration in profiles/cpu_iteration_tfi2d12x12.md)")
    return 1.0 / statistics.mean(est), cores, sample, statistics.mean(wall), pieces


def cpu_full_iteration():
    """One whole reference iteration on the host cores (no scaling) beside the
    bounded-sample estimate of the same host: the check of the extrapolation."""
    from oracle import pyoracle as orc

    orc.build()
    cores = os.cpu_count() or 1
    for rep in range(3):  # the bounded sample as the reference arm runs it: warm, the third call counts
        pieces = _cpu_iteration_pieces(orc, rep, cores, full=False)
    est = _cpu_estimate(pieces)
    t = time.perf_counter()
    full = _cpu_iteration_pieces(orc, 0, cores, full=True)
    total = time.perf_counter() - t
    return {"cores": cores, "full_iteration_s": total, "full_pieces_s": {k: v["s"] for k, v in full.items()},
            "estimate_s": est, "estimate_pieces_s": {k: v["s"] * v["scale"] for k, v in pieces.items()},
            "estimate_over_measured": est / total}


def suite(api, ctx, hbm_gbs):
    """Secondary workloads, reported beside the headline.

    xxz64: 1D XXZ chain N = 64, Delta = 1, periodic, Sz = 0, RBM alpha = 4 (P = 16,704),
    4096 chains x 32 recorded sweeps (+32 thermalisation) of anti-aligned neighbour
    exchanges -> 131,072 samples; times the sampler, E_loc and the O writer (HBM write
    bound: Ns P x 8 / 16 bytes) in complex64 and complex128.
    ff40: FeedForward Conv1D(1->12, K 5) -> LnCosh -> FC(480->16) -> LnCosh -> Sum on
    N = 40 spins (P = 7,740), forward + adjoint at batch 4096 / 16384 / 65536 with
    activations stored vs recomputed; O write bandwidth, TFI E_loc at h = 1.
    """
    out = {}
    n, m, chains, sweeps = 64, 256, 4096, 32
    for name, dt, prec in (("c64", api.C64, api.PREC_MIXED), ("c128", api.C128, api.PREC_FP64)):
        q = api.RBM(ctx, n, m, True, dt)
        q.init_random(W["seed"], 0.01)
        H = api.Hamiltonian.xxz(ctx, n, 1.0, 1.0, False)
        S = api.Sampler(q, chains, api.MOVE_EXCHANGE_NN, n // 2)
        sr = api.SR(q, H, S, api.SR_S, prec)
        S.sample(sweeps, 32, W["seed"], 0, True)
        S.sample(sweeps, 32, W["seed"], 1, True)
        t_s = ctx.stage_ms("sample")
        sr.construct()
        sr.construct()
        t_e, t_o = ctx.stage_ms("eloc"), ctx.stage_ms("O")
        ns = chains * sweeps
        bytes_o = ns * q.dim * (8 if dt == api.C64 else 16)
        out[f"xxz64_{name}"] = {"samples": ns, "P": q.dim, "sample_ms": t_s, "samples_per_s": ns / (t_s * 1e-3),
                                "proposals_per_s": chains * (sweeps + 32) * n / (t_s * 1e-3), "eloc_ms": t_e,
                                "O_ms": t_o, "O_GBps": bytes_o / (t_o * 1e-3) / 1e9,
                                "O_frac_of_hbm": bytes_o / (t_o * 1e-3) / 1e9 / hbm_gbs}
        for x in (sr, S, H, q):
            x.close()
    f = api.FeedForward(ctx, 40, 12, 5, 16)
    f.init_random(W["seed"])
    ff = {}
    for batch in (4096, 16384, 65536):
        f.random_batch(batch, W["seed"])
        row = {}
        for mode, budget in (("store", 1 << 62), ("recompute", 0)):
            f.forward(budget, copy=False)
            f.adjoint(copy=False)
            f.forward(budget, copy=False)
            tf = ctx.stage_ms(8)
            f.adjoint(copy=False)
            ta = ctx.stage_ms(9)
            row[mode] = {"forward_ms": tf, "adjoint_ms": ta,
                         "O_GBps": batch * f.dim * 4 / (ta * 1e-3) / 1e9}
        f.eloc_tfi(-1.0, -1.0, copy=False)
        f.eloc_tfi(-1.0, -1.0, copy=False)
        row["eloc_ms"] = ctx.stage_ms(10)
        ff[str(batch)] = row
    f.close()
    out["ff40"] = ff
    out["config_a_tfi16"] = config_a(api, ctx)
    out["batch64"] = batch64(api)
    out["j1j2_64"] = j1j2_64(api, ctx)
    out["ngd_ap_j1j2_20"] = ngd_ap(api, ctx)
    return out


def config_a(api, ctx, epochs=200):
    """The small plain configuration (Examples/RBMTFI.cpp call pattern): TFI chain
    N = 16, J = -1, h = -1, RBM alpha = 2 (P = 560), complex128 N(0, 0.01^2), 16
    chains re-randomised every epoch with 64 thermalisation + 64 recorded sweeps
    (1024 samples, S-form), LLT shift 1e-3, SGD 0.01, 200 epochs, FP64 throughout;
    and the same optimisation by exact summation over the 2^16 states
    (RunRBMExact).  Host wall time around the synchronous calls; energies per site
    of the last 50 epochs (sampled) and the last epoch (exact)."""
    import numpy as np

    n, m, seed = 16, 32, W["seed"]
    out = {}
    q = api.RBM(ctx, n, m, True, api.C128)
    q.init_random(seed, 0.01)
    H = api.Hamiltonian.tfi(ctx, n, -1.0, -1.0)
    S = api.Sampler(q, 16)
    sr = api.SR(q, H, S, api.SR_AUTO, api.PREC_FP64)
    t0 = time.perf_counter()
    es = [sr.iteration(64, 64, seed, ll, 1e-3, 0.01, reinit=True).energy / n for ll in range(epochs)]
    dt = time.perf_counter() - t0
    out["sampled"] = {"epochs": epochs, "iters_per_s": epochs / dt, "ms_per_iteration": 1e3 * dt / epochs,
                      "tail50_energy_per_site": float(np.mean(es[-50:])),
                      "tail50_sem": float(np.std(es[-50:], ddof=1) / np.sqrt(50)), "first": es[0]}
    for x in (sr, S):
        x.close()
    q.init_random(seed, 0.01)
    t0 = time.perf_counter()
    ee = [api.exact_iteration(q, H, 1e-3, 0.01)[0] / n for _ in range(epochs)]
    dt = time.perf_counter() - t0
    out["exact_summation"] = {"epochs": epochs, "iters_per_s": epochs / dt, "ms_per_iteration": 1e3 * dt / epochs,
                              "last_energy_per_site": ee[-1], "first": ee[0]}
    for x in (H, q):
        x.close()
    return out


def j1j2_64(api, ctx):
    """J1J2 chain N = 64 (J2 = 0.5, sign rule), RBM alpha = 4, complex64, Sz = 0:
    4096 chains x 32 recorded sweeps (+32 thermalisation) with the HamiltonianSweeper
    (proposals from the antiparallel NN / NNN bonds, w1 / w2 correction) against
    neighbour-pair exchanges; E_loc over the 131,072 samples (term table)."""
    n, m, chains, sweeps = 64, 256, 4096, 32
    res = {}
    q = api.RBM(ctx, n, m, True, api.C64)
    q.init_random(W["seed"], 0.01)
    H = api.Hamiltonian.j1j2(ctx, n, 1.0, 0.5, True)
    for name, move in (("hamiltonian_sweeper", api.MOVE_HAMILTONIAN), ("exchange_nn", api.MOVE_EXCHANGE_NN)):
        S = api.Sampler(q, chains, move, n // 2)
        if move == api.MOVE_HAMILTONIAN:
            S.set_hamiltonian(H)
        S.sample(sweeps, 32, W["seed"], 0, True)
        S.sample(sweeps, 32, W["seed"], 1, True)
        t_s = ctx.stage_ms("sample")
        row = {"sample_ms": t_s, "proposals_per_s": chains * (sweeps + 32) * n / (t_s * 1e-3),
               "accept_rate": float(S.get_accepts().sum()) / (chains * (sweeps + 32) * n)}
        if move == api.MOVE_HAMILTONIAN:
            sr = api.SR(q, H, S, api.SR_S, api.PREC_MIXED)
            sr.construct()
            sr.construct()
            row["eloc_ms"] = ctx.stage_ms("eloc")
            row["eloc_samples_per_s"] = chains * sweeps / (row["eloc_ms"] * 1e-3)
            sr.close()
        res[name] = row
        S.close()
    H.close()
    q.close()
    return res


def ngd_ap(api, ctx, iters=3):
    """Examples/AmplitudePhase.cpp at N = 20: J1J2(20, 1, 0.44, sign rule), Jz basis
    (184,756 configurations), RBM alpha = 2 without bias (P_amp = 800) and the
    example's phase network Conv1D 1->12->10->8->6->4->2 (kernel 5, LeakyHardTanh
    0.01), FullyConnected(40 -> 1), SoftSign (P_phase = 1,500); one NGDExact epoch
    (construct, both LLT solves, SGD) per iteration, host wall time around the
    synchronous call."""
    n = 20
    layers = []
    for a, b in [(1, 12), (12, 10), (10, 8), (8, 6), (6, 4), (4, 2)]:
        layers += [("conv1d", a, b, 5), ("leakyhardtanh", 0.01)]
    layers += [("fc", 2 * n, 1, False), ("softsign",)]
    q = api.AmplitudePhase(ctx, n, 2 * n, False, layers)
    q.init_random(W["seed"], 0.01, api.INIT_XAVIER)
    H = api.Hamiltonian.j1j2(ctx, n, 1.0, 0.44, True)
    g = api.NGDExact(q, H, api.BASIS_JZ, n // 2)
    g.iteration(10.0, 0.05)  # warm-up
    t0 = time.perf_counter()
    for ll in range(iters):
        e, gn, vn = g.iteration(max(10.0 * 0.9 ** (ll + 1), 1e-3), 0.05)
    dt = (time.perf_counter() - t0) / iters
    res = {"basis": g.basis_size, "P_amp": q.dim_amp, "P_phase": q.dim_phase, "ms_per_epoch": dt * 1e3,
           "epochs_per_s": 1.0 / dt, "energy_per_site": e / n,
           "gram_flop_per_epoch": 2.0 * g.basis_size * (q.dim_amp ** 2 + q.dim_phase ** 2)}
    for x in (g, H, q):
        x.close()
    return res


# DRAM bytes (read + write) of the Ns = 8192, P = 41,904 Gram launch, from one
# ncu capture (1 pass: dram__bytes_read.sum 40.33 GB, dram__bytes_write.sum 0.53 GB);
# the algorithmic minimum is the 5.49 GB of BF16 operand planes plus the 0.54 GB
# lower triangle of T.
GRAM_TRAFFIC_BYTES = 40.33e9 + 0.53e9


def batch_problems(seed, count=64):
    """The 64 independent TFI-1D problems of the batching workload: N from
    {16, 20, 24, 32, 48, 64}, h ~ U[0.5, 1.5], alpha from {1, 2, 4}, complex64,
    Ns = ceil64(256 + (N - 16) 1792 / 48) samples as Ns / 8 chains x 8 sweeps,
    T-form SR (seeded numpy draws)."""
    import numpy as np

    rng = np.random.default_rng(seed)
    out = []
    for _ in range(count):
        n = int(rng.choice([16, 20, 24, 32, 48, 64]))
        h = float(rng.uniform(0.5, 1.5))
        alpha = int(rng.choice([1, 2, 4]))
        ns = int(np.ceil((256 + (n - 16) * 1792 / 48) / 64) * 64)
        out.append((n, alpha, h, ns // 8))
    return out


def batch64(api, iters=5):
    """Aggregate iterations/s (all 64 problems advanced once): the mixed path as one
    batch (eager first call, then one CUDA graph replay per iteration, problems on
    their own streams) against the FP64-plain path as 64 sequential yq_vmc_iteration
    calls.  Host wall time around synchronous calls; thermalised chains (first call
    reinitialises with 32 discarded sweeps, later calls 8 + 8)."""
    import numpy as np

    res = {}
    probs = batch_problems(W["seed"] + 17)
    for prec in ("mixed", "fp64"):
        objs = []
        for k, (n, alpha, h, chains) in enumerate(probs):
            c = api.Context(0)
            q = api.RBM(c, n, alpha * n, True, api.C64 if prec == "mixed" else api.C128)
            q.init_random(W["seed"] + k, 0.01)
            H = api.Hamiltonian.tfi(c, n, -1.0, -h)
            S = api.Sampler(q, chains)
            sr = api.SR(q, H, S, api.SR_T, api.PREC_MIXED if prec == "mixed" else api.PREC_FP64)
            objs.append((c, q, H, S, sr))
        ir = 2 if prec == "mixed" else 0
        if prec == "mixed":
            master = api.Context(0)
            B = api.Batch(master, [o[4] for o in objs])
            B.iteration(8, 32, W["seed"], 0, 1e-3, 0.01, reinit=True, ir_steps=ir)  # eager + capture
            B.iteration(8, 8, W["seed"], 1, 1e-3, 0.01, reinit=False, ir_steps=ir)  # new parameters: recapture
            B.iteration(8, 8, W["seed"], 2, 1e-3, 0.01, reinit=False, ir_steps=ir)  # replay (warm)
            t0 = time.perf_counter()
            for it in range(iters):
                r = B.iteration(8, 8, W["seed"], 3 + it, 1e-3, 0.01, reinit=False, ir_steps=ir)
            dt = (time.perf_counter() - t0) / iters
            B.close()
            master.close()
            e = [x.energy / probs[k][0] for k, x in enumerate(r)]
        else:
            for k, o in enumerate(objs):
                o[4].iteration(8, 32, W["seed"] + k, 0, 1e-3, 0.01, reinit=True)
            t0 = time.perf_counter()
            for it in range(iters):
                r = [o[4].iteration(8, 8, W["seed"] + k, 1 + it, 1e-3, 0.01, reinit=False) for k, o in enumerate(objs)]
            dt = (time.perf_counter() - t0) / iters
            e = [x.energy / probs[k][0] for k, x in enumerate(r)]
        res[prec] = {"ms_per_batch_iteration": dt * 1e3, "batch_iters_per_s": 1.0 / dt,
                     "problem_iters_per_s": len(probs) / dt, "mean_energy_per_site": float(np.mean(e))}
        for c, q, H, S, sr in objs:
            for x in (sr, S, H, q, c):
                x.close()
    res["problems"] = len(probs)
    res["mixed_batch_over_fp64_sequential"] = res["mixed"]["batch_iters_per_s"] / res["fp64"]["batch_iters_per_s"]
    return res


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--precision", default="both", choices=["both", "mixed", "fp64"])
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-suite", action="store_true", help="skip the secondary workloads")
    ap.add_argument("--cpu-full-iteration", action="store_true",
                    help="with --impl reference: time one whole CPU iteration beside the bounded-sample estimate")
    args = ap.parse_args()
    ws, rank, lrank, pg = _dist()
    warmup = max(3, args.warmup)

    if args.impl == "reference":
        if rank != 0:
            return
        if args.cpu_full_iteration:
            print(json.dumps({"impl": "reference", "workload": W["workload"], **cpu_full_iteration()}))
            return
        v, cores, sample, step_s, pieces = cpu_sample(steps=args.steps, warmup=warmup)
        print(json.dumps({"impl": "reference", "metric": METRIC, "value": v, "unit": "iters/s", "n_gpus": 0,
                          "steps": args.steps, "warmup": warmup, "ms_per_step": 1e3 * step_s,
                          "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
                          "data": "synthetic",
                          "config": {"workload": W["workload"], "Ns": W["chains"] * W["n_sweeps"],
                                     "chains": W["chains"], "inputs": "larger than L2"},
                          "extrapolated": {"value_is": "whole-iteration rate estimated from each step's bounded "
                                                       "sample; ms_per_step is the measured time of one step",
                                           "estimate_ms_per_iteration": 1e3 / v,
                                           "pieces": {k: {"timed": x["timed"], "ms": 1e3 * x["s"],
                                                          "scale": x["scale"]} for k, x in pieces.items()},
                                           "check": "profiles/cpu_iteration_tfi2d12x12.md"},
                          "cpu_baseline": {"value": v, "unit": "iters/s", "cores": cores, "kind": "port",
                                           "sample": sample},
                          "e2e": {"value": v, "unit": "iters/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}))
        return

    from yannq_b200 import api

    ctx = api.Context(lrank)
    dev_peaks = ctx.measure_peaks()
    res = {}
    precs = ["mixed", "fp64"] if args.precision == "both" else [args.precision]
    for prec in precs:
        res[prec] = _run_precision(api, ctx, prec, args.steps, warmup, pg, lrank, with_e2e=(prec == precs[0]))
    head = res[precs[0]]
    peaks, src = _peaks()
    Ns, P = head["Ns"], head["P"]
    if precs[0] == "mixed":
        flops = 12.0 * Ns * Ns * P  # three BF16 products of the complex Hermitian lower triangle (4 Ns^2 P each)
        t_ms = head["stages_ms"]["gram"]
        ach = flops / (t_ms * 1e-3) / 1e12
        # the Gram is timed inside a ~70 ms step: the sustained BF16 figure is its roof
        pk = peaks.get("bf16_tflops_sustained") or peaks.get("bf16_tflops")
        roof = {"kernel": "herk_tc_kernel (tcgen05 BF16x3 Gram T = O~O~^H, Re and Im per CTA)", "bound": "tensor",
                "achieved": ach, "peak": pk, "unit": "TFLOP/s", "frac": ach / pk,
                "frac_of_burst": ach / peaks.get("bf16_tflops"),
                "peak_source": src + (" (sustained)" if peaks.get("bf16_tflops_sustained") else ""),
                "traffic": GRAM_TRAFFIC_BYTES if (Ns, P) == (8192, 41904) else None,
                "traffic_source": "ncu dram__bytes_read.sum + dram__bytes_write.sum of one Ns = 8192 Gram launch "
                                  "(profiles/herk_tc_kernel_gram_tfi2d12x12.md)"}
    else:
        flops = 4.0 * Ns * Ns * P
        t_ms = head["stages_ms"]["gram"]
        ach = flops / (t_ms * 1e-3) / 1e12
        pk = max(dev_peaks["fp64_simt_tflops"], dev_peaks["fp64_dmma_tflops"])
        roof = {"kernel": "gemm_z_dmma_kernel (FP64 tensor-core DMMA T = O~O~^H)", "bound": "fp64", "achieved": ach,
                "peak": pk, "unit": "TFLOP/s", "frac": ach / pk, "peak_source": "measured by yq_measure_peaks",
                "traffic": None}
    value = ws * 1e3 / head["ms_per_step"]
    line = {"metric": METRIC, "value": value, "unit": "iters/s", "n_gpus": ws, "steps": args.steps, "warmup": warmup,
            "ms_per_step": head["ms_per_step"], "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": "c64+bf16x3+f64" if precs[0] == "mixed" else "c128",
            "data": "synthetic (seeded Philox parameters and chains)",
            "config": {"workload": W["workload"], "precision": precs[0], "N": W["lx"] * W["ly"], "M": Ns and
                       W["alpha"] * W["lx"] * W["ly"], "P": P, "Ns": Ns, "chains": W["chains"],
                       "sweeps": f"{W['n_discard']} discard + {W['n_sweeps']} recorded per step, {W['therm']} therm",
                       "sr": "T-form, shift 1e-3, Cholesky", "parallelism": f"replicas{ws}",
                       "inputs": "larger than L2 (O~ and operands >= 2.7 GB)",
                       "sampler_chains_per_cta": head.get("chains_per_cta")},
            "gpu_launches": head["launches"], "clocks": head["clocks"], "roofline": roof,
            "stages_ms": head["stages_ms"], "energy_per_site": head["energy_per_site"], "device_peaks": dev_peaks,
            "accept_rate": head["accept_rate"]}
    if "e2e_ms" in head:
        line["e2e"] = {"value": ws * 1e3 / head["e2e_ms"], "unit": "iters/s", "h2d_bytes_per_step": head["h2d_bytes"],
                       "d2h_bytes_per_step": head["d2h_bytes"]}
    if len(precs) == 2:
        f = res["fp64"]
        line["fp64_plain"] = {"value": ws * 1e3 / f["ms_per_step"], "ms_per_step": f["ms_per_step"],
                              "stages_ms": f["stages_ms"], "energy_per_site": f["energy_per_site"],
                              "gpu_launches": f["launches"]}
        line["mixed_over_fp64"] = f["ms_per_step"] / head["ms_per_step"]
    if not args.no_suite:
        line["suite"] = suite(api, ctx, peaks.get("hbm_gbs", 6553.9))
    if rank == 0 and ws == 1 and not args.no_cpu_baseline:
        v, cores, sample, _, _ = cpu_sample(steps=1, warmup=0)
        line["cpu_baseline"] = {"value": v, "unit": "iters/s", "cores": cores, "kind": "port", "sample": sample}
    ctx.close()
    if rank == 0:
        print(json.dumps(line))
    if pg:
        pg.destroy_process_group()


if __name__ == "__main__":
    main()
