"""Reduced-size runs of the VMC step for kernel profiling (ncu captures).

    python -m yannq_b200.profile_cases --case iteration --chains 1024 --sweeps 2 --precision mixed

runs the precision workload's machine (12 x 12 TFI, RBM alpha = 2) for
`--iters` iterations with fewer recorded sweeps, so that one capture of each
kernel (sampler, local energy, O writer, tcgen05 Gram, Cholesky) ends quickly
while its inputs stay larger than L2 (O~ of 2048 x 41,904 complex64 = 0.69 GB,
BF16 operand planes 1.4 GB).

    python -m yannq_b200.profile_cases --case sampler_scaling

times the complex64 sampler of the same lattice (1024 chains, 8 + 8 local sweeps
per call, chains kept) at M = 288, 192, 144, 96, 64, 32 hidden units, i.e. 9 down
to 1 hidden units per lane: device ms of the sample stage, best of three calls.

    python -m yannq_b200.profile_cases --case xxz_o --chains 4096 --sweeps 4 --precision mixed

builds the S-form SR of the kernel-throughput machine (XXZ chain N = 64, Delta = 1,
Sz = 0, RBM alpha = 4, P = 16,704; neighbour exchanges) on chains x sweeps samples,
so that the centred O writer (o_writer_kernel) writes a few GB: 16,384 x 16,704
complex64 = 2.2 GB.
"""
import argparse
import os
import sys

sys.path.insert(0, os.path.dirname(os.path.dirname(os.path.abspath(__file__))))


def main():
    from yannq_b200 import api

    ap = argparse.ArgumentParser()
    ap.add_argument("--case", default="iteration", choices=["iteration", "sampler_scaling", "xxz_o"])
    ap.add_argument("--chains", type=int, default=1024)
    ap.add_argument("--sweeps", type=int, default=2)
    ap.add_argument("--discard", type=int, default=8)
    ap.add_argument("--iters", type=int, default=2)
    ap.add_argument("--precision", default="mixed", choices=["mixed", "fp64"])
    a = ap.parse_args()
    ctx = api.Context(0)
    n, m = 144, 288
    if a.case == "sampler_scaling":
        for mm in (288, 192, 144, 96, 64, 32):
            q = api.RBM(ctx, n, mm, True, api.C64)
            q.init_random(5, 0.01)
            S = api.Sampler(q, a.chains, api.MOVE_LOCAL)
            S.sample(8, 8, 1, 0, True)
            ts = []
            for e in range(1, 4):
                S.sample(8, 8, 1, e, False)
                ts.append(ctx.stage_ms("sample"))
            print(f"M {mm:4d}  units per lane {(mm + 31) // 32:2d}  sample {min(ts):.3f} ms  "
                  f"chains per CTA {S.chains_per_cta()}  warps per chain {S.warps_per_chain()}")
            S.close()
            q.close()
        ctx.close()
        return
    if a.case == "xxz_o":
        q = api.RBM(ctx, 64, 256, True, api.C64 if a.precision == "mixed" else api.C128)
        q.init_random(20261203, 0.01)
        H = api.Hamiltonian.xxz(ctx, 64, 1.0, 1.0, False)
        S = api.Sampler(q, a.chains, api.MOVE_EXCHANGE_NN, 32)
        S.sample(a.sweeps, 32, 20261203, 0, True)
        sr = api.SR(q, H, S, api.SR_S, api.PREC_MIXED if a.precision == "mixed" else api.PREC_FP64)
        for _ in range(a.iters):
            sr.construct()
            print(f"O stage {ctx.stage_ms('O'):.3f} ms for {a.chains * a.sweeps} x {q.dim} samples x parameters")
        for x in (sr, S, H, q, ctx):
            x.close()
        return
    q = api.RBM(ctx, n, m, True, api.C64 if a.precision == "mixed" else api.C128)
    q.init_random(20261203, 0.01)
    H = api.Hamiltonian.tfi2d(ctx, 12, 12, -1.0, -3.0)
    S = api.Sampler(q, a.chains)
    sr = api.SR(q, H, S, api.SR_T, api.PREC_MIXED if a.precision == "mixed" else api.PREC_FP64)
    for it in range(a.iters):
        r = sr.iteration(a.sweeps, a.discard, 20261203, it, 1e-3, 0.01, reinit=(it == 0),
                         ir_steps=2 if a.precision == "mixed" else 0)
        print(f"iter {it}: E/N = {r.energy / n:.8f}  |v| = {r.update_norm:.4e}  acc = {r.accept_rate:.3f}  "
              f"total {ctx.stage_ms('total'):.2f} ms")
    for x in (sr, S, H, q, ctx):
        x.close()


if __name__ == "__main__":
    main()
