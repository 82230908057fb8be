"""Reduced-size runs of the VMC step for kernel profiling (ncu captures).

    python -m yannq_b200.profile_cases --case iteration --chains 1024 --sweeps 2 --precision mixed

runs the precision workload's machine (12 x 12 TFI, RBM alpha = 2) for
`--iters` iterations with fewer recorded sweeps, so that one capture of each
kernel (sampler, local energy, O writer, tcgen05 Gram, Cholesky) ends quickly
while its inputs stay larger than L2 (O~ of 2048 x 41,904 complex64 = 0.69 GB,
BF16 operand planes 1.4 GB).
"""
import argparse
import os
import sys

sys.path.insert(0, os.path.dirname(os.path.dirname(os.path.abspath(__file__))))


def main():
    from yannq_b200 import api

    ap = argparse.ArgumentParser()
    ap.add_argument("--case", default="iteration", choices=["iteration"])
    ap.add_argument("--chains", type=int, default=1024)
    ap.add_argument("--sweeps", type=int, default=2)
    ap.add_argument("--discard", type=int, default=8)
    ap.add_argument("--iters", type=int, default=2)
    ap.add_argument("--precision", default="mixed", choices=["mixed", "fp64"])
    a = ap.parse_args()
    ctx = api.Context(0)
    n, m = 144, 288
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
