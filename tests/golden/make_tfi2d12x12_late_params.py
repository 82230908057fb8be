"""Writes tfi2d12x12_late_params.npy (needs a B200): the FP64 path's parameters
after 300 iterations of the bench workload -- 12 x 12 periodic TFI, J = -1,
h = -3, RBM alpha = 2 (P = 41,904) from N(0, 0.01^2) with seed 20261203, 1024
persistent chains (64 thermalisation sweeps, then 8 + 8 sweeps per iteration),
T-form SR with shift 1e-3, SGD 0.01 -- stored as complex64.  These are the
converged parameters at which the mixed and FP64 SR steps are compared on the
same samples (tests/test_gpu_precision.py), where T is ill-conditioned.  The same
parameters start every seed pair of `python -m yannq_b200.precision_run --steady`,
which writes them with --save-params.

    python tests/golden/make_tfi2d12x12_late_params.py
"""
import os
import sys

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)


def main():
    import numpy as np

    from yannq_b200 import api
    from yannq_b200.precision_run import DISCARD, LR, SEED, SHIFT, SWEEPS, THERM, _problem

    ctx = api.Context(0)
    q, H, S, sr = _problem(api, ctx, "fp64", SEED)
    for it in range(300):
        sr.iteration(SWEEPS, THERM + DISCARD if it == 0 else DISCARD, SEED, it, SHIFT, LR, reinit=it == 0)
    p = q.get_params()
    for x in (sr, S, H, q, ctx):
        x.close()
    np.save(os.path.join(os.path.dirname(os.path.abspath(__file__)), "tfi2d12x12_late_params.npy"),
            p.astype(np.complex64))


if __name__ == "__main__":
    main()
