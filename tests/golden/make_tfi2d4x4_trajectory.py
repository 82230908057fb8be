"""Writes tfi2d4x4_trajectory.json: the oracle's restated RunRBM loop
(oracle/pyoracle.py run_rbm, Runners/RunRBM.hpp:151-221) on the precision
workload's model at a lattice the CPU restatement runs in minutes -- 2D TFI on a
periodic 4 x 4 torus, J = -1, h = -3 (H = -sum ZZ - 3 sum X), RBM alpha = 2
(M = 32, P = 560), complex128 parameters N(0, 0.01^2) from seed 20261203, 1024
chains re-randomised every epoch with 64 thermalisation sweeps, 8 recorded sweeps
(8192 samples, so the S-form), LLT with shift 1e-3, SGD rate 0.01, 300 epochs --
and the exact ground energy of the torus (Lanczos over the 2^16 basis).

    python tests/golden/make_tfi2d4x4_trajectory.py
"""
import json
import os
import sys

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)

LX, LY, ALPHA, SEED, CHAINS, THERM, SWEEPS, SHIFT, LR, EPOCHS = 4, 4, 2, 20261203, 1024, 64, 8, 1e-3, 0.01, 300


def main():
    from oracle import pyoracle as orc

    orc.build()
    n = LX * LY
    m = ALPHA * n
    ham = orc.Ham.tfi2d(LX, LY, -1.0, -3.0)
    p = orc.init_params(n, m, SEED, 0.01)
    out, _ = orc.run_rbm(ham, m, p, CHAINS, EPOCHS, SWEEPS, THERM, SEED, SHIFT, LR)
    doc = {"lx": LX, "ly": LY, "n": n, "m": m, "seed": SEED, "chains": CHAINS, "n_discard": THERM,
           "n_sweeps": SWEEPS, "shift": SHIFT, "lr": LR, "epochs": EPOCHS, "ed_energy": orc.ed_ground(ham),
           "energies": [o["energy"] for o in out]}
    with open(os.path.join(os.path.dirname(os.path.abspath(__file__)), "tfi2d4x4_trajectory.json"), "w") as f:
        json.dump(doc, f)


if __name__ == "__main__":
    main()
