"""Writes config_a_trajectory.json: the oracle's restated RunRBM loop
(oracle/pyoracle.py run_rbm, Runners/RunRBM.hpp:151-221) on the small plain
configuration -- TFI chain N = 16, periodic, J = -1, h = -1 (H = -sum ZZ - sum X),
RBM alpha = 2 (M = 32) with complex128 parameters N(0, 0.01^2) from seed 20261203,
16 chains re-randomised every epoch, 64 thermalisation + 64 recorded sweeps (1024
samples), S-form LLT with shift 1e-3, SGD rate 0.01, 200 epochs -- and the exact
ground energy of the chain (Lanczos over the 2^16 basis).

    python tests/golden/make_config_a_trajectory.py
"""
import json
import os
import sys

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)

N, M, SEED, CHAINS, THERM, SWEEPS, SHIFT, LR, EPOCHS = 16, 32, 20261203, 16, 64, 64, 1e-3, 0.01, 200


def main():
    import numpy as np

    from oracle import pyoracle as orc

    orc.build()
    ham = orc.Ham.tfi(N, -1.0, -1.0)
    p = orc.init_params(N, M, SEED, 0.01)
    out, pf = orc.run_rbm(ham, M, p, CHAINS, EPOCHS, SWEEPS, THERM, SEED, SHIFT, LR)
    doc = {"n": N, "m": M, "seed": SEED, "chains": CHAINS, "n_discard": THERM, "n_sweeps": SWEEPS, "shift": SHIFT,
           "lr": LR, "epochs": EPOCHS, "ed_energy": orc.ed_ground(ham),
           "energies": [o["energy"] for o in out], "update_norms": [o["nv"] for o in out],
           "final_params_re": np.real(pf).tolist(), "final_params_im": np.imag(pf).tolist()}
    with open(os.path.join(os.path.dirname(os.path.abspath(__file__)), "config_a_trajectory.json"), "w") as f:
        json.dump(doc, f)


if __name__ == "__main__":
    main()
