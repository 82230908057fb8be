"""Writes the RBM checkpoint fixtures of tests/golden/ from the oracle's restatement
of the reference's cereal format (oracle/pyoracle.py rbm_archive):

    python tests/golden/make_rbm_archives.py

Each fixture is a small machine with fixed parameter values (entry k of the
reference layout [W col-major | a | b] is (k + 1) / 8 - 1j * k / 16, exactly
representable in float and double), so the bytes can also be checked by hand.
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))

CASES = [
    # name, n, m, use_bias, elem (0 complex<float>, 1 complex<double>, 2 double, 3 float)
    ("rbm_c128_n3_m2_bias.bin", 3, 2, True, 1),
    ("rbm_c64_n3_m2_bias.bin", 3, 2, True, 0),
    ("rbm_c128_n2_m4_nobias.bin", 2, 4, False, 1),
    ("rbm_f64_n3_m2_bias.bin", 3, 2, True, 2),
]


def params(n, m, use_bias, real):
    P = n * m + (n + m if use_bias else 0)
    k = np.arange(P, dtype=np.float64)
    return (k + 1) / 8 + (0 if real else -1j * k / 16)


def main():
    from oracle import pyoracle as orc

    for name, n, m, bias, elem in CASES:
        data = orc.rbm_archive(n, m, params(n, m, bias, elem >= 2), bias, elem)
        with open(os.path.join(HERE, name), "wb") as f:
            f.write(data)
        print(name, len(data))


if __name__ == "__main__":
    main()
