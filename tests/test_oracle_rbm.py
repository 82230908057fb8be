"""Pins the oracle's RBM math to the reference's own unit tests.

Each test re-expresses a reference test (cited) against the restatement in
oracle/oracle.hpp, plus the Random123 known-answer vectors for the RNG.
"""
import cmath
import math

import numpy as np
import pytest


def test_philox_known_answers(orc):
    # Random123 kat_vectors, philox4x32 with 10 rounds (Salmon et al., SC'11)
    kat = [
        ([0, 0, 0, 0], [0, 0], [0x6627E8D5, 0xE169C58D, 0xBC57AC4C, 0x9B00DBD8]),
        ([0xFFFFFFFF] * 4, [0xFFFFFFFF] * 2, [0x408F276D, 0x41C83B0E, 0xA20BC7C6, 0x6D5451FD]),
        ([0x243F6A88, 0x85A308D3, 0x13198A2E, 0x03707344], [0xA4093822, 0x299F31D0],
         [0xD16CFE09, 0x94FDCCEB, 0x5001E420, 0x24126EA1]),
    ]
    for ctr, key, want in kat:
        assert list(orc.philox(ctr, key)) == want


def test_logcosh_complex_grid(orc):
    # Tests/TestUtility.cpp:13-32: complex logCosh vs log(cosh) on [-10, 10]^2, 1e-7
    for x in np.linspace(-10, 10, 41):
        for y in np.linspace(-10, 10, 41):
            z = complex(x, y)
            got = orc.logcosh(z)
            ref = cmath.log(cmath.cosh(z))
            # compare modulo 2 pi i
            assert abs(cmath.exp(got - ref) - 1) < 1e-7


def test_logcosh_real_branch(orc):
    for x in [0.0, 1e-3, 3.0, 11.99, 12.0, 12.01, 40.0, -50.0]:
        want = abs(x) - math.log(2) if abs(x) > 12 else math.log(math.cosh(x))
        assert orc.logcosh_real(x) == pytest.approx(want, rel=1e-14, abs=1e-15)


def _rbm(orc, n, m, seed, sd):
    return orc.init_params(n, m, seed, sd)


def _same_ratio(a, b, tol):
    # Tests/TestRBMStates.cpp:26-60 IsSameRatio: equal modulo 2 pi i
    d = a - b
    k = round(d.imag / (2 * math.pi))
    return abs(d.real) < tol and abs(d.imag - 2 * math.pi * k) < tol


@pytest.mark.parametrize("seed", [1, 2, 3])
def test_logratio_against_logpsi(orc, seed):
    # Tests/TestRBMStates.cpp:93-212: N = M = 10, weights N(0, 1)
    n = m = 10
    p = _rbm(orc, n, m, seed, 1.0)
    rng = np.random.default_rng(seed)
    for _ in range(20):
        s = rng.choice([-1, 1], size=n).astype(np.int8)
        th = orc.theta(n, m, p, s)
        lp = orc.logpsi(n, m, p, s)
        for flips in ([int(rng.integers(n))], list(rng.choice(n, 2, replace=False)),
                      list(rng.choice(n, 4, replace=False))):
            s2 = s.copy()
            s2[flips] *= -1
            want = orc.logpsi(n, m, p, s2) - lp
            got = orc.logratio(n, m, p, s, th, flips)
            assert _same_ratio(got, want, 1e-6)


def test_theta_cache_after_flips(orc):
    # Tests/TestRBMStates.cpp:214-236: after 100 flips theta equals a fresh calcTheta
    n = m = 10
    p = _rbm(orc, n, m, 7, 1.0)
    rng = np.random.default_rng(0)
    s = rng.choice([-1, 1], size=n).astype(np.int8)
    th = orc.theta(n, m, p, s)
    for _ in range(100):
        k = int(rng.integers(3))
        flips = list(rng.choice(n, k + 1, replace=False))
        orc.flip(n, m, p, s, th, flips)
    fresh = orc.theta(n, m, p, s)
    assert np.max(np.abs(th - fresh)) < 1e-10


def test_logderiv_finite_difference(orc):
    # Tests/TestRBM.cpp:184-230: logDeriv vs central differences (holomorphic derivative)
    n, m = 8, 12
    p = _rbm(orc, n, m, 11, 0.3)
    rng = np.random.default_rng(5)
    s = rng.choice([-1, 1], size=n).astype(np.int8)
    th = orc.theta(n, m, p, s)
    O = orc.logderiv(n, m, p, s, th)
    h = 1e-6
    err = 0.0
    for k in range(len(p)):
        pp, pm = p.copy(), p.copy()
        pp[k] += h
        pm[k] -= h
        fd = (orc.logpsi(n, m, pp, s) - orc.logpsi(n, m, pm, s)) / (2 * h)
        err += abs(fd - O[k])
    assert err / (n * m) < 1e-6


def test_coeff_matches_logcoeff(orc):
    n, m = 6, 9
    p = _rbm(orc, n, m, 3, 0.5)
    s = np.array([1, -1, 1, 1, -1, -1], np.int8)
    assert cmath.exp(orc.logpsi(n, m, p, s)) == pytest.approx(orc.psi(n, m, p, s), rel=1e-12)


def test_param_init_statistics_and_order(orc):
    # Machines/RBM.hpp:325-349: a, b, then W; sd scales N(0, 1) draws
    n, m = 16, 32
    p1 = orc.init_params(n, m, 20261203, 0.01)
    p2 = orc.init_params(n, m, 20261203, 0.02)
    assert np.allclose(p2, 2 * p1)
    x = np.concatenate([p1.real, p1.imag]) / 0.01
    assert abs(x.mean()) < 0.1 and abs(x.std() - 1) < 0.1
    p3 = orc.init_params(n, m, 20261204, 0.01)
    assert not np.allclose(p1, p3)


def test_random_sigma_fixed_magnetisation(orc):
    # Utilities/Utility.hpp:77-88 randomSigma(n, nup): exactly nup entries equal -1
    seen = set()
    for c in range(200):
        s = orc.random_sigma(12, 6, 99, 0, c)
        assert (s == -1).sum() == 6 and set(np.unique(s)) <= {-1, 1}
        seen.add(s.tobytes())
    assert len(seen) > 150
