"""Pins the oracle's AmplitudePhase machine (Machines/AmplitudePhase.hpp, a real
RBM amplitude and a FeedForward phase) and its NGDExact restatement
(GroundState/NGDExact.hpp:123-189).

* The reference's only test of the machine (Tests/TestAmplitudePhase.cpp)
  includes a file that does not exist; its network (Conv1D stacks with
  LeakyReLU, FullyConnected, Tanh) is used here.  logDeriv is checked against
  central differences of log psi for networks that use every layer type (Conv1D
  with and without bias and stride, FullyConnected, every activation except
  Sigmoid, whose Jacobian the reference writes without the incoming gradient and
  which is therefore checked against its written form).
* NGDExact: energy, gradient, oloc and both correlation matrices against a
  direct numpy evaluation of the reference's formulas over the basis.
* The RunAmplitudePhaseExact loop (LLT of corrMat + lambda I per block, SGD)
  lowers the J1J2 energy towards exact diagonalisation.
"""
import numpy as np
import pytest

LAYERS_ALL = [
    [[0, 1, 3, 3, 1, 1], [11, 0, 0, 0, 1, 0], [0, 3, 2, 3, 2, 0], [19, 0, 0, 0, 1, 0], [1, 6, 4, 0, 1, 1],
     [12, 0, 0, 0, 1, 0], [1, 4, 3, 0, 1, 0], [16, 0, 0, 0, 1, 0], [1, 3, 2, 0, 1, 1], [13, 0, 0, 0, 1, 0],
     [1, 2, 2, 0, 1, 0], [20, 0, 0, 0, 1, 0], [1, 2, 1, 0, 1, 1], [21, 0, 0, 0, 1, 0]],
    [0, 0, 0, 0.02, 0, 1.7, 0, 0.05, 0, 0, 0, 0, 0, 1.3],
]
LAYERS_KINKS = [
    [[0, 1, 4, 5, 1, 0], [15, 0, 0, 0, 1, 0], [0, 4, 2, 3, 1, 1], [17, 0, 0, 0, 1, 0], [1, 12, 3, 0, 1, 1],
     [18, 0, 0, 0, 1, 0], [1, 3, 1, 0, 1, 0], [10, 0, 0, 0, 1, 0]],
    [0, 0, 0, 0, 0, 0, 0, 0],
]


def _ref_net(n):
    # Tests/TestAmplitudePhase.cpp:22-37 (LeakyReLU slope 0.1 default), at width n
    d, x = [], []
    for a, b in [(1, 12), (12, 10), (10, 8), (8, 6), (6, 4), (4, 2)]:
        d += [[0, a, b, 5, 1, 0], [16, 0, 0, 0, 1, 0]]
        x += [0, 0.1]
    d += [[1, 2 * n, 1, 0, 1, 0], [12, 0, 0, 0, 1, 0]]
    x += [0, 1.0]
    return d, x


@pytest.mark.parametrize("case", ["all", "kinks", "reference_net"])
def test_log_deriv_central_differences(orc, case):
    n = 6
    if case == "all":
        desc, xs = LAYERS_ALL
        m, bias, sd = 6, True, 0.3
    elif case == "kinks":
        desc, xs = LAYERS_KINKS
        m, bias, sd = 12, False, 0.4
    else:
        desc, xs = _ref_net(n)
        m, bias, sd = 4 * n, False, 0.05
    ap = orc.AP(n, m, bias, desc, xs)
    p = orc.ap_init(ap, 11, sd, 0)
    rng = np.random.default_rng(2)
    for _ in range(3):
        s = rng.choice(np.array([-1, 1], np.int8), n)
        d = orc.ap_log_deriv(ap, p, s)[0]
        eps = 1e-6
        for c in range(ap.dim):
            q1, q2 = p.copy(), p.copy()
            q1[c] += eps
            q2[c] -= eps
            fd = (orc.ap_log_psi(ap, q1, s)[0] - orc.ap_log_psi(ap, q2, s)[0]) / (2 * eps)
            assert abs(fd - d[c]) < 2e-6 * max(1.0, abs(d[c])), (case, c, fd, d[c])


def test_sigmoid_restated_as_written(orc):
    # activations.hpp:215-229: forward exp(z) + 1 (inverse() results discarded),
    # Jacobian (1 - A) A without the incoming gradient
    n = 4
    desc = [[1, 4, 1, 0, 1, 0], [14, 0, 0, 0, 1, 0]]
    ap = orc.AP(n, 2, False, desc, [0, 0])
    p = orc.ap_init(ap, 3, 0.1, 1)
    s = np.array([1, -1, -1, 1], np.int8)
    z = float(p[ap.Pa:] @ s)
    a = np.exp(z) + 1.0
    assert orc.ap_log_psi(ap, p, s)[0].imag == pytest.approx(np.pi * a, rel=1e-14)
    d = orc.ap_log_deriv(ap, p, s)[0]
    np.testing.assert_allclose(d[ap.Pa:].imag, np.pi * s * (1.0 - a) * a, rtol=1e-13)


def _dense(orc, ham, basis):
    idx = {int(b): i for i, b in enumerate(basis)}
    H = np.zeros((len(basis), len(basis)))
    for j, b in enumerate(basis):
        r, v = orc.ham_column(ham, int(b))
        for rr, vv in zip(r, v):
            if int(rr) in idx:
                H[j, idx[int(rr)]] += vv  # ConstructSparseMat.hpp:43-51: (row = idx, col = j)
    return H


@pytest.mark.parametrize("case", ["j1j2_jz", "tfi_full"])
def test_ngd_exact_against_numpy(orc, case):
    n = 8
    if case == "j1j2_jz":
        ham, bk, nup = orc.Ham.j1j2(n, 1.0, 0.4, True), 1, 4
    else:
        ham, bk, nup = orc.Ham.tfi(n, -1.0, -0.7), 0, 0
    # Conv1D(1, 2, 3, bias), LeakyHardTanh, Conv1D(2, 2, 3, stride 2), LnCosh, FC(8, 3, bias), SoftSign,
    # FC(3, 1), Tanh
    ap = orc.AP(n, 8, True, [[0, 1, 2, 3, 1, 1], [19, 0, 0, 0, 1, 0], [0, 2, 2, 3, 2, 0], [11, 0, 0, 0, 1, 0],
                            [1, 8, 3, 0, 1, 1], [20, 0, 0, 0, 1, 0], [1, 3, 1, 0, 1, 0], [12, 0, 0, 0, 1, 0]],
                [0, 0.01, 0, 0, 0, 0, 0, 1.0])
    p = orc.ap_init(ap, 7, 0.2, 1)
    res = orc.ngd_exact(ham, ap, p, bk, nup)
    basis = orc.basis(n, bk, nup)
    S = np.array([orc.sigma_of(int(b), n) for b in basis])
    lp = orc.ap_log_psi(ap, p, S)
    psi = np.exp(lp - lp.real.max())
    psi /= np.linalg.norm(psi)
    H = _dense(orc, ham, basis)
    k = H @ psi
    E = np.real(np.vdot(psi, k))
    D = orc.ap_log_deriv(ap, p, S)
    Da, Dp = D[:, :ap.Pa].real, D[:, ap.Pa:].imag
    w = np.abs(psi) ** 2
    oa, op = w @ Da, w @ Dp
    g = np.conj(psi) * k
    grad = np.concatenate([2 * Da.T @ g.real - 2 * E * oa, 2 * Dp.T @ g.imag])
    Ca = Da.T @ (w[:, None] * Da) - np.outer(oa, oa)
    Cp = Dp.T @ (w[:, None] * Dp) - np.outer(op, op)
    assert res["energy"] == pytest.approx(E, rel=1e-12)
    np.testing.assert_allclose(res["grad"], grad, atol=1e-11 * np.abs(grad).max())
    np.testing.assert_allclose(res["oloc_amp"], oa, atol=1e-12)
    np.testing.assert_allclose(res["oloc_phase"], op, atol=1e-12)
    np.testing.assert_allclose(res["corr_amp"], Ca, atol=1e-12 * np.abs(Ca).max())
    np.testing.assert_allclose(res["corr_phase"], Cp, atol=1e-12 * np.abs(Cp).max())


def test_oracle_run_amplitude_phase_descends(orc):
    """Runners/RunAmplitudePhase.hpp:92-119 in Python on the oracle: J1J2 N = 8."""
    n = 8
    ham = orc.Ham.j1j2(n, 1.0, 0.2, True)
    ap = orc.AP(n, 2 * n, False, [[0, 1, 2, 3, 1, 0], [19, 0, 0, 0, 1, 0], [1, 2 * n, 1, 0, 1, 0],
                                  [20, 0, 0, 0, 1, 0]], [0, 0.01, 0, 0])
    p = orc.ap_init(ap, 5, 0.01, 1)
    e0 = orc.ed_ground(ham, 1, 4)
    es = []
    for ll in range(40):
        r = orc.ngd_exact(ham, ap, p, 1, 4)
        lam = max(10.0 * 0.9 ** ll, 1e-3)
        va = np.linalg.solve(r["corr_amp"] + lam * np.eye(ap.Pa), r["grad"][:ap.Pa])
        vp = np.linalg.solve(r["corr_phase"] + lam * np.eye(ap.Pp), r["grad"][ap.Pa:])
        p = p - 0.05 * np.concatenate([va, vp])
        es.append(r["energy"])
    assert es[-1] < es[0] - 0.5
    assert es[-1] >= e0 - 1e-9
