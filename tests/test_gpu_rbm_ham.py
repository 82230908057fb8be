"""GPU parity of the RBM and Hamiltonian kernels against the oracle (C-ABI calls).

FP64 path: theta and parameter initialisation bit-exact; log psi, log ratios,
log derivatives and E_loc within 1e-12 relative; flip enumeration bit-exact.
complex64 path: within 1e-5 relative.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

TOL64 = 1e-12
TOL32 = 5e-5  # complex64: relative to max(|value|, 1)


@pytest.fixture(scope="module")
def ctx():
    from yannq_b200 import api

    c = api.Context(0)
    yield c
    c.close()


def _rbm(api, ctx, orc, n, m, seed, sd, dtype):
    q = api.RBM(ctx, n, m, True, dtype)
    p = orc.init_params(n, m, seed, sd)
    q.set_params(p)
    return q, p


def _rand_sigma(rng, ns, n):
    return rng.choice(np.array([-1, 1], np.int8), size=(ns, n))


def test_init_params_bit_exact(ctx, orc):
    from yannq_b200 import api

    for n, m in [(16, 32), (144, 288)]:
        q = api.RBM(ctx, n, m, True, api.C128)
        q.init_random(20261203, 0.01)
        np.testing.assert_array_equal(q.get_params(), orc.init_params(n, m, 20261203, 0.01))
        q.close()


@pytest.mark.parametrize("n,m", [(10, 10), (16, 32), (64, 256), (144, 288)])
def test_theta_bit_exact(ctx, orc, n, m):
    from yannq_b200 import api

    q, p = _rbm(api, ctx, orc, n, m, 5, 0.3, api.C128)
    rng = np.random.default_rng(n)
    s = _rand_sigma(rng, 17, n)
    got = q.theta(s)
    want = np.array([orc.theta(n, m, p, x) for x in s])
    np.testing.assert_array_equal(got, want)
    q.close()


@pytest.mark.parametrize("dtype", [1, 0])
def test_log_psi_and_ratios(ctx, orc, dtype):
    from yannq_b200 import api

    n = m = 10
    q, p = _rbm(api, ctx, orc, n, m, 7, 1.0, dtype)  # Tests/TestRBMStates.cpp: N = M = 10, N(0, 1)
    rng = np.random.default_rng(1)
    s = _rand_sigma(rng, 64, n)
    th = np.array([orc.theta(n, m, p, x) for x in s])
    tol = TOL64 if dtype == api.C128 else TOL32
    lp = q.log_psi(s)
    want = np.array([orc.logpsi(n, m, p, x) for x in s])
    assert np.max(np.abs(np.exp(lp - want) - 1)) < 1e-12  # log psi is always evaluated in FP64
    for nf in (1, 2):
        flips = np.array([rng.choice(n, nf, replace=False) for _ in range(len(s))], np.int32)
        got = q.log_ratio(s, th, flips)
        ref = np.array([orc.logratio(n, m, p, x, t, f) for x, t, f in zip(s, th, flips)])
        # compare modulo 2 pi i (Tests/TestRBMStates.cpp IsSameRatio)
        assert np.max(np.abs(np.exp(got - ref) - 1)) < tol


@pytest.mark.parametrize("dtype", [1, 0])
def test_k_flip_and_state_ratios(ctx, orc, dtype):
    """logRatio(vector<int>) and logRatio(other state) (States/RBMState.hpp:107-149)
    as Tests/TestRBMStates.cpp:93-237 checks them -- N = M = 10, weights N(0, 1) --
    against the oracle's k-flip ratio and the difference of exact log psi, modulo
    2 pi i, for 1 to 10 flips; the flipped state's theta cache after 100 flips
    equals a fresh calcTheta (:214-236), so the state ratio can use either."""
    from yannq_b200 import api

    n = m = 10
    q, p = _rbm(api, ctx, orc, n, m, 11, 1.0, dtype)
    rng = np.random.default_rng(3)
    s = _rand_sigma(rng, 48, n)
    th = np.array([orc.theta(n, m, p, x) for x in s])
    # weights are evaluated in the machine's type, so the complex64 machine agrees at its tolerance
    tol = TOL64 if dtype == api.C128 else 2e-4
    for k in range(1, n + 1):
        flips = np.array([rng.choice(n, k, replace=False) for _ in range(len(s))], np.int32)
        got = q.log_ratio_k(s, th, flips)
        ref = np.array([orc.logratio(n, m, p, x, t, f) for x, t, f in zip(s, th, flips)])
        assert np.max(np.abs(np.exp(got - ref) - 1)) < tol, k
        s2 = s.copy()
        for r, f in enumerate(flips):
            s2[r, f] *= -1
        exact = np.array([orc.logpsi(n, m, p, b) - orc.logpsi(n, m, p, a) for a, b in zip(s, s2)])
        assert np.max(np.abs(np.exp(got - exact) - 1)) < tol, k
    # state vs state: random pairs, theta of the second state from 100 incremental flips
    s_b = _rand_sigma(rng, len(s), n)
    th_b = np.array([orc.theta(n, m, p, x) for x in s_b])
    for r in range(len(s)):
        sig, t = s_b[r].copy(), th_b[r].copy()
        for f in rng.integers(0, n, 100):
            orc.flip(n, m, p, sig, t, [int(f)])
        assert np.max(np.abs(t - orc.theta(n, m, p, sig))) < 1e-6  # TestRBMStates.cpp:214-236
        s_b[r], th_b[r] = sig, t
    got = q.log_ratio_states(s, th, s_b, th_b)
    exact = np.array([orc.logpsi(n, m, p, b) - orc.logpsi(n, m, p, a) for a, b in zip(s, s_b)])
    assert np.max(np.abs(np.exp(got - exact) - 1)) < max(tol, 1e-9)
    q.close()


def test_log_deriv(ctx, orc):
    from yannq_b200 import api

    n, m = 12, 24
    q, p = _rbm(api, ctx, orc, n, m, 3, 0.5, api.C128)
    rng = np.random.default_rng(2)
    s = _rand_sigma(rng, 9, n)
    th = np.array([orc.theta(n, m, p, x) for x in s])
    got = q.log_deriv(s, th)
    want = np.array([orc.logderiv(n, m, p, x, t) for x, t in zip(s, th)])
    assert np.max(np.abs(got - want)) <= TOL64 * max(1.0, np.max(np.abs(want)))


HAMS = [
    ("tfi", lambda o: o.Ham.tfi(12, -1.0, -1.0)),
    ("tfi_h", lambda o: o.Ham.tfi(12, 1.0, 0.2)),
    ("xxz", lambda o: o.Ham.xxz(12, 1.0, 1.0, True)),
    ("xxz_d", lambda o: o.Ham.xxz(10, 0.7, 1.3, False)),
    ("tfi2d", lambda o: o.Ham.tfi2d(3, 4, -1.0, -3.0)),
    ("xxx", lambda o: o.Ham.xxx(12)),
    ("j1j2_sign", lambda o: o.Ham.j1j2(12, 1.0, 0.5, True)),
    ("j1j2", lambda o: o.Ham.j1j2(11, -0.8, 0.3, False)),
    ("xyznnn", lambda o: o.Ham.xyznnn(10, 0.3, 0.7)),
    ("kitaev4x2_field", lambda o: o.Ham.kitaev_hex(4, 2, 1.0, 1.0, 1.0, 0.2)),
    ("kitaev4x4_aniso", lambda o: o.Ham.kitaev_hex(4, 4, 0.2, 0.4, 0.6)),
    ("kitaev2x4_field", lambda o: o.Ham.kitaev_hex(2, 4, 0.5, -0.7, 0.9, -0.3)),
]


def _dev_ham(api, ctx, h):
    """The device Hamiltonian of an oracle descriptor."""
    if h.kind == 2:
        return api.Hamiltonian.tfi2d(ctx, h.lx, h.ly, h.J, h.h)
    if h.kind == 1:
        return api.Hamiltonian.xxz(ctx, h.n, h.J, h.h, h.sign < 0)
    if h.kind == 3:
        return api.Hamiltonian.xxx(ctx, h.n)
    if h.kind == 4:
        return api.Hamiltonian.j1j2(ctx, h.n, h.J, h.h, h.sign < 0)
    if h.kind == 5:
        return api.Hamiltonian.xyznnn(ctx, h.n, h.J, h.h)
    if h.kind == 6:
        return api.Hamiltonian.kitaev_hex(ctx, h.lx, h.ly, h.J, h.jy, h.jz, h.h)
    return api.Hamiltonian.tfi(ctx, h.n, h.J, h.h)


@pytest.mark.parametrize("name,mk", HAMS, ids=[h[0] for h in HAMS])
def test_flip_enumeration_bit_exact(ctx, orc, name, mk):
    """Every configuration of the 2^n basis: the device's (mask, coeff) list and
    diagonal equal the oracle's state-form enumeration, which equals the
    reference column form (tests/test_oracle_ham.py)."""
    from yannq_b200 import api

    h = mk(orc)
    H = _dev_ham(api, ctx, h)
    n = h.n
    cols = np.arange(1 << n)
    sig = np.array([orc.sigma_of(c, n) for c in cols])
    a, b, c, d = H.enumerate(sig)
    assert a.shape[1] == len(orc.ham_enumerate(h, sig[0])[1])
    for k in range(0, len(cols), 7 if n <= 12 else 61):
        dg, masks, coeffs = orc.ham_enumerate(h, sig[k])
        gm = np.array([(1 << int(x)) | ((1 << int(y)) if y >= 0 else 0) for x, y in zip(a[k], b[k])], np.uint64)
        np.testing.assert_array_equal(gm, masks)
        np.testing.assert_array_equal(c[k], coeffs)
        assert d[k] == dg
    H.close()


@pytest.mark.parametrize("name,mk", HAMS, ids=[h[0] for h in HAMS])
@pytest.mark.parametrize("dtype", [1, 0])
def test_eloc_parity(ctx, orc, name, mk, dtype):
    from yannq_b200 import api

    h = mk(orc)
    n, m = h.n, 2 * h.n
    q, p = _rbm(api, ctx, orc, n, m, 11, 0.2, dtype)
    H = _dev_ham(api, ctx, h)
    rng = np.random.default_rng(3)
    s = _rand_sigma(rng, 200, n)
    th = np.array([orc.theta(n, m, p, x) for x in s])
    got = H.eloc(q, s, th)
    want = orc.eloc(h, m, p, s, th)
    tol = TOL64 if dtype == api.C128 else TOL32
    # relative to each sample's magnitude (psi-ratios can be >> 1 at these weights)
    rel = np.abs(got - want) / np.maximum(np.abs(want), 1.0)
    assert np.max(rel) < tol, np.max(rel)
    H.close()
    q.close()


def test_eloc_full_size_2d(ctx, orc):
    """12 x 12 torus, alpha = 2 (the precision workload's machine): FP64 kernel vs oracle."""
    from yannq_b200 import api

    h = orc.Ham.tfi2d(12, 12, -1.0, -3.0)
    n, m = 144, 288
    q, p = _rbm(api, ctx, orc, n, m, 20261203, 0.01, api.C128)
    H = _dev_ham(api, ctx, h)
    rng = np.random.default_rng(4)
    s = _rand_sigma(rng, 32, n)
    th = np.array([orc.theta(n, m, p, x) for x in s])
    got = H.eloc(q, s, th)
    want = orc.eloc(h, m, p, s, th)
    assert np.max(np.abs(got - want)) / (4 * n) < TOL64


@pytest.mark.parametrize("name,mk,m", [
    ("j1j2_64", lambda o: o.Ham.j1j2(64, 1.0, 0.45, True), 128),
    ("xyznnn_48", lambda o: o.Ham.xyznnn(48, 0.6, -0.4), 96),
    ("kitaev_12x12", lambda o: o.Ham.kitaev_hex(12, 12, 1.0, 0.8, 0.6, 0.1), 288),
], ids=["j1j2_64", "xyznnn_48", "kitaev_12x12"])
@pytest.mark.parametrize("dtype", [1, 0])
def test_eloc_term_tables_large(ctx, orc, name, mk, m, dtype):
    """Term-table kinds at sizes where one block covers several table strides."""
    from yannq_b200 import api

    h = mk(orc)
    n = h.n
    q, p = _rbm(api, ctx, orc, n, m, 5, 0.05, dtype)
    H = _dev_ham(api, ctx, h)
    rng = np.random.default_rng(9)
    s = _rand_sigma(rng, 48, n)
    th = np.array([orc.theta(n, m, p, x) for x in s])
    got = H.eloc(q, s, th)
    want = orc.eloc(h, m, p, s, th)
    tol = TOL64 if dtype == api.C128 else TOL32
    rel = np.abs(got - want) / np.maximum(np.abs(want), 1.0)
    assert np.max(rel) < tol, np.max(rel)
    a, b, c, d = H.enumerate(s)
    for k in range(0, len(s), 5):
        dg, masks, coeffs = orc.ham_enumerate(h, s[k], cap=8 * n)
        np.testing.assert_array_equal(c[k], coeffs)
        assert d[k] == dg
    H.close()
    q.close()


def test_term_table_arguments(ctx):
    from yannq_b200 import api

    with pytest.raises(api.YQError):
        api.Hamiltonian.j1j2(ctx, 2, 1.0, 0.5)
    with pytest.raises(api.YQError):
        api.Hamiltonian.kitaev_hex(ctx, 3, 4, 1.0, 1.0, 1.0)
    with pytest.raises(api.YQError):
        api.Hamiltonian(ctx, api.HAM_KITAEV_HEX, 16, 1.0, 0.0)
    for mk, k in [(lambda: api.Hamiltonian.xxx(ctx, 10), 10), (lambda: api.Hamiltonian.j1j2(ctx, 10, 1, 0.2), 20),
                  (lambda: api.Hamiltonian.kitaev_hex(ctx, 4, 4, 1, 1, 1), 32),
                  (lambda: api.Hamiltonian.tfi2d(ctx, 3, 4, -1, -1), 12)]:
        H = mk()
        assert H.num_offdiag == k
        H.close()
