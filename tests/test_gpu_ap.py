"""AmplitudePhase and NGDExact on the device against the oracle (C-ABI calls).

* Parameter initialisation bit-exact; log psi and logDeriv within 1e-12 for
  networks using every layer type.
* NGDExact::constructExact: energy within 1e-11 relative, gradient, oloc and
  both correlation matrices within 1e-10 of their largest entry (the device sums
  over the basis in another order), full and Jz bases, odd basis sizes.
* One RunAmplitudePhaseExact epoch: the updated parameters match the oracle's
  construct + numpy LLT + SGD within 1e-9; a short run descends towards the
  exact ground energy of the J1J2 chain.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def ctx():
    from yannq_b200 import api

    c = api.Context(0)
    yield c
    c.close()


NETS = {
    # every layer type but Sigmoid, Conv1D with bias and stride 2 (n = 6)
    "all": [("conv1d", 1, 3, 3, 1, True), ("lncosh",), ("conv1d", 3, 2, 3, 2, False), ("leakyhardtanh", 0.02),
            ("fc", 6, 4, True), ("tanh", 1.7), ("fc", 4, 3, False), ("leakyrelu", 0.05), ("fc", 3, 2, True),
            ("weaktanh",), ("fc", 2, 2, False), ("softsign",), ("fc", 2, 1, True), ("cos", 1.3)],
    "kinks": [("conv1d", 1, 4, 5), ("relu",), ("conv1d", 4, 2, 3, 1, True), ("hardtanh",), ("fc", 12, 3, True),
              ("softshrink",), ("fc", 3, 1, False), ("identity",)],
    "sigmoid": [("fc", 6, 1, False), ("sigmoid",)],
}


def _pair(api, orc, ctx, n, m, bias, layers):
    q = api.AmplitudePhase(ctx, n, m, bias, layers)
    o = orc.AP(n, m, bias, q.desc, q.xs)
    assert (o.Pa, o.Pp) == (q.dim_amp, q.dim_phase)
    return q, o


@pytest.mark.parametrize("net", list(NETS))
def test_log_psi_and_deriv(ctx, orc, net):
    from yannq_b200 import api

    n = 6
    q, o = _pair(api, orc, ctx, n, 9, net != "kinks", NETS[net])
    q.init_random(17, 0.2, api.INIT_LECUN)
    p = q.get_params()
    np.testing.assert_array_equal(p, orc.ap_init(o, 17, 0.2, 0))
    rng = np.random.default_rng(5)
    s = rng.choice(np.array([-1, 1], np.int8), size=(33, n))  # odd batch: a lone last pair
    got, want = q.log_psi(s), orc.ap_log_psi(o, p, s)
    assert np.max(np.abs(got - want)) <= 1e-12 * max(1.0, np.max(np.abs(want)))
    gd, wd = q.log_deriv(s), orc.ap_log_deriv(o, p, s)
    assert np.max(np.abs(gd - wd)) <= 1e-12 * max(1.0, np.max(np.abs(wd)))
    q.close()


def _ngd_case(api, orc, ctx, name):
    if name == "j1j2_jz":
        n, bk, nup = 10, api.BASIS_JZ, 5
        ho = orc.Ham.j1j2(n, 1.0, 0.4, True)
        hd = api.Hamiltonian.j1j2(ctx, n, 1.0, 0.4, True)
    elif name == "tfi_full_odd":  # 2^9 configurations, odd network width
        n, bk, nup = 9, api.BASIS_FULL, 0
        ho = orc.Ham.tfi(n, -1.0, -0.7)
        hd = api.Hamiltonian.tfi(ctx, n, -1.0, -0.7)
    elif name == "xxz_jz_odd_dim":  # C(7, 3) = 35 configurations
        n, bk, nup = 7, api.BASIS_JZ, 3
        ho = orc.Ham.xxz(n, 1.0, 0.8, True)
        hd = api.Hamiltonian.xxz(ctx, n, 1.0, 0.8, True)
    else:  # kitaev 4 x 2 with a field, full basis
        n, bk, nup = 8, api.BASIS_FULL, 0
        ho = orc.Ham.kitaev_hex(4, 2, 1.0, 0.8, 0.6, 0.2)
        hd = api.Hamiltonian.kitaev_hex(ctx, 4, 2, 1.0, 0.8, 0.6, 0.2)
    layers = [("conv1d", 1, 3, 3, 1, True), ("leakyhardtanh", 0.01), ("conv1d", 3, 2, 5), ("softsign",),
              ("fc", 2 * n, 1, True), ("tanh", 1.0)]
    q, o = _pair(api, orc, ctx, n, 2 * n, True, layers)
    q.init_random(23, 0.1, api.INIT_XAVIER)
    return n, bk, nup, ho, hd, q, o


def _rel(a, b):
    return np.max(np.abs(a - b)) / max(np.max(np.abs(b)), 1e-300)


@pytest.mark.parametrize("name", ["j1j2_jz", "tfi_full_odd", "xxz_jz_odd_dim", "kitaev_full"])
def test_ngd_construct(ctx, orc, name):
    from yannq_b200 import api

    n, bk, nup, ho, hd, q, o = _ngd_case(api, orc, ctx, name)
    p = q.get_params()
    ref = orc.ngd_exact(ho, o, p, bk, nup)
    g = api.NGDExact(q, hd, bk, nup)
    e = g.construct()
    assert e == pytest.approx(ref["energy"], rel=1e-11)
    assert _rel(g.get(api.NGD_GRAD), ref["grad"]) < 1e-10
    assert _rel(g.get(api.NGD_OLOC_AMP), ref["oloc_amp"]) < 1e-10
    assert _rel(g.get(api.NGD_OLOC_PHASE), ref["oloc_phase"]) < 1e-10
    assert _rel(g.get(api.NGD_CORR_AMP), ref["corr_amp"]) < 1e-10
    assert _rel(g.get(api.NGD_CORR_PHASE), ref["corr_phase"]) < 1e-10
    g.close()
    hd.close()
    q.close()


def test_ngd_construct_split_gram(ctx, orc):
    """A basis of 2^14 configurations (8,192 row pairs): the correlation matrices
    are computed in K-chunks on side streams and summed."""
    from yannq_b200 import api

    n = 14
    ho = orc.Ham.tfi(n, -1.0, -0.9)
    hd = api.Hamiltonian.tfi(ctx, n, -1.0, -0.9)
    layers = [("conv1d", 1, 2, 3, 1, True), ("lncosh",), ("fc", 2 * n, 2, True), ("tanh", 1.0), ("fc", 2, 1, False)]
    q, o = _pair(api, orc, ctx, n, n, True, layers)
    q.init_random(29, 0.1, api.INIT_XAVIER)
    p = q.get_params()
    ref = orc.ngd_exact(ho, o, p, api.BASIS_FULL, 0)
    g = api.NGDExact(q, hd, api.BASIS_FULL, 0)
    for _ in range(2):  # partials are rewritten, not accumulated, on every construct
        e = g.construct()
        assert e == pytest.approx(ref["energy"], rel=1e-11)
        assert _rel(g.get(api.NGD_GRAD), ref["grad"]) < 1e-10
        assert _rel(g.get(api.NGD_CORR_AMP), ref["corr_amp"]) < 1e-10
        assert _rel(g.get(api.NGD_CORR_PHASE), ref["corr_phase"]) < 1e-10
    g.close()
    hd.close()
    q.close()


def test_ngd_iteration_matches_oracle_step(ctx, orc):
    from yannq_b200 import api

    n, bk, nup, ho, hd, q, o = _ngd_case(api, orc, ctx, "j1j2_jz")
    p = q.get_params()
    ref = orc.ngd_exact(ho, o, p, bk, nup)
    lam, lr = 0.5, 0.05
    va = np.linalg.solve(ref["corr_amp"] + lam * np.eye(o.Pa), ref["grad"][:o.Pa])
    vp = np.linalg.solve(ref["corr_phase"] + lam * np.eye(o.Pp), ref["grad"][o.Pa:])
    want = p - lr * np.concatenate([va, vp])
    g = api.NGDExact(q, hd, bk, nup)
    e, gn, vn = g.iteration(lam, lr, api.NGD_ALL)
    assert e == pytest.approx(ref["energy"], rel=1e-11)
    assert gn == pytest.approx(np.linalg.norm(ref["grad"]), rel=1e-10)
    assert vn == pytest.approx(np.linalg.norm(np.concatenate([va, vp])), rel=1e-8)
    assert np.max(np.abs(q.get_params() - want)) < 1e-9 * max(1.0, np.max(np.abs(want)))
    # amplitude-only epoch leaves the phase block alone
    before = q.get_params()
    g.iteration(lam, lr, api.NGD_AMP)
    after = q.get_params()
    np.testing.assert_array_equal(after[o.Pa:], before[o.Pa:])
    assert np.any(after[:o.Pa] != before[:o.Pa])
    g.close()
    hd.close()
    q.close()


def test_run_amplitude_phase_descends(ctx, orc):
    """Examples/AmplitudePhase.cpp pattern (J1J2 with the sign rule, Jz basis,
    lambda 10 * 0.9^ll down to 1e-3) on N = 10."""
    from yannq_b200 import api

    n = 10
    hd = api.Hamiltonian.j1j2(ctx, n, 1.0, 0.2, True)
    layers = [("conv1d", 1, 4, 5), ("leakyhardtanh", 0.01), ("conv1d", 4, 2, 5), ("leakyhardtanh", 0.01),
              ("fc", 2 * n, 1, False), ("softsign",)]
    q = api.AmplitudePhase(ctx, n, 2 * n, False, layers)
    q.init_random(2026, 0.01, api.INIT_XAVIER)
    g = api.NGDExact(q, hd, api.BASIS_JZ, n // 2)
    es = [g.iteration(max(10.0 * 0.9 ** ll, 1e-3), 0.05)[0] for ll in range(60)]
    e0 = orc.ed_ground(orc.Ham.j1j2(n, 1.0, 0.2, True), 1, n // 2)
    assert es[-1] < es[0] - 1.0
    assert es[-1] >= e0 - 1e-9
    g.close()
    hd.close()
    q.close()


def test_ap_arguments(ctx, orc):
    from yannq_b200 import api

    with pytest.raises(api.YQError):
        api.AmplitudePhase(ctx, 6, 6, True, [("fc", 5, 1)])  # width mismatch
    with pytest.raises(api.YQError):
        api.AmplitudePhase(ctx, 6, 6, True, [("fc", 6, 2)])  # two outputs
    with pytest.raises(api.YQError):
        api.AmplitudePhase(ctx, 6, 6, True, [("conv1d", 4, 2, 3), ("fc", 2, 1)])  # 6 % 4 != 0
    q = api.AmplitudePhase(ctx, 6, 6, True, [("fc", 6, 1)])
    H = api.Hamiltonian.tfi(ctx, 6, -1.0, -1.0)
    with pytest.raises(api.YQError):
        api.NGDExact(q, H, api.BASIS_JZ, 3)  # TFI does not conserve Sz
    H8 = api.Hamiltonian.tfi(ctx, 8, -1.0, -1.0)
    with pytest.raises(api.YQError):
        api.NGDExact(q, H8)
    for x in (H, H8, q):
        x.close()
