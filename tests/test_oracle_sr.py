"""Pins the oracle's sampler, SR step and FeedForward derivative.

* SR (GroundState/SRMat.hpp:89-237): S-mode LLT against numpy; CG (Eigen
  semantics) against LLT; the sample-space dual (T-mode) against S-mode.
* Sampler (Samplers/SamplerMT.hpp + LocalSweeper/SwapSweeper): the histogram of
  samples matches |psi|^2 from exact enumeration (chi^2), exchange moves keep
  the magnetisation, and the recorded theta is the incrementally updated cache.
* FeedForward backward (Machines/FeedForward.hpp:186-205): central differences
  as in Tests/TestFeedForward.cpp:16-79 and Tests/TestConvLayer.cpp:14-53.
"""
import numpy as np
import pytest


def _samples(orc, n, m, p, chains=64, sweeps=8, discard=16, move=0, nup=-1, seed=5):
    s, th, cs, acc = orc.sample(n, m, p, chains, move=move, nup=nup, seed=seed, n_sweeps=sweeps, n_discard=discard)
    return s, th


def test_sr_s_mode_llt_matches_numpy(orc):
    n, m = 6, 12
    ham = orc.Ham.tfi(n, -1.0, -1.0)
    p = orc.init_params(n, m, 1, 0.1)
    s, th = _samples(orc, n, m, p, chains=32, sweeps=8)
    r = orc.sr_step(ham, m, p, s, th, 1e-3, orc.SR_S, orc.SOLVE_LLT)
    assert r["status"] == 0
    O = np.array([orc.logderiv(n, m, p, a, b) for a, b in zip(s, th)])
    E = orc.eloc(ham, m, p, s, th)
    ol = O.mean(0)
    Oc = O - ol
    F = Oc.conj().T @ E / len(s)
    S = Oc.conj().T @ Oc / len(s) + 1e-3 * np.eye(O.shape[1])
    v = np.linalg.solve(S, F)
    assert np.allclose(r["grad"], F, rtol=1e-12, atol=1e-14)
    assert np.allclose(r["v"], v, rtol=1e-8, atol=1e-10)
    assert r["energy"] == pytest.approx(E.real.mean(), rel=1e-13)
    assert r["energy_var"] == pytest.approx((E.real ** 2).mean() - E.real.mean() ** 2, rel=1e-9, abs=1e-12)


def test_sr_cg_and_t_mode_agree_with_llt(orc):
    n, m = 6, 12
    ham = orc.Ham.tfi(n, -1.0, -1.0)
    p = orc.init_params(n, m, 2, 0.1)
    s, th = _samples(orc, n, m, p, chains=8, sweeps=4)  # Ns = 32 < P = 90
    a = orc.sr_step(ham, m, p, s, th, 1e-2, orc.SR_S, orc.SOLVE_LLT)
    b = orc.sr_step(ham, m, p, s, th, 1e-2, orc.SR_S, orc.SOLVE_CG, cgtol=1e-12)
    c = orc.sr_step(ham, m, p, s, th, 1e-2, orc.SR_T, orc.SOLVE_LLT)
    assert np.allclose(b["v"], a["v"], rtol=1e-8, atol=1e-9)
    assert np.allclose(c["v"], a["v"], rtol=1e-8, atol=1e-9)
    assert b["cg_relres"] < 1e-12


def test_cholesky_restatement(orc):
    rng = np.random.default_rng(0)
    X = rng.normal(size=(40, 60)) + 1j * rng.normal(size=(40, 60))
    A = X @ X.conj().T / 60 + 1e-3 * np.eye(40)
    b = rng.normal(size=40) + 1j * rng.normal(size=40)
    st, x = orc.cholesky_solve(A, b)
    assert st == 0
    assert np.allclose(A @ x, b, atol=1e-9)
    st, _ = orc.cholesky_solve(-A, b)
    assert st == 1


def _exact_probs(orc, n, m, p):
    basis = orc.basis(n)
    psi = np.array([orc.psi(n, m, p, orc.sigma_of(b, n)) for b in basis])
    pr = np.abs(psi) ** 2
    return pr / pr.sum()


def _index(s):
    return int(sum(((1 - int(x)) // 2) << i for i, x in enumerate(s)))


@pytest.mark.parametrize("move", [0, 1, 2])
def test_sampler_distribution(orc, move):
    n, m = 6, 6
    p = orc.init_params(n, m, 3, 0.25)
    nup = -1 if move == 0 else 3
    s, th = _samples(orc, n, m, p, chains=256, sweeps=40, discard=100, move=move, nup=nup, seed=17)
    pr = _exact_probs(orc, n, m, p)
    if move:
        assert np.all((s == -1).sum(1) == 3)
        mask = np.array([bin(b).count("1") == 3 for b in range(1 << n)])
        pr = np.where(mask, pr, 0)
        pr /= pr.sum()
    counts = np.bincount([_index(x) for x in s], minlength=1 << n)
    N = len(s)
    sel = pr * N > 20
    chi2 = (((counts[sel] - N * pr[sel]) ** 2) / (N * pr[sel])).sum()
    dof = sel.sum() - 1
    # samples within a chain are correlated; allow a generous factor over dof
    assert chi2 < 4 * dof + 30, (chi2, dof)
    # recorded theta is the incrementally updated cache (SamplerMT.hpp:169-170)
    for k in range(0, N, 97):
        assert np.allclose(th[k], orc.theta(n, m, p, s[k]), atol=1e-12)


def test_sampler_is_deterministic(orc):
    n, m = 10, 20
    p = orc.init_params(n, m, 9, 0.05)
    a = _samples(orc, n, m, p, chains=16, sweeps=4, seed=123)
    b = _samples(orc, n, m, p, chains=16, sweeps=4, seed=123)
    c = _samples(orc, n, m, p, chains=16, sweeps=4, seed=124)
    assert np.array_equal(a[0], b[0]) and np.array_equal(a[1], b[1])
    assert not np.array_equal(a[0], c[0])


def test_vmc_loop_descends_towards_ed(orc):
    # Runners/RunRBM.hpp:123-222 restated for a few SR + SGD iterations
    n, m = 8, 16
    ham = orc.Ham.tfi(n, -1.0, -1.0)
    p = orc.init_params(n, m, 20261203, 0.01)
    e0 = orc.ed_ground(ham)
    es = []
    for it in range(30):
        s, th, _, _ = orc.sample(n, m, p, 16, seed=1, epoch=it, n_sweeps=64, n_discard=32)
        r = orc.sr_step(ham, m, p, s, th, 1e-3, orc.SR_S, orc.SOLVE_LLT)
        p = p - 0.05 * r["v"]
        es.append(r["energy"])
    assert np.mean(es[-5:]) < es[0]
    assert np.mean(es[-5:]) >= e0 - 0.05 * abs(e0)


FF = dict(L=12, conv_out=4, conv_k=5, fc_out=6)


def test_ff_backward_finite_difference(orc):
    rng = np.random.default_rng(3)
    P = orc.ff_dim(**FF)
    p = rng.normal(scale=0.3, size=P)
    s = rng.choice([-1, 1], size=FF["L"]).astype(np.int8)
    der = orc.ff_backward(FF["L"], FF["conv_out"], FF["conv_k"], FF["fc_out"], p, s)
    h = 1e-5
    fd = np.zeros(P)
    for k in range(P):
        pp, pm = p.copy(), p.copy()
        pp[k] += h
        pm[k] -= h
        fd[k] = (orc.ff_forward(FF["L"], FF["conv_out"], FF["conv_k"], FF["fc_out"], pp, s)
                 - orc.ff_forward(FF["L"], FF["conv_out"], FF["conv_k"], FF["fc_out"], pm, s)) / (2 * h)
    assert np.max(np.abs(fd - der)) / max(1e-12, np.max(np.abs(der))) < 1e-6


def test_ff_forward_matches_numpy(orc):
    rng = np.random.default_rng(4)
    L, C, K, F = FF["L"], FF["conv_out"], FF["conv_k"], FF["fc_out"]
    p = rng.normal(scale=0.3, size=orc.ff_dim(**FF))
    s = rng.choice([-1, 1], size=L).astype(np.int8)
    ker = p[: K * C].reshape(C, K)  # column-major (K x C)
    z1 = np.zeros((C, L))
    for oc in range(C):
        for r in range(L):
            z1[oc, r] = sum(ker[oc, ki] * s[(r + ki - K // 2) % L] for ki in range(K))
    a1 = np.log(np.cosh(z1)).reshape(-1)
    Wfc = p[K * C:].reshape(F, L * C).T  # (I x F) column-major
    z2 = Wfc.T @ a1
    want = np.log(np.cosh(z2)).sum()
    assert orc.ff_forward(L, C, K, F, p, s) == pytest.approx(want, rel=1e-12)


def test_oracle_tempering_samples_follow_psi2(orc):
    """The oracle's restated SamplerMT with nTmps = 4 records beta = 1 chains whose
    configurations follow |psi|^2 (chi^2 on a 6-spin RBM)."""
    from scipy import stats

    n, m, ntemps, per = 6, 12, 4, 32
    p = orc.init_params(n, m, 25, 0.5)
    s, _, _, slots, _ = orc.sample_pt(n, m, p, per * ntemps, ntemps, seed=11, n_sweeps=400, n_discard=100)
    assert sorted(slots[:ntemps].tolist()) == list(range(ntemps))
    idx = np.array([orc.index_of(x) for x in s[::4]])
    lp = np.array([orc.logpsi(n, m, p, orc.sigma_of(k, n)).real for k in range(1 << n)])
    w = np.exp(2 * (lp - lp.max()))
    w /= w.sum()
    chi2, pval = stats.chisquare(np.bincount(idx, minlength=1 << n), len(idx) * w)
    assert pval > 1e-4, (chi2, pval)


HAM_SWEEPER_CASES = [
    # (name, Ham factory, n, nup, allowed(index) -> bool)
    ("tfi6", lambda o: o.Ham.tfi(6, -1.0, -1.0), 6, -1, lambda b: True),
    ("j1j2_6_sign", lambda o: o.Ham.j1j2(6, 1.0, 0.5, True), 6, 3, lambda b: bin(b).count("1") == 3),
    ("xyznnn6", lambda o: o.Ham.xyznnn(6, 0.3, 0.7), 6, 3, lambda b: bin(b).count("1") % 2 == 1),
    ("kitaev4x2_field", lambda o: o.Ham.kitaev_hex(4, 2, 0.5, 0.7, 0.9, 0.3), 8, -1, lambda b: True),
]


@pytest.mark.parametrize("name,mk,n,nup,allowed", HAM_SWEEPER_CASES, ids=[c[0] for c in HAM_SWEEPER_CASES])
def test_hamiltonian_sweeper_distribution(orc, name, mk, n, nup, allowed):
    """Samplers/HamiltonianSweeper.hpp:22-50: proposals drawn uniformly from
    offDiagonals(sigma) with the w1 / w2 correction sample |psi|^2 on the sector
    the moves connect (pair flips keep the magnetisation where only antiparallel
    pairs flip, and its parity where parallel pairs flip too)."""
    m = n
    ham = mk(orc)
    p = orc.init_params(n, m, 41, 0.3)
    s, th, _, acc = orc.sample(n, m, p, 256, move=orc.MOVE_HAMILTONIAN, nup=nup, seed=23, n_sweeps=60,
                               n_discard=100, ham=ham)
    assert acc.sum() > 0
    pr = _exact_probs(orc, n, m, p)
    mask = np.array([allowed(b) for b in range(1 << n)])
    pr = np.where(mask, pr, 0)
    pr /= pr.sum()
    idx = np.array([_index(x) for x in s])
    assert mask[idx].all()
    counts = np.bincount(idx, minlength=1 << n)
    N = len(s)
    sel = pr * N > 20
    chi2 = (((counts[sel] - N * pr[sel]) ** 2) / (N * pr[sel])).sum()
    dof = sel.sum() - 1
    assert chi2 < 4 * dof + 30, (chi2, dof)
    for k in range(0, N, 211):
        assert np.allclose(th[k], orc.theta(n, m, p, s[k]), atol=1e-12)


def test_hamiltonian_sweeper_list_sizes_vary(orc):
    """The chi^2 case j1j2_6_sign exercises the w1 / w2 correction: its
    offDiagonals list (antiparallel bonds) changes size with the state, while
    XYZNNN's (a != b, every coefficient non-zero) and TFIsing's do not."""
    n = 6

    def sizes(ham):
        out = set()
        for b in range(1 << n):
            d, masks, coeffs = orc.ham_enumerate(ham, orc.sigma_of(b, n))
            out.add(int(np.count_nonzero(coeffs)))
        return out

    assert len(sizes(orc.Ham.j1j2(n, 1.0, 0.5, True))) > 1
    assert sizes(orc.Ham.xyznnn(n, 0.3, 0.7)) == {2 * n}


def test_runner_restatement_without_momentum_is_the_sr_step_loop(orc):
    """pyoracle.run_rbm (Runners/RunRBM.hpp:151-221) with beta1 = beta2 = 0 and no
    clip is the loop of C++ oracle SR steps (S-form LLT) on the same samples."""
    n, m = 8, 16
    ham = orc.Ham.tfi(n, -1.0, -1.0)
    p = orc.init_params(n, m, 20261203, 0.01)
    out, pf = orc.run_rbm(ham, m, p, 16, 3, 16, 16, 7, 1e-3, 0.01)
    pp = p.copy()
    for it in range(3):
        s, th, _, _ = orc.sample(n, m, pp, 16, seed=7, epoch=it, n_sweeps=16, n_discard=16)
        ref = orc.sr_step(ham, m, pp, s, th, 1e-3, orc.SR_S, orc.SOLVE_LLT)
        assert out[it]["energy"] == pytest.approx(ref["energy"], rel=1e-12)
        assert np.linalg.norm(out[it]["v"] - ref["v"]) <= 1e-10 * np.linalg.norm(ref["v"])
        pp = pp - 0.01 * ref["v"]
    assert np.max(np.abs(pf - pp)) <= 1e-12


def test_obs_avg_semantics(orc):
    """ObsAvg (RunRBM.hpp:13-37): starting from zero, getAvg after t updates is the
    bias-corrected exponential average; a constant input averages to itself and
    beta = 0 returns the last input."""
    a = orc.ObsAvg(0.9, np.zeros(3))
    xs = [np.array([1.0, 2.0, 3.0]) * (k + 1) for k in range(4)]
    for x in xs:
        a.update(x)
    w = np.array([0.9 ** (3 - k) * 0.1 for k in range(4)])
    assert np.allclose(a.get_avg(), sum(wk * x for wk, x in zip(w, xs)) / (1 - 0.9 ** 4), rtol=1e-14)
    c = orc.ObsAvg(0.95, np.zeros(2))
    for _ in range(5):
        c.update(np.array([2.0, -1.0]))
    assert np.allclose(c.get_avg(), [2.0, -1.0], rtol=1e-14)
    z = orc.ObsAvg(0.0, np.zeros(1))
    z.update(np.array([5.0]))
    z.update(np.array([7.0]))
    assert z.get_avg()[0] == 7.0


@pytest.mark.parametrize("beta1,beta2,clip", [(0.9, 0.0, 0.0), (0.0, 0.9, 0.0), (0.0, 0.0, 0.05)])
def test_runner_options_change_the_trajectory(orc, beta1, beta2, clip):
    """Each RunRBM option (gradient momentum, Fisher averaging, update clip) moves
    the parameters away from the plain loop, and the clip bounds the step."""
    n, m = 6, 12
    ham = orc.Ham.tfi(n, -1.0, -1.0)
    p = orc.init_params(n, m, 3, 0.05)
    plain, p0 = orc.run_rbm(ham, m, p, 16, 3, 16, 16, 11, 1e-3, 0.05)
    opt, p1 = orc.run_rbm(ham, m, p, 16, 3, 16, 16, 11, 1e-3, 0.05, beta1=beta1, beta2=beta2, grad_clip=clip)
    assert plain[0]["energy"] == opt[0]["energy"]  # same parameters, same samples at epoch 0
    assert np.max(np.abs(p1 - p0)) > 1e-8
    if clip:
        assert all(np.linalg.norm(o["v"]) <= clip * (1 + 1e-12) for o in opt)
