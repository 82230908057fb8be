"""GPU parity of the sampler and the SR step against the oracle (C-ABI calls).

* FP64 sampler: with the same Philox streams the device chains equal the
  oracle's restated SamplerMT draw for draw (sigma bit-exact, theta within
  1e-13 relative) for local, any-pair and neighbour-pair moves.
* complex64 sampler: chi^2 against exact |psi|^2.
* SR (FP64): E_loc, oloc, F, S/T and the solution v against the oracle's
  restated SRMat on identical samples; S-mode LLT, T-mode dual and CG agree.
* A whole yq_vmc_iteration trajectory (sample, SR, SGD) tracks the oracle loop.
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


def _mk(api, ctx, orc, n, m, seed, sd, dtype):
    q = api.RBM(ctx, n, m, True, dtype)
    p = orc.init_params(n, m, seed, sd)
    q.set_params(p)
    return q, p


@pytest.mark.parametrize("move,nup", [(0, -1), (1, 5), (2, 5)])
def test_sampler_fp64_matches_oracle_draw_for_draw(ctx, orc, move, nup):
    from yannq_b200 import api

    n, m = 10, 20
    q, p = _mk(api, ctx, orc, n, m, 21, 0.3, api.C128)
    S = api.Sampler(q, 32, move, nup)
    S.sample(6, 4, seed=99, epoch=3, reinit=True)
    s, th = S.get_samples()
    os_, oth, ocs, oacc = orc.sample(n, m, p, 32, move=move, nup=nup, seed=99, epoch=3, reinit=True, n_sweeps=6,
                                     n_discard=4)
    np.testing.assert_array_equal(s, os_)
    assert np.max(np.abs(th - oth)) <= 1e-13 * max(1.0, np.max(np.abs(oth)))
    np.testing.assert_array_equal(S.get_accepts(), oacc)
    np.testing.assert_array_equal(S.get_chains(), ocs)
    # continue the chains without re-initialisation
    S.sample(3, 0, seed=99, epoch=4, reinit=False)
    s2, _ = S.get_samples()
    os2, _, _, _ = orc.sample(n, m, p, 32, move=move, nup=nup, seed=99, epoch=4, reinit=False, n_sweeps=3,
                              n_discard=0, chain_sigma=ocs)
    np.testing.assert_array_equal(s2, os2)
    S.close()
    q.close()


def test_sampler_fp64_full_size_draw_for_draw(ctx, orc):
    """12 x 12 lattice, alpha = 2: the first 8 chains of the precision workload."""
    from yannq_b200 import api

    n, m = 144, 288
    q, p = _mk(api, ctx, orc, n, m, 20261203, 0.01, api.C128)
    S = api.Sampler(q, 8, 0, -1)
    S.sample(2, 2, seed=20261203, epoch=0, reinit=True)
    s, th = S.get_samples()
    os_, oth, _, _ = orc.sample(n, m, p, 8, seed=20261203, epoch=0, reinit=True, n_sweeps=2, n_discard=2)
    np.testing.assert_array_equal(s, os_)
    assert np.max(np.abs(th - oth)) <= 1e-13 * max(1.0, np.max(np.abs(oth)))


@pytest.mark.parametrize("move", [0, 2])
def test_sampler_c64_distribution(ctx, orc, move):
    from yannq_b200 import api

    n, m = 6, 6
    q, p = _mk(api, ctx, orc, n, m, 3, 0.25, api.C64)
    nup = -1 if move == 0 else 3
    S = api.Sampler(q, 512, move, nup)
    S.sample(40, 100, seed=17, epoch=0, reinit=True)
    s, _ = S.get_samples(theta=False)
    basis = orc.basis(n)
    psi = np.array([orc.psi(n, m, p, orc.sigma_of(b, n)) for b in basis])
    pr = np.abs(psi) ** 2
    if move:
        pr = np.where([bin(b).count("1") == 3 for b in range(1 << n)], pr, 0)
        assert np.all((s == -1).sum(1) == 3)
    pr /= pr.sum()
    counts = np.bincount([orc.index_of(x) for x in s], minlength=1 << n)
    N = len(s)
    sel = pr * N > 20
    chi2 = (((counts[sel] - N * pr[sel]) ** 2) / (N * pr[sel])).sum()
    dof = sel.sum() - 1
    assert chi2 < 4 * dof + 30, (chi2, dof)


def _sr_case(api, ctx, orc, ham_o, n, m, chains, sweeps, mode):
    q, p = _mk(api, ctx, orc, n, m, 8, 0.1, api.C128)
    s, th, _, _ = orc.sample(n, m, p, chains, seed=5, n_sweeps=sweeps, n_discard=20)
    if ham_o.kind == 0:
        H = api.Hamiltonian.tfi(ctx, n, ham_o.J, ham_o.h)
    else:
        H = api.Hamiltonian.xxz(ctx, n, ham_o.J, ham_o.h, ham_o.sign < 0)
    S = api.Sampler(q, chains)
    S.put_samples(s, th)
    sr = api.SR(q, H, S, mode, api.PREC_FP64)
    sr.construct()
    return q, p, s, th, H, S, sr


@pytest.mark.parametrize("mode", [1, 2])
def test_sr_fp64_matches_oracle(ctx, orc, mode):
    from yannq_b200 import api

    n, m = 8, 16
    h = orc.Ham.tfi(n, -1.0, -1.0)
    # S-mode: Ns = 256 > P = 152; T-mode forced on the same samples
    q, p, s, th, H, S, sr = _sr_case(api, ctx, orc, h, n, m, 32, 8, mode)
    P = q.dim
    ref = orc.sr_step(h, m, p, s, th, 1e-3, orc.SR_S, orc.SOLVE_LLT)
    e, var = sr.energy()
    assert e == pytest.approx(ref["energy"], rel=1e-12)
    assert var == pytest.approx(ref["energy_var"], rel=1e-9, abs=1e-12)
    np.testing.assert_allclose(sr.get(0, len(s)), ref["elocs"], rtol=1e-12, atol=1e-12)
    np.testing.assert_allclose(sr.get(1, P), ref["oloc"], rtol=1e-12, atol=1e-14)
    np.testing.assert_allclose(sr.get(2, P), ref["grad"], rtol=1e-10, atol=1e-13)
    v, _, _ = sr.solve(1e-3, api.SOLVE_LLT)
    assert np.max(np.abs(v - ref["v"])) <= 1e-9 * np.max(np.abs(ref["v"]))
    for x in (sr, S, H, q):
        x.close()


def test_sr_matrix_and_cg(ctx, orc):
    from yannq_b200 import api

    n, m = 6, 12
    h = orc.Ham.xxz(n, 1.0, 1.0, True)
    q, p, s, th, H, S, sr = _sr_case(api, ctx, orc, h, n, m, 16, 4, api.SR_T)  # Ns = 64 < P = 90
    O = np.array([orc.logderiv(n, m, p, a, b) for a, b in zip(s, th)])
    Oc = O - O.mean(0)
    T = sr.matrix()
    Tw = Oc @ Oc.conj().T / len(s)
    low = np.tril_indices(len(s))
    assert np.max(np.abs(T[low] - Tw[low])) < 1e-12 * np.max(np.abs(Tw))
    ref = orc.sr_step(h, m, p, s, th, 1e-2, orc.SR_S, orc.SOLVE_LLT)
    v_llt, _, _ = sr.solve(1e-2, api.SOLVE_LLT)
    v_cg, it, rr = sr.solve(1e-2, api.SOLVE_CG, 1e-12)
    assert rr < 1e-12 and it > 0
    for v in (v_llt, v_cg):
        assert np.max(np.abs(v - ref["v"])) <= 1e-8 * np.max(np.abs(ref["v"]))
    for x in (sr, S, H, q):
        x.close()


def test_not_positive_definite_is_reported(ctx, orc):
    """Shift 0 with Ns < P makes T singular (rank <= Ns - 1 after centring): the
    Cholesky reports YQ_E_NOT_PD instead of returning garbage."""
    from yannq_b200 import api

    n, m = 6, 12
    h = orc.Ham.tfi(n, -1.0, -1.0)
    q, p, s, th, H, S, sr = _sr_case(api, ctx, orc, h, n, m, 8, 4, api.SR_T)
    with pytest.raises(api.YQError) as e:
        sr.solve(0.0, api.SOLVE_LLT)
    assert e.value.code == api.E_NOT_PD
    v, _, _ = sr.solve(1e-3, api.SOLVE_LLT)  # the context stays usable
    assert np.all(np.isfinite(v))
    for x in (sr, S, H, q):
        x.close()


def test_vmc_iterations_track_oracle_loop(ctx, orc):
    """Runners/RunRBM.hpp:151-221 on the device vs the oracle loop, FP64:
    identical samples each iteration, parameters within 1e-9 after 3 updates."""
    from yannq_b200 import api

    n, m = 8, 16
    h = orc.Ham.tfi(n, -1.0, -1.0)
    q, p = _mk(api, ctx, orc, n, m, 20261203, 0.01, api.C128)
    H = api.Hamiltonian.tfi(ctx, n, -1.0, -1.0)
    S = api.Sampler(q, 16)
    sr = api.SR(q, H, S, api.SR_AUTO, api.PREC_FP64)
    pp = p.copy()
    for it in range(3):
        r = sr.iteration(n_sweeps=16, n_discard=16, seed=7, epoch=it, shift=1e-3, lr=0.01, reinit=True)
        s, th, _, _ = orc.sample(n, m, pp, 16, seed=7, epoch=it, n_sweeps=16, n_discard=16)
        ref = orc.sr_step(h, m, pp, s, th, 1e-3, orc.SR_T, orc.SOLVE_LLT)
        pp = pp - 0.01 * ref["v"]
        assert r.energy == pytest.approx(ref["energy"], rel=1e-11)
        got = q.get_params()
        assert np.max(np.abs(got - pp)) < 1e-9 * np.max(np.abs(pp))
        assert r.update_norm == pytest.approx(np.linalg.norm(ref["v"]), rel=1e-8)
    for x in (sr, S, H, q):
        x.close()


def test_vmc_converges_towards_ed(ctx, orc):
    from yannq_b200 import api

    n, m = 10, 20
    e0 = orc.ed_ground(orc.Ham.tfi(n, -1.0, -1.0))
    q = api.RBM(ctx, n, m, True, api.C128)
    q.init_random(1, 0.01)
    H = api.Hamiltonian.tfi(ctx, n, -1.0, -1.0)
    S = api.Sampler(q, 64)
    sr = api.SR(q, H, S, api.SR_AUTO, api.PREC_FP64)
    es = [sr.iteration(16, 16, 3, it, 1e-3, 0.05).energy for it in range(60)]
    assert np.mean(es[-10:]) < es[0]
    assert abs(np.mean(es[-10:]) - e0) / abs(e0) < 0.02


def test_sampler_autotuned_launch_shape(ctx, orc):
    """The autotuner picks 1, 2 or 4 chains per CTA once per configuration; a
    second sampler with the same configuration reuses the choice, and the chains
    are the same whatever the choice (each warp owns one chain)."""
    from yannq_b200 import api

    n, m, chains = 10, 20, 48
    p = orc.init_params(n, m, 3, 0.1)
    out = []
    for _ in range(2):
        q = api.RBM(ctx, n, m, True, api.C128)
        q.set_params(p)
        S = api.Sampler(q, chains)
        S.sample(4, 4, seed=9, epoch=0, reinit=True)
        out.append((S.chains_per_cta(), S.get_samples()[0]))
        S.close()
        q.close()
    assert out[0][0] in (1, 2, 4)
    assert out[1][0] == out[0][0]
    assert np.array_equal(out[0][1], out[1][1])


_SHAPE_SCRIPT = r"""
import hashlib, sys
sys.path.insert(0, sys.argv[1])
from yannq_b200 import api
ctx = api.Context(0)
h = hashlib.sha256()
for dtype, move, nup, m in ((api.C64, 0, -1, 40), (api.C128, 1, 8, 20), (api.C64, 0, -1, 288)):
    q = api.RBM(ctx, 16, m, True, dtype)
    q.init_random(11, 0.1)
    S = api.Sampler(q, 96, move, nup)
    S.sample(3, 2, seed=5, epoch=0, reinit=True)
    S.sample(3, 2, seed=5, epoch=1, reinit=False)
    s, th = S.get_samples()
    h.update(s.tobytes()); h.update(th.tobytes()); h.update(S.get_accepts().tobytes())
    print("shape", S.chains_per_cta(), file=sys.stderr)
    S.close(); q.close()
ctx.close()
print(h.hexdigest())
"""


def test_sampler_launch_shapes_give_identical_chains():
    """YQ_CHAINS_PER_CTA = 1, 2 and 4 (read once per process, so one process each)
    give bit-identical samples, theta and acceptance counts: each warp owns one chain
    and its own Philox counters, whatever the block it runs in."""
    import os
    import subprocess
    import sys

    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    digests = {}
    for v in ("1", "2", "4"):
        env = dict(os.environ, YQ_CHAINS_PER_CTA=v)
        out = subprocess.run([sys.executable, "-c", _SHAPE_SCRIPT, root], env=env, capture_output=True, text=True,
                             timeout=300)
        assert out.returncode == 0, out.stderr
        assert out.stderr.count(f"shape {v}") == 3, out.stderr
        digests[v] = out.stdout.strip()
    assert digests["1"] == digests["2"] == digests["4"], digests


@pytest.mark.parametrize("move,nup,ntemps", [(0, -1, 4), (1, 5, 2), (0, -1, 8)])
def test_tempering_fp64_matches_oracle_draw_for_draw(ctx, orc, move, nup, ntemps):
    """SamplerMT with nTmps > 1: every chain sweeps at its beta, temperatures swap
    within groups after every sweep, the beta = 1 chains are recorded; device and
    oracle agree draw for draw, swap for swap, and across a second call."""
    from yannq_b200 import api

    n, m, per = 10, 20, 4
    nc = per * ntemps
    q, p = _mk(api, ctx, orc, n, m, 23, 0.4, api.C128)
    S = api.Sampler(q, nc, move, nup)
    S.set_tempering(ntemps)
    S.sample(6, 5, seed=77, epoch=2, reinit=True)
    s, th = S.get_samples()
    os_, oth, ocs, osl, oacc = orc.sample_pt(n, m, p, nc, ntemps, move=move, nup=nup, seed=77, epoch=2, reinit=True,
                                             n_sweeps=6, n_discard=5)
    assert s.shape == (per * 6, n)
    np.testing.assert_array_equal(s, os_)
    assert np.max(np.abs(th - oth)) <= 1e-13 * max(1.0, np.max(np.abs(oth)))
    np.testing.assert_array_equal(S.get_slots(), osl)
    np.testing.assert_array_equal(S.get_accepts(), oacc)
    assert len(set(osl.tolist())) == ntemps
    if ntemps >= 4:  # temperatures moved (a two-slot ladder may return to where it started)
        assert not np.array_equal(osl, np.arange(nc) % ntemps)
    S.sample(4, 0, seed=77, epoch=3, reinit=False)
    s2, _ = S.get_samples()
    os2, _, _, osl2, _ = orc.sample_pt(n, m, p, nc, ntemps, move=move, nup=nup, seed=77, epoch=3, reinit=False,
                                       n_sweeps=4, n_discard=0, chain_sigma=ocs, slot=osl)
    np.testing.assert_array_equal(s2, os2)
    np.testing.assert_array_equal(S.get_slots(), osl2)
    S.close()
    q.close()


def test_tempering_complex64_distribution(ctx, orc):
    """The beta = 1 samples of a tempered complex64 sampler follow |psi|^2 (chi^2)."""
    from scipy import stats
    from yannq_b200 import api

    n, m, ntemps, per = 6, 12, 4, 64
    q, p = _mk(api, ctx, orc, n, m, 24, 0.5, api.C64)
    S = api.Sampler(q, per * ntemps)
    S.set_tempering(ntemps)
    S.sample(200, 100, seed=5, epoch=0, reinit=True)
    s, _ = S.get_samples()
    idx = np.array([orc.index_of(x) for x in s])
    counts = np.bincount(idx, minlength=1 << n)
    lp = np.array([orc.logpsi(n, m, p, orc.sigma_of(k, n)).real for k in range(1 << n)])
    w = np.exp(2 * (lp - lp.max()))
    w /= w.sum()
    # consecutive sweeps of one chain are correlated: compare against a conservative
    # effective sample size (every 4th sample)
    chi2, pval = stats.chisquare(np.bincount(idx[::4], minlength=1 << n), len(idx[::4]) * w)
    assert pval > 1e-4, (chi2, pval)
    S.close()
    q.close()


def _dev_ham(api, ctx, h):
    """The device Hamiltonian of an oracle descriptor."""
    if h.kind == 0:
        return api.Hamiltonian.tfi(ctx, h.n, h.J, h.h)
    if h.kind == 1:
        return api.Hamiltonian.xxz(ctx, h.n, h.J, h.h, h.sign < 0)
    if h.kind == 2:
        return api.Hamiltonian.tfi2d(ctx, h.lx, h.ly, h.J, h.h)
    if h.kind == 3:
        return api.Hamiltonian.xxx(ctx, h.n)
    if h.kind == 4:
        return api.Hamiltonian.j1j2(ctx, h.n, h.J, h.h, h.sign < 0)
    if h.kind == 5:
        return api.Hamiltonian.xyznnn(ctx, h.n, h.J, h.h)
    return api.Hamiltonian.kitaev_hex(ctx, h.lx, h.ly, h.J, h.jy, h.jz, h.h)


HAM_SWEEPER = [
    ("tfi10", lambda o: o.Ham.tfi(10, -1.0, -1.0), -1),
    ("tfi2d_3x4", lambda o: o.Ham.tfi2d(3, 4, -1.0, -3.0), -1),
    ("xxz10_sign", lambda o: o.Ham.xxz(10, 1.0, 1.0, True), 5),
    ("xxx10", lambda o: o.Ham.xxx(10), 5),
    ("j1j2_10_sign", lambda o: o.Ham.j1j2(10, 1.0, 0.5, True), 5),
    ("xyznnn10", lambda o: o.Ham.xyznnn(10, 0.3, 0.7), -1),
    ("kitaev4x2_field", lambda o: o.Ham.kitaev_hex(4, 2, 0.5, 0.7, 0.9, 0.3), -1),
    ("kitaev4x4_nofield", lambda o: o.Ham.kitaev_hex(4, 4, 0.2, 0.4, 0.6), -1),
]


@pytest.mark.parametrize("name,mk,nup", HAM_SWEEPER, ids=[c[0] for c in HAM_SWEEPER])
def test_hamiltonian_sweeper_fp64_draw_for_draw(ctx, orc, name, mk, nup):
    """Samplers/HamiltonianSweeper.hpp:22-50 on the device (warp ballots over the
    offDiagonals list) against the oracle's restatement, same Philox streams."""
    from yannq_b200 import api

    h = mk(orc)
    n = h.n
    m = 2 * n
    q, p = _mk(api, ctx, orc, n, m, 27, 0.3, api.C128)
    H = _dev_ham(api, ctx, h)
    S = api.Sampler(q, 32, api.MOVE_HAMILTONIAN, nup)
    S.set_hamiltonian(H)
    S.sample(6, 4, seed=7, epoch=2, reinit=True)
    s, th = S.get_samples()
    os_, oth, ocs, oacc = orc.sample(n, m, p, 32, move=orc.MOVE_HAMILTONIAN, nup=nup, seed=7, epoch=2, reinit=True,
                                     n_sweeps=6, n_discard=4, ham=h)
    np.testing.assert_array_equal(s, os_)
    assert np.max(np.abs(th - oth)) <= 1e-13 * max(1.0, np.max(np.abs(oth)))
    np.testing.assert_array_equal(S.get_accepts(), oacc)
    assert oacc.sum() > 0
    S.sample(3, 0, seed=7, epoch=3, reinit=False)
    s2, _ = S.get_samples()
    os2, _, _, _ = orc.sample(n, m, p, 32, move=orc.MOVE_HAMILTONIAN, nup=nup, seed=7, epoch=3, reinit=False,
                              n_sweeps=3, n_discard=0, chain_sigma=ocs, ham=h)
    np.testing.assert_array_equal(s2, os2)
    S.close()
    H.close()
    q.close()


def test_hamiltonian_sweeper_tempering_draw_for_draw(ctx, orc):
    from yannq_b200 import api

    h = orc.Ham.j1j2(10, 1.0, 0.5, True)
    n, m, nt = 10, 20, 4
    q, p = _mk(api, ctx, orc, n, m, 28, 0.3, api.C128)
    H = _dev_ham(api, ctx, h)
    S = api.Sampler(q, 16 * nt, api.MOVE_HAMILTONIAN, 5)
    S.set_hamiltonian(H)
    S.set_tempering(nt)
    S.sample(5, 3, seed=8, epoch=1, reinit=True)
    s, _ = S.get_samples()
    os_, _, _, osl, _ = orc.sample_pt(n, m, p, 16 * nt, nt, move=orc.MOVE_HAMILTONIAN, nup=5, seed=8, epoch=1,
                                      n_sweeps=5, n_discard=3, ham=h)
    np.testing.assert_array_equal(s, os_)
    np.testing.assert_array_equal(S.get_slots(), osl)
    S.close()
    H.close()
    q.close()


@pytest.mark.parametrize("name,mk,nup,allowed", [
    ("j1j2_6_sign", lambda o: o.Ham.j1j2(6, 1.0, 0.5, True), 3, lambda b: bin(b).count("1") == 3),
    ("kitaev4x2_field", lambda o: o.Ham.kitaev_hex(4, 2, 0.5, 0.7, 0.9, 0.3), -1, lambda b: True),
], ids=["j1j2_6_sign", "kitaev4x2_field"])
def test_hamiltonian_sweeper_c64_distribution(ctx, orc, name, mk, nup, allowed):
    from yannq_b200 import api

    h = mk(orc)
    n = m = h.n
    q, p = _mk(api, ctx, orc, n, m, 41, 0.3, api.C64)
    H = _dev_ham(api, ctx, h)
    S = api.Sampler(q, 512, api.MOVE_HAMILTONIAN, nup)
    S.set_hamiltonian(H)
    S.sample(40, 100, seed=19, epoch=0, reinit=True)
    s, _ = S.get_samples(theta=False)
    basis = orc.basis(n)
    pr = np.abs(np.array([orc.psi(n, m, p, orc.sigma_of(b, n)) for b in basis])) ** 2
    mask = np.array([allowed(b) for b in range(1 << n)])
    pr = np.where(mask, pr, 0)
    pr /= pr.sum()
    idx = np.array([orc.index_of(x) for x in s])
    assert mask[idx].all()
    counts = np.bincount(idx, minlength=1 << n)
    N = len(s)
    sel = pr * N > 20
    chi2 = (((counts[sel] - N * pr[sel]) ** 2) / (N * pr[sel])).sum()
    dof = sel.sum() - 1
    assert chi2 < 4 * dof + 30, (chi2, dof)
    S.close()
    H.close()
    q.close()


def test_hamiltonian_sweeper_arguments(ctx, orc):
    from yannq_b200 import api

    q, _ = _mk(api, ctx, orc, 8, 8, 1, 0.1, api.C128)
    S = api.Sampler(q, 8, api.MOVE_HAMILTONIAN)
    with pytest.raises(api.YQError):
        S.sample(1, 0, seed=1, epoch=0, reinit=True)  # no Hamiltonian attached
    H10 = api.Hamiltonian.tfi(ctx, 10, -1.0, -1.0)
    with pytest.raises(api.YQError):
        S.set_hamiltonian(H10)  # size differs
    L = api.Sampler(q, 8, api.MOVE_LOCAL)
    H = api.Hamiltonian.tfi(ctx, 8, -1.0, -1.0)
    with pytest.raises(api.YQError):
        L.set_hamiltonian(H)  # not a HamiltonianSweeper sampler
    for x in (S, L, H10, H, q):
        x.close()
