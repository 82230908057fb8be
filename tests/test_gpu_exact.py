"""Exact summation (GroundState/SRMatExact.hpp:97-132) and exact sampling
(Samplers/ExactSampler.hpp:49-79) on the device against the oracle.

Complex128 machine: E and Var within 1e-11 relative; oloc, F and S within 1e-10
of their largest entry (the device sums over the basis in another order).
Complex64 machine (E_loc in the machine's FP32 product form): E within 1e-5
relative, F within 1e-4 of its largest entry.  Exact sampler: the oracle's
restatement, fed the same Philox stream, draws the same basis positions (a draw
could differ only where u * total lands within rounding of a CDF step); and a
chi^2 test of the complex64 sampler against |psi|^2.
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


def _max_rel(a, b):
    return np.max(np.abs(a - b)) / max(np.max(np.abs(b)), 1e-300)


CASES = [
    # (name, oracle ham, device ham factory, n, m, basis kind, nup)
    ("tfi10_full", lambda o: o.Ham.tfi(10, -1.0, -1.0), lambda a, c: a.Hamiltonian.tfi(c, 10, -1.0, -1.0), 10, 20, 0, 0),
    ("xxz10_jz", lambda o: o.Ham.xxz(10, 1.0, 1.0, True), lambda a, c: a.Hamiltonian.xxz(c, 10, 1.0, 1.0, True), 10, 20,
     1, 5),
    ("tfi2d_3x3_full", lambda o: o.Ham.tfi2d(3, 3, -1.0, -3.0), lambda a, c: a.Hamiltonian.tfi2d(c, 3, 3, -1.0, -3.0),
     9, 18, 0, 0),
    ("j1j2_12_jz", lambda o: o.Ham.j1j2(12, 1.0, 0.5, True), lambda a, c: a.Hamiltonian.j1j2(c, 12, 1.0, 0.5, True),
     12, 12, 1, 6),
    ("xxx10_jz", lambda o: o.Ham.xxx(10), lambda a, c: a.Hamiltonian.xxx(c, 10), 10, 10, 1, 5),
    ("xyznnn10_full", lambda o: o.Ham.xyznnn(10, 0.3, 0.7), lambda a, c: a.Hamiltonian.xyznnn(c, 10, 0.3, 0.7), 10, 10,
     0, 0),
    ("kitaev4x2_full", lambda o: o.Ham.kitaev_hex(4, 2, 1.0, 0.8, 0.6, 0.2),
     lambda a, c: a.Hamiltonian.kitaev_hex(c, 4, 2, 1.0, 0.8, 0.6, 0.2), 8, 16, 0, 0),
]


@pytest.mark.parametrize("name,oham,dham,n,m,kind,nup", CASES)
def test_exact_summation_fp64(ctx, orc, name, oham, dham, n, m, kind, nup):
    from yannq_b200 import api

    p = orc.init_params(n, m, 31, 0.1)
    ref = orc.exact(oham(orc), m, p, basis_kind=kind, nup=nup)
    q = api.RBM(ctx, n, m, True, api.C128)
    q.set_params(p)
    H = dham(api, ctx)
    got = api.exact(q, H, kind, nup)
    assert got["energy"] == pytest.approx(ref["energy"], rel=1e-11)
    assert got["energy_var"] == pytest.approx(ref["energy_var"], rel=1e-9, abs=1e-11)
    assert _max_rel(got["oloc"], ref["oloc"]) < 1e-10
    assert _max_rel(got["grad"], ref["grad"]) < 1e-10
    assert _max_rel(got["S"], ref["S"]) < 1e-10
    H.close()
    q.close()


def test_exact_summation_complex64(ctx, orc):
    from yannq_b200 import api

    n, m = 10, 20
    p = orc.init_params(n, m, 32, 0.1)
    ref = orc.exact(orc.Ham.tfi(n, -1.0, -1.0), m, p)
    q = api.RBM(ctx, n, m, True, api.C64)
    q.set_params(p)
    H = api.Hamiltonian.tfi(ctx, n, -1.0, -1.0)
    got = api.exact(q, H)
    assert got["energy"] == pytest.approx(ref["energy"], rel=1e-5)
    assert _max_rel(got["grad"], ref["grad"]) < 1e-4
    assert _max_rel(got["S"], ref["S"]) < 1e-10  # O and weights are FP64 for either machine
    H.close()
    q.close()


def test_exact_summation_large_basis(ctx, orc):
    """2^17 configurations: more rows than one launch's grid.y, F and oloc only."""
    from yannq_b200 import api

    n, m = 17, 17
    p = orc.init_params(n, m, 33, 0.05)
    ref = orc.exact(orc.Ham.tfi(n, -1.0, -0.7), m, p, with_S=False)
    q = api.RBM(ctx, n, m, True, api.C128)
    q.set_params(p)
    H = api.Hamiltonian.tfi(ctx, n, -1.0, -0.7)
    got = api.exact(q, H, with_S=False)
    assert got["energy"] == pytest.approx(ref["energy"], rel=1e-11)
    assert _max_rel(got["oloc"], ref["oloc"]) < 1e-10
    assert _max_rel(got["grad"], ref["grad"]) < 1e-10
    H.close()
    q.close()


def test_exact_jz_needs_conserving_hamiltonian(ctx, orc):
    from yannq_b200 import api

    q = api.RBM(ctx, 8, 8, True, api.C128)
    q.set_params(orc.init_params(8, 8, 1, 0.1))
    for H in (api.Hamiltonian.tfi(ctx, 8, -1.0, -1.0), api.Hamiltonian.xyznnn(ctx, 8, 0.3, 0.7),
              api.Hamiltonian.kitaev_hex(ctx, 4, 2, 1.0, 1.0, 1.0)):
        with pytest.raises(api.YQError):
            api.exact(q, H, api.BASIS_JZ, 4)
        H.close()
    H = api.Hamiltonian.xyznnn(ctx, 8, 0.5, 0.5)  # a == b: the parallel-pair flips vanish
    api.exact(q, H, api.BASIS_JZ, 4)
    H.close()
    q.close()


@pytest.mark.parametrize("kind,nup", [(0, -1), (1, 6)])
def test_exact_sampler_matches_oracle(ctx, orc, kind, nup):
    from yannq_b200 import api

    n, m, ns = 12, 24, 4000
    p = orc.init_params(n, m, 34, 0.2)
    q = api.RBM(ctx, n, m, True, api.C128)
    q.set_params(p)
    S = api.Sampler(q, 16, api.MOVE_LOCAL if nup < 0 else api.MOVE_EXCHANGE_ANY, nup)
    for epoch in (0, 1):
        pos = S.sample_exact(ns, seed=20261203, epoch=epoch, positions=True)
        opos, oidx, dim = orc.exact_sample(n, m, p, ns, 20261203, epoch, basis_kind=kind, nup=max(nup, 0))
        assert np.array_equal(pos, opos.astype(np.uint64))
        sig, th = S.get_samples()
        want = np.array([orc.sigma_of(v, n) for v in oidx])
        assert np.array_equal(sig, want)
        th_ref = np.array([orc.theta(n, m, p, s) for s in want])
        assert np.max(np.abs(th - th_ref)) < 1e-12
    S.close()
    q.close()


def test_exact_sampler_chi2_complex64(ctx, orc):
    from scipy import stats
    from yannq_b200 import api

    n, m, ns = 6, 12, 200000
    p = orc.init_params(n, m, 35, 0.4)
    q = api.RBM(ctx, n, m, True, api.C64)
    q.set_params(p)
    S = api.Sampler(q, 8)
    pos = S.sample_exact(ns, seed=7, positions=True)
    counts = np.bincount(pos.astype(np.int64), minlength=1 << n)
    lp = np.array([orc.logpsi(n, m, p, orc.sigma_of(k, n)).real for k in range(1 << n)])
    w = np.exp(2 * (lp - lp.max()))
    w /= w.sum()
    chi2, pval = stats.chisquare(counts, ns * w)
    assert pval > 1e-4, (chi2, pval)
    S.close()
    q.close()
