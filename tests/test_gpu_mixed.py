"""Mixed-precision SR path: tcgen05 BF16x3 Gram matrix and the refined solve.

The Hermitian T = O~ O~^H / Ns formed on the tensor cores is checked against an
FP64 numpy product of the oracle's O~ (stated tolerance 3e-5 of max |T|: BF16x3
keeps ~16 significand bits per operand and accumulates in FP32); the refined
solution v against the FP64 oracle solve (2e-4 relative: complex64 O~ plus two
FP64 refinement steps).
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

TOL_T = 3e-5
TOL_V = 2e-4


@pytest.fixture(scope="module")
def ctx():
    from yannq_b200 import api

    c = api.Context(0)
    yield c
    c.close()


def _case(api, ctx, orc, n, m, chains, sweeps, seed=8, sd=0.1):
    p = orc.init_params(n, m, seed, sd)
    s, th, _, _ = orc.sample(n, m, p, chains, seed=5, n_sweeps=sweeps, n_discard=20)
    q = api.RBM(ctx, n, m, True, api.C64)
    q.set_params(p)
    H = api.Hamiltonian.tfi(ctx, n, -1.0, -1.0)
    S = api.Sampler(q, chains)
    S.put_samples(s, th)
    sr = api.SR(q, H, S, api.SR_T, api.PREC_MIXED)
    sr.construct()
    return p, s, th, q, H, S, sr


def _t_ref(orc, n, m, p, s, th):
    O = np.array([orc.logderiv(n, m, p, a, b) for a, b in zip(s, th)])
    Oc = O - O.mean(0)
    return Oc @ Oc.conj().T / len(s)


# P = nm + n + m: 152, 560, 636 and 90 (even, not a multiple of 4) take the
# two-column O writer, 175 (odd) the one-column writer.
@pytest.mark.parametrize("n,m,chains,sweeps", [(8, 16, 16, 8), (16, 32, 64, 8), (12, 48, 40, 7), (10, 15, 24, 5),
                                               (6, 12, 20, 6)])
def test_tensor_core_gram(ctx, orc, n, m, chains, sweeps):
    from yannq_b200 import api

    p, s, th, q, H, S, sr = _case(api, ctx, orc, n, m, chains, sweeps)
    T = sr.matrix()
    Tw = _t_ref(orc, n, m, p, s, th)
    low = np.tril_indices(len(s))
    err = np.max(np.abs(T[low] - Tw[low])) / np.max(np.abs(Tw))
    assert err < TOL_T, err
    for x in (sr, S, H, q):
        x.close()


# Ns < P: T-form.  P = 560 takes the pair kernels of O~^H y and O~ x, P = 175 the
# one-column kernels.
@pytest.mark.parametrize("n,m,chains", [(16, 32, 32), (10, 15, 12)])
def test_mixed_solve_matches_fp64(ctx, orc, n, m, chains):
    from yannq_b200 import api

    p, s, th, q, H, S, sr = _case(api, ctx, orc, n, m, chains, 8)
    ref = orc.sr_step(orc.Ham.tfi(n, -1.0, -1.0), m, p, s, th, 1e-3, orc.SR_T, orc.SOLVE_LLT)
    v, _, _ = sr.solve(1e-3, api.SOLVE_LLT)
    err = np.max(np.abs(v - ref["v"])) / np.max(np.abs(ref["v"]))
    assert err < TOL_V, err
    e, _ = sr.energy()
    assert e == pytest.approx(ref["energy"], rel=1e-5)
    for x in (sr, S, H, q):
        x.close()


def test_mixed_full_size_properties(ctx, orc):
    """12 x 12 lattice, 8192 samples: T is Hermitian PSD-shifted (the Cholesky
    succeeds), the update is finite and its norm is close to the FP64 path's on
    the same samples."""
    from yannq_b200 import api

    n, m = 144, 288
    p = orc.init_params(n, m, 20261203, 0.01)
    out = {}
    for prec, dt in (("mixed", api.C64), ("fp64", api.C128)):
        q = api.RBM(ctx, n, m, True, dt)
        q.set_params(p)
        H = api.Hamiltonian.tfi2d(ctx, 12, 12, -1.0, -3.0)
        S = api.Sampler(q, 1024)
        sr = api.SR(q, H, S, api.SR_T, api.PREC_MIXED if prec == "mixed" else api.PREC_FP64)
        if prec == "mixed":
            S.sample(8, 32, seed=3, epoch=0, reinit=True)
            sig, th = S.get_samples()
        else:
            S.put_samples(sig, th)
        sr.construct()
        v, _, _ = sr.solve(1e-3, api.SOLVE_LLT)
        out[prec] = (v, sr.energy()[0])
        for x in (sr, S, H, q):
            x.close()
    vm, em = out["mixed"]
    vf, ef = out["fp64"]
    assert np.all(np.isfinite(vm))
    assert abs(em - ef) / abs(ef) < 1e-5
    assert np.linalg.norm(vm - vf) / np.linalg.norm(vf) < 1e-3


@pytest.mark.parametrize("chains,sweeps", [(100, 12), (64, 9)])
def test_mixed_panel_cholesky_matches_fp64(ctx, orc, chains, sweeps):
    """T larger than one 512-wide Cholesky panel: the tensor-core trailing updates
    (ragged 704- and 192-row trailing blocks for Ns = 1200, identity padding up to
    a multiple of 64) followed by refinement reproduce the FP64 oracle solve."""
    from yannq_b200 import api

    n, m = 36, 72
    p, s, th, q, H, S, sr = _case(api, ctx, orc, n, m, chains, sweeps, seed=11, sd=0.05)
    ref = orc.sr_step(orc.Ham.tfi(n, -1.0, -1.0), m, p, s, th, 1e-3, orc.SR_T, orc.SOLVE_LLT)
    v, _, _ = sr.solve(1e-3, api.SOLVE_LLT)
    err = np.max(np.abs(v - ref["v"])) / np.max(np.abs(ref["v"]))
    assert err < TOL_V, err
    for x in (sr, S, H, q):
        x.close()


# S-form of the complex64 machine (Ns >= P): the centred O~ rows of the complex64
# writer (32 bytes per thread; P = 152 even, 175 odd) feed the FP64-accumulating
# Gram; S and F against numpy products of the oracle's FP64 rows.
@pytest.mark.parametrize("n,m,chains", [(8, 16, 48), (10, 15, 40)])
def test_complex64_s_form_matches_oracle(ctx, orc, n, m, chains):
    from yannq_b200 import api

    p = orc.init_params(n, m, 8, 0.1)
    s, th, _, _ = orc.sample(n, m, p, chains, seed=5, n_sweeps=8, n_discard=20)
    q = api.RBM(ctx, n, m, True, api.C64)
    q.set_params(p)
    H = api.Hamiltonian.tfi(ctx, n, -1.0, -1.0)
    S = api.Sampler(q, chains)
    S.put_samples(s, th)
    sr = api.SR(q, H, S, api.SR_S, api.PREC_MIXED)
    sr.construct()
    O = orc.logderiv_rows(n, m, p, s, th)
    Oc = O - O.mean(0)
    e = orc.eloc(orc.Ham.tfi(n, -1.0, -1.0), m, p, s, th)
    F = Oc.conj().T @ (e - e.mean()) / len(s)
    Sm = Oc.conj().T @ Oc / len(s)
    got_F = sr.get(2, q.dim)
    assert np.max(np.abs(got_F - F)) / np.max(np.abs(F)) < 5e-5
    got_S = sr.matrix()
    low = np.tril_indices(q.dim)
    assert np.max(np.abs(got_S[low] - Sm[low])) / np.max(np.abs(Sm)) < 5e-6
    for x in (sr, S, H, q):
        x.close()
