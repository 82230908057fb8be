"""The runner loop of Runners/RunRBM.hpp:151-221 on the device (yq_vmc_iteration)
against the oracle's restatement (pyoracle.run_rbm), FP64, for the options a
RunRBM user sets: ObsAvg momentum of the gradient and of the Fisher matrix
(setMomentum, :13-37, :73-77, :180-202), the update clip (setGradClip, :79-82,
:204-209) and the CG branch with its cgErr (:183-191).  Samples are drawn from the
same Philox streams, so every epoch sees the oracle's samples; stated tolerances:
energy 1e-11 relative, parameters 1e-9 relative to their largest entry."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

N, M, SEED, SHIFT, LR = 8, 16, 7, 1e-3, 0.02


@pytest.fixture(scope="module")
def ctx():
    from yannq_b200 import api

    c = api.Context(0)
    yield c
    c.close()


def _problem(api, ctx, orc, chains, mode):
    q = api.RBM(ctx, N, M, True, api.C128)
    p = orc.init_params(N, M, 20261203, 0.05)
    q.set_params(p)
    H = api.Hamiltonian.tfi(ctx, N, -1.0, -1.0)
    S = api.Sampler(q, chains)
    sr = api.SR(q, H, S, mode, api.PREC_FP64)
    return q, p, H, S, sr


def _run(api, orc, objs, chains, epochs, sweeps, solver=0, **opt):
    q, p, H, S, sr = objs
    res = [sr.iteration(sweeps, 16, SEED, ll, SHIFT, LR, reinit=True, solver=solver, cg_tol=1e-13)
           for ll in range(epochs)]
    ref, pf = orc.run_rbm(orc.Ham.tfi(N, -1.0, -1.0), M, p, chains, epochs, sweeps, 16, SEED, SHIFT, LR,
                          use_cg=solver == api.SOLVE_CG, **opt)
    got = q.get_params()
    for ll in range(epochs):
        assert res[ll].energy == pytest.approx(ref[ll]["energy"], rel=1e-11), ll
        assert res[ll].update_norm == pytest.approx(ref[ll]["nv"], rel=1e-8), ll
    assert np.max(np.abs(got - pf)) <= 1e-9 * np.max(np.abs(pf))
    return res, ref


@pytest.mark.parametrize("beta1,beta2", [(0.9, 0.0), (0.0, 0.95), (0.9, 0.95)])
def test_momentum_s_form_matches_oracle_runner(ctx, orc, beta1, beta2):
    """S-form (Ns = 256 > P = 152): gradient and Fisher-matrix averages in the LLT branch."""
    from yannq_b200 import api

    objs = _problem(api, ctx, orc, 16, api.SR_AUTO)
    objs[4].set_momentum(beta1, beta2)
    _run(api, orc, objs, 16, 4, 16, beta1=beta1, beta2=beta2)
    for x in objs[4], objs[3], objs[2], objs[0]:
        x.close()


def test_gradient_momentum_t_form_woodbury(ctx, orc):
    """T-form (Ns = 64 < P = 152): the averaged gradient is no longer O~^H y, and
    (S + lambda)^{-1} g is solved through (T + lambda)^{-1} by the Woodbury identity."""
    from yannq_b200 import api

    objs = _problem(api, ctx, orc, 8, api.SR_T)
    objs[4].set_momentum(0.8, 0.0)
    _run(api, orc, objs, 8, 4, 8, beta1=0.8)
    for x in objs[4], objs[3], objs[2], objs[0]:
        x.close()


def test_fisher_average_needs_the_s_form(ctx, orc):
    from yannq_b200 import api

    objs = _problem(api, ctx, orc, 8, api.SR_T)
    objs[4].set_momentum(0.0, 0.9)
    with pytest.raises(api.YQError) as e:
        objs[4].iteration(8, 16, SEED, 0, SHIFT, LR)
    assert e.value.code == api.E_UNSUPPORTED
    with pytest.raises(api.YQError) as e:
        objs[4].set_momentum(1.0, 0.0)
    assert e.value.code == api.E_ARG
    for x in objs[4], objs[3], objs[2], objs[0]:
        x.close()


@pytest.mark.parametrize("mode", ["S", "T"])
def test_grad_clip_matches_oracle_runner(ctx, orc, mode):
    """setGradClip: |v| above the clip is scaled to the clip (the reported norm is
    the unclipped one, as the callback's nv)."""
    from yannq_b200 import api

    chains, sweeps = (16, 16) if mode == "S" else (8, 8)
    objs = _problem(api, ctx, orc, chains, api.SR_S if mode == "S" else api.SR_T)
    objs[4].set_grad_clip(0.5)
    res, ref = _run(api, orc, objs, chains, 3, sweeps, grad_clip=0.5)
    assert max(r["nv"] for r in ref) > 0.5  # the clip acted
    for x in objs[4], objs[3], objs[2], objs[0]:
        x.close()


def test_cg_branch_with_momentum(ctx, orc):
    """useCG with beta2 = 0: CG on the averaged gradient (tolerance 1e-13), cgErr =
    |apply(v) - grad| of the device's own v."""
    from yannq_b200 import api

    objs = _problem(api, ctx, orc, 16, api.SR_S)
    objs[4].set_momentum(0.5, 0.0)
    res, ref = _run(api, orc, objs, 16, 3, 16, solver=api.SOLVE_CG, beta1=0.5)
    for r in res:
        assert 0.0 <= r.cg_err < 1e-9
    for x in objs[4], objs[3], objs[2], objs[0]:
        x.close()


def test_batches_reject_momentum(ctx, orc):
    from yannq_b200 import api

    objs = _problem(api, ctx, orc, 8, api.SR_T)
    objs[4].set_momentum(0.9, 0.0)
    B = api.Batch(ctx, [objs[4]])
    with pytest.raises(api.YQError) as e:
        B.iteration(8, 8, SEED, 0, SHIFT, LR)
    assert e.value.code == api.E_UNSUPPORTED
    B.close()
    for x in objs[4], objs[3], objs[2], objs[0]:
        x.close()
