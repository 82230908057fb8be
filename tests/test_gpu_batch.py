"""Batched iterations of independent problems (yq_batch_*): the eager first call
and the captured-graph replays give, problem by problem, the same energies and
parameters as running each problem alone through yq_vmc_iteration with the
batch's seed + position and consecutive epochs (the same kernels on the same
inputs; stated tolerance 1e-12 relative), and, for the FP64 batch, the same as
the oracle's restated loop per problem (SamplerMT with persistent chains,
SRMat T-form, SGD: energies 1e-11, parameters 1e-9 relative)."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

# (n, alpha, h, chains) per precision; one batch per precision keeps the
# refinement steps uniform inside a batch
PROBLEMS = {
    "fp64": [(8, 1, 0.5, 16), (10, 4, 1.5, 16), (6, 2, 1.0, 8)],
    "mixed": [(12, 2, 1.0, 32), (16, 2, 0.8, 64)],
}
SWEEPS, DISCARD, SEED, SHIFT, LR, ITERS = 4, 8, 20261203, 1e-3, 0.01, 4


def _build(api, orc, k, spec, prec):
    n, alpha, h, chains = spec
    m = alpha * n
    ctx = api.Context(0)
    q = api.RBM(ctx, n, m, True, api.C64 if prec == "mixed" else api.C128)
    q.set_params(orc.init_params(n, m, 100 + k, 0.05))
    H = api.Hamiltonian.tfi(ctx, n, -1.0, -h)
    S = api.Sampler(q, chains)
    sr = api.SR(q, H, S, api.SR_T, api.PREC_MIXED if prec == "mixed" else api.PREC_FP64)
    return [ctx, q, H, S, sr]


def _close(objs):
    ctx, q, H, S, sr = objs
    for x in (sr, S, H, q, ctx):
        x.close()


@pytest.mark.parametrize("prec", ["fp64", "mixed"])
def test_batch_matches_single_problems(orc, prec):
    from yannq_b200 import api

    ir = 2 if prec == "mixed" else 0
    specs = PROBLEMS[prec]
    single = []
    for k, spec in enumerate(specs):
        objs = _build(api, orc, k, spec, prec)
        es = [objs[4].iteration(SWEEPS, DISCARD, SEED + k, it, SHIFT, LR, reinit=(it == 0), ir_steps=ir).energy
              for it in range(ITERS)]
        single.append((np.array(es), objs[1].get_params()))
        _close(objs)

    built = [_build(api, orc, k, spec, prec) for k, spec in enumerate(specs)]
    master = api.Context(0)
    B = api.Batch(master, [o[4] for o in built])
    got = [B.iteration(SWEEPS, DISCARD, SEED, it, SHIFT, LR, reinit=(it == 0), ir_steps=ir) for it in range(ITERS)]
    for k in range(len(specs)):
        es = np.array([got[it][k].energy for it in range(ITERS)])
        assert np.allclose(es, single[k][0], rtol=1e-12, atol=0), (k, es, single[k][0])
        assert all(got[it][k].status == 0 for it in range(ITERS))
        p = built[k][1].get_params()
        assert np.max(np.abs(p - single[k][1])) <= 1e-12 * np.max(np.abs(single[k][1]))
    if prec == "fp64":
        for k, (n, alpha, h, chains) in enumerate(specs):
            m = alpha * n
            ham = orc.Ham.tfi(n, -1.0, -h)
            pp = orc.init_params(n, m, 100 + k, 0.05)
            cs = None
            for it in range(ITERS):
                s, th, cs, _ = orc.sample(n, m, pp, chains, seed=SEED + k, epoch=it, reinit=(it == 0),
                                          n_sweeps=SWEEPS, n_discard=DISCARD, chain_sigma=cs)
                ref = orc.sr_step(ham, m, pp, s, th, SHIFT, orc.SR_T, orc.SOLVE_LLT)
                assert got[it][k].energy == pytest.approx(ref["energy"], rel=1e-11), (k, it)
                pp = pp - LR * ref["v"]
            p = built[k][1].get_params()
            assert np.max(np.abs(p - pp)) <= 1e-9 * np.max(np.abs(pp)), k
    # changed parameters: eager call and a new capture
    r = B.iteration(SWEEPS, DISCARD, SEED, ITERS, SHIFT, 0.5 * LR, reinit=False, ir_steps=ir)
    r2 = B.iteration(SWEEPS, DISCARD, SEED, ITERS + 1, SHIFT, 0.5 * LR, reinit=False, ir_steps=ir)
    assert all(np.isfinite(x.energy) for x in r + r2)
    B.close()
    for o in built:
        _close(o)
    master.close()
