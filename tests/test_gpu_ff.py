"""FeedForward machine on the device vs the FP64 oracle (Machines/FeedForward.hpp).

FP32 kernels: log psi within 1e-5 relative, the adjoint (log-derivative rows)
within 2e-5 of max |O| of the oracle's backward and within 1e-3 of FP64 central
differences (step 1e-4, as the differentiation workload asks); activation store
and recompute give the same rows; E_loc of the TFI chain by single-flip updates
within 1e-5 relative of full oracle forwards.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

L, CH, K, F = 40, 12, 5, 16  # the differentiation workload's network


@pytest.fixture(scope="module")
def ctx():
    from yannq_b200 import api

    c = api.Context(0)
    yield c
    c.close()


def _net(api, ctx, seed=3):
    f = api.FeedForward(ctx, L, CH, K, F)
    f.init_random(seed)
    return f, f.get_params()


def test_init_is_xavier(ctx):
    from yannq_b200 import api

    f, p = _net(api, ctx)
    kc = K * CH
    assert p[:kc].std() == pytest.approx(np.sqrt(2.0 / (K + CH * K)), rel=0.2)
    assert p[kc:].std() == pytest.approx(np.sqrt(2.0 / (L * CH + F)), rel=0.05)
    f.close()


def test_forward_and_adjoint_match_oracle(ctx, orc):
    from yannq_b200 import api

    f, p = _net(api, ctx)
    rng = np.random.default_rng(0)
    s = rng.choice(np.array([-1, 1], np.int8), size=(37, L))
    f.set_batch(s)
    lp = f.forward(act_budget_bytes=1 << 40)
    O_store = f.adjoint()
    f.forward(act_budget_bytes=0)  # activations not kept: the adjoint recomputes them
    O_recomp = f.adjoint()
    ref_lp, ref_O = orc.ff_batch(L, CH, K, F, p, s)
    assert np.max(np.abs(lp - ref_lp) / np.abs(ref_lp)) < 1e-5
    assert np.max(np.abs(O_store - ref_O)) < 2e-5 * np.max(np.abs(ref_O))
    np.testing.assert_array_equal(O_store, O_recomp)
    f.close()


@pytest.mark.parametrize("net_seed,cfg_seed", [(5, 1), (11, 2), (23, 3), (37, 4)])
def test_adjoint_vs_central_differences(ctx, orc, net_seed, cfg_seed):
    """The adjoint row against central differences of the oracle's forward pass,
    for several networks and spin configurations."""
    from yannq_b200 import api

    f, p = _net(api, ctx, seed=net_seed)
    rng = np.random.default_rng(cfg_seed)
    s = rng.choice(np.array([-1, 1], np.int8), size=(1, L))
    f.set_batch(s)
    f.forward()
    O = f.adjoint()[0]
    h = 1e-4
    idx = np.concatenate([np.arange(K * CH), rng.choice(np.arange(K * CH, len(p)), 200, replace=False)])
    for k in idx:
        pp, pm = p.copy(), p.copy()
        pp[k] += h
        pm[k] -= h
        fd = (orc.ff_forward(L, CH, K, F, pp, s[0]) - orc.ff_forward(L, CH, K, F, pm, s[0])) / (2 * h)
        assert abs(O[k] - fd) < 1e-3 * max(1.0, abs(fd)), (k, O[k], fd)
    f.close()


@pytest.mark.parametrize("hfield", [0.5, 1.0, 1.5])
def test_eloc_tfi_matches_full_forwards(ctx, orc, hfield):
    from yannq_b200 import api

    f, p = _net(api, ctx, seed=7)
    rng = np.random.default_rng(2)
    s = rng.choice(np.array([-1, 1], np.int8), size=(16, L))
    f.set_batch(s)
    got = f.eloc_tfi(-1.0, -hfield)
    for b in range(len(s)):
        lp = orc.ff_forward(L, CH, K, F, p, s[b])
        e = 0.0
        for i in range(L):
            e += -1.0 * s[b, i] * s[b, (i + 1) % L]
            t = s[b].copy()
            t[i] *= -1
            e += -hfield * np.exp(orc.ff_forward(L, CH, K, F, p, t) - lp)
        assert abs(got[b].real - e) < 1e-5 * max(1.0, abs(e))
    f.close()
