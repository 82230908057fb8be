"""The bounded device waits run out cleanly.

The persistent tile Cholesky and the triangular solves wait on flags published by
other CTAs, each wait limited to a number of polls; when one gives up it records
YQ_E_TIMEOUT in the context's status word and raises an abort word that every
other CTA checks before it takes work or while it waits.  Here the flag of the
first work item is never set (its counter starts past it), the limit is a few
thousand polls, and the test checks that the call returns YQ_E_TIMEOUT within
seconds, that no CTA published anything after the abort, and that the same
context then runs an ordinary SR solve correctly.  No kernel traps or faults.
"""
import ctypes as C
import time

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("which", [0, 1], ids=["tile_factorisation", "forward_solve"])
def test_unpublished_flag_times_out_and_context_stays_usable(orc, which):
    from yannq_b200 import api

    ctx = api.Context(0)
    published = C.c_int(-1)
    t0 = time.perf_counter()
    rc = api.lib().yq_debug_wait_timeout(ctx.h, which, 4096, C.byref(published))
    dt = time.perf_counter() - t0
    assert rc == api.E_TIMEOUT, (rc, api.last_error())
    assert "timed out" in api.last_error()
    assert published.value == 0
    assert dt < 30.0
    # the status word was read and cleared; the context runs a normal S-form solve
    n, m = 8, 16
    h = orc.Ham.tfi(n, -1.0, -1.0)
    p = orc.init_params(n, m, 3, 0.1)
    s, th, _, _ = orc.sample(n, m, p, 32, seed=4, n_sweeps=8, n_discard=16)
    q = api.RBM(ctx, n, m, True, api.C128)
    q.set_params(p)
    H = api.Hamiltonian.tfi(ctx, n, -1.0, -1.0)
    S = api.Sampler(q, 32)
    S.put_samples(s, th)
    sr = api.SR(q, H, S, api.SR_S, api.PREC_FP64)
    sr.construct()
    v, _, _ = sr.solve(1e-3, api.SOLVE_LLT)
    ref = orc.sr_step(h, m, p, s, th, 1e-3, orc.SR_S, orc.SOLVE_LLT)
    assert np.max(np.abs(v - ref["v"])) <= 1e-9 * np.max(np.abs(ref["v"]))
    for x in (sr, S, H, q, ctx):
        x.close()
