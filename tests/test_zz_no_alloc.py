"""The no-allocation entry point yq_rbm_oloc_noalloc.

It serves callers that cannot let the library allocate device memory: they
pass device buffers they own, and the call keeps its temporary partial sums in a
fixed array compiled into the library.  This test hands it device buffers
(allocated here by torch, standing in for such a caller's own allocator) and
checks its output against the existing SR object's oloc (yq_sr_get) on two calls
in a row with different sample sets, so the second call also shows that what the
first call left in the shared array does not leak into the result.  It lives in
its own file so that a run stopping at the first failure has already run every
other test.
"""
import ctypes as C

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

TOL64 = 1e-12  # FP64 parity tolerance used by the other GPU tests
TOL32 = 5e-5   # complex64 tolerance used by the other GPU tests


def _reference_oloc(api, q, ctx, sigma, theta, prec):
    H = api.Hamiltonian.tfi(ctx, q.n, -1.0, -1.0)
    S = api.Sampler(q, 1)
    S.put_samples(sigma, theta)
    sr = api.SR(q, H, S, api.SR_T if prec == api.PREC_MIXED else api.SR_AUTO, prec)
    sr.construct()
    want = sr.get(1, q.dim)
    for x in (sr, S, H):
        x.close()
    return want


@pytest.mark.parametrize("dtype", [1, 0])
def test_oloc_noalloc_matches_sr_oloc_on_two_calls(orc, dtype):
    import torch

    from yannq_b200 import api

    n, m = 16, 32
    ctx = api.Context(0)
    q = api.RBM(ctx, n, m, True, dtype)
    p = orc.init_params(n, m, 20261203, 0.2)
    q.set_params(p)
    prec = api.PREC_FP64 if dtype == api.C128 else api.PREC_MIXED
    tol = TOL64 if dtype == api.C128 else TOL32
    cdt = np.complex128 if dtype == api.C128 else np.complex64
    out = torch.zeros(2 * q.dim, dtype=torch.float64, device="cuda")
    for call, (chains, seed) in enumerate([(64, 5), (24, 9)]):
        sigma, theta, _, _ = orc.sample(n, m, p, chains, seed=seed, n_sweeps=8, n_discard=16)
        want = _reference_oloc(api, q, ctx, sigma, theta, prec)
        d_sigma = torch.from_numpy(np.ascontiguousarray(sigma)).cuda()
        th = np.ascontiguousarray(theta.astype(cdt))
        d_theta = torch.from_numpy(th.view(np.float64 if dtype == api.C128 else np.float32)).cuda()
        torch.cuda.synchronize()
        rc = api.lib().yq_rbm_oloc_noalloc(q.h, len(sigma), C.c_void_p(d_sigma.data_ptr()),
                                           C.c_void_p(d_theta.data_ptr()), C.c_void_p(out.data_ptr()))
        api.check(rc)
        ctx.synchronize()
        got = out.cpu().numpy().view(np.complex128)
        err = np.max(np.abs(got - want)) / max(1.0, np.max(np.abs(want)))
        assert err < tol, (call, err)
    q.close()
    ctx.close()


def test_oloc_noalloc_rejects_machines_beyond_the_scratch(orc):
    import torch

    from yannq_b200 import api

    ctx = api.Context(0)
    q = api.RBM(ctx, 1000, 1000, True, api.C128)  # (n + 1) (m + 1) > 262144
    buf = torch.zeros(16, dtype=torch.float64, device="cuda")
    rc = api.lib().yq_rbm_oloc_noalloc(q.h, 1, C.c_void_p(buf.data_ptr()), C.c_void_p(buf.data_ptr()),
                                       C.c_void_p(buf.data_ptr()))
    assert rc == api.E_ARG and "4 MiB" in api.last_error()
    q.close()
    ctx.close()
