"""The no-allocation entry point yq_rbm_oloc_noalloc.

It serves callers that cannot let the library allocate device memory: they
pass device buffers they own, and the call keeps its temporary partial sums in a
fixed array compiled into the library.  This test hands it device buffers
(allocated here by torch, standing in for such a caller's own allocator) and
checks, on two calls in a row with different sample sets (so the second call
also shows that what the first call left in the shared array does not leak into
the result), for machines with and without biases:

* its output against the oracle's column mean of the logDeriv rows
  (Machines/RBM.hpp:390-406, GroundState/SRMat.hpp:97-98) and against the SR
  object's oloc (yq_sr_get), at the tolerance of the other GPU tests;
* that the library made no device allocation during the call (yq_alloc_count).

It lives in its own file so that a run stopping at the first failure has already
run every other test.
"""
import ctypes as C

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

TOL64 = 1e-12  # FP64 parity tolerance used by the other GPU tests
TOL32 = 5e-5   # complex64 tolerance used by the other GPU tests


def _sr_oloc(api, q, ctx, sigma, theta, prec):
    H = api.Hamiltonian.tfi(ctx, q.n, -1.0, -1.0)
    S = api.Sampler(q, 1)
    S.put_samples(sigma, theta)
    sr = api.SR(q, H, S, api.SR_T if prec == api.PREC_MIXED else api.SR_AUTO, prec)
    sr.construct()
    want = sr.get(1, q.dim)
    for x in (sr, S, H):
        x.close()
    return want


@pytest.mark.parametrize("use_bias", [True, False])
@pytest.mark.parametrize("dtype", [1, 0])
def test_oloc_noalloc_matches_oracle_on_two_calls(orc, dtype, use_bias):
    import torch

    from yannq_b200 import api

    n, m = 16, 40
    ctx = api.Context(0)
    q = api.RBM(ctx, n, m, use_bias, dtype)
    p = orc.init_params(n, m, 20261203, 0.2, use_bias)
    q.set_params(p)
    prec = api.PREC_FP64 if dtype == api.C128 else api.PREC_MIXED
    tol = TOL64 if dtype == api.C128 else TOL32
    cdt = np.complex128 if dtype == api.C128 else np.complex64
    out = torch.zeros(2 * q.dim, dtype=torch.float64, device="cuda")
    for call, (chains, seed) in enumerate([(64, 5), (24, 9)]):
        sigma, theta, _, _ = orc.sample(n, m, p, chains, seed=seed, n_sweeps=8, n_discard=16, use_bias=use_bias)
        want = orc.logderiv_rows(n, m, p, sigma, theta, use_bias).mean(axis=0)
        d_sigma = torch.from_numpy(np.ascontiguousarray(sigma)).cuda()
        th = np.ascontiguousarray(theta.astype(cdt))
        d_theta = torch.from_numpy(th.view(np.float64 if dtype == api.C128 else np.float32)).cuda()
        torch.cuda.synchronize()
        a0 = api.alloc_count()
        rc = api.lib().yq_rbm_oloc_noalloc(q.h, len(sigma), C.c_void_p(d_sigma.data_ptr()),
                                           C.c_void_p(d_theta.data_ptr()), C.c_void_p(out.data_ptr()))
        api.check(rc)
        ctx.synchronize()
        assert api.alloc_count() == a0, "the no-allocation entry point allocated device memory"
        got = out.cpu().numpy().view(np.complex128)
        scale = max(1.0, np.max(np.abs(want)))
        err = np.max(np.abs(got - want)) / scale
        assert err < tol, (call, err)
        sr_oloc = _sr_oloc(api, q, ctx, sigma, theta, prec)
        assert np.max(np.abs(got - sr_oloc)) / scale < tol, call
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
