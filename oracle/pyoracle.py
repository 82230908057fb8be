"""ctypes front end of the CPU oracle (oracle/liboracle.so).

TEST INFRASTRUCTURE ONLY: imported by tests/, by the smoke check and by the
CPU-baseline leg of bench.py, never by the product package.  Complex arrays
cross the boundary as numpy complex128 (interleaved doubles).
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB_PATH = os.path.join(_HERE, "liboracle.so")

# Hamiltonian kinds (oracle.hpp)
TFI, XXZ, TFI2D, XXX, J1J2, XYZNNN, KITAEV_HEX = 0, 1, 2, 3, 4, 5, 6
MOVE_LOCAL, MOVE_EXCHANGE_ANY, MOVE_EXCHANGE_NN, MOVE_HAMILTONIAN = 0, 1, 2, 3
SR_S, SR_T = 0, 1
SOLVE_LLT, SOLVE_CG = 0, 1


def build(quiet: bool = True) -> str:
    """Compile liboracle.so with the committed Makefile (no-op when up to date)."""
    out = subprocess.run(["make", "-C", _HERE], capture_output=True, text=True)
    if out.returncode != 0:
        raise RuntimeError("oracle build failed:\n" + out.stdout + out.stderr)
    return _LIB_PATH


_lib = None


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(_LIB_PATH):
            build()
        _lib = C.CDLL(_LIB_PATH)
        _declare(_lib)
    return _lib


def _p(a):
    return a.ctypes.data_as(C.c_void_p) if a is not None else None


def _declare(L):
    vp, i, d, u64, u32 = C.c_void_p, C.c_int, C.c_double, C.c_uint64, C.c_uint32
    sig = {
        "orc_philox": (None, [vp, vp, vp]),
        "orc_logcosh": (None, [vp, vp]),
        "orc_logcosh_real": (d, [d]),
        "orc_init_params": (None, [i, i, i, u64, d, vp]),
        "orc_theta": (None, [i, i, i, vp, vp, vp]),
        "orc_logpsi": (None, [i, i, i, vp, vp, vp]),
        "orc_psi": (None, [i, i, i, vp, vp, vp]),
        "orc_logratio": (None, [i, i, i, vp, vp, vp, i, vp, vp]),
        "orc_flip": (None, [i, i, i, vp, vp, vp, i, vp]),
        "orc_logderiv": (None, [i, i, i, vp, vp, vp, vp]),
        "orc_logderiv_batch": (None, [i, i, i, vp, i, vp, vp, vp, i]),
        "orc_ham_enumerate": (d, [i, i, i, i, vp, vp, vp, vp, i, vp]),
        "orc_ham_column": (i, [i, i, i, i, vp, u64, vp, vp, i]),
        "orc_eloc": (None, [i, i, i, i, vp, i, i, vp, i, vp, vp, vp, i]),
        "orc_random_sigma": (None, [i, i, u64, u32, u32, vp]),
        "orc_sample": (None, [i, i, i, vp, i, i, i, u64, u32, i, i, i, i, vp, vp, vp, vp, i, i, i, i, vp]),
        "orc_sample_pt": (None, [i, i, i, vp, i, i, i, i, u64, u32, i, i, i, i, vp, vp, vp, vp, vp, i, i, i, i, vp]),
        "orc_sr_step": (i, [i, i, i, i, vp, i, i, vp, i, vp, vp, d, i, i, d, vp, vp, vp, vp, vp, i]),
        "orc_cholesky_solve": (i, [i, vp, vp]),
        "orc_exact": (i, [i, i, i, i, vp, i, i, vp, i, i, vp, vp, vp, vp, i]),
        "orc_exact_sample": (i, [i, i, i, vp, i, i, i, u64, u32, vp, vp, i]),
        "orc_basis": (i, [i, i, i, vp, i]),
        "orc_ed_ground": (d, [i, i, i, i, vp, i, i, i, i]),
        "orc_ap_dims": (i, [i, i, i, i, vp, vp, vp]),
        "orc_ap_init": (None, [i, i, i, i, vp, vp, u64, d, i, vp]),
        "orc_ap_log_psi": (None, [i, i, i, i, vp, vp, vp, i, vp, vp]),
        "orc_ap_log_deriv": (None, [i, i, i, i, vp, vp, vp, i, vp, vp]),
        "orc_ngd_exact": (i, [i, i, i, i, vp, i, i, i, vp, vp, vp, i, i, i, vp, vp, vp, vp, vp, vp, i]),
        "orc_ff_forward": (d, [i, i, i, i, vp, vp]),
        "orc_ff_backward": (None, [i, i, i, i, vp, vp, vp]),
        "orc_ff_batch": (None, [i, i, i, i, vp, i, vp, vp, vp, i]),
    }
    for name, (res, args) in sig.items():
        f = getattr(L, name)
        f.restype = res
        f.argtypes = args


# ---------------------------------------------------------------------------
class Ham:
    """Hamiltonian descriptor with the reference's sign conventions.

    TFI:    E_loc = sum_i J s_i s_{i+1} + h ratio(i)         (TFIsing(n, J, h))
    XXZ:    E_loc = sum_i J Delta zz_i + sign J (1 - zz_i) ratio(i, i+1)
    TFI2D:  E_loc = sum_i J s_i (s_right + s_down) + h ratio(i)  on an lx x ly torus
    XXX:    XXX(n)                      J = h = 0
    J1J2:   J1J2(n, J1, J2, signRule)   J = J1, h = J2
    XYZNNN: XYZNNN(n, a, b)             J = a, h = b
    KITAEV_HEX: KitaevHex(n_, m_, Jx, Jy, Jz) plus field h; lx = n_, ly = m_
    """

    def __init__(self, kind, n, J, h, sign=1.0, lx=0, ly=0, jy=0.0, jz=0.0):
        self.kind, self.n, self.J, self.h, self.sign, self.lx, self.ly = kind, n, J, h, sign, lx, ly
        self.jy, self.jz = jy, jz
        self._hp = np.array([J, h, sign, jy, jz], dtype=np.float64)

    @classmethod
    def tfi(cls, n, J, h):
        return cls(TFI, n, J, h)

    @classmethod
    def xxz(cls, n, J, delta, sign_rule=False):
        return cls(XXZ, n, J, delta, -1.0 if sign_rule else 1.0)

    @classmethod
    def tfi2d(cls, lx, ly, J, h):
        return cls(TFI2D, lx * ly, J, h, 1.0, lx, ly)

    @classmethod
    def xxx(cls, n):
        return cls(XXX, n, 0.0, 0.0)

    @classmethod
    def j1j2(cls, n, J1, J2, sign_rule=False):
        return cls(J1J2, n, J1, J2, -1.0 if sign_rule else 1.0)

    @classmethod
    def xyznnn(cls, n, a, b):
        return cls(XYZNNN, n, a, b)

    @classmethod
    def kitaev_hex(cls, ncol, nrow, Jx, Jy, Jz, h=0.0):
        return cls(KITAEV_HEX, ncol * nrow, Jx, h, 1.0, ncol, nrow, Jy, Jz)

    def args(self):
        return (self.kind, self.n, self.lx, self.ly, _p(self._hp))


def rbm_dim(n, m, use_bias=True):
    return n * m + (n + m if use_bias else 0)


def philox(ctr, key):
    c = np.asarray(ctr, dtype=np.uint32)
    k = np.asarray(key, dtype=np.uint32)
    o = np.zeros(4, dtype=np.uint32)
    lib().orc_philox(_p(c), _p(k), _p(o))
    return o


def logcosh(z):
    zz = np.asarray([complex(z).real, complex(z).imag], dtype=np.float64)
    o = np.zeros(2)
    lib().orc_logcosh(_p(zz), _p(o))
    return complex(o[0], o[1])


def logcosh_real(x):
    return lib().orc_logcosh_real(float(x))


def init_params(n, m, seed, sd, use_bias=True):
    p = np.zeros(rbm_dim(n, m, use_bias), dtype=np.complex128)
    lib().orc_init_params(n, m, int(use_bias), seed, sd, _p(p))
    return p


def _s8(sigma):
    return np.ascontiguousarray(sigma, dtype=np.int8)


def theta(n, m, params, sigma, use_bias=True):
    th = np.zeros(m, dtype=np.complex128)
    lib().orc_theta(n, m, int(use_bias), _p(params), _p(_s8(sigma)), _p(th))
    return th


def logpsi(n, m, params, sigma, use_bias=True):
    o = np.zeros(2)
    lib().orc_logpsi(n, m, int(use_bias), _p(params), _p(_s8(sigma)), _p(o))
    return complex(o[0], o[1])


def psi(n, m, params, sigma, use_bias=True):
    o = np.zeros(2)
    lib().orc_psi(n, m, int(use_bias), _p(params), _p(_s8(sigma)), _p(o))
    return complex(o[0], o[1])


def logratio(n, m, params, sigma, th, flips, use_bias=True):
    f = np.asarray(flips, dtype=np.int32)
    o = np.zeros(2)
    lib().orc_logratio(n, m, int(use_bias), _p(params), _p(_s8(sigma)), _p(th), len(f), _p(f), _p(o))
    return complex(o[0], o[1])


def flip(n, m, params, sigma, th, flips, use_bias=True):
    """In place on sigma (int8 array) and th (complex128 array)."""
    f = np.asarray(flips, dtype=np.int32)
    lib().orc_flip(n, m, int(use_bias), _p(params), _p(sigma), _p(th), len(f), _p(f))


def logderiv(n, m, params, sigma, th, use_bias=True):
    o = np.zeros(rbm_dim(n, m, use_bias), dtype=np.complex128)
    lib().orc_logderiv(n, m, int(use_bias), _p(params), _p(_s8(sigma)), _p(th), _p(o))
    return o


def logderiv_rows(n, m, params, sigma, th, use_bias=True, nthreads=0):
    """constructDelta (GroundState/utils.hpp:12-51): logDeriv rows of a batch, Ns x P."""
    sigma = _s8(sigma)
    ns = sigma.shape[0]
    th = np.ascontiguousarray(th, dtype=np.complex128)
    o = np.zeros((ns, rbm_dim(n, m, use_bias)), dtype=np.complex128)
    lib().orc_logderiv_batch(n, m, int(use_bias), _p(params), ns, _p(sigma), _p(th), _p(o), nthreads or os.cpu_count())
    return o


def ham_enumerate(ham, sigma, cap=4096):
    masks = np.zeros(cap, dtype=np.uint64)
    coeffs = np.zeros(cap)
    cnt = C.c_int(0)
    d = lib().orc_ham_enumerate(*ham.args(), _p(_s8(sigma)), _p(masks), _p(coeffs), cap, C.byref(cnt))
    return d, masks[: cnt.value].copy(), coeffs[: cnt.value].copy()


def ham_column(ham, col, cap=4096):
    rows = np.zeros(cap, dtype=np.uint64)
    vals = np.zeros(cap)
    c = lib().orc_ham_column(*ham.args(), int(col), _p(rows), _p(vals), cap)
    return rows[:c].copy(), vals[:c].copy()


def eloc(ham, m, params, sigma, th, use_bias=True, nthreads=0):
    sigma = _s8(sigma)
    ns = sigma.shape[0]
    th = np.ascontiguousarray(th, dtype=np.complex128)
    o = np.zeros(ns, dtype=np.complex128)
    lib().orc_eloc(*ham.args(), m, int(use_bias), _p(params), ns, _p(sigma), _p(th), _p(o), nthreads or os.cpu_count())
    return o


def random_sigma(n, nup, seed, epoch, chain):
    s = np.zeros(n, dtype=np.int8)
    lib().orc_random_sigma(n, nup, seed, epoch, chain, _p(s))
    return s


def _ham_tail(ham):
    return (ham.kind, ham.lx, ham.ly, _p(ham._hp)) if ham is not None else (0, 0, 0, None)


def sample(n, m, params, n_chains, move=MOVE_LOCAL, nup=-1, seed=0, epoch=0, reinit=True, n_sweeps=1,
           n_discard=0, sweep_len=0, chain_sigma=None, use_bias=True, nthreads=0, ham=None):
    """Restated SamplerMT (nTmps = 1).  Returns (sigma[Ns, n], theta[Ns, m], chain_sigma, acc).
    move MOVE_HAMILTONIAN takes its proposals from `ham` (HamiltonianSweeper)."""
    cs = np.zeros((n_chains, n), dtype=np.int8) if chain_sigma is None else np.ascontiguousarray(chain_sigma, np.int8)
    ns = n_chains * n_sweeps
    osig = np.zeros((ns, n), dtype=np.int8)
    oth = np.zeros((ns, m), dtype=np.complex128)
    acc = np.zeros(n_chains, dtype=np.uint64)
    lib().orc_sample(n, m, int(use_bias), _p(params), n_chains, move, nup, seed, epoch, int(reinit), n_sweeps,
                     n_discard, sweep_len, _p(cs), _p(osig), _p(oth), _p(acc), nthreads or os.cpu_count(),
                     *_ham_tail(ham))
    return osig, oth, cs, acc


def sample_pt(n, m, params, n_chains, ntemps, move=MOVE_LOCAL, nup=-1, seed=0, epoch=0, reinit=True, n_sweeps=1,
              n_discard=0, sweep_len=0, chain_sigma=None, slot=None, use_bias=True, nthreads=0, ham=None):
    """Restated SamplerMT with nTmps = ntemps > 1 (temperature swaps between the
    chains of a group).  Returns (sigma[groups * n_sweeps, n], theta, chain_sigma, slot, acc)."""
    cs = np.zeros((n_chains, n), dtype=np.int8) if chain_sigma is None else np.ascontiguousarray(chain_sigma, np.int8)
    sl = np.zeros(n_chains, dtype=np.int32) if slot is None else np.ascontiguousarray(slot, np.int32)
    ns = (n_chains // ntemps) * n_sweeps
    osig = np.zeros((ns, n), dtype=np.int8)
    oth = np.zeros((ns, m), dtype=np.complex128)
    acc = np.zeros(n_chains, dtype=np.uint64)
    lib().orc_sample_pt(n, m, int(use_bias), _p(params), n_chains, ntemps, move, nup, seed, epoch, int(reinit),
                        n_sweeps, n_discard, sweep_len, _p(cs), _p(sl), _p(osig), _p(oth), _p(acc),
                        nthreads or os.cpu_count(), *_ham_tail(ham))
    return osig, oth, cs, sl, acc


def sr_step(ham, m, params, sigma, th, shift, mode=SR_S, solver=SOLVE_LLT, cgtol=1e-4, use_bias=True, nthreads=0):
    sigma = _s8(sigma)
    ns, n = sigma.shape
    P = rbm_dim(n, m, use_bias)
    th = np.ascontiguousarray(th, dtype=np.complex128)
    v = np.zeros(P, np.complex128)
    g = np.zeros(P, np.complex128)
    ol = np.zeros(P, np.complex128)
    el = np.zeros(ns, np.complex128)
    st = np.zeros(4)
    status = lib().orc_sr_step(*ham.args(), m, int(use_bias), _p(params), ns, _p(sigma), _p(th), shift, mode, solver,
                               cgtol, _p(v), _p(g), _p(ol), _p(el), _p(st), nthreads or os.cpu_count())
    return dict(status=status, v=v, grad=g, oloc=ol, elocs=el, energy=st[0], energy_var=st[1],
                cg_iters=int(st[2]), cg_relres=st[3])


class ObsAvg:
    """Runners/RunRBM.hpp:13-37: obs = beta obs + (1 - beta) x per update; getAvg
    divides by 1 - beta^t (t = number of updates)."""

    def __init__(self, beta, ini):
        self.beta, self.t, self.obs = beta, 0, np.array(ini, dtype=np.complex128)

    def update(self, x):
        self.obs = self.beta * self.obs + (1.0 - self.beta) * x
        self.t += 1

    def get_avg(self):
        return self.obs / (1.0 - self.beta ** self.t)


def run_rbm(ham, m, params, n_chains, epochs, n_sweeps, n_discard, seed, shift, lr, beta1=0.0, beta2=0.0,
            grad_clip=0.0, use_cg=False, use_bias=True, move=MOVE_LOCAL, nup=-1, nthreads=0):
    """Runners/RunRBM.hpp:151-221 restated for epochs ll = 0 .. epochs-1 with a fixed
    lambda (`shift`) and SGD rate (`lr`): randomize + sample (Philox epoch ll),
    constructFromSamples (E_loc, centred logDeriv rows, energyGrad), then

      gradAvg.update(grad); g = gradAvg.getAvg()                    (:180-181)
      CG branch (use_cg and beta2 == 0):  v = (S + lambda)^{-1} g,
          cgErr = |apply(v) - g|                                    (:183-191)
      LLT branch: gradAvg.update(grad) again; fisherAvg.update(S);
          v = LLT(fisherAvg.getAvg() + lambda I).solve(g)           (:192-202)
      nv = |v|; v *= clip / nv if clip != 0 and nv > clip          (:204-209)
      params -= lr v                                                (SGD, :211-216)

    The CG branch is solved exactly here (numpy), the limit of Eigen's CG as its
    tolerance goes to 0.  Returns (per-epoch dicts energy / nv / cg_err / v, params)."""
    n = ham.n
    P = rbm_dim(n, m, use_bias)
    p = np.array(params, dtype=np.complex128)
    g_avg = ObsAvg(beta1, np.zeros(P))
    f_avg = ObsAvg(beta2, np.zeros((P, P)))
    out = []
    for ll in range(epochs):
        s, th, _, _ = sample(n, m, p, n_chains, move=move, nup=nup, seed=seed, epoch=ll, reinit=True,
                             n_sweeps=n_sweeps, n_discard=n_discard, use_bias=use_bias, nthreads=nthreads)
        O = logderiv_rows(n, m, p, s, th, use_bias, nthreads)
        el = eloc(ham, m, p, s, th, use_bias, nthreads)
        ns = len(s)
        Oc = O - O.mean(axis=0)
        grad = Oc.conj().T @ el / ns
        S = Oc.conj().T @ Oc / ns
        g_avg.update(grad)
        g = g_avg.get_avg()
        A = S + shift * np.eye(P)
        if use_cg and beta2 == 0.0:
            v = np.linalg.solve(A, g)
            cg_err = float(np.linalg.norm(A @ v - g))
        else:
            g_avg.update(grad)
            f_avg.update(S)
            st, v = cholesky_solve(f_avg.get_avg() + shift * np.eye(P), g)  # Eigen::LLT restated
            assert st == 0, "LLT met a non-positive pivot"
            cg_err = 0.0
        nv = float(np.linalg.norm(v))
        if grad_clip != 0.0 and nv > grad_clip:
            v = v * (grad_clip / nv)
        p = p - lr * v
        out.append(dict(energy=float(el.real.mean()), nv=nv, cg_err=cg_err, v=v))
    return out, p


def cholesky_solve(A, b):
    A = np.array(A, dtype=np.complex128, order="C")
    x = np.array(b, dtype=np.complex128)
    st = lib().orc_cholesky_solve(A.shape[0], _p(A), _p(x))
    return st, x


def exact(ham, m, params, basis_kind=0, nup=0, with_S=True, use_bias=True, nthreads=0):
    P = rbm_dim(ham.n, m, use_bias)
    st = np.zeros(2)
    ol = np.zeros(P, np.complex128)
    g = np.zeros(P, np.complex128)
    S = np.zeros((P, P), np.complex128) if with_S else None
    dim = lib().orc_exact(*ham.args(), m, int(use_bias), _p(params), basis_kind, nup, _p(st), _p(ol), _p(g), _p(S),
                          nthreads or os.cpu_count())
    return dict(energy=st[0], energy_var=st[1], oloc=ol, grad=g, S=S, dim=dim)


def exact_sample(n, m, params, nsamples, seed, epoch=0, basis_kind=0, nup=0, use_bias=True, nthreads=0):
    """Samplers/ExactSampler.hpp:49-79 restated: basis positions and configuration
    indices of `nsamples` draws from |psi|^2 (exact-sampler Philox stream)."""
    pos = np.zeros(nsamples, np.uint32)
    idx = np.zeros(nsamples, np.uint64)
    dim = lib().orc_exact_sample(n, m, int(use_bias), _p(params), basis_kind, nup, nsamples, seed, epoch, _p(pos),
                                 _p(idx), nthreads or os.cpu_count())
    return pos, idx, dim


def sigma_of(index, n):
    """Utilities/Utility.hpp:91-99 toSigma: bit i set <=> sigma_i = -1."""
    index = int(index)
    return np.array([1 - 2 * ((index >> i) & 1) for i in range(n)], dtype=np.int8)


def index_of(sigma):
    """Utilities/Utility.hpp:102-110 toValue."""
    return int(sum(((1 - int(x)) // 2) << i for i, x in enumerate(sigma)))


def basis(n, basis_kind=0, nup=0):
    from math import comb
    cap = (1 << n) if basis_kind == 0 else comb(n, nup)
    out = np.zeros(cap, dtype=np.uint64)
    c = lib().orc_basis(n, basis_kind, nup, _p(out), cap)
    return out[:c]


def ed_ground(ham, basis_kind=0, nup=0, maxit=300, nthreads=0):
    return lib().orc_ed_ground(*ham.args(), basis_kind, nup, maxit, nthreads or os.cpu_count())


def ff_dim(L, conv_out, conv_k, fc_out):
    return conv_k * conv_out + L * conv_out * fc_out


def ff_forward(L, conv_out, conv_k, fc_out, params, sigma):
    p = np.ascontiguousarray(params, dtype=np.float64)
    return lib().orc_ff_forward(L, conv_out, conv_k, fc_out, _p(p), _p(_s8(sigma)))


def ff_backward(L, conv_out, conv_k, fc_out, params, sigma):
    p = np.ascontiguousarray(params, dtype=np.float64)
    der = np.zeros(ff_dim(L, conv_out, conv_k, fc_out))
    lib().orc_ff_backward(L, conv_out, conv_k, fc_out, _p(p), _p(_s8(sigma)), _p(der))
    return der


def ff_batch(L, conv_out, conv_k, fc_out, params, sigma, want_der=True, nthreads=0):
    p = np.ascontiguousarray(params, dtype=np.float64)
    sigma = _s8(sigma)
    B = sigma.shape[0]
    lp = np.zeros(B)
    der = np.zeros((B, ff_dim(L, conv_out, conv_k, fc_out))) if want_der else None
    lib().orc_ff_batch(L, conv_out, conv_k, fc_out, _p(p), B, _p(sigma), _p(lp), _p(der), nthreads or os.cpu_count())
    return lp, der


# ---------------------------------------------------------------------------
# RBM checkpoints: the cereal BinaryOutputArchive image of std::unique_ptr<RBM<T>>
# (Runners/RunRBM.hpp:155-164, Runners/AbstractRunner.hpp:83-94).  cereal is not
# vendored; the layout is restated from its published binary-archive rules
# (little-endian raw values, no names, no header; a unique_ptr is one "valid" byte
# and the pointee; a versioned class writes its u32 version before its first
# instance) applied to Serializers/SerializeRBM.hpp:20-82 (useBias, N, M, W, then
# a and b if useBias) and Serializers/SerializeEigen.hpp:8-35 (i32 rows, i32 cols,
# raw column-major data).
ARCHIVE_ELEM = {0: ("<f4", True), 1: ("<f8", True), 2: ("<f8", False), 3: ("<f4", False)}


def rbm_archive(n, m, params, use_bias=True, elem=1, version=1):
    """bytes of the archive; params in the reference layout [W (m x n col-major) | a | b]."""
    import struct

    fmt, cplx = ARCHIVE_ELEM[elem]
    p = np.asarray(params, np.complex128)

    def values(x):
        x = np.asarray(x, np.complex128)
        if cplx:
            return np.stack([x.real, x.imag], axis=-1).astype(fmt).tobytes()
        assert np.all(x.imag == 0)
        return x.real.astype(fmt).tobytes()

    nm = n * m
    out = struct.pack("<BIBII", 1, version, int(bool(use_bias)), n, m)
    out += struct.pack("<ii", m, n) + values(p[:nm])
    if use_bias:
        out += struct.pack("<ii", n, 1) + values(p[nm:nm + n])
        out += struct.pack("<ii", m, 1) + values(p[nm + n:nm + n + m])
    return out


def rbm_unarchive(data, elem=1):
    """(n, m, use_bias, params) from an archive."""
    import struct

    fmt, cplx = ARCHIVE_ELEM[elem]
    valid, _version, bias, n, m = struct.unpack_from("<BIBII", data, 0)
    assert valid == 1
    at = struct.calcsize("<BIBII")
    es = np.dtype(fmt).itemsize * (2 if cplx else 1)

    def block(rows, cols):
        nonlocal at
        r, c = struct.unpack_from("<ii", data, at)
        assert (r, c) == (rows, cols)
        at += 8
        raw = np.frombuffer(data, dtype=fmt, count=rows * cols * (2 if cplx else 1), offset=at)
        at += rows * cols * es
        raw = raw.astype(np.float64)
        return raw[0::2] + 1j * raw[1::2] if cplx else raw + 0j

    parts = [block(m, n)]
    if bias:
        parts += [block(n, 1), block(m, 1)]
    assert at == len(data)
    return n, m, bool(bias), np.concatenate(parts)


# ---------------------------------------------------------------------------
# AmplitudePhase (Machines/AmplitudePhase.hpp) and NGDExact (GroundState/NGDExact.hpp).
class AP:
    """Shape of an AmplitudePhase machine: RBM<double>(n, m, use_bias) amplitude and
    a phase network given as desc (L x 6 ints: type, a, b, k, stride, bias) and xs
    (L doubles) in the oracle's LayerType numbering."""

    def __init__(self, n, m, use_bias, desc, xs):
        self.n, self.m, self.use_bias = n, m, bool(use_bias)
        self.desc = np.ascontiguousarray(desc, np.int32).reshape(-1, 6)
        self.xs = np.ascontiguousarray(xs, np.float64).reshape(-1)
        dims = np.zeros(2, np.uint64)
        if lib().orc_ap_dims(n, m, int(use_bias), len(self.xs), _p(self.desc), _p(self.xs), _p(dims)) != 0:
            raise ValueError("bad phase network")
        self.Pa, self.Pp = int(dims[0]), int(dims[1])
        self.dim = self.Pa + self.Pp

    def args(self):
        return (self.n, self.m, int(self.use_bias), len(self.xs), _p(self.desc), _p(self.xs))


def ap_init(ap, seed, sigma_amp, mode=1):
    p = np.zeros(ap.dim)
    lib().orc_ap_init(*ap.args(), seed, sigma_amp, mode, _p(p))
    return p


def ap_log_psi(ap, params, sigma):
    s = _s8(sigma).reshape(-1, ap.n)
    out = np.zeros(s.shape[0], np.complex128)
    lib().orc_ap_log_psi(*ap.args(), _p(np.ascontiguousarray(params, np.float64)), s.shape[0], _p(s), _p(out))
    return out


def ap_log_deriv(ap, params, sigma):
    s = _s8(sigma).reshape(-1, ap.n)
    out = np.zeros((s.shape[0], ap.dim), np.complex128)
    lib().orc_ap_log_deriv(*ap.args(), _p(np.ascontiguousarray(params, np.float64)), s.shape[0], _p(s), _p(out))
    return out


def ngd_exact(ham, ap, params, basis_kind=0, nup=0, with_corr=True, nthreads=0):
    """NGDExact::constructExact: dict of energy, grad, oloc_amp, oloc_phase, corr_amp, corr_phase."""
    g = np.zeros(ap.dim)
    oa, op = np.zeros(ap.Pa), np.zeros(ap.Pp)
    ca = np.zeros((ap.Pa, ap.Pa)) if with_corr else None
    cp = np.zeros((ap.Pp, ap.Pp)) if with_corr else None
    e = C.c_double()
    k, lx, ly, hp = ham.kind, ham.lx, ham.ly, _p(ham._hp)
    lib().orc_ngd_exact(k, ham.n, lx, ly, hp, ap.m, int(ap.use_bias), len(ap.xs), _p(ap.desc), _p(ap.xs),
                        _p(np.ascontiguousarray(params, np.float64)), basis_kind, nup, int(with_corr), C.byref(e),
                        _p(g), _p(oa), _p(op), _p(ca), _p(cp), nthreads or os.cpu_count())
    return {"energy": e.value, "grad": g, "oloc_amp": oa, "oloc_phase": op, "corr_amp": ca, "corr_phase": cp}
