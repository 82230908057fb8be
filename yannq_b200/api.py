"""ctypes binding of libyannq_b200.so (include/yannq_b200.h).

This is the Python-side harness over the C ABI used by the tests and by
bench.py; the product is the shared library and its C/C++ headers.  There is no
fallback: importing this module fails if the library is missing.
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "libyannq_b200.so")

OK, E_ARG, E_CUDA, E_NOMEM, E_NOT_PD, E_NONFINITE, E_TIMEOUT, E_STATE, E_UNSUPPORTED = range(9)
C64, C128 = 0, 1
ARCHIVE_C64, ARCHIVE_C128, ARCHIVE_F64, ARCHIVE_F32 = 0, 1, 2, 3
LAYER_TYPES = {"conv1d": 0, "fc": 1, "identity": 10, "lncosh": 11, "tanh": 12, "weaktanh": 13, "sigmoid": 14,
               "relu": 15, "leakyrelu": 16, "hardtanh": 17, "softshrink": 18, "leakyhardtanh": 19, "softsign": 20,
               "cos": 21}
INIT_LECUN, INIT_XAVIER, INIT_HE = 0, 1, 2
NGD_GRAD, NGD_OLOC_AMP, NGD_OLOC_PHASE, NGD_CORR_AMP, NGD_CORR_PHASE = 0, 1, 2, 3, 4
NGD_AMP, NGD_PHASE, NGD_ALL = 0, 1, 2
HAM_TFI, HAM_XXZ, HAM_TFI2D, HAM_XXX, HAM_J1J2, HAM_XYZNNN, HAM_KITAEV_HEX = 0, 1, 2, 3, 4, 5, 6
MOVE_LOCAL, MOVE_EXCHANGE_ANY, MOVE_EXCHANGE_NN, MOVE_HAMILTONIAN = 0, 1, 2, 3
SR_AUTO, SR_S, SR_T = 0, 1, 2
PREC_FP64, PREC_MIXED = 0, 1
SOLVE_LLT, SOLVE_CG = 0, 1
BASIS_FULL, BASIS_JZ = 0, 1
STAGES = {"sample": 0, "eloc": 1, "O": 2, "gram": 3, "solve": 4, "update": 5, "total": 6, "mean": 7}


class YQError(RuntimeError):
    def __init__(self, code, msg):
        super().__init__(f"yannq_b200 error {code}: {msg}")
        self.code = code


class IterParams(C.Structure):
    _fields_ = [("n_sweeps", C.c_int), ("n_discard", C.c_int), ("reinit", C.c_int), ("seed", C.c_uint64),
                ("epoch", C.c_uint32), ("shift", C.c_double), ("lr", C.c_double), ("solver", C.c_int),
                ("cg_tol", C.c_double), ("ir_steps", C.c_int)]


class IterResult(C.Structure):
    _fields_ = [("energy", C.c_double), ("energy_var", C.c_double), ("update_norm", C.c_double),
                ("cg_err", C.c_double), ("accept_rate", C.c_double), ("status", C.c_int)]


# every symbol declared in include/yannq_b200.h with its argument types
_vp, _i, _d, _u64, _u32, _sz = C.c_void_p, C.c_int, C.c_double, C.c_uint64, C.c_uint32, C.c_size_t
SIGNATURES = {
    "yq_last_error": [C.c_char_p, _sz],
    "yq_version": [],
    "yq_launch_count": [_vp],
    "yq_alloc_count": [_vp],
    "yq_host_alloc": [_sz, _vp],
    "yq_host_free": [_vp],
    "yq_ctx_create": [_i, _vp],
    "yq_ctx_destroy": [_vp],
    "yq_ctx_synchronize": [_vp],
    "yq_ctx_stage_ms": [_vp, _i, _vp],
    "yq_measure_peaks": [_vp, _vp],
    "yq_rbm_create": [_vp, _i, _i, _i, _i, _vp],
    "yq_rbm_destroy": [_vp],
    "yq_rbm_dim": [_vp, _vp],
    "yq_rbm_archive_size": [_vp, _i, _vp],
    "yq_rbm_save_archive": [_vp, _i, _vp, C.c_size_t, _vp],
    "yq_rbm_load_archive": [_vp, _i, _vp, C.c_size_t],
    "yq_rbm_archive_shape": [_vp, C.c_size_t, _vp, _vp, _vp],
    "yq_rbm_save": [_vp, _i, C.c_char_p],
    "yq_rbm_load": [_vp, _i, C.c_char_p],
    "yq_rbm_file_shape": [C.c_char_p, _vp, _vp, _vp],
    "yq_ap_create": [_vp, _i, _i, _i, _i, _vp, _vp, _vp],
    "yq_ap_destroy": [_vp],
    "yq_ap_dims": [_vp, _vp, _vp],
    "yq_ap_set_params": [_vp, _vp],
    "yq_ap_get_params": [_vp, _vp],
    "yq_ap_update_params": [_vp, _vp],
    "yq_ap_init_random": [_vp, C.c_uint64, _d, _i],
    "yq_ap_log_psi": [_vp, _i, _vp, _vp],
    "yq_ap_log_deriv": [_vp, _i, _vp, _vp],
    "yq_ngd_create": [_vp, _vp, _i, _i, _vp],
    "yq_ngd_destroy": [_vp],
    "yq_ngd_basis_size": [_vp, _vp],
    "yq_ngd_construct": [_vp, _vp],
    "yq_ngd_get": [_vp, _i, _vp],
    "yq_ngd_iteration": [_vp, _d, _d, _i, _vp, _vp, _vp],
    "yq_rbm_set_params": [_vp, _vp],
    "yq_rbm_get_params": [_vp, _vp],
    "yq_rbm_update_params": [_vp, _vp],
    "yq_rbm_init_random": [_vp, _u64, _d],
    "yq_rbm_theta": [_vp, _i, _vp, _vp],
    "yq_rbm_log_psi": [_vp, _i, _vp, _vp],
    "yq_rbm_log_ratio": [_vp, _i, _vp, _vp, _i, _vp, _vp],
    "yq_rbm_log_deriv": [_vp, _i, _vp, _vp, _vp],
    "yq_rbm_log_ratio_k": [_vp, _i, _vp, _vp, _i, _vp, _vp],
    "yq_rbm_log_ratio_states": [_vp, _i, _vp, _vp, _vp, _vp, _vp],
    "yq_rbm_oloc_noalloc": [_vp, _i, _vp, _vp, _vp],
    "yq_ham_create": [_vp, _i, _i, _i, _i, _d, _d, _i, _vp],
    "yq_ham_create_kitaev_hex": [_vp, _i, _i, _d, _d, _d, _d, _vp],
    "yq_ham_destroy": [_vp],
    "yq_ham_num_offdiag": [_vp, _vp],
    "yq_ham_enumerate": [_vp, _i, _vp, _vp, _vp, _vp, _vp],
    "yq_eloc": [_vp, _vp, _i, _vp, _vp, _vp],
    "yq_sampler_create": [_vp, _i, _i, _i, _i, _vp],
    "yq_sampler_destroy": [_vp],
    "yq_sampler_set_hamiltonian": [_vp, _vp],
    "yq_sampler_set_resync": [_vp, _i],
    "yq_sampler_set_chains": [_vp, _vp],
    "yq_sampler_get_chains": [_vp, _vp],
    "yq_sample": [_vp, _i, _i, _u64, _u32, _i],
    "yq_sampler_num_samples": [_vp, _vp],
    "yq_sampler_get_samples": [_vp, _vp, _vp],
    "yq_sampler_get_accepts": [_vp, _vp],
    "yq_sampler_put_samples": [_vp, _i, _vp, _vp],
    "yq_sampler_sample_exact": [_vp, _i, _u64, _u32, _vp],
    "yq_sampler_chains_per_cta": [_vp, _vp],
    "yq_sampler_warps_per_chain": [_vp, _vp],
    "yq_sampler_set_tempering": [_vp, _i],
    "yq_sampler_get_slots": [_vp, _vp],
    "yq_exact": [_vp, _vp, _i, _i, _vp, _vp, _vp, _vp],
    "yq_exact_iteration": [_vp, _vp, _i, _i, _d, _d, _vp],
    "yq_batch_create": [_vp, _i, _vp, _vp],
    "yq_batch_iteration": [_vp, _vp, _vp],
    "yq_batch_destroy": [_vp],
    "yq_debug_wait_timeout": [_vp, _i, C.c_uint, _vp],
    "yq_sr_create": [_vp, _vp, _vp, _i, _i, _vp],
    "yq_sr_destroy": [_vp],
    "yq_sr_construct": [_vp],
    "yq_sr_energy": [_vp, _vp, _vp],
    "yq_sr_get": [_vp, _i, _vp],
    "yq_sr_solve": [_vp, _d, _i, _d, _vp, _vp, _vp],
    "yq_sr_set_solve_steps": [_vp, _i],
    "yq_sr_matrix": [_vp, _vp, _vp],
    "yq_sr_set_momentum": [_vp, _d, _d],
    "yq_sr_set_grad_clip": [_vp, _d],
    "yq_vmc_iteration": [_vp, _vp, _vp],
    "yq_ff_create": [_vp, _i, _i, _i, _i, _vp],
    "yq_ff_destroy": [_vp],
    "yq_ff_dim": [_vp, _vp],
    "yq_ff_set_params": [_vp, _vp],
    "yq_ff_get_params": [_vp, _vp],
    "yq_ff_init_random": [_vp, _u64],
    "yq_ff_set_batch": [_vp, _i, _vp],
    "yq_ff_random_batch": [_vp, _i, _u64],
    "yq_ff_forward": [_vp, _sz, _vp],
    "yq_ff_adjoint": [_vp, _vp],
    "yq_ff_eloc_tfi": [_vp, _d, _d, _vp],
}

_lib = None


def lib():
    """Load libyannq_b200.so (raises if it was not built)."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise ImportError(f"{LIB_PATH} is missing: build it with `make -C yannq_b200/csrc` "
                              "(or __graft_entry__.build())")
        L = C.CDLL(LIB_PATH)
        for name, args in SIGNATURES.items():
            f = getattr(L, name)
            f.argtypes = args
            f.restype = C.c_char_p if name == "yq_version" else C.c_int
        _lib = L
    return _lib


def last_error():
    buf = C.create_string_buffer(4096)
    lib().yq_last_error(buf, 4096)
    return buf.value.decode()


def check(code):
    if code != OK:
        raise YQError(code, last_error())


def exact(rbm, ham, basis_kind=0, nup=0, with_S=True):
    """SRMatExact::constructExact + eloc/elocVar/oloc/energyGrad/corrMat
    (GroundState/SRMatExact.hpp:97-132) on the device."""
    P = rbm.dim
    st = np.zeros(2)
    ol = np.zeros(P, np.complex128)
    g = np.zeros(P, np.complex128)
    S = np.zeros((P, P), np.complex128) if with_S else None
    check(lib().yq_exact(rbm.h, ham.h, basis_kind, nup, _p(st), _p(ol), _p(g), _p(S) if with_S else None))
    return dict(energy=st[0], energy_var=st[1], oloc=ol, grad=g, S=S)


def exact_iteration(rbm, ham, shift, lr, basis_kind=0, nup=0):
    """One RunRBMExact epoch (Runners/RunRBMExact.hpp:46-80) on the device: returns
    (E, Var, |v|), the energy before the update."""
    out = np.zeros(3)
    check(lib().yq_exact_iteration(rbm.h, ham.h, basis_kind, nup, shift, lr, _p(out)))
    return float(out[0]), float(out[1]), float(out[2])


def alloc_count():
    v = C.c_uint64()
    check(lib().yq_alloc_count(C.byref(v)))
    return v.value


def launch_count():
    v = C.c_uint64()
    check(lib().yq_launch_count(C.byref(v)))
    return v.value


class PinnedArray:
    """numpy view of a page-locked host buffer from yq_host_alloc."""

    def __init__(self, shape, dtype):
        self.dtype = np.dtype(dtype)
        nbytes = int(np.prod(shape)) * self.dtype.itemsize
        ptr = C.c_void_p()
        check(lib().yq_host_alloc(nbytes, C.byref(ptr)))
        self.ptr = ptr
        buf = (C.c_char * nbytes).from_address(ptr.value)
        self.array = np.frombuffer(buf, dtype=self.dtype).reshape(shape)

    def free(self):
        if self.ptr:
            self.array = None
            check(lib().yq_host_free(self.ptr))
            self.ptr = None


def _p(a):
    return None if a is None else a.ctypes.data_as(C.c_void_p)


def _s8(x):
    return np.ascontiguousarray(x, dtype=np.int8)


def _c128(x):
    return np.ascontiguousarray(x, dtype=np.complex128)


class Context:
    def __init__(self, device=0):
        h = C.c_void_p()
        check(lib().yq_ctx_create(device, C.byref(h)))
        self.h = h

    def close(self):
        if self.h:
            check(lib().yq_ctx_destroy(self.h))
            self.h = None

    def synchronize(self):
        check(lib().yq_ctx_synchronize(self.h))

    def stage_ms(self, stage):
        v = C.c_float()
        check(lib().yq_ctx_stage_ms(self.h, STAGES.get(stage, stage), C.byref(v)))
        return v.value

    def measure_peaks(self):
        out = np.zeros(4)
        check(lib().yq_measure_peaks(self.h, _p(out)))
        return {"fp64_simt_tflops": out[0], "fp32_simt_tflops": out[1], "fp64_dmma_tflops": out[2],
                "logcosh_c128_geval_s": out[3]}


class RBM:
    """RBM<complex<float|double>>(n, m, useBias) on the device (Machines/RBM.hpp)."""

    def __init__(self, ctx, n, m, use_bias=True, dtype=C128):
        self.ctx, self.n, self.m, self.use_bias, self.dtype = ctx, n, m, use_bias, dtype
        h = C.c_void_p()
        check(lib().yq_rbm_create(ctx.h, n, m, int(use_bias), dtype, C.byref(h)))
        self.h = h
        d = C.c_size_t()
        check(lib().yq_rbm_dim(h, C.byref(d)))
        self.dim = d.value

    def close(self):
        if self.h:
            check(lib().yq_rbm_destroy(self.h))
            self.h = None

    def set_params(self, p):
        p = _c128(p)
        assert p.shape == (self.dim,)
        check(lib().yq_rbm_set_params(self.h, _p(p)))

    def get_params(self, out=None):
        out = np.zeros(self.dim, np.complex128) if out is None else out
        check(lib().yq_rbm_get_params(self.h, _p(out)))
        return out

    def update_params(self, d):
        check(lib().yq_rbm_update_params(self.h, _p(_c128(d))))

    def archive(self, elem=None):
        """The cereal image of unique_ptr<RBM<T>> (Serializers/SerializeRBM.hpp) as bytes;
        elem defaults to the machine's own type."""
        elem = self.dtype if elem is None else elem
        size = C.c_size_t()
        check(lib().yq_rbm_archive_size(self.h, elem, C.byref(size)))
        buf = (C.c_uint8 * size.value)()
        got = C.c_size_t()
        check(lib().yq_rbm_save_archive(self.h, elem, buf, size.value, C.byref(got)))
        return bytes(buf[:got.value])

    def load_archive(self, data, elem=None):
        elem = self.dtype if elem is None else elem
        buf = (C.c_uint8 * len(data)).from_buffer_copy(data)
        check(lib().yq_rbm_load_archive(self.h, elem, buf, len(data)))

    def save(self, path, elem=None):
        check(lib().yq_rbm_save(self.h, self.dtype if elem is None else elem, os.fsencode(path)))

    def load(self, path, elem=None):
        check(lib().yq_rbm_load(self.h, self.dtype if elem is None else elem, os.fsencode(path)))

    def init_random(self, seed, sd):
        check(lib().yq_rbm_init_random(self.h, seed, sd))

    def theta(self, sigma):
        s = _s8(sigma).reshape(-1, self.n)
        out = np.zeros((s.shape[0], self.m), np.complex128)
        check(lib().yq_rbm_theta(self.h, s.shape[0], _p(s), _p(out)))
        return out

    def log_psi(self, sigma):
        s = _s8(sigma).reshape(-1, self.n)
        out = np.zeros(s.shape[0], np.complex128)
        check(lib().yq_rbm_log_psi(self.h, s.shape[0], _p(s), _p(out)))
        return out

    def log_ratio(self, sigma, theta, flips):
        s = _s8(sigma).reshape(-1, self.n)
        th = _c128(theta).reshape(s.shape[0], self.m)
        f = np.ascontiguousarray(flips, dtype=np.int32).reshape(s.shape[0], -1)
        out = np.zeros(s.shape[0], np.complex128)
        check(lib().yq_rbm_log_ratio(self.h, s.shape[0], _p(s), _p(th), f.shape[1], _p(f), _p(out)))
        return out

    def log_ratio_k(self, sigma, theta, flips):
        """logRatio(vector<int>) (States/RBMState.hpp:107-125): flips is ns x k."""
        s = _s8(sigma).reshape(-1, self.n)
        th = _c128(theta).reshape(s.shape[0], self.m)
        f = np.ascontiguousarray(flips, dtype=np.int32).reshape(s.shape[0], -1)
        out = np.zeros(s.shape[0], np.complex128)
        check(lib().yq_rbm_log_ratio_k(self.h, s.shape[0], _p(s), _p(th), f.shape[1], _p(f), _p(out)))
        return out

    def log_ratio_states(self, sigma, theta, sigma_other, theta_other):
        """logRatio(other state) (States/RBMState.hpp:136-149)."""
        s = _s8(sigma).reshape(-1, self.n)
        th = _c128(theta).reshape(s.shape[0], self.m)
        so = _s8(sigma_other).reshape(s.shape[0], self.n)
        tho = _c128(theta_other).reshape(s.shape[0], self.m)
        out = np.zeros(s.shape[0], np.complex128)
        check(lib().yq_rbm_log_ratio_states(self.h, s.shape[0], _p(s), _p(th), _p(so), _p(tho), _p(out)))
        return out

    def log_deriv(self, sigma, theta):
        s = _s8(sigma).reshape(-1, self.n)
        th = _c128(theta).reshape(s.shape[0], self.m)
        out = np.zeros((s.shape[0], self.dim), np.complex128)
        check(lib().yq_rbm_log_deriv(self.h, s.shape[0], _p(s), _p(th), _p(out)))
        return out


class Hamiltonian:
    def __init__(self, ctx, kind, n, J, h, sign_rule=False, lx=0, ly=0, _handle=None):
        self.ctx, self.kind, self.n = ctx, kind, n
        if _handle is None:
            hh = C.c_void_p()
            check(lib().yq_ham_create(ctx.h, kind, n, lx, ly, J, h, int(sign_rule), C.byref(hh)))
            _handle = hh
        self.h = _handle

    @classmethod
    def tfi(cls, ctx, n, J, h):
        return cls(ctx, HAM_TFI, n, J, h)

    @classmethod
    def xxz(cls, ctx, n, J, delta, sign_rule=False):
        return cls(ctx, HAM_XXZ, n, J, delta, sign_rule)

    @classmethod
    def tfi2d(cls, ctx, lx, ly, J, h):
        return cls(ctx, HAM_TFI2D, lx * ly, J, h, False, lx, ly)

    @classmethod
    def xxx(cls, ctx, n):
        """Hamiltonians/XXX.hpp: XXX(n)."""
        return cls(ctx, HAM_XXX, n, 0.0, 0.0)

    @classmethod
    def j1j2(cls, ctx, n, J1, J2, sign_rule=False):
        """Hamiltonians/J1J2.hpp: J1J2(n, J1, J2, signRule)."""
        return cls(ctx, HAM_J1J2, n, J1, J2, sign_rule)

    @classmethod
    def xyznnn(cls, ctx, n, a, b):
        """Hamiltonians/XYZNNN.hpp: XYZNNN(n, a, b)."""
        return cls(ctx, HAM_XYZNNN, n, a, b)

    @classmethod
    def kitaev_hex(cls, ctx, ncol, nrow, Jx, Jy, Jz, h=0.0):
        """Hamiltonians/KitaevHex.hpp: KitaevHex(ncol, nrow, Jx, Jy, Jz) with field h."""
        hh = C.c_void_p()
        check(lib().yq_ham_create_kitaev_hex(ctx.h, ncol, nrow, Jx, Jy, Jz, h, C.byref(hh)))
        return cls(ctx, HAM_KITAEV_HEX, ncol * nrow, Jx, h, _handle=hh)

    def close(self):
        if self.h:
            check(lib().yq_ham_destroy(self.h))
            self.h = None

    @property
    def num_offdiag(self):
        k = C.c_int()
        check(lib().yq_ham_num_offdiag(self.h, C.byref(k)))
        return k.value

    def enumerate(self, sigma):
        s = _s8(sigma).reshape(-1, self.n)
        ns, K = s.shape[0], self.num_offdiag
        a = np.zeros((ns, K), np.int32)
        b = np.zeros((ns, K), np.int32)
        c = np.zeros((ns, K))
        d = np.zeros(ns)
        check(lib().yq_ham_enumerate(self.h, ns, _p(s), _p(a), _p(b), _p(c), _p(d)))
        return a, b, c, d

    def eloc(self, rbm, sigma, theta):
        s = _s8(sigma).reshape(-1, self.n)
        th = _c128(theta).reshape(s.shape[0], rbm.m)
        out = np.zeros(s.shape[0], np.complex128)
        check(lib().yq_eloc(self.h, rbm.h, s.shape[0], _p(s), _p(th), _p(out)))
        return out


def archive_shape(data):
    """(N, M, useBias) of an RBM archive."""
    n, m, b = C.c_int(), C.c_int(), C.c_int()
    buf = (C.c_uint8 * len(data)).from_buffer_copy(data)
    check(lib().yq_rbm_archive_shape(buf, len(data), C.byref(n), C.byref(m), C.byref(b)))
    return n.value, m.value, bool(b.value)


def file_shape(path):
    n, m, b = C.c_int(), C.c_int(), C.c_int()
    check(lib().yq_rbm_file_shape(os.fsencode(path), C.byref(n), C.byref(m), C.byref(b)))
    return n.value, m.value, bool(b.value)


class Sampler:
    def __init__(self, rbm, n_chains, move=MOVE_LOCAL, nup=-1, sweep_len=0):
        self.rbm, self.n_chains = rbm, n_chains
        h = C.c_void_p()
        check(lib().yq_sampler_create(rbm.h, n_chains, move, nup, sweep_len, C.byref(h)))
        self.h = h

    def close(self):
        if self.h:
            check(lib().yq_sampler_destroy(self.h))
            self.h = None

    def set_hamiltonian(self, ham):
        """HamiltonianSweeper proposals (Samplers/HamiltonianSweeper.hpp) from `ham`,
        which must stay open while the sampler uses it."""
        check(lib().yq_sampler_set_hamiltonian(self.h, ham.h))
        self._ham = ham

    def set_resync(self, every):
        check(lib().yq_sampler_set_resync(self.h, every))

    def set_chains(self, sigma):
        check(lib().yq_sampler_set_chains(self.h, _p(_s8(sigma))))

    def get_chains(self):
        out = np.zeros((self.n_chains, self.rbm.n), np.int8)
        check(lib().yq_sampler_get_chains(self.h, _p(out)))
        return out

    def sample(self, n_sweeps, n_discard, seed, epoch=0, reinit=True):
        check(lib().yq_sample(self.h, n_sweeps, n_discard, seed, epoch, int(reinit)))

    def num_samples(self):
        v = C.c_int()
        check(lib().yq_sampler_num_samples(self.h, C.byref(v)))
        return v.value

    def get_samples(self, theta=True):
        ns = self.num_samples()
        s = np.zeros((ns, self.rbm.n), np.int8)
        th = np.zeros((ns, self.rbm.m), np.complex128) if theta else None
        check(lib().yq_sampler_get_samples(self.h, _p(s), _p(th)))
        return s, th

    def set_tempering(self, ntemps):
        """SamplerMT with nTmps = ntemps (parallel tempering between the chains of each group)."""
        check(lib().yq_sampler_set_tempering(self.h, ntemps))

    def get_slots(self):
        out = np.zeros(self.n_chains, np.int32)
        check(lib().yq_sampler_get_slots(self.h, _p(out)))
        return out

    def warps_per_chain(self):
        v = C.c_int()
        check(lib().yq_sampler_warps_per_chain(self.h, C.byref(v)))
        return v.value

    def chains_per_cta(self):
        v = C.c_int()
        check(lib().yq_sampler_chains_per_cta(self.h, C.byref(v)))
        return v.value

    def get_accepts(self):
        out = np.zeros(self.n_chains, np.uint64)
        check(lib().yq_sampler_get_accepts(self.h, _p(out)))
        return out

    def put_samples(self, sigma, theta):
        s = _s8(sigma)
        th = _c128(theta)
        check(lib().yq_sampler_put_samples(self.h, s.shape[0], _p(s), _p(th)))

    def sample_exact(self, ns, seed, epoch=0, positions=False):
        """ExactSampler::sample (Samplers/ExactSampler.hpp:49-79): ns draws from |psi|^2
        over the full basis (nup < 0) or the fixed-Sz basis; returns the drawn basis
        positions when asked."""
        pos = np.zeros(ns, np.uint64) if positions else None
        check(lib().yq_sampler_sample_exact(self.h, ns, seed, epoch, _p(pos) if positions else None))
        return pos


class SR:
    def __init__(self, rbm, ham, sampler, mode=SR_AUTO, precision=PREC_FP64):
        self.rbm = rbm
        h = C.c_void_p()
        check(lib().yq_sr_create(rbm.h, ham.h, sampler.h, mode, precision, C.byref(h)))
        self.h = h

    def close(self):
        if self.h:
            check(lib().yq_sr_destroy(self.h))
            self.h = None

    def construct(self):
        check(lib().yq_sr_construct(self.h))

    def energy(self):
        e, v = C.c_double(), C.c_double()
        check(lib().yq_sr_energy(self.h, C.byref(e), C.byref(v)))
        return e.value, v.value

    def get(self, which, size):
        out = np.zeros(size, np.complex128)
        check(lib().yq_sr_get(self.h, which, _p(out)))
        return out

    def set_solve_steps(self, steps):
        check(lib().yq_sr_set_solve_steps(self.h, int(steps)))

    def solve(self, shift, solver=SOLVE_LLT, cg_tol=1e-4):
        v = np.zeros(self.rbm.dim, np.complex128)
        it, rr = C.c_int(), C.c_double()
        check(lib().yq_sr_solve(self.h, shift, solver, cg_tol, _p(v), C.byref(it), C.byref(rr)))
        return v, it.value, rr.value

    def matrix(self):
        d = C.c_int()
        check(lib().yq_sr_matrix(self.h, C.byref(d), None))
        out = np.zeros((d.value, d.value), np.complex128)
        check(lib().yq_sr_matrix(self.h, C.byref(d), _p(out)))
        return out

    def set_momentum(self, beta1, beta2=0.0):
        """RunRBM::setMomentum (Runners/RunRBM.hpp:73-77), applied by iteration()."""
        check(lib().yq_sr_set_momentum(self.h, beta1, beta2))

    def set_grad_clip(self, clip):
        """RunRBM::setGradClip (Runners/RunRBM.hpp:79-82), applied by iteration()."""
        check(lib().yq_sr_set_grad_clip(self.h, clip))

    def iteration(self, n_sweeps, n_discard, seed, epoch, shift, lr, reinit=True, solver=SOLVE_LLT, cg_tol=1e-4,
                  ir_steps=0):
        p = IterParams(n_sweeps, n_discard, int(reinit), seed, epoch, shift, lr, solver, cg_tol, ir_steps)
        r = IterResult()
        check(lib().yq_vmc_iteration(self.h, C.byref(p), C.byref(r)))
        return r


class Batch:
    """Independent SR problems advanced together; calls after the first replay one
    captured CUDA graph (yq_batch_* in include/yannq_b200.h)."""

    def __init__(self, ctx, srs):
        self.srs = list(srs)
        arr = (C.c_void_p * len(self.srs))(*[s.h.value if isinstance(s.h, C.c_void_p) else s.h for s in self.srs])
        h = C.c_void_p()
        check(lib().yq_batch_create(ctx.h, len(self.srs), arr, C.byref(h)))
        self.h = h

    def iteration(self, n_sweeps, n_discard, seed, epoch, shift, lr, reinit=True, ir_steps=0):
        p = IterParams(n_sweeps, n_discard, int(reinit), seed, epoch, shift, lr, SOLVE_LLT, 1e-4, ir_steps)
        res = (IterResult * len(self.srs))()
        check(lib().yq_batch_iteration(self.h, C.byref(p), res))
        return list(res)

    def close(self):
        if self.h:
            check(lib().yq_batch_destroy(self.h))
            self.h = None


class FeedForward:
    """Conv1D(1 -> channels, kernel, periodic) -> LnCosh -> FC(L channels -> fc_out) -> LnCosh -> Sum, FP32."""

    def __init__(self, ctx, L, channels, kernel, fc_out):
        self.ctx, self.L = ctx, L
        h = C.c_void_p()
        check(lib().yq_ff_create(ctx.h, L, channels, kernel, fc_out, C.byref(h)))
        self.h = h
        d = C.c_size_t()
        check(lib().yq_ff_dim(h, C.byref(d)))
        self.dim = d.value
        self.batch = 0

    def close(self):
        if self.h:
            check(lib().yq_ff_destroy(self.h))
            self.h = None

    def set_params(self, p):
        check(lib().yq_ff_set_params(self.h, _p(np.ascontiguousarray(p, dtype=np.float64))))

    def get_params(self):
        out = np.zeros(self.dim)
        check(lib().yq_ff_get_params(self.h, _p(out)))
        return out

    def init_random(self, seed):
        check(lib().yq_ff_init_random(self.h, seed))

    def set_batch(self, sigma):
        s = _s8(sigma).reshape(-1, self.L)
        self.batch = s.shape[0]
        check(lib().yq_ff_set_batch(self.h, self.batch, _p(s)))

    def random_batch(self, batch, seed):
        self.batch = batch
        check(lib().yq_ff_random_batch(self.h, batch, seed))

    def forward(self, act_budget_bytes=1 << 62, copy=True):
        out = np.zeros(self.batch) if copy else None
        check(lib().yq_ff_forward(self.h, act_budget_bytes, _p(out)))
        return out

    def adjoint(self, copy=True):
        out = np.zeros((self.batch, self.dim)) if copy else None
        check(lib().yq_ff_adjoint(self.h, _p(out)))
        return out

    def eloc_tfi(self, J, h, copy=True):
        out = np.zeros(self.batch, np.complex128) if copy else None
        check(lib().yq_ff_eloc_tfi(self.h, J, h, _p(out)))
        return out


# ---------------------------------------------------------------------------
def encode_layers(spec):
    """Phase-network layers in the C ABI's encoding from a list such as
    [("conv1d", in_ch, out_ch, kernel[, stride[, bias]]), ("leakyhardtanh", 0.01),
     ("fc", in_dim, out_dim[, bias]), ("softsign",)].  Returns (desc, xs)."""
    desc, xs = [], []
    for layer in spec:
        kind, args = layer[0], list(layer[1:])
        t = LAYER_TYPES[kind]
        if kind == "conv1d":
            a, b, k = args[:3]
            stride = args[3] if len(args) > 3 else 1
            bias = args[4] if len(args) > 4 else False
            desc.append([t, a, b, k, stride, int(bool(bias))])
            xs.append(0.0)
        elif kind == "fc":
            a, b = args[:2]
            bias = args[2] if len(args) > 2 else True
            desc.append([t, a, b, 0, 1, int(bool(bias))])
            xs.append(0.0)
        else:
            default = {"tanh": 1.0, "leakyrelu": 0.1, "leakyhardtanh": 0.01, "cos": 1.0}.get(kind, 0.0)
            desc.append([t, 0, 0, 0, 1, 0])
            xs.append(float(args[0]) if args else default)
    return np.ascontiguousarray(desc, np.int32), np.ascontiguousarray(xs, np.float64)


class AmplitudePhase:
    """Machines/AmplitudePhase.hpp on the device: real RBM amplitude, FeedForward phase."""

    def __init__(self, ctx, n, m, use_bias, layers):
        self.ctx, self.n, self.m, self.use_bias = ctx, n, m, bool(use_bias)
        self.desc, self.xs = encode_layers(layers) if not isinstance(layers, tuple) else layers
        h = C.c_void_p()
        check(lib().yq_ap_create(ctx.h, n, m, int(use_bias), len(self.xs), _p(self.desc), _p(self.xs), C.byref(h)))
        self.h = h
        a, b = C.c_size_t(), C.c_size_t()
        check(lib().yq_ap_dims(h, C.byref(a), C.byref(b)))
        self.dim_amp, self.dim_phase = a.value, b.value
        self.dim = self.dim_amp + self.dim_phase

    def close(self):
        if self.h:
            check(lib().yq_ap_destroy(self.h))
            self.h = None

    def set_params(self, p):
        p = np.ascontiguousarray(p, np.float64)
        assert p.size == self.dim
        check(lib().yq_ap_set_params(self.h, _p(p)))

    def get_params(self):
        p = np.zeros(self.dim)
        check(lib().yq_ap_get_params(self.h, _p(p)))
        return p

    def update_params(self, d):
        d = np.ascontiguousarray(d, np.float64)
        check(lib().yq_ap_update_params(self.h, _p(d)))

    def init_random(self, seed, sigma_amp, mode=INIT_XAVIER):
        check(lib().yq_ap_init_random(self.h, seed, sigma_amp, mode))

    def log_psi(self, sigma):
        s = _s8(sigma).reshape(-1, self.n)
        out = np.zeros(s.shape[0], np.complex128)
        check(lib().yq_ap_log_psi(self.h, s.shape[0], _p(s), _p(out)))
        return out

    def log_deriv(self, sigma):
        s = _s8(sigma).reshape(-1, self.n)
        out = np.zeros((s.shape[0], self.dim), np.complex128)
        check(lib().yq_ap_log_deriv(self.h, s.shape[0], _p(s), _p(out)))
        return out


class NGDExact:
    """GroundState/NGDExact.hpp on the device; iteration() is one epoch of
    RunAmplitudePhaseExact (Runners/RunAmplitudePhase.hpp)."""

    def __init__(self, ap, ham, basis_kind=BASIS_FULL, nup=0):
        self.ap, self.ham = ap, ham
        h = C.c_void_p()
        check(lib().yq_ngd_create(ap.h, ham.h, basis_kind, nup, C.byref(h)))
        self.h = h
        d = C.c_uint64()
        check(lib().yq_ngd_basis_size(h, C.byref(d)))
        self.basis_size = d.value

    def close(self):
        if self.h:
            check(lib().yq_ngd_destroy(self.h))
            self.h = None

    def construct(self):
        e = C.c_double()
        check(lib().yq_ngd_construct(self.h, C.byref(e)))
        return e.value

    def get(self, what):
        a = self.ap
        size = {NGD_GRAD: a.dim, NGD_OLOC_AMP: a.dim_amp, NGD_OLOC_PHASE: a.dim_phase,
                NGD_CORR_AMP: a.dim_amp ** 2, NGD_CORR_PHASE: a.dim_phase ** 2}[what]
        out = np.zeros(size)
        check(lib().yq_ngd_get(self.h, what, _p(out)))
        if what == NGD_CORR_AMP:
            return out.reshape(a.dim_amp, a.dim_amp)
        if what == NGD_CORR_PHASE:
            return out.reshape(a.dim_phase, a.dim_phase)
        return out

    def iteration(self, lam, lr, mode=NGD_ALL):
        e, g, v = C.c_double(), C.c_double(), C.c_double()
        check(lib().yq_ngd_iteration(self.h, lam, lr, mode, C.byref(e), C.byref(g), C.byref(v)))
        return e.value, g.value, v.value
