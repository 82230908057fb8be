// Product-form psi-ratios of the RBM, shared by the sampler, the local-energy
// kernel and the test entry points.
//
// With t_j = tanh(theta_j), x = 2 s_k W_jk and cosh even / sinh odd,
//   cosh(theta_j - x) / cosh(theta_j) = cosh(2 W_jk) (1 - s_k t_j tanh(2 W_jk)),
// so the reference's log-ratio (States/RBMState.hpp:48-63, 2M complex logcosh
// per call) equals
//   -2 a_k s_k + L_k + log prod_j (1 - s_k t_j tau_jk),
//   L_k = sum_j logcosh(2 W_jk),  tau = tanh(2 W)   (both refreshed per parameter update).
// For two flips (States/RBMState.hpp:78-94) tanh's addition formula gives the
// factor 1 + tx ty - t (tx + ty) with tx = s_k tau_jk, ty = s_l tau_jl.
#pragma once
#include "common.cuh"

namespace yq {

template <typename R>
__device__ __forceinline__ cplx<R> one() {
    return mk(R(1), R(0));
}

// log of a scaled product as a complex number: log|p| + e ln 2 + i arg p
template <typename R>
__device__ __forceinline__ c128 log_scaled(const ScaledProd<R>& P) {
    double pr = double(P.p.re), pi = double(P.p.im);
    return mk(0.5 * log(pr * pr + pi * pi) + double(P.e) * 0.69314718055994530942, atan2(pi, pr));
}
// value of exp(base) * p * 2^e
template <typename R>
__device__ __forceinline__ c128 value_scaled(c128 base, const ScaledProd<R>& P) {
    c128 eb = cexp(mk(base.re + double(P.e) * 0.69314718055994530942, base.im));
    return eb * cast<double>(P.p);
}

template <typename R>
__device__ __forceinline__ void renorm_if(ScaledProd<R>& P, int j, int chunk_mask) {
    if ((j & chunk_mask) == chunk_mask) P.renorm();
}

template <typename R>
struct RenormChunk {
    static constexpr int mask = 7;
};
template <>
struct RenormChunk<float> {
    static constexpr int mask = 3;
};

// Cancellation guard.  1 - s t tau loses relative accuracy when |t tau| ~ 1 and
// the difference is small (both tanh near +-1): the relative error grows as
// |t tau| / |d|.  Below |d| < |t tau| / 256 the factor is re-evaluated in the
// reference's well-conditioned logcosh form,
//   d = cosh(theta - x) / (cosh(theta) cosh(x)),   x = 2 s W,
// and for two flips d = cosh(theta - x - y) / (cosh(theta) cosh(x) cosh(y)).
// Threshold on |d|^2 / |t tau|^2: relative error amplification <= 256 in FP64
// (~6e-14), <= 16 in FP32 (~1e-6).
template <typename R>
struct Cancel {
    static constexpr double thr2 = 1.0 / 65536.0;
};
template <>
struct Cancel<float> {
    static constexpr double thr2 = 1.0 / 256.0;
};

template <typename R>
__device__ __noinline__ cplx<R> exact_factor1(cplx<R> th, R sk, cplx<R> w) {
    c128 t = cast<double>(th);
    c128 x = (2.0 * double(sk)) * cast<double>(w);
    c128 l = clogcosh(t - x) - clogcosh(t) - clogcosh(x);
    return cast<R>(cexp(l));
}
template <typename R>
__device__ __noinline__ cplx<R> exact_factor2(cplx<R> th, R sk, cplx<R> wk, R sl, cplx<R> wl) {
    c128 t = cast<double>(th);
    c128 x = (2.0 * double(sk)) * cast<double>(wk);
    c128 y = (2.0 * double(sl)) * cast<double>(wl);
    c128 l = clogcosh(t - x - y) - clogcosh(t) - clogcosh(x) - clogcosh(y);
    return cast<R>(cexp(l));
}

// One-flip factor for hidden unit j.
template <typename R>
__device__ __forceinline__ cplx<R> factor1(cplx<R> tj, cplx<R> tau, R sk, cplx<R> thj, const cplx<R>* wkj,
                                           bool& exact) {
    cplx<R> tt = tj * tau;
    cplx<R> d = mk(R(1) - sk * tt.re, -sk * tt.im);
    exact = norm2(d) < R(Cancel<R>::thr2) * norm2(tt);
    if (exact) d = exact_factor1(thj, sk, *wkj);
    return d;
}
// Two-flip factor for hidden unit j (tx = s_k tau_jk, ty = s_l tau_jl).
template <typename R>
__device__ __forceinline__ cplx<R> factor2(cplx<R> tj, cplx<R> tx, cplx<R> ty, R sk, R sl, cplx<R> thj,
                                           const cplx<R>* wkj, const cplx<R>* wlj, bool& exact) {
    cplx<R> a = tx * ty, b = tj * (tx + ty);
    cplx<R> d = one<R>() + a - b;
    R big = fmax(R(1), fmax(norm2(a), norm2(b)));
    exact = norm2(d) < R(Cancel<R>::thr2) * big;
    if (exact) d = exact_factor2(thj, sk, *wkj, sl, *wlj);
    return d;
}

// prod_j (1 - s_k t_j tau_jk) with tau given transposed (tauT[j * n + k]); t and theta
// with stride ts; W column-major (m x n).  For complex64 the tau loads of four
// consecutive units are issued before their factors are formed (the rare
// re-evaluation in logcosh form is a call the compiler does not move loads across):
// E_loc of the 12 x 12 workload 0.95 -> 0.82 ms.  Complex128 keeps one unit at a time
// (four raised its registers to 112 and its E_loc from 0.99 to 1.13 ms).  The
// product keeps its order either way.
template <typename R>
struct ProdUnroll {
    static constexpr int value = sizeof(R) == 4 ? 4 : 1;
};
template <typename R>
__device__ __forceinline__ ScaledProd<R> prod1(int k, R sk, int n, int m, const cplx<R>* t, const cplx<R>* th,
                                              int ts, const cplx<R>* tauT, const cplx<R>* W) {
    constexpr int PU = ProdUnroll<R>::value;
    ScaledProd<R> P;
    P.init();
    for (int j0 = 0; j0 < m; j0 += PU) {
        cplx<R> tv[PU];
#pragma unroll
        for (int u = 0; u < PU; ++u) tv[u] = j0 + u < m ? tauT[size_t(j0 + u) * n + k] : one<R>();
#pragma unroll
        for (int u = 0; u < PU; ++u) {
            const int j = j0 + u;
            if (j < m) {
                bool ex;
                cplx<R> d = factor1<R>(t[size_t(j) * ts], tv[u], sk, th[size_t(j) * ts], W + size_t(k) * m + j, ex);
                P.p = P.p * d;
                renorm_if(P, j, RenormChunk<R>::mask);
            }
        }
    }
    P.renorm();
    return P;
}

template <typename R>
__device__ __forceinline__ ScaledProd<R> prod2(int k, R sk, int l, R sl, int n, int m, const cplx<R>* t,
                                              const cplx<R>* th, int ts, const cplx<R>* tauT, const cplx<R>* W) {
    constexpr int PU = ProdUnroll<R>::value;
    ScaledProd<R> P;
    P.init();
    for (int j0 = 0; j0 < m; j0 += PU) {
        cplx<R> tk[PU], tl[PU];
#pragma unroll
        for (int u = 0; u < PU; ++u) {
            tk[u] = j0 + u < m ? tauT[size_t(j0 + u) * n + k] : one<R>();
            tl[u] = j0 + u < m ? tauT[size_t(j0 + u) * n + l] : one<R>();
        }
#pragma unroll
        for (int u = 0; u < PU; ++u) {
            const int j = j0 + u;
            if (j < m) {
                const cplx<R> tx = sk * tk[u], ty = sl * tl[u];
                bool ex;
                cplx<R> d = factor2<R>(t[size_t(j) * ts], tx, ty, sk, sl, th[size_t(j) * ts], W + size_t(k) * m + j,
                                       W + size_t(l) * m + j, ex);
                P.p = P.p * d;
                renorm_if(P, j, RenormChunk<R>::mask);
            }
        }
    }
    P.renorm();
    return P;
}

// exponent base of a one-flip ratio: L_k - 2 a_k s_k (FP64)
__device__ __forceinline__ c128 base1(const c128* Lk, const c128* a, int k, double sk) {
    c128 r = Lk[k];
    if (a) r = r - (2.0 * sk) * a[k];
    return r;
}

}  // namespace yq
