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

// prod_j (1 - s_k t_j tau_jk) with tau given transposed (tauT[j * n + k]), t with stride ts.
template <typename R>
__device__ __forceinline__ ScaledProd<R> prod1(int k, R sk, int n, int m, const cplx<R>* t, int ts,
                                              const cplx<R>* tauT) {
    ScaledProd<R> P;
    P.init();
    for (int j = 0; j < m; ++j) {
        cplx<R> tt = t[size_t(j) * ts] * tauT[size_t(j) * n + k];
        cplx<R> d = mk(R(1) - sk * tt.re, -sk * tt.im);
        P.p = P.p * d;
        renorm_if(P, j, RenormChunk<R>::mask);
    }
    P.renorm();
    return P;
}

template <typename R>
__device__ __forceinline__ ScaledProd<R> prod2(int k, R sk, int l, R sl, int n, int m, const cplx<R>* t, int ts,
                                              const cplx<R>* tauT) {
    ScaledProd<R> P;
    P.init();
    for (int j = 0; j < m; ++j) {
        cplx<R> tx = sk * tauT[size_t(j) * n + k];
        cplx<R> ty = sl * tauT[size_t(j) * n + l];
        cplx<R> tj = t[size_t(j) * ts];
        cplx<R> d = one<R>() + tx * ty - tj * (tx + ty);
        P.p = P.p * d;
        renorm_if(P, j, RenormChunk<R>::mask);
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
