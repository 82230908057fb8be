// RBM machine on the device: derived arrays for product-form ratios, theta,
// log psi, log ratios and log derivatives over batches (Machines/RBM.hpp,
// States/RBMState.hpp).
#include "internal.hpp"
#include "ratio.cuh"

namespace yq {

// ---------------------------------------------------------------------------
// Per-parameter-update preparation: W in the compute type, tau = tanh(2W) in both
// column-major (sampler: column k contiguous) and transposed (local energy: site k
// contiguous for fixed j) layouts, and L_k = sum_j logcosh(2 W_jk) in FP64.
template <typename R>
__global__ void prep_columns_kernel(const c128* __restrict__ p64, int n, int m, cplx<R>* __restrict__ W,
                                    cplx<R>* __restrict__ tau, cplx<R>* __restrict__ tauT, c128* __restrict__ Lk) {
    const int warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int lane = threadIdx.x & 31;
    if (warp >= n) return;
    const int k = warp;
    c128 acc = mk(0.0, 0.0);
    for (int j = lane; j < m; j += 32) {
        c128 w = p64[size_t(k) * m + j];
        c128 w2 = mk(2.0 * w.re, 2.0 * w.im);
        c128 tz = ctanh(w2);
        W[size_t(k) * m + j] = cast<R>(w);
        tau[size_t(k) * m + j] = cast<R>(tz);
        tauT[size_t(j) * n + k] = cast<R>(tz);
        acc = acc + clogcosh(w2);
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        acc.re += __shfl_xor_sync(0xffffffffu, acc.re, o);
        acc.im += __shfl_xor_sync(0xffffffffu, acc.im, o);
    }
    if (lane == 0) Lk[k] = acc;
}

template <typename R>
__global__ void prep_bias_kernel(const c128* __restrict__ p64, int n, int m, bool bias, cplx<R>* a, cplx<R>* b) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    size_t nm = size_t(n) * m;
    if (i < n) a[i] = bias ? cast<R>(p64[nm + i]) : mk(R(0), R(0));
    if (i < m) b[i] = bias ? cast<R>(p64[nm + n + i]) : mk(R(0), R(0));
}

template <typename R>
static void prepare_t(yq_rbm_s* q) {
    const int threads = 256;
    cudaStream_t st = q->ctx->stream;
    prep_columns_kernel<R><<<cdiv_u(size_t(q->n) * 32, threads), threads, 0, st>>>(
        q->p64.as<c128>(), q->n, q->m, q->W.as<cplx<R>>(), q->tau.as<cplx<R>>(), q->tauT.as<cplx<R>>(),
        q->Lk.as<c128>());
    YQ_LAUNCH_CHECK();
    int mx = q->n > q->m ? q->n : q->m;
    prep_bias_kernel<R><<<cdiv_u(mx, threads), threads, 0, st>>>(q->p64.as<c128>(), q->n, q->m, q->use_bias,
                                                                  q->a.as<cplx<R>>(), q->b.as<cplx<R>>());
    YQ_LAUNCH_CHECK();
}

void rbm_prepare(yq_rbm_s* q) {
    if (q->prepared == q->version) return;
    if (q->dtype == YQ_C64)
        prepare_t<float>(q);
    else
        prepare_t<double>(q);
    q->prepared = q->version;
}

// ---------------------------------------------------------------------------
// theta = W sigma + b in FP64 (RBM.hpp:137-141), i ascending then + b, matching
// the oracle's summation order bit for bit.
template <typename OutT>
__global__ void theta_kernel(const c128* __restrict__ p64, int n, int m, bool bias, const int8_t* __restrict__ sigma,
                             OutT* __restrict__ theta) {
    extern __shared__ int8_t s_sig[];
    const int s = blockIdx.y;
    for (int i = threadIdx.x; i < n; i += blockDim.x) s_sig[i] = sigma[size_t(s) * n + i];
    __syncthreads();
    const int j = blockIdx.x * blockDim.x + threadIdx.x;
    if (j >= m) return;
    double ar = 0., ai = 0.;
    for (int i = 0; i < n; ++i) {
        c128 w = p64[size_t(i) * m + j];
        double sv = double(s_sig[i]);
        ar += w.re * sv;
        ai += w.im * sv;
    }
    if (bias) {
        c128 bb = p64[size_t(n) * m + n + j];
        ar += bb.re;
        ai += bb.im;
    }
    OutT o;
    o.re = ar;
    o.im = ai;
    theta[size_t(s) * m + j] = o;
}

void rbm_theta(yq_rbm_s* q, int ns, const int8_t* d_sigma, void* d_theta, bool out_c128) {
    if (ns <= 0) return;
    dim3 grid(cdiv_u(q->m, 128), ns);
    if (out_c128 || q->dtype == YQ_C128)
        theta_kernel<c128><<<grid, 128, q->n, q->ctx->stream>>>(q->p64.as<c128>(), q->n, q->m, q->use_bias, d_sigma,
                                                                reinterpret_cast<c128*>(d_theta));
    else
        theta_kernel<c64><<<grid, 128, q->n, q->ctx->stream>>>(q->p64.as<c128>(), q->n, q->m, q->use_bias, d_sigma,
                                                               reinterpret_cast<c64*>(d_theta));
    YQ_LAUNCH_CHECK();
}

// log psi = a.sigma + sum_j logcosh(theta_j) (RBM.hpp:367-378), FP64, thread per sample.
__global__ void log_psi_kernel(const c128* __restrict__ p64, int n, int m, bool bias, int ns,
                               const int8_t* __restrict__ sigma, c128* __restrict__ out) {
    int s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= ns) return;
    const int8_t* sg = sigma + size_t(s) * n;
    c128 r = mk(0., 0.);
    size_t nm = size_t(n) * m;
    if (bias)
        for (int i = 0; i < n; ++i) r = r + double(sg[i]) * p64[nm + i];
    for (int j = 0; j < m; ++j) {
        double ar = 0., ai = 0.;
        for (int i = 0; i < n; ++i) {
            c128 w = p64[size_t(i) * m + j];
            ar += w.re * sg[i];
            ai += w.im * sg[i];
        }
        c128 th = mk(ar, ai);
        if (bias) th = th + p64[nm + n + j];
        r = r + clogcosh(th);
    }
    out[s] = r;
}

void rbm_log_psi(yq_rbm_s* q, int ns, const int8_t* d_sigma, c128* d_out) {
    if (ns <= 0) return;
    log_psi_kernel<<<cdiv_u(ns, 128), 128, 0, q->ctx->stream>>>(q->p64.as<c128>(), q->n, q->m, q->use_bias, ns,
                                                                 d_sigma, d_out);
    YQ_LAUNCH_CHECK();
}

// ---------------------------------------------------------------------------
// Test entry: product-form log ratio of one or two flips, thread per sample,
// with the same device routines the local-energy kernel runs.
template <typename R>
__global__ void log_ratio_kernel(int n, int m, int ns, const int8_t* __restrict__ sigma, const c128* __restrict__ theta,
                                 int nflip, const int* __restrict__ flips, const cplx<R>* __restrict__ tauT,
                                 const c128* __restrict__ Lk, const c128* __restrict__ a, const cplx<R>* __restrict__ W,
                                 cplx<R>* __restrict__ tws, c128* __restrict__ out) {
    int s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= ns) return;
    cplx<R>* t = tws + size_t(s) * 2 * m;
    cplx<R>* th = t + m;
    for (int j = 0; j < m; ++j) {
        t[j] = cast<R>(ctanh(theta[size_t(s) * m + j]));
        th[j] = cast<R>(theta[size_t(s) * m + j]);
    }
    const int8_t* sg = sigma + size_t(s) * n;
    int k = flips[size_t(s) * nflip];
    R sk = R(sg[k]);
    if (nflip == 1) {
        ScaledProd<R> P = prod1<R>(k, sk, n, m, t, th, 1, tauT, W);
        out[s] = base1(Lk, a, k, double(sk)) + log_scaled(P);
    } else {
        int l = flips[size_t(s) * nflip + 1];
        R sl = R(sg[l]);
        ScaledProd<R> P = prod2<R>(k, sk, l, sl, n, m, t, th, 1, tauT, W);
        out[s] = base1(Lk, a, k, double(sk)) + base1(Lk, a, l, double(sl)) + log_scaled(P);
    }
}

void rbm_log_ratio(yq_rbm_s* q, int ns, const int8_t* d_sigma, const void* d_theta, int nflip, const int* d_flips,
                   c128* d_out) {
    if (ns <= 0) return;
    rbm_prepare(q);
    DevBuf tws;
    tws.ensure(size_t(ns) * 2 * q->m * q->csize());
    const c128* a = q->use_bias ? q->p64.as<c128>() + size_t(q->n) * q->m : nullptr;
    if (q->dtype == YQ_C64)
        log_ratio_kernel<float><<<cdiv_u(ns, 64), 64, 0, q->ctx->stream>>>(
            q->n, q->m, ns, d_sigma, reinterpret_cast<const c128*>(d_theta), nflip, d_flips, q->tauT.as<c64>(),
            q->Lk.as<c128>(), a, q->W.as<c64>(), tws.as<c64>(), d_out);
    else
        log_ratio_kernel<double><<<cdiv_u(ns, 64), 64, 0, q->ctx->stream>>>(
            q->n, q->m, ns, d_sigma, reinterpret_cast<const c128*>(d_theta), nflip, d_flips, q->tauT.as<c128>(),
            q->Lk.as<c128>(), a, q->W.as<c128>(), tws.as<c128>(), d_out);
    YQ_LAUNCH_CHECK();
    YQ_CUDA(cudaStreamSynchronize(q->ctx->stream));
}

// logRatio(vector) -- States/RBMState.hpp:107-125, k distinct flips per sample, in
// the reference's form: -2 sum_e a_e s_e + sum_j [logCosh(theta_j - 2 sum_e s_e W_je)
// - logCosh(theta_j)], evaluated in FP64 from the machine's weights (W in the
// compute type, m x n column-major; a the FP64 master values).
template <typename R>
__global__ void log_ratio_k_kernel(int n, int m, int ns, int k, const int8_t* __restrict__ sigma,
                                   const c128* __restrict__ theta, const int* __restrict__ flips,
                                   const cplx<R>* __restrict__ W, const c128* __restrict__ a, c128* __restrict__ out) {
    const int s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= ns) return;
    const int8_t* sg = sigma + size_t(s) * n;
    const int* f = flips + size_t(s) * k;
    c128 res = mk(0., 0.);
    if (a)
        for (int e = 0; e < k; ++e) res = res - (2.0 * double(sg[f[e]])) * a[f[e]];
    for (int j = 0; j < m; ++j) {
        const c128 th = theta[size_t(s) * m + j];
        c128 t = th;
        for (int e = 0; e < k; ++e) t = t - (2.0 * double(sg[f[e]])) * cast<double>(W[size_t(f[e]) * m + j]);
        res = res + (clogcosh(t) - clogcosh(th));
    }
    out[s] = res;
}

// logRatio(other) -- States/RBMState.hpp:136-149: a^T (s' - s) + sum_j [logCosh(theta'_j)
// - logCosh(theta_j)] between two states of the same machine.
__global__ void log_ratio_states_kernel(int n, int m, int ns, const int8_t* __restrict__ sa,
                                        const c128* __restrict__ tha, const int8_t* __restrict__ sb,
                                        const c128* __restrict__ thb, const c128* __restrict__ a,
                                        c128* __restrict__ out) {
    const int s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= ns) return;
    c128 res = mk(0., 0.);
    if (a)
        for (int i = 0; i < n; ++i) res = res + double(sb[size_t(s) * n + i] - sa[size_t(s) * n + i]) * a[i];
    for (int j = 0; j < m; ++j) res = res + (clogcosh(thb[size_t(s) * m + j]) - clogcosh(tha[size_t(s) * m + j]));
    out[s] = res;
}

void rbm_log_ratio_k(yq_rbm_s* q, int ns, const int8_t* d_sigma, const c128* d_theta, int k, const int* d_flips,
                     c128* d_out) {
    if (ns <= 0) return;
    rbm_prepare(q);
    const c128* a = q->use_bias ? q->p64.as<c128>() + size_t(q->n) * q->m : nullptr;
    if (q->dtype == YQ_C64)
        log_ratio_k_kernel<float><<<cdiv_u(ns, 64), 64, 0, q->ctx->stream>>>(q->n, q->m, ns, k, d_sigma, d_theta,
                                                                            d_flips, q->W.as<c64>(), a, d_out);
    else
        log_ratio_k_kernel<double><<<cdiv_u(ns, 64), 64, 0, q->ctx->stream>>>(q->n, q->m, ns, k, d_sigma, d_theta,
                                                                             d_flips, q->W.as<c128>(), a, d_out);
    YQ_LAUNCH_CHECK();
}

void rbm_log_ratio_states(yq_rbm_s* q, int ns, const int8_t* d_sa, const c128* d_tha, const int8_t* d_sb,
                          const c128* d_thb, c128* d_out) {
    if (ns <= 0) return;
    const c128* a = q->use_bias ? q->p64.as<c128>() + size_t(q->n) * q->m : nullptr;
    log_ratio_states_kernel<<<cdiv_u(ns, 64), 64, 0, q->ctx->stream>>>(q->n, q->m, ns, d_sa, d_tha, d_sb, d_thb, a,
                                                                      d_out);
    YQ_LAUNCH_CHECK();
}

// O row = [s_i tanh(theta_j) | s | tanh(theta)] (RBM.hpp:390-406), c128 output.
__global__ void log_deriv_kernel(int n, int m, bool bias, int ns, const int8_t* __restrict__ sigma,
                                 const c128* __restrict__ theta, c128* __restrict__ out) {
    const int s = blockIdx.y;
    const size_t P = bias ? size_t(n) * m + n + m : size_t(n) * m;
    const size_t nm = size_t(n) * m;
    for (size_t p = size_t(blockIdx.x) * blockDim.x + threadIdx.x; p < P; p += size_t(gridDim.x) * blockDim.x) {
        c128 v;
        if (p < nm) {
            int i = int(p / m), j = int(p % m);
            v = double(sigma[size_t(s) * n + i]) * ctanh(theta[size_t(s) * m + j]);
        } else if (p < nm + n) {
            v = mk(double(sigma[size_t(s) * n + (p - nm)]), 0.0);
        } else {
            v = ctanh(theta[size_t(s) * m + (p - nm - n)]);
        }
        out[size_t(s) * P + p] = v;
    }
}

void rbm_log_deriv(yq_rbm_s* q, int ns, const int8_t* d_sigma, const void* d_theta, c128* d_out) {
    if (ns <= 0) return;
    dim3 grid(64, ns);
    log_deriv_kernel<<<grid, 256, 0, q->ctx->stream>>>(q->n, q->m, q->use_bias, ns, d_sigma,
                                                       reinterpret_cast<const c128*>(d_theta), d_out);
    YQ_LAUNCH_CHECK();
}

// ---------------------------------------------------------------------------
// Machines/RBM.hpp:325-349 draw order with Philox + Box-Muller normals
// (identical to the oracle's init_params).
static double normal_pair(uint64_t seed, uint32_t idx, double* second) {
    U4 x = draw(seed, idx, 0u, 0u, TAG_PARAM);
    const double u1 = 1.0 - draw_u53(x.x, x.y);
    const double u2 = draw_u53(x.z, x.w);
    const double r = std::sqrt(-2.0 * std::log(u1));
    const double ang = 6.283185307179586476925286766559 * u2;
    *second = r * std::sin(ang);
    return r * std::cos(ang);
}

void rbm_init_params_host(int n, int m, bool bias, uint64_t seed, double sd, c128* p) {
    uint32_t e = 0;
    auto drawc = [&](c128& out) {
        double im;
        double re = normal_pair(seed, e++, &im);
        out = mk(sd * re, sd * im);
    };
    const size_t nm = size_t(n) * m;
    if (bias) {
        for (int i = 0; i < n; ++i) drawc(p[nm + i]);
        for (int j = 0; j < m; ++j) drawc(p[nm + n + j]);
    }
    for (int i = 0; i < n; ++i)
        for (int j = 0; j < m; ++j) drawc(p[size_t(i) * m + j]);
}

}  // namespace yq
