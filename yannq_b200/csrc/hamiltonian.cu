// Hamiltonians on the device: off-diagonal flip enumeration and the local energy
// E_loc(sigma) = sum_terms coeff * psi(sigma')/psi(sigma) + diagonal
// (Hamiltonians/TFIsing.hpp:28-39, Hamiltonians/XXZ.hpp:37-49, and the 2D TFI
// model built on the same concept), reusing the sample's theta cache.
#include "internal.hpp"
#include "ratio.cuh"

namespace yq {

struct HamDesc {
    int kind, n, lx, ly;
    double J, h, sign;
};

__device__ __forceinline__ int right_of(const HamDesc& H, int i) {
    if (H.kind == YQ_HAM_TFI2D) {
        int x = i % H.lx, y = i / H.lx;
        return (x + 1) % H.lx + H.lx * y;
    }
    return (i + 1) % H.n;
}
__device__ __forceinline__ int down_of(const HamDesc& H, int i) {
    int x = i % H.lx, y = i / H.lx;
    return x + H.lx * ((y + 1) % H.ly);
}

// Contribution of site i to the diagonal, in the reference's evaluation order.
__device__ __forceinline__ double diag_term(const HamDesc& H, const int8_t* s, int i) {
    if (H.kind == YQ_HAM_TFI) return H.J * s[i] * s[(i + 1) % H.n];
    if (H.kind == YQ_HAM_XXZ) {
        int zz = s[i] * s[(i + 1) % H.n];
        return H.J * H.h * zz;
    }
    double d = H.J * s[i] * s[right_of(H, i)];
    return d + H.J * s[i] * s[down_of(H, i)];
}
// The i-th off-diagonal request: flip site a (and b >= 0) with coefficient c.
__device__ __forceinline__ void offdiag_term(const HamDesc& H, const int8_t* s, int i, int& a, int& b, double& c) {
    a = i;
    if (H.kind == YQ_HAM_XXZ) {
        b = (i + 1) % H.n;
        int zz = s[i] * s[b];
        c = H.sign * H.J * (1 - zz);
    } else {
        b = -1;
        c = H.h;
    }
}

__global__ void enumerate_kernel(HamDesc H, int ns, const int8_t* __restrict__ sigma, int* __restrict__ oa,
                                 int* __restrict__ ob, double* __restrict__ oc, double* __restrict__ od) {
    int smp = blockIdx.x * blockDim.x + threadIdx.x;
    if (smp >= ns) return;
    const int8_t* s = sigma + size_t(smp) * H.n;
    double diag = 0.;
    for (int i = 0; i < H.n; ++i) {
        if (H.kind == YQ_HAM_TFI2D) {
            diag += H.J * s[i] * s[right_of(H, i)];
            diag += H.J * s[i] * s[down_of(H, i)];
        } else {
            diag += diag_term(H, s, i);
        }
        int a, b;
        double c;
        offdiag_term(H, s, i, a, b, c);
        oa[size_t(smp) * H.n + i] = a;
        ob[size_t(smp) * H.n + i] = b;
        oc[size_t(smp) * H.n + i] = c;
    }
    od[smp] = diag;
}

static HamDesc desc(const yq_ham_s* H) { return HamDesc{H->kind, H->n, H->lx, H->ly, H->J, H->h, H->sign}; }

void ham_enumerate(yq_ham_s* H, int ns, const int8_t* d_sigma, int* d_a, int* d_b, double* d_c, double* d_diag) {
    if (ns <= 0) return;
    enumerate_kernel<<<cdiv_u(ns, 128), 128, 0, H->ctx->stream>>>(desc(H), ns, d_sigma, d_a, d_b, d_c, d_diag);
    YQ_LAUNCH_CHECK();
}

// ---------------------------------------------------------------------------
template <typename R>
struct ElocArgs {
    HamDesc H;
    int m, ns, nstride;
    const int8_t* sigma;
    const cplx<R>* theta;
    const cplx<R>* tauT;
    const cplx<R>* W;
    const c128* Lk;
    const c128* a;  // visible bias (FP64) or null
    c128* out;
    int* status;
};

template <typename R>
__global__ void __launch_bounds__(256) eloc_kernel(ElocArgs<R> A) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    cplx<R>* t = reinterpret_cast<cplx<R>*>(smem_raw);
    cplx<R>* th = t + A.m;
    int8_t* s = reinterpret_cast<int8_t*>(smem_raw + 2 * sizeof(cplx<R>) * A.m);
    __shared__ c128 red[8];
    const int n = A.H.n, m = A.m;
    const int tid = threadIdx.x, nt = blockDim.x;
    for (int smp = blockIdx.x; smp < A.ns; smp += gridDim.x) {
        for (int i = tid; i < n; i += nt) s[i] = A.sigma[size_t(smp) * n + i];
        for (int j = tid; j < m; j += nt) {
            cplx<R> v = A.theta[size_t(smp) * m + j];
            th[j] = v;
            t[j] = ctanh(v);
        }
        __syncthreads();
        c128 acc = mk(0., 0.);
        for (int i = tid; i < n; i += nt) {
            acc.re += diag_term(A.H, s, i);
            int ka, kb;
            double c;
            offdiag_term(A.H, s, i, ka, kb, c);
            if (c == 0.0) continue;  // zero coefficient: the reference multiplies the ratio by 0
            c128 val;
            if (kb < 0) {
                ScaledProd<R> P = prod1<R>(ka, R(s[ka]), n, m, t, th, 1, A.tauT, A.W);
                val = value_scaled(base1(A.Lk, A.a, ka, double(s[ka])), P);
            } else {
                ScaledProd<R> P = prod2<R>(ka, R(s[ka]), kb, R(s[kb]), n, m, t, th, 1, A.tauT, A.W);
                val = value_scaled(base1(A.Lk, A.a, ka, double(s[ka])) + base1(A.Lk, A.a, kb, double(s[kb])), P);
            }
            acc = acc + c * val;
        }
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) {
            acc.re += __shfl_xor_sync(0xffffffffu, acc.re, o);
            acc.im += __shfl_xor_sync(0xffffffffu, acc.im, o);
        }
        if ((tid & 31) == 0) red[tid >> 5] = acc;
        __syncthreads();
        if (tid == 0) {
            c128 r = red[0];
            for (int w = 1; w < (nt >> 5); ++w) r = r + red[w];
            A.out[smp] = r;
            if (!isfinite(r.re) || !isfinite(r.im)) atomicOr(A.status, DS_NONFINITE);
        }
        __syncthreads();
    }
}

template <typename R>
static void eloc_t(yq_ham_s* H, yq_rbm_s* q, int ns, const int8_t* d_sigma, const void* d_theta, c128* d_out) {
    ElocArgs<R> A;
    A.H = desc(H);
    A.m = q->m;
    A.ns = ns;
    A.nstride = (H->n + 15) & ~15;
    A.sigma = d_sigma;
    A.theta = reinterpret_cast<const cplx<R>*>(d_theta);
    A.tauT = q->tauT.as<cplx<R>>();
    A.W = q->W.as<cplx<R>>();
    A.Lk = q->Lk.as<c128>();
    A.a = q->use_bias ? q->p64.as<c128>() + size_t(q->n) * q->m : nullptr;
    A.out = d_out;
    A.status = H->ctx->status.as<int>();
    int threads = ((H->n + 31) / 32) * 32;
    if (threads > 256) threads = 256;
    if (threads < 64) threads = 64;
    size_t smem = 2 * sizeof(cplx<R>) * q->m + A.nstride;
    if (smem > 48 * 1024)
        YQ_CUDA(cudaFuncSetAttribute(eloc_kernel<R>, cudaFuncAttributeMaxDynamicSharedMemorySize, int(smem)));
    int blocks = ns < 148 * 16 ? ns : 148 * 16;
    eloc_kernel<R><<<blocks, threads, smem, H->ctx->stream>>>(A);
    YQ_LAUNCH_CHECK();
}

void ham_eloc(yq_ham_s* H, yq_rbm_s* q, int ns, const int8_t* d_sigma, const void* d_theta, c128* d_out) {
    YQ_CHECK_ARG(H->n == q->n, "eloc: Hamiltonian and RBM sizes differ");
    if (ns <= 0) return;
    rbm_prepare(q);
    if (q->dtype == YQ_C64)
        eloc_t<float>(H, q, ns, d_sigma, d_theta, d_out);
    else
        eloc_t<double>(H, q, ns, d_sigma, d_theta, d_out);
}

}  // namespace yq
