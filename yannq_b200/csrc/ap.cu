// AmplitudePhase machine and exact natural-gradient descent on the device.
//
//   AmplitudePhase  Machines/AmplitudePhase.hpp:9-178: psi(s) = sqrt(A(s)) exp(i pi phi(s))
//                   with A(s) = exp(a.s + sum_j logCosh(theta_j)) from a real
//                   RBM<double> (Machines/RBM.hpp:367-406) and phi(s) the output of
//                   a FeedForward<double> (Machines/FeedForward.hpp:132-205) built
//                   from Conv1D (layers/Conv1D.hpp:144-225), FullyConnected
//                   (layers/FullyConnected.hpp) and the activation layers
//                   (layers/ActivationLayer.hpp, layers/activations.hpp).
//   NGDExact        GroundState/NGDExact.hpp:123-189 over a basis:
//                     p = |psi|^2 (normalised), k = H psi, E = Re <psi|k>,
//                     o_amp = sum p D_amp, o_phase = sum p D_phase,
//                     grad_amp = 2 D_amp^T Re(conj(psi) k) - 2 E o_amp,
//                     grad_phase = 2 D_phase^T Im(conj(psi) k),
//                     C_x = D_x^T diag(p) D_x - o_x o_x^T,
//                   with D_amp = RBM logDeriv / 2 and D_phase = pi * backward.
//   iteration       Runners/RunAmplitudePhase.hpp:92-119: both blocks solved by
//                   LLT of C_x + lambda I, then the SGD update -lr v.
//
// Layout: the derivative rows of two consecutive configurations share one
// complex element (real part: configuration 2k, imaginary part: 2k + 1), so the
// FP64 complex DMMA Hermitian product of the centred, sqrt(p)-scaled rows yields
// the real correlation matrix as its real part at half the cost of an embedding
// with zero imaginary parts.  Blocks of the derivative kernels take such a pair,
// so every store is a full 16-byte element.
#include <algorithm>
#include <cmath>
#include <cstring>
#include <memory>
#include <string>
#include <vector>

#include "ap.hpp"
#include "basis.cuh"
#include "chol.hpp"
#include "gemm64.cuh"
#include "internal.hpp"

namespace yq {

void record_error(const std::string& msg);

// Layer types (the numbering of the C ABI).
enum : int {
    L_CONV1D = 0, L_FC = 1,
    A_IDENTITY = 10, A_LNCOSH = 11, A_TANH = 12, A_WEAKTANH = 13, A_SIGMOID = 14, A_RELU = 15, A_LEAKYRELU = 16,
    A_HARDTANH = 17, A_SOFTSHRINK = 18, A_LEAKYHARDTANH = 19, A_SOFTSIGN = 20, A_COS = 21
};

struct LayerDev {
    int type, a, b, k, stride, bias;
    double x;
    int in_size, out_size, in_len, out_len;
    long long off;  // parameter offset within the phase block
    int in_act, out_act;  // offsets of the layer's input and output in the activation buffer
};

constexpr int AP_THREADS = 128;
constexpr int MAX_LAYERS = 64;

}  // namespace yq

struct yq_ap_s {
    yq_ctx_s* ctx = nullptr;
    int n = 0, m = 0;
    bool bias = true;
    size_t Pa = 0, Pp = 0;
    std::vector<yq::LayerDev> layers;
    int act_total = 0, max_width = 0;
    yq::DevBuf p64;      // Pa + Pp doubles
    yq::DevBuf dlayers;  // layers on the device
};

struct yq_ngd_s {
    yq_ap_s* q = nullptr;
    yq_ham_s* H = nullptr;
    int kind = 0, nup = 0;
    uint64_t dim = 0, dim2 = 0;
    yq::DevBuf binom, index, sigma;
    yq::DevBuf logA, phi, p, psi, kv, ya, yb;  // per configuration
    yq::DevBuf Da, Dp;                           // packed derivative rows
    yq::DevBuf part, scal;                       // reductions
    yq::DevBuf grad, oloc;                       // Pa + Pp doubles each
    yq::DevBuf Ca, Cp;                           // c128 dim_pad x dim_pad (lower, real part used)
    yq::DevBuf La, LaH, Lp, LpH, Ga, Gp, rhs, chol_work, cpart, va, vp;
    int pad_a = 0, pad_p = 0;
    double energy = 0.;
    bool constructed = false;
    // K-split of the two Gram matrices: side streams, fork / join events, partials
    static constexpr int NSIDE = 8;
    cudaStream_t side[NSIDE] = {};
    cudaEvent_t fork = nullptr, join[NSIDE] = {};
    int split_a = 1, split_p = 1;
    yq::DevBuf Cpart;
    ~yq_ngd_s() {
        for (int i = 0; i < NSIDE; ++i) {
            if (join[i]) cudaEventDestroy(join[i]);
            if (side[i]) cudaStreamDestroy(side[i]);
        }
        if (fork) cudaEventDestroy(fork);
    }
};

namespace yq {
namespace {

// ---------------------------------------------------------------------------
// Amplitude: theta, log A and D_amp for the configuration pair (2 pr, 2 pr + 1).
struct AmpArgs {
    int n, m;
    bool bias;
    uint64_t count;  // configurations
    const int8_t* sigma;
    const double* p;  // amplitude parameters [W col-major m x n | a | b]
    double* logA;     // count, or null
    c128* D;          // packed rows, Pa per pair
    size_t Pa;
};

__global__ void __launch_bounds__(AP_THREADS) amp_kernel(AmpArgs A) {
    extern __shared__ double sm_amp[];
    double* t = sm_amp;  // 2 x m tanh(theta)
    __shared__ double red[2][AP_THREADS / 32];
    const int tid = threadIdx.x, n = A.n, m = A.m;
    const size_t nm = size_t(n) * m;
    const uint64_t npairs = (A.count + 1) / 2;
    for (uint64_t pr = blockIdx.x; pr < npairs; pr += gridDim.x) {
        double lsum[2] = {0., 0.};
        for (int h = 0; h < 2; ++h) {
            const uint64_t k = 2 * pr + h;
            if (k >= A.count) {
                for (int j = tid; j < m; j += blockDim.x) t[h * m + j] = 0.;
                continue;
            }
            const int8_t* s = A.sigma + k * n;
            for (int j = tid; j < m; j += blockDim.x) {
                double th = A.bias ? A.p[nm + n + j] : 0.0;
                for (int i = 0; i < n; ++i) th += A.p[size_t(j) + size_t(i) * m] * double(s[i]);
                t[h * m + j] = tanh(th);
                lsum[h] += logcosh_real(th);
            }
            if (A.bias)
                for (int i = tid; i < n; i += blockDim.x) lsum[h] += A.p[nm + i] * double(s[i]);
        }
        if (A.logA) {
#pragma unroll
            for (int h = 0; h < 2; ++h) {
                double v = lsum[h];
#pragma unroll
                for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
                if ((tid & 31) == 0) red[h][tid >> 5] = v;
            }
        }
        __syncthreads();
        if (A.logA && tid < 2) {
            const uint64_t k = 2 * pr + tid;
            if (k < A.count) {
                double v = 0.;
                for (int w = 0; w < int(blockDim.x >> 5); ++w) v += red[tid][w];
                A.logA[k] = v;
            }
        }
        // D_amp = RBM logDeriv / 2: [s_i tanh(theta_j) | s_i | tanh(theta_j)]
        const int8_t* s0 = A.sigma + (2 * pr) * n;
        const bool has1 = 2 * pr + 1 < A.count;
        const int8_t* s1 = has1 ? s0 + n : s0;
        c128* row = A.D + pr * A.Pa;
        for (size_t e = tid; e < nm; e += blockDim.x) {
            const int i = int(e / m), j = int(e % m);
            row[e] = mk(0.5 * double(s0[i]) * t[j], has1 ? 0.5 * double(s1[i]) * t[m + j] : 0.0);
        }
        if (A.bias) {
            for (int i = tid; i < n; i += blockDim.x) row[nm + i] = mk(0.5 * double(s0[i]), has1 ? 0.5 * double(s1[i]) : 0.0);
            for (int j = tid; j < m; j += blockDim.x) row[nm + n + j] = mk(0.5 * t[j], has1 ? 0.5 * t[m + j] : 0.0);
        }
        __syncthreads();
    }
}

// ---------------------------------------------------------------------------
// Phase network: forward (FeedForward::makeData) and backward with dout = 1
// (FeedForward.hpp:186-205) for a configuration pair; writes phi and pi * der.
struct PhaseArgs {
    int n, nlayers, act_total, max_width;
    uint64_t count;
    const int8_t* sigma;
    const LayerDev* layers;
    const double* p;  // phase parameters
    double* phi;      // count, or null
    c128* D;          // packed rows, Pp per pair
    size_t Pp;
};

__device__ __forceinline__ double act_fwd(int type, double x, double z) {
    switch (type) {
        case A_IDENTITY: return z;
        case A_LNCOSH: return logcosh_real(z);
        case A_TANH: return x * tanh(z / x);
        case A_WEAKTANH: return z - tanh(z) / 2.0;
        case A_SIGMOID: return exp(z) + 1.;  // activations.hpp:215-220 as written
        case A_RELU: return fmax(z, 0.0);
        case A_LEAKYRELU: return z > 0 ? z : x * z;
        case A_HARDTANH: return fabs(z) > 1.0 ? copysign(1.0, z) : z;
        case A_SOFTSHRINK: return fabs(z) < 1.0 ? 0.0 : (z - copysign(1.0, z));
        case A_LEAKYHARDTANH: {
            double v = fabs(z) > 1.0 ? copysign(1.0, z) : z;
            v += fabs(z) < 1.0 ? 0.0 : x * (z - copysign(1.0, z));
            return v;
        }
        case A_SOFTSIGN: return z / (fabs(z) + 1.0);
        default: return x * cos(z * M_PI / x);  // A_COS
    }
}
__device__ __forceinline__ double act_jac(int type, double x, double z, double a, double f) {
    switch (type) {
        case A_IDENTITY: return f;
        case A_LNCOSH: return f * tanh(z);
        case A_TANH: return f * (1. - a * a / (x * x));
        case A_WEAKTANH: {
            const double t = tanh(z);
            return f * (1.0 + t * t) / 2.0;
        }
        case A_SIGMOID: return (1. - a) * a;  // activations.hpp:226-229 as written (F unused)
        case A_RELU: return z > 0 ? f : 0.0;
        case A_LEAKYRELU: return z > 0 ? f : x * f;
        case A_HARDTANH: return fabs(z) > 1.0 ? 0.0 : f;
        case A_SOFTSHRINK: return fabs(z) < 1.0 ? 0.0 : f;
        case A_LEAKYHARDTANH: return fabs(z) > 1.0 ? x * f : f;
        case A_SOFTSIGN: {
            const double d = 1.0 + fabs(z);
            return (1.0 / (d * d)) * f;
        }
        default: return -M_PI * sin(M_PI * z / x) * f;  // A_COS
    }
}

// input index of Conv1D output position r for kernel tap ki (Conv1D.hpp:159-160)
__device__ __forceinline__ int conv_src(const LayerDev& L, int r, int ki) {
    return (r * L.stride + ki - L.k / 2 + L.in_len) % L.in_len;
}

__global__ void __launch_bounds__(AP_THREADS) phase_kernel(PhaseArgs A) {
    extern __shared__ double sm_ph[];
    // per half h: activations [act_total], dout [max_width], din [max_width]
    const int stride_h = A.act_total + 2 * A.max_width;
    const int tid = threadIdx.x, nt = blockDim.x;
    const uint64_t npairs = (A.count + 1) / 2;
    for (uint64_t pr = blockIdx.x; pr < npairs; pr += gridDim.x) {
        const bool has1 = 2 * pr + 1 < A.count;
        for (int e = tid; e < 2 * A.n; e += nt) {
            const int h = e / A.n, i = e % A.n;
            const uint64_t k = has1 ? 2 * pr + h : 2 * pr;
            sm_ph[h * stride_h + i] = double(A.sigma[k * A.n + i]);
        }
        __syncthreads();
        // ---- forward
        for (int l = 0; l < A.nlayers; ++l) {
            const LayerDev L = A.layers[l];
            const double* w = A.p + L.off;
            for (int e = tid; e < 2 * L.out_size; e += nt) {
                const int h = e / L.out_size, o = e % L.out_size;
                const double* in = sm_ph + h * stride_h + L.in_act;
                double v;
                if (L.type == L_CONV1D) {
                    const int oc = o / L.out_len, r = o % L.out_len;
                    v = 0.;
                    for (int ic = 0; ic < L.a; ++ic)
                        for (int ki = 0; ki < L.k; ++ki)
                            v += w[size_t(ki + ic * L.k) + size_t(oc) * L.a * L.k] * in[conv_src(L, r, ki) + ic * L.in_len];
                    if (L.bias) v += w[size_t(L.a) * L.b * L.k + oc];
                } else if (L.type == L_FC) {
                    double t = 0.;
                    for (int i = 0; i < L.a; ++i) t += w[size_t(i) + size_t(o) * L.a] * in[i];
                    v = (L.bias ? w[size_t(L.a) * L.b + o] : 0.0) + t;
                } else {
                    v = act_fwd(L.type, L.x, in[o]);
                }
                sm_ph[h * stride_h + L.out_act + o] = v;
            }
            __syncthreads();
        }
        if (A.phi && tid < 2 && (tid == 0 || has1)) {
            const LayerDev& last = A.layers[A.nlayers - 1];
            A.phi[2 * pr + tid] = sm_ph[tid * stride_h + last.out_act];
        }
        // ---- backward, dout = 1
        if (tid < 2) sm_ph[tid * stride_h + A.act_total] = 1.0;
        __syncthreads();
        c128* row = A.D + pr * A.Pp;
        for (int l = A.nlayers - 1; l >= 0; --l) {
            const LayerDev L = A.layers[l];
            const double* w = A.p + L.off;
            // dout of this layer at [act_total], din written to [act_total + max_width]
            for (int e = tid; e < 2 * L.in_size; e += nt) {
                const int h = e / L.in_size, i = e % L.in_size;
                const double* base = sm_ph + h * stride_h;
                const double* dout = base + A.act_total;
                double v;
                if (L.type == L_CONV1D) {
                    const int ic = i / L.in_len, q = i % L.in_len;
                    v = 0.;
                    for (int oc = 0; oc < L.b; ++oc)
                        for (int ki = 0; ki < L.k; ++ki) {
                            const double wk = w[size_t(ki + ic * L.k) + size_t(oc) * L.a * L.k];
                            if (L.stride == 1) {
                                const int r = (q - ki + L.k / 2 + 2 * L.in_len) % L.in_len;
                                v += wk * dout[r + oc * L.out_len];
                            } else {
                                for (int r = 0; r < L.out_len; ++r)
                                    if (conv_src(L, r, ki) == q) v += wk * dout[r + oc * L.out_len];
                            }
                        }
                } else if (L.type == L_FC) {
                    double t = 0.;
                    for (int o = 0; o < L.b; ++o) t += w[size_t(i) + size_t(o) * L.a] * dout[o];
                    v = t;
                } else {
                    v = act_jac(L.type, L.x, base[L.in_act + i], base[L.out_act + i], dout[i]);
                }
                sm_ph[h * stride_h + A.act_total + A.max_width + i] = v;
            }
            // parameter derivatives of this layer (both halves into one element)
            if (L.type == L_CONV1D || L.type == L_FC) {
                const long long np = (L.type == L_CONV1D) ? (long long)L.a * L.b * L.k + (L.bias ? L.b : 0)
                                                          : (long long)L.a * L.b + (L.bias ? L.b : 0);
                c128* d = row + L.off;
                for (long long e = tid; e < np; e += nt) {
                    double g[2];
#pragma unroll
                    for (int h = 0; h < 2; ++h) {
                        const double* base = sm_ph + h * stride_h;
                        const double* dout = base + A.act_total;
                        const double* prev = base + L.in_act;
                        double v = 0.;
                        if (L.type == L_CONV1D) {
                            const long long nw = (long long)L.a * L.b * L.k;
                            if (e < nw) {
                                const int rowi = int(e % (L.a * L.k)), oc = int(e / (L.a * L.k));
                                const int ic = rowi / L.k, ki = rowi % L.k;
                                for (int r = 0; r < L.out_len; ++r)
                                    v += prev[conv_src(L, r, ki) + ic * L.in_len] * dout[r + oc * L.out_len];
                            } else {
                                const int oc = int(e - nw);
                                for (int r = 0; r < L.out_len; ++r) v += dout[r + oc * L.out_len];
                            }
                        } else {
                            const long long nw = (long long)L.a * L.b;
                            if (e < nw) {
                                v = prev[e % L.a] * dout[e / L.a];
                            } else {
                                v = dout[e - nw];
                            }
                        }
                        g[h] = M_PI * v;  // logDerivPhase = pi * backward
                    }
                    d[e] = mk(g[0], has1 ? g[1] : 0.0);
                }
            }
            __syncthreads();
            // din becomes the next (earlier) layer's dout
            for (int e = tid; e < 2 * L.in_size; e += nt) {
                const int h = e / L.in_size, i = e % L.in_size;
                sm_ph[h * stride_h + A.act_total + i] = sm_ph[h * stride_h + A.act_total + A.max_width + i];
            }
            __syncthreads();
        }
    }
}

// ---------------------------------------------------------------------------
// Reductions (fixed grids, fixed order).
constexpr int RED = 256;

__global__ void max_partial_kernel(uint64_t n, const double* __restrict__ x, double* __restrict__ part) {
    __shared__ double red[8];
    double v = -INFINITY;
    for (uint64_t i = uint64_t(blockIdx.x) * blockDim.x + threadIdx.x; i < n; i += uint64_t(gridDim.x) * blockDim.x)
        v = fmax(v, x[i]);
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v = fmax(v, __shfl_xor_sync(0xffffffffu, v, o));
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = v;
    __syncthreads();
    if (threadIdx.x == 0) {
        double t = -INFINITY;
        for (int w = 0; w < int(blockDim.x >> 5); ++w) t = fmax(t, red[w]);
        part[blockIdx.x] = t;
    }
}

// w = exp(logA - max) and its partial sums
__global__ void weight_kernel(uint64_t n, const double* __restrict__ logA, const double* __restrict__ mpart,
                              double* __restrict__ w, double* __restrict__ zpart) {
    __shared__ double red[8];
    __shared__ double mx;
    if (threadIdx.x == 0) {
        double t = -INFINITY;
        for (int b = 0; b < RED; ++b) t = fmax(t, mpart[b]);
        mx = t;
    }
    __syncthreads();
    double z = 0.;
    for (uint64_t i = uint64_t(blockIdx.x) * blockDim.x + threadIdx.x; i < n; i += uint64_t(gridDim.x) * blockDim.x) {
        const double v = exp(logA[i] - mx);
        w[i] = v;
        z += v;
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) z += __shfl_xor_sync(0xffffffffu, z, o);
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = z;
    __syncthreads();
    if (threadIdx.x == 0) {
        double t = 0.;
        for (int k = 0; k < int(blockDim.x >> 5); ++k) t += red[k];
        zpart[blockIdx.x] = t;
    }
}

// p = w / Z, psi = sqrt(p) exp(i pi phi)
__global__ void psi_kernel(uint64_t n, const double* __restrict__ zpart, double* __restrict__ p,
                           const double* __restrict__ phi, c128* __restrict__ psi) {
    __shared__ double zs;
    if (threadIdx.x == 0) {
        double t = 0.;
        for (int b = 0; b < RED; ++b) t += zpart[b];
        zs = t;
    }
    __syncthreads();
    for (uint64_t i = uint64_t(blockIdx.x) * blockDim.x + threadIdx.x; i < n; i += uint64_t(gridDim.x) * blockDim.x) {
        const double pi_ = p[i] / zs;
        p[i] = pi_;
        double sn, cs;
        sincos(M_PI * phi[i], &sn, &cs);
        const double r = sqrt(pi_);
        psi[i] = mk(r * cs, r * sn);
    }
}

// partial sums of conj(psi) k; ya = Re, yb = Im of conj(psi) k per configuration
__global__ void energy_kernel(uint64_t n, const c128* __restrict__ psi, const c128* __restrict__ kv,
                              double* __restrict__ ya, double* __restrict__ yb, double* __restrict__ epart) {
    __shared__ double red[8];
    double e = 0.;
    for (uint64_t i = uint64_t(blockIdx.x) * blockDim.x + threadIdx.x; i < n; i += uint64_t(gridDim.x) * blockDim.x) {
        const c128 a = psi[i], b = kv[i];
        const double re = a.re * b.re + a.im * b.im, im = a.re * b.im - a.im * b.re;
        ya[i] = re;
        yb[i] = im;
        e += re;
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) e += __shfl_xor_sync(0xffffffffu, e, o);
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = e;
    __syncthreads();
    if (threadIdx.x == 0) {
        double t = 0.;
        for (int k = 0; k < int(blockDim.x >> 5); ++k) t += red[k];
        epart[blockIdx.x] = t;
    }
}
__global__ void sum_final_kernel(const double* __restrict__ part, int nparts, double* __restrict__ out) {
    if (threadIdx.x == 0 && blockIdx.x == 0) {
        double t = 0.;
        for (int b = 0; b < nparts; ++b) t += part[b];
        *out = t;
    }
}

// Weighted column sums of packed rows: out1[c] = sum_k y1[k] X(k, c),
// out2[c] = sum_k y2[k] X(k, c), X(2k', c) = Z(k', c).re, X(2k'+1, c) = Z(k', c).im.
__global__ void packed_colsum_partial_kernel(size_t P, uint64_t count, uint64_t chunk, const c128* __restrict__ Z,
                                             const double* __restrict__ y1, const double* __restrict__ y2,
                                             double* __restrict__ part /* [nsplit][2][P] */) {
    const size_t c = size_t(blockIdx.x) * blockDim.x + threadIdx.x;
    if (c >= P) return;
    const uint64_t npairs = (count + 1) / 2;
    const uint64_t p0 = uint64_t(blockIdx.y) * chunk, p1 = min(npairs, p0 + chunk);
    double s1 = 0., s2 = 0.;
    for (uint64_t k = p0; k < p1; ++k) {
        const c128 z = Z[k * P + c];
        const uint64_t e = 2 * k, o = 2 * k + 1;
        s1 += y1[e] * z.re;
        s2 += y2[e] * z.re;
        if (o < count) {
            s1 += y1[o] * z.im;
            s2 += y2[o] * z.im;
        }
    }
    part[(size_t(blockIdx.y) * 2) * P + c] = s1;
    part[(size_t(blockIdx.y) * 2 + 1) * P + c] = s2;
}
__global__ void packed_colsum_final_kernel(size_t P, int nsplit, const double* __restrict__ part, double* __restrict__ o1,
                                           double* __restrict__ o2) {
    const size_t c = size_t(blockIdx.x) * blockDim.x + threadIdx.x;
    if (c >= P) return;
    double s1 = 0., s2 = 0.;
    for (int b = 0; b < nsplit; ++b) {
        s1 += part[(size_t(b) * 2) * P + c];
        s2 += part[(size_t(b) * 2 + 1) * P + c];
    }
    o1[c] = s1;
    o2[c] = s2;
}

// grad = 2 g - 2 E o (amplitude) or 2 g (phase), in place over g
__global__ void grad_kernel(size_t P, const double* __restrict__ e, const double* __restrict__ o, double* __restrict__ g,
                            int centre) {
    const size_t c = size_t(blockIdx.x) * blockDim.x + threadIdx.x;
    if (c >= P) return;
    g[c] = centre ? 2.0 * g[c] - 2.0 * (*e) * o[c] : 2.0 * g[c];
}

// Z(k', c) <- sqrt(p) (X - o_c) for both halves; the missing half of an odd count stays 0
__global__ void centre_scale_kernel(size_t P, uint64_t count, const double* __restrict__ p, const double* __restrict__ o,
                                    c128* __restrict__ Z) {
    const uint64_t npairs = (count + 1) / 2;
    const uint64_t total = npairs * P;
    for (uint64_t e = uint64_t(blockIdx.x) * blockDim.x + threadIdx.x; e < total; e += uint64_t(gridDim.x) * blockDim.x) {
        const uint64_t k = e / P;
        const size_t c = size_t(e % P);
        c128 z = Z[e];
        const uint64_t i0 = 2 * k, i1 = 2 * k + 1;
        z.re = sqrt(p[i0]) * (z.re - o[c]);
        z.im = i1 < count ? sqrt(p[i1]) * (z.im - o[c]) : 0.0;
        Z[e] = z;
    }
}

// G = Re(C) + lambda I on the lower triangle, identity on the padding, zero imaginary parts
__global__ void shift_pad_kernel(int P, int pad, const c128* __restrict__ C, c128* __restrict__ G, double lambda) {
    const size_t total = size_t(pad) * pad;
    for (size_t e = size_t(blockIdx.x) * blockDim.x + threadIdx.x; e < total; e += size_t(gridDim.x) * blockDim.x) {
        const int r = int(e / pad), c = int(e % pad);
        double v = 0.;
        if (r < P && c < P) {
            if (c <= r) v = C[e].re + (r == c ? lambda : 0.0);
        } else if (r == c) {
            v = 1.0;
        }
        G[e] = mk(v, 0.0);
    }
}

// params += -lr v  (Optimizers/SGD.hpp:48-54 getUpdate, AmplitudePhase::updateParams)
__global__ void sgd_kernel(size_t P, const c128* __restrict__ va, size_t Pa, const c128* __restrict__ vp, double lr,
                           int use_a, int use_p, double* __restrict__ params) {
    const size_t c = size_t(blockIdx.x) * blockDim.x + threadIdx.x;
    if (c >= P) return;
    double v = 0.;
    if (c < Pa) {
        if (use_a) v = va[c].re;
    } else if (use_p) {
        v = vp[c - Pa].re;
    }
    params[c] += -lr * v;
}

// ---------------------------------------------------------------------------
// Host helpers.
double normal_first(uint64_t seed, uint32_t idx) {
    U4 x = draw(seed, idx, 0u, 0u, TAG_PARAM);
    const double u1 = 1.0 - draw_u53(x.x, x.y);
    const double u2 = draw_u53(x.z, x.w);
    return std::sqrt(-2.0 * std::log(u1)) * std::cos(6.283185307179586476925286766559 * u2);
}

unsigned grid_for(uint64_t work, unsigned per_block, unsigned cap) {
    return unsigned(std::max<uint64_t>(1, std::min<uint64_t>(cap, (work + per_block - 1) / per_block)));
}

size_t phase_smem(const yq_ap_s* q) { return size_t(2) * (q->act_total + 2 * q->max_width) * sizeof(double); }

// D_amp and log A of `count` configurations into packed rows (Pa per pair)
void run_amp(yq_ap_s* q, uint64_t count, const int8_t* sigma, double* logA, c128* D, cudaStream_t st) {
    if (count == 0) return;
    AmpArgs A{q->n, q->m, q->bias, count, sigma, q->p64.as<double>(), logA, D, q->Pa};
    const size_t smem = size_t(2) * q->m * sizeof(double);
    amp_kernel<<<grid_for((count + 1) / 2, 1, 148 * 16), AP_THREADS, smem, st>>>(A);
    YQ_LAUNCH_CHECK();
}

void run_phase(yq_ap_s* q, uint64_t count, const int8_t* sigma, double* phi, c128* D, cudaStream_t st) {
    if (count == 0) return;
    PhaseArgs A{q->n, int(q->layers.size()), q->act_total, q->max_width, count, sigma, q->dlayers.as<LayerDev>(),
                q->p64.as<double>() + q->Pa, phi, D, q->Pp};
    // layer offsets are relative to the phase block
    const size_t smem = phase_smem(q);
    if (smem > 48 * 1024)
        YQ_CUDA(cudaFuncSetAttribute(phase_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, int(smem)));
    phase_kernel<<<grid_for((count + 1) / 2, 1, 148 * 16), AP_THREADS, smem, st>>>(A);
    YQ_LAUNCH_CHECK();
}

void packed_colsums(const c128* Z, size_t P, uint64_t count, const double* y1, const double* y2, DevBuf& part,
                    double* o1, double* o2, cudaStream_t st) {
    const uint64_t npairs = (count + 1) / 2;
    const unsigned gx = unsigned((P + 127) / 128);
    const int nsplit = int(std::max<uint64_t>(1, std::min<uint64_t>(std::min<uint64_t>(256, npairs), uint64_t(8 * 148) / gx + 1)));
    const uint64_t chunk = (npairs + nsplit - 1) / nsplit;
    part.ensure(size_t(nsplit) * 2 * P * sizeof(double));
    packed_colsum_partial_kernel<<<dim3(gx, unsigned(nsplit)), 128, 0, st>>>(P, count, chunk, Z, y1, y2,
                                                                              part.as<double>());
    packed_colsum_final_kernel<<<gx, 128, 0, st>>>(P, nsplit, part.as<double>(), o1, o2);
    YQ_LAUNCH_CHECK();
}

template <class Fn>
int guard_ap(Fn&& fn) {
    try {
        fn();
        return YQ_OK;
    } catch (const Error& e) {
        record_error(e.what());
        return e.code;
    } catch (const std::bad_alloc&) {
        record_error("host allocation failed");
        return YQ_E_NOMEM;
    } catch (const std::exception& e) {
        record_error(e.what());
        return YQ_E_ARG;
    }
}

void need(const void* p, const char* what) {
    if (!p) throw Error(YQ_E_ARG, std::string("null argument: ") + what);
}

void check_sigma_pm1(const int8_t* s, size_t count) {
    for (size_t i = 0; i < count; ++i)
        if (s[i] != 1 && s[i] != -1) throw Error(YQ_E_ARG, "sigma entries must be +1 or -1");
}

// C = sum of the split partials (every element; only the lower triangle is read)
__global__ void sum_partials_kernel(size_t count, int nparts, const c128* __restrict__ parts, c128* __restrict__ C) {
    for (size_t e = size_t(blockIdx.x) * blockDim.x + threadIdx.x; e < count; e += size_t(gridDim.x) * blockDim.x) {
        c128 acc = parts[e];
        for (int k = 1; k < nparts; ++k) acc = acc + parts[size_t(k) * count + e];
        C[e] = acc;
    }
}

// The real correlation matrices as the real parts of Z^H Z over the packed rows.
// One DMMA CTA computes one 64 x 64 tile of the lower triangle over all K = dim2
// rows, and P of a few hundred to a few thousand gives fewer tiles than the GPU
// has SMs, so K is split into chunks computed on side streams into partial
// matrices that are then summed in a fixed order.
void grams(yq_ngd_s* g, cudaStream_t st) {
    yq_ap_s* q = g->q;
    const size_t Pa = q->Pa, Pp = q->Pp;
    const uint64_t K = g->dim2;
    if (g->split_a * g->split_p == 1) {
        gram_fp64<double>(g->Da.as<c128>(), Pa, 1, int(Pa), int(K), g->Ca.as<c128>(), size_t(g->pad_a), 1.0, 0, 0.0, st);
        if (Pp)
            gram_fp64<double>(g->Dp.as<c128>(), Pp, 1, int(Pp), int(K), g->Cp.as<c128>(), size_t(g->pad_p), 1.0, 0, 0.0,
                              st);
        return;
    }
    const size_t na = size_t(g->pad_a) * g->pad_a, np = size_t(g->pad_p) * g->pad_p;
    c128* pa = g->Cpart.as<c128>();
    c128* pp = pa + size_t(g->split_a) * na;
    YQ_CUDA(cudaEventRecord(g->fork, st));
    int job = 0;
    auto run = [&](const c128* Z, size_t P, int split, c128* parts, size_t cnt, int pad) {
        const uint64_t chunk = (K + split - 1) / split;
        for (int k = 0; k < split; ++k) {
            const uint64_t k0 = std::min<uint64_t>(K, uint64_t(k) * chunk), kc = std::min<uint64_t>(chunk, K - k0);
            cudaStream_t ss = g->side[job % yq_ngd_s::NSIDE];
            if (job < yq_ngd_s::NSIDE) YQ_CUDA(cudaStreamWaitEvent(ss, g->fork, 0));
            if (kc > 0)
                gram_fp64<double>(Z + k0 * P, P, 1, int(P), int(kc), parts + size_t(k) * cnt, size_t(pad), 1.0, 0, 0.0,
                                  ss);
            else
                YQ_CUDA(cudaMemsetAsync(parts + size_t(k) * cnt, 0, cnt * sizeof(c128), ss));
            ++job;
        }
    };
    run(g->Da.as<c128>(), Pa, g->split_a, pa, na, g->pad_a);
    if (Pp) run(g->Dp.as<c128>(), Pp, g->split_p, pp, np, g->pad_p);
    for (int i = 0; i < std::min(job, int(yq_ngd_s::NSIDE)); ++i) {
        YQ_CUDA(cudaEventRecord(g->join[i], g->side[i]));
        YQ_CUDA(cudaStreamWaitEvent(st, g->join[i], 0));
    }
    sum_partials_kernel<<<grid_for(na, 256, 148 * 16), 256, 0, st>>>(na, g->split_a, pa, g->Ca.as<c128>());
    if (Pp) sum_partials_kernel<<<grid_for(np, 256, 148 * 16), 256, 0, st>>>(np, g->split_p, pp, g->Cp.as<c128>());
    YQ_LAUNCH_CHECK();
}

// NGDExact::constructExact on the device
void ngd_construct(yq_ngd_s* g) {
    yq_ap_s* q = g->q;
    cudaStream_t st = q->ctx->stream;
    const uint64_t dim = g->dim;
    const size_t Pa = q->Pa, Pp = q->Pp;
    run_amp(q, dim, g->sigma.as<int8_t>(), g->logA.as<double>(), g->Da.as<c128>(), st);
    run_phase(q, dim, g->sigma.as<int8_t>(), g->phi.as<double>(), g->Dp.as<c128>(), st);
    double* part = g->part.as<double>();
    double* scal = g->scal.as<double>();  // [0] energy
    max_partial_kernel<<<RED, 256, 0, st>>>(dim, g->logA.as<double>(), part);
    weight_kernel<<<RED, 256, 0, st>>>(dim, g->logA.as<double>(), part, g->p.as<double>(), part + RED);
    psi_kernel<<<grid_for(dim, 256, 148 * 16), 256, 0, st>>>(dim, part + RED, g->p.as<double>(), g->phi.as<double>(),
                                                           g->psi.as<c128>());
    YQ_LAUNCH_CHECK();
    ham_apply_basis(g->H, dim, g->kind, g->nup, g->kind == YQ_BASIS_JZ ? g->binom.as<uint64_t>() : nullptr,
                    g->index.as<uint64_t>(), g->sigma.as<int8_t>(), g->psi.as<c128>(), g->kv.as<c128>(), st);
    energy_kernel<<<RED, 256, 0, st>>>(dim, g->psi.as<c128>(), g->kv.as<c128>(), g->ya.as<double>(),
                                       g->yb.as<double>(), part + 2 * RED);
    sum_final_kernel<<<1, 32, 0, st>>>(part + 2 * RED, RED, scal);
    YQ_LAUNCH_CHECK();
    double* grad = g->grad.as<double>();
    double* oloc = g->oloc.as<double>();
    packed_colsums(g->Da.as<c128>(), Pa, dim, g->p.as<double>(), g->ya.as<double>(), g->cpart, oloc, grad, st);
    packed_colsums(g->Dp.as<c128>(), Pp, dim, g->p.as<double>(), g->yb.as<double>(), g->cpart, oloc + Pa, grad + Pa,
                   st);
    grad_kernel<<<grid_for(Pa, 256, 1u << 20), 256, 0, st>>>(Pa, scal, oloc, grad, 1);
    grad_kernel<<<grid_for(Pp, 256, 1u << 20), 256, 0, st>>>(Pp, scal, oloc + Pa, grad + Pa, 0);
    // centred, sqrt(p)-scaled rows and their real Gram matrices (lower triangles)
    centre_scale_kernel<<<grid_for(g->dim2 * Pa, 256, 148 * 32), 256, 0, st>>>(Pa, dim, g->p.as<double>(), oloc,
                                                                             g->Da.as<c128>());
    centre_scale_kernel<<<grid_for(g->dim2 * Pp, 256, 148 * 32), 256, 0, st>>>(Pp, dim, g->p.as<double>(), oloc + Pa,
                                                                             g->Dp.as<c128>());
    YQ_LAUNCH_CHECK();
    grams(g, st);
    YQ_CUDA(cudaMemcpyAsync(&g->energy, scal, sizeof(double), cudaMemcpyDeviceToHost, st));
    YQ_CUDA(cudaStreamSynchronize(st));
    g->constructed = true;
}

// LLT of (C + lambda I) for one block: solution into g->sol (c128, pad entries)
void solve_block(yq_ngd_s* g, DevBuf& C, DevBuf& G, int P, int pad, DevBuf& L, DevBuf& LH, const double* rhs_dev,
                 double lambda, c128* out) {
    yq_ctx_s* ctx = g->q->ctx;
    cudaStream_t st = ctx->stream;
    G.ensure(size_t(pad) * pad * sizeof(c128));
    shift_pad_kernel<<<grid_for(size_t(pad) * pad, 256, 148 * 32), 256, 0, st>>>(P, pad, C.as<c128>(), G.as<c128>(),
                                                                               lambda);
    YQ_LAUNCH_CHECK();
    const size_t nb = size_t(pad) / CHOL_NB;
    L.ensure(nb * CHOL_NB * CHOL_NB * sizeof(c128));
    LH.ensure(nb * CHOL_NB * CHOL_NB * sizeof(c128));
    g->chol_work.ensure(chol_tile_scratch_bytes(pad));
    chol_factor_tiled(G.as<c128>(), pad, size_t(pad), L.as<c128>(), LH.as<c128>(), ctx->status.as<int>(),
                      g->chol_work.p, ctx->sm_count, st);
    // right-hand side: the gradient block as complex, zero padding
    std::vector<double> h(static_cast<size_t>(P));
    YQ_CUDA(cudaMemcpyAsync(h.data(), rhs_dev, size_t(P) * sizeof(double), cudaMemcpyDeviceToHost, st));
    YQ_CUDA(cudaStreamSynchronize(st));
    std::vector<c128> b(size_t(pad), mk(0., 0.));
    for (int i = 0; i < P; ++i) b[size_t(i)] = mk(h[size_t(i)], 0.);
    g->rhs.ensure(size_t(pad) * sizeof(c128));
    YQ_CUDA(cudaMemcpyAsync(g->rhs.p, b.data(), size_t(pad) * sizeof(c128), cudaMemcpyHostToDevice, st));
    chol_solve_tiled(G.as<c128>(), pad, size_t(pad), L.as<c128>(), LH.as<c128>(), g->rhs.as<c128>(), out,
                     ctx->status.as<int>(), g->chol_work.p, ctx->sm_count, st);
    YQ_CUDA(cudaStreamSynchronize(st));
}

void read_lower_real(const DevBuf& C, int P, int pad, cudaStream_t st, double* out) {
    std::vector<c128> h(size_t(pad) * pad);
    YQ_CUDA(cudaMemcpyAsync(h.data(), C.p, h.size() * sizeof(c128), cudaMemcpyDeviceToHost, st));
    YQ_CUDA(cudaStreamSynchronize(st));
    for (int r = 0; r < P; ++r)
        for (int c = 0; c <= r; ++c) {
            const double v = h[size_t(r) * pad + c].re;
            out[size_t(r) * P + c] = v;
            out[size_t(c) * P + r] = v;
        }
}

}  // namespace
}  // namespace yq

using namespace yq;

extern "C" {

int yq_ap_create(yq_ctx ctx, int n, int m, int use_bias, int nlayers, const int* layers, const double* layer_x,
                 yq_ap* out) {
    return guard_ap([&] {
        need(ctx, "ctx");
        need(out, "out");
        *out = nullptr;
        if (n < 1 || m < 1 || n > 4096 || m > 65535) throw Error(YQ_E_ARG, "ap: need 1 <= n <= 4096, 1 <= m");
        if (nlayers < 1 || nlayers > MAX_LAYERS) throw Error(YQ_E_ARG, "ap: need 1 to 64 phase layers");
        need(layers, "layers");
        need(layer_x, "layer_x");
        auto q = std::make_unique<yq_ap_s>();
        q->ctx = ctx;
        q->n = n;
        q->m = m;
        q->bias = use_bias != 0;
        q->Pa = size_t(n) * m + (q->bias ? size_t(n + m) : 0);
        int size = n, act = n;  // the input occupies [0, n) of the activation buffer
        long long off = 0;
        q->max_width = n;
        for (int l = 0; l < nlayers; ++l) {
            LayerDev L{};
            L.type = layers[6 * l];
            L.a = layers[6 * l + 1];
            L.b = layers[6 * l + 2];
            L.k = layers[6 * l + 3];
            L.stride = layers[6 * l + 4];
            L.bias = layers[6 * l + 5] ? 1 : 0;
            L.x = layer_x[l];
            L.in_size = size;
            L.in_act = act - size;
            L.off = off;
            long long np = 0;
            if (L.type == L_CONV1D) {  // Conv1D(inChannels, outChannels, kernelSize, stride, useBias)
                if (L.a < 1 || L.b < 1 || L.k < 1 || L.stride < 1 || size % L.a)
                    throw Error(YQ_E_ARG, "ap: Conv1D needs channels >= 1, kernel >= 1, stride >= 1 and an input "
                                          "that is a multiple of the input channels");
                L.in_len = size / L.a;
                if (L.k / 2 > L.in_len) throw Error(YQ_E_ARG, "ap: Conv1D kernel wider than twice the input length");
                L.out_len = L.in_len / L.stride;
                if (L.out_len < 1) throw Error(YQ_E_ARG, "ap: Conv1D stride longer than the input");
                L.out_size = L.out_len * L.b;
                np = (long long)L.a * L.b * L.k + (L.bias ? L.b : 0);
            } else if (L.type == L_FC) {  // FullyConnected(inputDim, outputDim, useBias)
                if (L.a != size || L.b < 1) throw Error(YQ_E_ARG, "ap: FullyConnected input width differs");
                L.out_size = L.b;
                np = (long long)L.a * L.b + (L.bias ? L.b : 0);
            } else if (L.type >= A_IDENTITY && L.type <= A_COS) {
                if ((L.type == A_TANH || L.type == A_COS) && L.x == 0.0)
                    throw Error(YQ_E_ARG, "ap: Tanh and Cos need a non-zero constant");
                L.out_size = size;
            } else {
                throw Error(YQ_E_ARG, "ap: unknown layer type " + std::to_string(L.type));
            }
            if (L.out_size > 8192) throw Error(YQ_E_ARG, "ap: layers wider than 8192 values are not built");
            L.out_act = act;
            act += L.out_size;
            off += np;
            size = L.out_size;
            q->max_width = std::max(q->max_width, std::max(L.in_size, L.out_size));
            q->layers.push_back(L);
        }
        if (size != 1) throw Error(YQ_E_ARG, "ap: the phase network must end in a single output");
        q->act_total = act;
        q->Pp = size_t(off);
        if (phase_smem(q.get()) > 200 * 1024)
            throw Error(YQ_E_UNSUPPORTED, "ap: the phase network's activations exceed the shared-memory budget");
        q->p64.ensure((q->Pa + q->Pp) * sizeof(double));
        YQ_CUDA(cudaMemsetAsync(q->p64.p, 0, (q->Pa + q->Pp) * sizeof(double), ctx->stream));
        q->dlayers.ensure(q->layers.size() * sizeof(LayerDev));
        YQ_CUDA(cudaMemcpyAsync(q->dlayers.p, q->layers.data(), q->layers.size() * sizeof(LayerDev),
                                cudaMemcpyHostToDevice, ctx->stream));
        YQ_CUDA(cudaStreamSynchronize(ctx->stream));
        *out = q.release();
    });
}

int yq_ap_destroy(yq_ap q) {
    return guard_ap([&] { delete q; });
}

int yq_ap_dims(yq_ap q, size_t* dim_amp, size_t* dim_phase) {
    return guard_ap([&] {
        need(q, "ap");
        if (dim_amp) *dim_amp = q->Pa;
        if (dim_phase) *dim_phase = q->Pp;
    });
}

int yq_ap_set_params(yq_ap q, const double* params) {
    return guard_ap([&] {
        need(q, "ap");
        need(params, "params");
        YQ_CUDA(cudaMemcpyAsync(q->p64.p, params, (q->Pa + q->Pp) * sizeof(double), cudaMemcpyHostToDevice,
                                q->ctx->stream));
        YQ_CUDA(cudaStreamSynchronize(q->ctx->stream));
    });
}

int yq_ap_get_params(yq_ap q, double* params) {
    return guard_ap([&] {
        need(q, "ap");
        need(params, "params");
        YQ_CUDA(cudaMemcpyAsync(params, q->p64.p, (q->Pa + q->Pp) * sizeof(double), cudaMemcpyDeviceToHost,
                                q->ctx->stream));
        YQ_CUDA(cudaStreamSynchronize(q->ctx->stream));
    });
}

int yq_ap_update_params(yq_ap q, const double* delta) {
    return guard_ap([&] {
        need(q, "ap");
        need(delta, "delta");
        const size_t P = q->Pa + q->Pp;
        std::vector<double> cur(P);
        YQ_CUDA(cudaMemcpyAsync(cur.data(), q->p64.p, P * sizeof(double), cudaMemcpyDeviceToHost, q->ctx->stream));
        YQ_CUDA(cudaStreamSynchronize(q->ctx->stream));
        for (size_t i = 0; i < P; ++i) cur[i] += delta[i];
        YQ_CUDA(cudaMemcpyAsync(q->p64.p, cur.data(), P * sizeof(double), cudaMemcpyHostToDevice, q->ctx->stream));
        YQ_CUDA(cudaStreamSynchronize(q->ctx->stream));
    });
}

int yq_ap_init_random(yq_ap q, uint64_t seed, double sigma_amp, int phase_mode) {
    return guard_ap([&] {
        need(q, "ap");
        if (phase_mode < 0 || phase_mode > 2) throw Error(YQ_E_ARG, "ap: phase mode is LeCun 0, Xavier 1 or He 2");
        const size_t P = q->Pa + q->Pp, nm = size_t(q->n) * q->m;
        std::vector<double> p(P, 0.0);
        uint32_t e = 0;
        // amplitude: RBM.hpp:325-349 order (a, b, W by columns)
        if (q->bias) {
            for (int i = 0; i < q->n; ++i) p[nm + i] = sigma_amp * normal_first(seed, e++);
            for (int j = 0; j < q->m; ++j) p[nm + q->n + j] = sigma_amp * normal_first(seed, e++);
        }
        for (int i = 0; i < q->n; ++i)
            for (int j = 0; j < q->m; ++j) p[size_t(i) * q->m + j] = sigma_amp * normal_first(seed, e++);
        // phase: FeedForward.hpp initializeRandom(re, mode), layer by layer
        for (const LayerDev& L : q->layers) {
            if (L.type != L_CONV1D && L.type != L_FC) continue;
            const double fin = L.type == L_CONV1D ? double(L.a) * L.k : double(L.a);
            const double fout = L.type == L_CONV1D ? double(L.b) * L.k : double(L.b);
            const double sd = phase_mode == 0 ? std::sqrt(1.0 / fin)
                              : phase_mode == 1 ? std::sqrt(2.0 / (fin + fout))
                                                : std::sqrt(2.0 / fin);
            const long long np = L.type == L_CONV1D ? (long long)L.a * L.b * L.k + (L.bias ? L.b : 0)
                                                    : (long long)L.a * L.b + (L.bias ? L.b : 0);
            for (long long k = 0; k < np; ++k) p[q->Pa + size_t(L.off + k)] = sd * normal_first(seed, e++);
        }
        YQ_CUDA(cudaMemcpyAsync(q->p64.p, p.data(), P * sizeof(double), cudaMemcpyHostToDevice, q->ctx->stream));
        YQ_CUDA(cudaStreamSynchronize(q->ctx->stream));
    });
}

int yq_ap_log_psi(yq_ap q, int ns, const int8_t* sigma, double* out) {
    return guard_ap([&] {
        need(q, "ap");
        need(sigma, "sigma");
        need(out, "out");
        if (ns < 0) throw Error(YQ_E_ARG, "ns < 0");
        if (ns == 0) return;
        check_sigma_pm1(sigma, size_t(ns) * q->n);
        cudaStream_t st = q->ctx->stream;
        const uint64_t pairs = (uint64_t(ns) + 1) / 2;
        DevBuf s, la, ph, Da, Dp;
        s.ensure(size_t(ns) * q->n);
        la.ensure(size_t(ns) * sizeof(double));
        ph.ensure(size_t(ns) * sizeof(double));
        Da.ensure(pairs * q->Pa * sizeof(c128));
        Dp.ensure(pairs * std::max<size_t>(1, q->Pp) * sizeof(c128));
        YQ_CUDA(cudaMemcpyAsync(s.p, sigma, size_t(ns) * q->n, cudaMemcpyHostToDevice, st));
        run_amp(q, uint64_t(ns), s.as<int8_t>(), la.as<double>(), Da.as<c128>(), st);
        run_phase(q, uint64_t(ns), s.as<int8_t>(), ph.as<double>(), Dp.as<c128>(), st);
        std::vector<double> a(static_cast<size_t>(ns)), f(static_cast<size_t>(ns));
        YQ_CUDA(cudaMemcpyAsync(a.data(), la.p, a.size() * sizeof(double), cudaMemcpyDeviceToHost, st));
        YQ_CUDA(cudaMemcpyAsync(f.data(), ph.p, f.size() * sizeof(double), cudaMemcpyDeviceToHost, st));
        YQ_CUDA(cudaStreamSynchronize(st));
        // log psi = log A / 2 + i pi phi   (AmplitudePhase::coeff)
        for (int k = 0; k < ns; ++k) {
            out[2 * k] = 0.5 * a[size_t(k)];
            out[2 * k + 1] = M_PI * f[size_t(k)];
        }
    });
}

int yq_ap_log_deriv(yq_ap q, int ns, const int8_t* sigma, double* out) {
    return guard_ap([&] {
        need(q, "ap");
        need(sigma, "sigma");
        need(out, "out");
        if (ns < 0) throw Error(YQ_E_ARG, "ns < 0");
        if (ns == 0) return;
        check_sigma_pm1(sigma, size_t(ns) * q->n);
        cudaStream_t st = q->ctx->stream;
        const uint64_t pairs = (uint64_t(ns) + 1) / 2;
        DevBuf s, Da, Dp;
        s.ensure(size_t(ns) * q->n);
        Da.ensure(pairs * q->Pa * sizeof(c128));
        Dp.ensure(pairs * std::max<size_t>(1, q->Pp) * sizeof(c128));
        YQ_CUDA(cudaMemcpyAsync(s.p, sigma, size_t(ns) * q->n, cudaMemcpyHostToDevice, st));
        run_amp(q, uint64_t(ns), s.as<int8_t>(), nullptr, Da.as<c128>(), st);
        run_phase(q, uint64_t(ns), s.as<int8_t>(), nullptr, Dp.as<c128>(), st);
        std::vector<c128> ha(pairs * q->Pa), hp(pairs * q->Pp);
        YQ_CUDA(cudaMemcpyAsync(ha.data(), Da.p, ha.size() * sizeof(c128), cudaMemcpyDeviceToHost, st));
        if (q->Pp) YQ_CUDA(cudaMemcpyAsync(hp.data(), Dp.p, hp.size() * sizeof(c128), cudaMemcpyDeviceToHost, st));
        YQ_CUDA(cudaStreamSynchronize(st));
        // rows [logDerivAmp | i logDerivPhase] (AmplitudePhase.hpp:52-59)
        const size_t P = q->Pa + q->Pp;
        for (int k = 0; k < ns; ++k) {
            double* row = out + 2 * size_t(k) * P;
            const size_t pr = size_t(k) / 2;
            const bool odd = k & 1;
            for (size_t c = 0; c < q->Pa; ++c) {
                const c128 z = ha[pr * q->Pa + c];
                row[2 * c] = odd ? z.im : z.re;
                row[2 * c + 1] = 0.0;
            }
            for (size_t c = 0; c < q->Pp; ++c) {
                const c128 z = hp[pr * q->Pp + c];
                row[2 * (q->Pa + c)] = 0.0;
                row[2 * (q->Pa + c) + 1] = odd ? z.im : z.re;
            }
        }
    });
}

int yq_ngd_create(yq_ap q, yq_ham H, int basis_kind, int nup, yq_ngd* out) {
    return guard_ap([&] {
        need(q, "ap");
        need(H, "ham");
        need(out, "out");
        *out = nullptr;
        if (H->n != q->n) throw Error(YQ_E_ARG, "ngd: Hamiltonian and machine sizes differ");
        if (basis_kind == YQ_BASIS_JZ && !H->conserves_sz)
            throw Error(YQ_E_ARG, "ngd: the Jz basis needs a Hamiltonian that conserves Sz (XXZ, XXX, J1J2)");
        if (H->ctx->device != q->ctx->device) throw Error(YQ_E_ARG, "ngd: Hamiltonian on another device");
        auto g = std::make_unique<yq_ngd_s>();
        g->q = q;
        g->H = H;
        g->kind = basis_kind;
        g->nup = nup;
        cudaStream_t st = q->ctx->stream;
        Basis b = make_basis(q->n, basis_kind, nup);
        g->dim = b.dim;
        g->dim2 = (b.dim + 1) / 2;
        if (basis_kind == YQ_BASIS_JZ) {
            g->binom.ensure(b.binom.size() * sizeof(uint64_t));
            YQ_CUDA(cudaMemcpyAsync(g->binom.p, b.binom.data(), b.binom.size() * sizeof(uint64_t),
                                    cudaMemcpyHostToDevice, st));
        }
        g->index.ensure(b.dim * sizeof(uint64_t));
        g->sigma.ensure(b.dim * q->n);
        basis_kernel<<<grid_for(b.dim, 256, 148 * 16), 256, 0, st>>>(
            b.dim, q->n, basis_kind, nup, basis_kind == YQ_BASIS_JZ ? g->binom.as<uint64_t>() : nullptr,
            g->index.as<uint64_t>(), g->sigma.as<int8_t>());
        YQ_LAUNCH_CHECK();
        for (DevBuf* d : {&g->logA, &g->phi, &g->p, &g->ya, &g->yb}) d->ensure(b.dim * sizeof(double));
        g->psi.ensure(b.dim * sizeof(c128));
        g->kv.ensure(b.dim * sizeof(c128));
        g->Da.ensure(g->dim2 * q->Pa * sizeof(c128));
        g->Dp.ensure(g->dim2 * std::max<size_t>(1, q->Pp) * sizeof(c128));
        g->part.ensure(3 * RED * sizeof(double));
        g->scal.ensure(8 * sizeof(double));
        g->grad.ensure((q->Pa + q->Pp) * sizeof(double));
        g->oloc.ensure((q->Pa + q->Pp) * sizeof(double));
        g->pad_a = int((q->Pa + CHOL_NB - 1) / CHOL_NB * CHOL_NB);
        g->pad_p = int((std::max<size_t>(1, q->Pp) + CHOL_NB - 1) / CHOL_NB * CHOL_NB);
        g->Ca.ensure(size_t(g->pad_a) * g->pad_a * sizeof(c128));
        g->Cp.ensure(size_t(g->pad_p) * g->pad_p * sizeof(c128));
        YQ_CUDA(cudaMemsetAsync(g->Ca.p, 0, size_t(g->pad_a) * g->pad_a * sizeof(c128), st));
        YQ_CUDA(cudaMemsetAsync(g->Cp.p, 0, size_t(g->pad_p) * g->pad_p * sizeof(c128), st));
        // K-split: enough chunks that both Grams together give about eight tiles per SM
        // (at most 8 chunks each, and chunks of at least 4096 rows)
        {
            const int sms = std::max(1, q->ctx->sm_count);
            auto tiles = [](size_t P) { const size_t t = (P + 63) / 64; return t * (t + 1) / 2; };
            const size_t ta = tiles(q->Pa), tp = q->Pp ? tiles(q->Pp) : 0;
            const size_t want = size_t(8) * sms;
            const int by_rows = int(std::max<uint64_t>(1, g->dim2 / 4096));
            const int split = int(std::min<size_t>(8, std::max<size_t>(1, (want + ta + tp - 1) / (ta + tp))));
            g->split_a = g->split_p = std::min(split, by_rows);
            if (g->split_a > 1) {
                YQ_CUDA(cudaEventCreateWithFlags(&g->fork, cudaEventDisableTiming));
                for (int i = 0; i < yq_ngd_s::NSIDE; ++i) {
                    YQ_CUDA(cudaStreamCreateWithFlags(&g->side[i], cudaStreamNonBlocking));
                    YQ_CUDA(cudaEventCreateWithFlags(&g->join[i], cudaEventDisableTiming));
                }
                const size_t cnt = size_t(g->split_a) * g->pad_a * g->pad_a + size_t(g->split_p) * g->pad_p * g->pad_p;
                g->Cpart.ensure(cnt * sizeof(c128));
                YQ_CUDA(cudaMemsetAsync(g->Cpart.p, 0, cnt * sizeof(c128), st));
            }
        }
        YQ_CUDA(cudaStreamSynchronize(st));
        *out = g.release();
    });
}

int yq_ngd_destroy(yq_ngd g) {
    return guard_ap([&] { delete g; });
}

int yq_ngd_basis_size(yq_ngd g, uint64_t* dim) {
    return guard_ap([&] {
        need(g, "ngd");
        need(dim, "dim");
        *dim = g->dim;
    });
}

int yq_ngd_construct(yq_ngd g, double* energy) {
    return guard_ap([&] {
        need(g, "ngd");
        ngd_construct(g);
        if (energy) *energy = g->energy;
        const int stt = g->q->ctx->read_status_and_clear();
        if (stt & DS_NONFINITE) throw Error(YQ_E_NONFINITE, "ngd: non-finite value");
    });
}

int yq_ngd_get(yq_ngd g, int what, double* out) {
    return guard_ap([&] {
        need(g, "ngd");
        need(out, "out");
        if (!g->constructed) throw Error(YQ_E_STATE, "ngd: construct first");
        yq_ap_s* q = g->q;
        cudaStream_t st = q->ctx->stream;
        switch (what) {
            case YQ_NGD_GRAD:
                YQ_CUDA(cudaMemcpyAsync(out, g->grad.p, (q->Pa + q->Pp) * sizeof(double), cudaMemcpyDeviceToHost, st));
                break;
            case YQ_NGD_OLOC_AMP:
                YQ_CUDA(cudaMemcpyAsync(out, g->oloc.p, q->Pa * sizeof(double), cudaMemcpyDeviceToHost, st));
                break;
            case YQ_NGD_OLOC_PHASE:
                YQ_CUDA(cudaMemcpyAsync(out, g->oloc.as<double>() + q->Pa, q->Pp * sizeof(double),
                                        cudaMemcpyDeviceToHost, st));
                break;
            case YQ_NGD_CORR_AMP: read_lower_real(g->Ca, int(q->Pa), g->pad_a, st, out); break;
            case YQ_NGD_CORR_PHASE: read_lower_real(g->Cp, int(q->Pp), g->pad_p, st, out); break;
            default: throw Error(YQ_E_ARG, "ngd: unknown quantity");
        }
        YQ_CUDA(cudaStreamSynchronize(st));
    });
}

int yq_ngd_iteration(yq_ngd g, double lambda, double lr, int mode, double* energy, double* grad_norm, double* v_norm) {
    return guard_ap([&] {
        need(g, "ngd");
        if (mode != YQ_NGD_AMP && mode != YQ_NGD_PHASE && mode != YQ_NGD_ALL) throw Error(YQ_E_ARG, "ngd: unknown mode");
        if (!(lambda > 0.0)) throw Error(YQ_E_ARG, "ngd: lambda must be > 0");
        yq_ap_s* q = g->q;
        yq_ctx_s* ctx = q->ctx;
        cudaStream_t st = ctx->stream;
        ngd_construct(g);
        const size_t P = q->Pa + q->Pp;
        std::vector<double> grad(P);
        YQ_CUDA(cudaMemcpyAsync(grad.data(), g->grad.p, P * sizeof(double), cudaMemcpyDeviceToHost, st));
        YQ_CUDA(cudaStreamSynchronize(st));
        const bool use_a = mode == YQ_NGD_AMP || mode == YQ_NGD_ALL;
        const bool use_p = (mode == YQ_NGD_PHASE || mode == YQ_NGD_ALL) && q->Pp > 0;
        DevBuf& va = g->va;
        DevBuf& vp = g->vp;
        va.ensure(size_t(g->pad_a) * sizeof(c128));
        vp.ensure(size_t(g->pad_p) * sizeof(c128));
        if (use_a)
            solve_block(g, g->Ca, g->Ga, int(q->Pa), g->pad_a, g->La, g->LaH, g->grad.as<double>(), lambda,
                        va.as<c128>());
        if (use_p)
            solve_block(g, g->Cp, g->Gp, int(q->Pp), g->pad_p, g->Lp, g->LpH, g->grad.as<double>() + q->Pa, lambda,
                        vp.as<c128>());
        const int stt = ctx->read_status_and_clear();
        if (stt & DS_TIMEOUT) throw Error(YQ_E_TIMEOUT, "ngd: a bounded device wait gave up");
        if (stt & DS_NOT_PD) throw Error(YQ_E_NOT_PD, "ngd: the correlation matrix plus shift is not positive definite");
        double vn = 0.;
        std::vector<c128> h(size_t(std::max(g->pad_a, g->pad_p)));
        if (use_a) {
            YQ_CUDA(cudaMemcpyAsync(h.data(), va.p, q->Pa * sizeof(c128), cudaMemcpyDeviceToHost, st));
            YQ_CUDA(cudaStreamSynchronize(st));
            for (size_t i = 0; i < q->Pa; ++i) vn += h[i].re * h[i].re;
        }
        if (use_p) {
            YQ_CUDA(cudaMemcpyAsync(h.data(), vp.p, q->Pp * sizeof(c128), cudaMemcpyDeviceToHost, st));
            YQ_CUDA(cudaStreamSynchronize(st));
            for (size_t i = 0; i < q->Pp; ++i) vn += h[i].re * h[i].re;
        }
        sgd_kernel<<<grid_for(P, 256, 1u << 20), 256, 0, st>>>(P, va.as<c128>(), q->Pa, vp.as<c128>(), lr, use_a ? 1 : 0,
                                                             use_p ? 1 : 0, q->p64.as<double>());
        YQ_LAUNCH_CHECK();
        YQ_CUDA(cudaStreamSynchronize(st));
        double gn = 0.;
        for (double x : grad) gn += x * x;
        if (energy) *energy = g->energy;
        if (grad_norm) *grad_norm = std::sqrt(gn);
        if (v_norm) *v_norm = std::sqrt(vn);
    });
}

}  // extern "C"
