// FeedForward machine on the device (Machines/FeedForward.hpp with the layers
// Conv1D (layers/Conv1D.hpp:144-225, one input channel, periodic, no bias),
// LnCosh (layers/activations.hpp:74-107), FullyConnected (layers/FullyConnected.hpp
// :150-179, no bias) and a Sum output (= fc_out x Mean, layers/Mean.hpp:92-125)).
//
//   forward:  z1 = conv(sigma), a1 = logcosh(z1), z2 = W^T a1, log psi = sum logcosh(z2)
//   adjoint:  d2 = tanh(z2); dW = a1 d2^T; d1 = (W d2) * tanh(z1); dker = corr(sigma, d1)
//             (FeedForward::backward with dout = 1, FeedForward.hpp:186-205), written as
//             the log-derivative row O = [dker (K x C) | dW ((L C) x F)].
// The adjoint reads the activations the forward stored when batch x (L C + F)
// floats fit the caller's budget, and recomputes them otherwise.
// E_loc of the TFI chain uses single-flip updates: flipping site i changes K
// conv outputs per channel, so log psi(sigma^i) - log psi(sigma) costs K C
// logcosh and K C F multiply-adds instead of a full forward pass.
#include <algorithm>
#include <cmath>
#include <vector>

#include "internal.hpp"

namespace yq {

void record_error(const std::string& msg);

namespace {
constexpr int FF_SB = 8;  // samples per block in the forward / adjoint kernels

__device__ __forceinline__ float logcoshf_ref(float x) {
    // Utilities/Utility.hpp:14-24
    const float xp = fabsf(x);
    return xp <= 12.f ? logf(coshf(xp)) : xp - 0.69314718055994530942f;
}

struct FFDims {
    int L, C, K, F, LC, KC;
    size_t P;
};

// z1 = conv(sigma), a1 = logcosh(z1) (each evaluated once) and z2 = W^T a1 for nsb
// <= FF_SB samples into shared memory.
__device__ void ff_forward_block(const FFDims& d, const float* __restrict__ ker, const float* __restrict__ Wfc,
                                 const float* s_sig /*[SB][L]*/, float* s_z1 /*[SB][LC]*/, float* s_a1 /*[SB][LC]*/,
                                 float* s_z2 /*[SB][F]*/, int nsb) {
    const int tid = threadIdx.x, nt = blockDim.x, warp = tid >> 5, lane = tid & 31, nw = nt >> 5;
    for (int e = tid; e < nsb * d.LC; e += nt) {
        const int s = e / d.LC, q = e % d.LC, oc = q / d.L, r = q % d.L;
        float acc = 0.f;
        for (int ki = 0; ki < d.K; ++ki) acc += ker[ki + d.K * oc] * s_sig[s * d.L + (r + ki - d.K / 2 + d.L) % d.L];
        s_z1[s * d.LC + q] = acc;
        s_a1[s * d.LC + q] = logcoshf_ref(acc);
    }
    __syncthreads();
    for (int pr = warp; pr < nsb * d.F; pr += nw) {
        const int s = pr / d.F, o = pr % d.F;
        float acc = 0.f;
        for (int i = lane; i < d.LC; i += 32) acc += s_a1[s * d.LC + i] * Wfc[i + size_t(d.LC) * o];
#pragma unroll
        for (int off = 16; off > 0; off >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, off);
        if (lane == 0) s_z2[s * d.F + o] = acc;
    }
    __syncthreads();
}

__global__ void ff_forward_kernel(FFDims d, int batch, const float* __restrict__ params,
                                  const int8_t* __restrict__ sigma, double* __restrict__ logpsi,
                                  float* __restrict__ acts) {
    extern __shared__ float sm[];
    float* s_sig = sm;                    // SB * L
    float* s_z1 = s_sig + FF_SB * d.L;    // SB * LC
    float* s_z2 = s_z1 + FF_SB * d.LC;    // SB * F
    float* s_a1 = s_z2 + FF_SB * d.F;     // SB * LC
    const int b0 = blockIdx.x * FF_SB, nsb = min(FF_SB, batch - b0);
    for (int e = threadIdx.x; e < nsb * d.L; e += blockDim.x) s_sig[e] = float(sigma[size_t(b0) * d.L + e]);
    __syncthreads();
    ff_forward_block(d, params, params + d.KC, s_sig, s_z1, s_a1, s_z2, nsb);
    if (threadIdx.x < nsb) {
        double lp = 0.;
        for (int o = 0; o < d.F; ++o) lp += double(logcoshf_ref(s_z2[threadIdx.x * d.F + o]));
        logpsi[b0 + threadIdx.x] = lp;
    }
    if (acts) {
        const int w = d.LC + d.F;
        for (int e = threadIdx.x; e < nsb * w; e += blockDim.x) {
            const int s = e / w, q = e % w;
            acts[size_t(b0 + s) * w + q] = q < d.LC ? s_z1[s * d.LC + q] : s_z2[s * d.F + q - d.LC];
        }
    }
}

__global__ void ff_adjoint_kernel(FFDims d, int batch, const float* __restrict__ params,
                                  const int8_t* __restrict__ sigma, const float* __restrict__ acts,
                                  float* __restrict__ O) {
    extern __shared__ float sm[];
    float* s_sig = sm;                    // SB * L
    float* s_z1 = s_sig + FF_SB * d.L;    // SB * LC   (z1, then reused for dz1)
    float* s_z2 = s_z1 + FF_SB * d.LC;    // SB * F    (z2, then d2)
    float* s_a1 = s_z2 + FF_SB * d.F;     // SB * LC
    const float* ker = params;
    const float* Wfc = params + d.KC;
    const int b0 = blockIdx.x * FF_SB, nsb = min(FF_SB, batch - b0);
    const int tid = threadIdx.x, nt = blockDim.x;
    for (int e = tid; e < nsb * d.L; e += nt) s_sig[e] = float(sigma[size_t(b0) * d.L + e]);
    if (acts) {
        const int w = d.LC + d.F;
        for (int e = tid; e < nsb * w; e += nt) {
            const int s = e / w, q = e % w;
            const float v = acts[size_t(b0 + s) * w + q];
            if (q < d.LC)
                s_z1[s * d.LC + q] = v;
            else
                s_z2[s * d.F + q - d.LC] = v;
        }
        __syncthreads();
        for (int e = tid; e < nsb * d.LC; e += nt) s_a1[e] = logcoshf_ref(s_z1[e]);
    } else {
        __syncthreads();
        ff_forward_block(d, ker, Wfc, s_sig, s_z1, s_a1, s_z2, nsb);
    }
    for (int e = tid; e < nsb * d.F; e += nt) s_z2[e] = tanhf(s_z2[e]);  // d2 = 1 * tanh(z2)
    __syncthreads();
    // FullyConnected.hpp:170-172: der_w = a1 d2^T, column-major (LC x F) after the conv block.
    // With KC, LC and P multiples of 4 the block is written as aligned float4 runs
    // of a1 (one 16-byte store per thread and step); otherwise one float at a time.
    if ((d.KC & 3) == 0 && (d.LC & 3) == 0 && (d.P & 3) == 0) {
        const int lc4 = d.LC >> 2, tot4 = lc4 * d.F;
        const float4* a14 = reinterpret_cast<const float4*>(s_a1);
        for (int e = tid; e < tot4; e += nt) {
            const int o = e / lc4, i4 = e - o * lc4;
            for (int s = 0; s < nsb; ++s) {
                const float4 a = a14[s * lc4 + i4];
                const float g = s_z2[s * d.F + o];
                *reinterpret_cast<float4*>(O + size_t(b0 + s) * d.P + d.KC + size_t(4) * e) =
                    make_float4(a.x * g, a.y * g, a.z * g, a.w * g);
            }
        }
    } else {
        for (int s = 0; s < nsb; ++s) {
            float* row = O + size_t(b0 + s) * d.P + d.KC;
            for (int e = tid; e < d.LC * d.F; e += nt) {
                const int o = e / d.LC, i = e % d.LC;
                row[e] = s_a1[s * d.LC + i] * s_z2[s * d.F + o];
            }
        }
    }
    // d1 = W d2, then the LnCosh Jacobian: dz1 = d1 * tanh(z1) (in place of z1); a
    // thread per input i keeps the block's samples in registers, so each weight is
    // read once per block
    for (int i = tid; i < d.LC; i += nt) {
        float acc[FF_SB];
#pragma unroll
        for (int s = 0; s < FF_SB; ++s) acc[s] = 0.f;
        for (int o = 0; o < d.F; ++o) {
            const float w = Wfc[i + size_t(d.LC) * o];
#pragma unroll
            for (int s = 0; s < FF_SB; ++s) acc[s] += w * s_z2[s * d.F + o];
        }
#pragma unroll
        for (int s = 0; s < FF_SB; ++s)
            if (s < nsb) s_z1[s * d.LC + i] = acc[s] * tanhf(s_z1[s * d.LC + i]);
    }
    __syncthreads();
    // Conv1D.hpp:197-212: dw(ki, oc) = sum_r in((r + ki - K/2) mod L) dz1(r + oc L)
    for (int e = tid; e < nsb * d.KC; e += nt) {
        const int s = e / d.KC, q = e % d.KC, oc = q / d.K, ki = q % d.K;
        float acc = 0.f;
        for (int r = 0; r < d.L; ++r) acc += s_sig[s * d.L + (r + ki - d.K / 2 + d.L) % d.L] * s_z1[s * d.LC + r + oc * d.L];
        O[size_t(b0 + s) * d.P + q] = acc;
    }
}

// E_loc for the TFI chain (Hamiltonians/TFIsing.hpp:28-39): one block per sample,
// thread i evaluates log psi(sigma^i) - log psi(sigma) by a local update.
__global__ void ff_eloc_tfi_kernel(FFDims d, int batch, double J, double h, const float* __restrict__ params,
                                   const int8_t* __restrict__ sigma, c128* __restrict__ eloc,
                                   int* __restrict__ status) {
    extern __shared__ float sm[];
    float* s_sig = sm;             // L
    float* s_z1 = s_sig + d.L;     // LC
    float* s_z2 = s_z1 + d.LC;     // F
    float* s_a1 = s_z2 + d.F;      // LC
    __shared__ double red[32];
    const float* ker = params;
    const float* Wfc = params + d.KC;
    const int b = blockIdx.x, tid = threadIdx.x;
    for (int e = tid; e < d.L; e += blockDim.x) s_sig[e] = float(sigma[size_t(b) * d.L + e]);
    __syncthreads();
    ff_forward_block(d, ker, Wfc, s_sig, s_z1, s_a1, s_z2, 1);
    double acc = 0.;
    for (int i = tid; i < d.L; i += blockDim.x) {
        const float si = s_sig[i];
        // diagonal: J s_i s_{i+1}
        acc += J * double(si) * double(s_sig[(i + 1) % d.L]);
        // off-diagonal ratio for flipping site i
        float dz2[64];
        for (int o = 0; o < d.F; ++o) dz2[o] = 0.f;
        for (int oc = 0; oc < d.C; ++oc)
            for (int ki = 0; ki < d.K; ++ki) {
                const int r = ((i - ki + d.K / 2) % d.L + d.L) % d.L;  // output positions that read input i
                const int q = r + oc * d.L;
                const float z = s_z1[q];
                const float zn = z - 2.f * si * ker[ki + d.K * oc];
                const float da = logcoshf_ref(zn) - logcoshf_ref(z);
                for (int o = 0; o < d.F; ++o) dz2[o] += Wfc[q + size_t(d.LC) * o] * da;
            }
        double lr = 0.;
        for (int o = 0; o < d.F; ++o)
            lr += double(logcoshf_ref(s_z2[o] + dz2[o])) - double(logcoshf_ref(s_z2[o]));
        acc += h * exp(lr);
    }
#pragma unroll
    for (int off = 16; off > 0; off >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, off);
    if ((tid & 31) == 0) red[tid >> 5] = acc;
    __syncthreads();
    if (tid == 0) {
        double e = 0.;
        for (int w = 0; w < int(blockDim.x >> 5); ++w) e += red[w];
        eloc[b] = mk(e, 0.0);
        if (!isfinite(e)) atomicOr(status, DS_NONFINITE);
    }
}

__global__ void ff_random_batch_kernel(int batch, int L, uint64_t seed, int8_t* __restrict__ sigma) {
    const size_t n = size_t(batch) * L;
    for (size_t e = size_t(blockIdx.x) * blockDim.x + threadIdx.x; e < n; e += size_t(gridDim.x) * blockDim.x) {
        U4 x = draw(seed, uint32_t(e % L), 0u, uint32_t(e / L), TAG_INIT);
        sigma[e] = (x.x & 1u) ? int8_t(-1) : int8_t(1);
    }
}

FFDims dims(const yq_ff_s* f) {
    return FFDims{f->L, f->C, f->K, f->F, f->L * f->C, f->K * f->C, f->P};
}

template <class Fn>
int guard_ff(Fn&& fn) {
    try {
        fn();
        return YQ_OK;
    } catch (const Error& e) {
        record_error(e.what());
        return e.code;
    } catch (const std::exception& e) {
        record_error(e.what());
        return YQ_E_ARG;
    }
}

void need_batch(const yq_ff_s* f) {
    if (f->batch <= 0) throw Error(YQ_E_STATE, "feedforward: set a batch first");
}

size_t fwd_smem(const FFDims& d) { return size_t(FF_SB) * (d.L + 2 * d.LC + d.F) * sizeof(float); }
size_t adj_smem(const FFDims& d) { return size_t(FF_SB) * (d.L + 2 * d.LC + d.F) * sizeof(float); }

void set_smem_attr(const void* fn, size_t bytes) {
    if (bytes > 48 * 1024) YQ_CUDA(cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, int(bytes)));
}
}  // namespace
}  // namespace yq

using namespace yq;

extern "C" {

int yq_ff_create(yq_ctx ctx, int L, int channels, int kernel, int fc_out, yq_ff* out) {
    return guard_ff([&] {
        if (!ctx || !out) throw Error(YQ_E_ARG, "ff_create: null argument");
        *out = nullptr;
        if (L < 2 || channels < 1 || kernel < 1 || kernel > L || fc_out < 1 || fc_out > 64 || L * channels > 8192)
            throw Error(YQ_E_ARG, "ff_create: need 2 <= L, 1 <= kernel <= L, 1 <= fc_out <= 64, L * channels <= 8192");
        auto* f = new yq_ff_s();
        f->ctx = ctx;
        f->L = L;
        f->C = channels;
        f->K = kernel;
        f->F = fc_out;
        f->P = size_t(kernel) * channels + size_t(L) * channels * fc_out;
        try {
            f->params.ensure(f->P * sizeof(float));
            YQ_CUDA(cudaMemsetAsync(f->params.p, 0, f->P * sizeof(float), ctx->stream));
        } catch (...) {
            delete f;
            throw;
        }
        *out = f;
    });
}

int yq_ff_destroy(yq_ff f) {
    return guard_ff([&] {
        if (!f) return;
        cudaStreamSynchronize(f->ctx->stream);
        delete f;
    });
}

int yq_ff_dim(yq_ff f, size_t* dim) {
    return guard_ff([&] {
        if (!f || !dim) throw Error(YQ_E_ARG, "ff_dim: null argument");
        *dim = f->P;
    });
}

int yq_ff_set_params(yq_ff f, const double* params) {
    return guard_ff([&] {
        if (!f || !params) throw Error(YQ_E_ARG, "ff_set_params: null argument");
        std::vector<float> v(params, params + f->P);
        YQ_CUDA(cudaMemcpyAsync(f->params.p, v.data(), f->P * sizeof(float), cudaMemcpyHostToDevice, f->ctx->stream));
        YQ_CUDA(cudaStreamSynchronize(f->ctx->stream));
        f->acts_valid = false;
    });
}

int yq_ff_get_params(yq_ff f, double* params) {
    return guard_ff([&] {
        if (!f || !params) throw Error(YQ_E_ARG, "ff_get_params: null argument");
        std::vector<float> v(f->P);
        YQ_CUDA(cudaMemcpyAsync(v.data(), f->params.p, f->P * sizeof(float), cudaMemcpyDeviceToHost, f->ctx->stream));
        YQ_CUDA(cudaStreamSynchronize(f->ctx->stream));
        std::copy(v.begin(), v.end(), params);
    });
}

// FeedForward::initializeRandom(re, Xavier) (FeedForward.hpp:42-73): per layer N(0, sqrt(2 / (fanIn + fanOut)))
// with Conv1D fanIn = K, fanOut = C K (Conv1D.hpp:227-234) and FullyConnected fanIn = L C, fanOut = F.
int yq_ff_init_random(yq_ff f, uint64_t seed) {
    return guard_ff([&] {
        if (!f) throw Error(YQ_E_ARG, "ff_init_random: null argument");
        std::vector<float> v(f->P);
        const double s_conv = std::sqrt(2.0 / (f->K + f->C * f->K));
        const double s_fc = std::sqrt(2.0 / (f->L * f->C + f->F));
        const size_t kc = size_t(f->K) * f->C;
        for (size_t e = 0; e < f->P; ++e) {
            U4 x = draw(seed, uint32_t(e), 0u, 0u, TAG_PARAM);
            const double u1 = 1.0 - draw_u53(x.x, x.y), u2 = draw_u53(x.z, x.w);
            const double z = std::sqrt(-2.0 * std::log(u1)) * std::cos(6.283185307179586476925286766559 * u2);
            v[e] = float(z * (e < kc ? s_conv : s_fc));
        }
        YQ_CUDA(cudaMemcpyAsync(f->params.p, v.data(), f->P * sizeof(float), cudaMemcpyHostToDevice, f->ctx->stream));
        YQ_CUDA(cudaStreamSynchronize(f->ctx->stream));
        f->acts_valid = false;
    });
}

int yq_ff_set_batch(yq_ff f, int batch, const int8_t* sigma) {
    return guard_ff([&] {
        if (!f || !sigma || batch < 1) throw Error(YQ_E_ARG, "ff_set_batch: null argument or batch < 1");
        for (size_t i = 0; i < size_t(batch) * f->L; ++i)
            if (sigma[i] != 1 && sigma[i] != -1) throw Error(YQ_E_ARG, "sigma entries must be +1 or -1");
        f->sigma.ensure(size_t(batch) * f->L);
        YQ_CUDA(cudaMemcpyAsync(f->sigma.p, sigma, size_t(batch) * f->L, cudaMemcpyHostToDevice, f->ctx->stream));
        YQ_CUDA(cudaStreamSynchronize(f->ctx->stream));
        f->batch = batch;
        f->acts_valid = false;
    });
}

int yq_ff_random_batch(yq_ff f, int batch, uint64_t seed) {
    return guard_ff([&] {
        if (!f || batch < 1) throw Error(YQ_E_ARG, "ff_random_batch: null argument or batch < 1");
        f->sigma.ensure(size_t(batch) * f->L);
        ff_random_batch_kernel<<<std::min(cdiv_u(size_t(batch) * f->L, 256), 148u * 16), 256, 0, f->ctx->stream>>>(
            batch, f->L, seed, f->sigma.as<int8_t>());
        YQ_LAUNCH_CHECK();
        f->batch = batch;
        f->acts_valid = false;
    });
}

int yq_ff_forward(yq_ff f, size_t act_budget_bytes, double* logpsi) {
    return guard_ff([&] {
        if (!f) throw Error(YQ_E_ARG, "ff_forward: null argument");
        need_batch(f);
        const FFDims d = dims(f);
        cudaStream_t st = f->ctx->stream;
        f->logpsi.ensure(size_t(f->batch) * sizeof(double));
        const size_t act_bytes = size_t(f->batch) * (d.LC + d.F) * sizeof(float);
        const bool store = act_bytes <= act_budget_bytes;
        if (store) f->acts.ensure(act_bytes);
        set_smem_attr(reinterpret_cast<const void*>(ff_forward_kernel), fwd_smem(d));
        f->ctx->stage_begin(ST_FF_FORWARD);
        ff_forward_kernel<<<cdiv_u(f->batch, FF_SB), 256, fwd_smem(d), st>>>(
            d, f->batch, f->params.as<float>(), f->sigma.as<int8_t>(), f->logpsi.as<double>(),
            store ? f->acts.as<float>() : nullptr);
        YQ_LAUNCH_CHECK();
        f->ctx->stage_end(ST_FF_FORWARD);
        f->acts_valid = store;
        if (logpsi) {
            YQ_CUDA(cudaMemcpyAsync(logpsi, f->logpsi.p, size_t(f->batch) * sizeof(double), cudaMemcpyDeviceToHost, st));
            YQ_CUDA(cudaStreamSynchronize(st));
        }
    });
}

int yq_ff_adjoint(yq_ff f, double* O) {
    return guard_ff([&] {
        if (!f) throw Error(YQ_E_ARG, "ff_adjoint: null argument");
        need_batch(f);
        const FFDims d = dims(f);
        cudaStream_t st = f->ctx->stream;
        f->O.ensure(size_t(f->batch) * f->P * sizeof(float));
        set_smem_attr(reinterpret_cast<const void*>(ff_adjoint_kernel), adj_smem(d));
        f->ctx->stage_begin(ST_FF_ADJOINT);
        ff_adjoint_kernel<<<cdiv_u(f->batch, FF_SB), 256, adj_smem(d), st>>>(
            d, f->batch, f->params.as<float>(), f->sigma.as<int8_t>(), f->acts_valid ? f->acts.as<float>() : nullptr,
            f->O.as<float>());
        YQ_LAUNCH_CHECK();
        f->ctx->stage_end(ST_FF_ADJOINT);
        if (O) {
            std::vector<float> tmp(size_t(f->batch) * f->P);
            YQ_CUDA(cudaMemcpyAsync(tmp.data(), f->O.p, tmp.size() * sizeof(float), cudaMemcpyDeviceToHost, st));
            YQ_CUDA(cudaStreamSynchronize(st));
            std::copy(tmp.begin(), tmp.end(), O);
        }
    });
}

int yq_ff_eloc_tfi(yq_ff f, double J, double h, double* eloc) {
    return guard_ff([&] {
        if (!f) throw Error(YQ_E_ARG, "ff_eloc_tfi: null argument");
        need_batch(f);
        const FFDims d = dims(f);
        cudaStream_t st = f->ctx->stream;
        f->eloc.ensure(size_t(f->batch) * sizeof(c128));
        const size_t smem = size_t(d.L + 2 * d.LC + d.F) * sizeof(float);
        set_smem_attr(reinterpret_cast<const void*>(ff_eloc_tfi_kernel), smem);
        const int threads = std::max(32, std::min(256, ((d.L + 31) / 32) * 32));
        f->ctx->stage_begin(ST_FF_ELOC);
        ff_eloc_tfi_kernel<<<f->batch, threads, smem, st>>>(d, f->batch, J, h, f->params.as<float>(),
                                                          f->sigma.as<int8_t>(), f->eloc.as<c128>(),
                                                          f->ctx->status.as<int>());
        YQ_LAUNCH_CHECK();
        f->ctx->stage_end(ST_FF_ELOC);
        if (eloc) {
            YQ_CUDA(cudaMemcpyAsync(eloc, f->eloc.p, size_t(f->batch) * sizeof(c128), cudaMemcpyDeviceToHost, st));
            YQ_CUDA(cudaStreamSynchronize(st));
        }
    });
}

}  // extern "C"
