// yq_rbm_oloc_noalloc: the column mean of the log-derivative rows, computed from
// samples the caller already holds on the device, without any device allocation.
//
// Why it exists: some callers cannot let a library call cudaMalloc -- a host
// framework that has reserved the device for its own allocator, or a service loop
// where an allocation's latency and implicit synchronisation are not acceptable.
// This entry point takes device input and output pointers from the caller and
// keeps its only temporary data (the partial sums of a two-stage reduction) in a
// fixed array in device global memory, compiled into the library.
//
// The array is NOALLOC_SCRATCH_BYTES (4 MiB) and every GPU that loads the library
// holds it until the process exits.  All calls share it: calls that overlap on the
// GPU (from different streams, contexts or threads) race on it and must be
// serialised by the caller.  Every partial slot a call reads was written earlier
// by the same call, so nothing has to be cleared between calls.
#include <algorithm>
#include <mutex>

#include "internal.hpp"

namespace yq {

constexpr size_t NOALLOC_SCRATCH_BYTES = size_t(4) << 20;
static __device__ __align__(256) unsigned char g_noalloc_scratch[NOALLOC_SCRATCH_BYTES];

void record_error(const std::string& msg);  // capi.cu

namespace {
// Partial sums over a chunk of samples of s_i tanh(theta_j) for i in [0, n]
// (i = n stands for s := 1, the b block) and j in [0, m] (j = m: t := 1, the a block),
// with tanh(theta) evaluated in place (the SR object keeps a tanh buffer instead).
template <typename R>
__global__ void oloc_partial_noalloc_kernel(int n, int m, int ns, int chunk, const int8_t* __restrict__ sigma,
                                            const cplx<R>* __restrict__ theta, c128* __restrict__ part) {
    const int j = blockIdx.x * 32 + (threadIdx.x & 31);
    const int i = blockIdx.y * 8 + (threadIdx.x >> 5);
    const int split = blockIdx.z;
    if (i > n || j > m) return;
    const int s0 = split * chunk, s1 = min(ns, s0 + chunk);
    double ar = 0., ai = 0.;
    for (int s = s0; s < s1; ++s) {
        const double sv = (i < n) ? double(sigma[size_t(s) * n + i]) : 1.0;
        if (j < m) {
            const cplx<R> tv = ctanh(theta[size_t(s) * m + j]);
            ar += sv * double(tv.re);
            ai += sv * double(tv.im);
        } else {
            ar += sv;
        }
    }
    part[size_t(split) * (n + 1) * (m + 1) + size_t(i) * (m + 1) + j] = mk(ar, ai);
}

__global__ void oloc_finish_noalloc_kernel(int n, int m, bool bias, int nsplit, double inv_ns,
                                           const c128* __restrict__ part, c128* __restrict__ oloc) {
    const size_t cnt = size_t(n + 1) * (m + 1);
    for (size_t q = size_t(blockIdx.x) * blockDim.x + threadIdx.x; q < cnt; q += size_t(gridDim.x) * blockDim.x) {
        c128 acc = mk(0., 0.);
        for (int sp = 0; sp < nsplit; ++sp) acc = acc + part[size_t(sp) * cnt + q];
        acc = inv_ns * acc;
        const int i = int(q / (m + 1)), j = int(q % (m + 1));
        const size_t nm = size_t(n) * m;
        if (i < n && j < m)
            oloc[size_t(i) * m + j] = acc;
        else if (bias && i < n && j == m)
            oloc[nm + i] = acc;
        else if (bias && i == n && j < m)
            oloc[nm + n + j] = acc;
    }
}

// Device address of the scratch array, looked up once per device (with that device current).
void* scratch_address(int device) {
    static std::mutex mu;
    static void* addr[64] = {};
    YQ_CHECK_ARG(device >= 0 && device < 64, "oloc_noalloc: device index out of range");
    std::lock_guard<std::mutex> lock(mu);
    if (!addr[device]) {
        void* p = nullptr;
        cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
        if (e != cudaSuccess || !p)
            throw Error(YQ_E_CUDA, std::string("oloc_noalloc: cudaGetSymbolAddress failed: ") + cudaGetErrorString(e));
        addr[device] = p;
    }
    return addr[device];
}

template <typename R>
void oloc_noalloc_t(yq_rbm_s* q, int ns, const int8_t* d_sigma, const void* d_theta, c128* d_oloc, c128* part) {
    const int n = q->n, m = q->m;
    const size_t cnt = size_t(n + 1) * (m + 1);
    const size_t cap = NOALLOC_SCRATCH_BYTES / sizeof(c128);
    dim3 g(cdiv_u(m + 1, 32), cdiv_u(n + 1, 8), 1);
    int nsplit = int(std::min<size_t>(64, cap / cnt));
    nsplit = std::max(1, std::min(nsplit, ns));
    const int chunk = (ns + nsplit - 1) / nsplit;
    g.z = nsplit;
    cudaStream_t st = q->ctx->stream;
    oloc_partial_noalloc_kernel<R><<<g, 256, 0, st>>>(n, m, ns, chunk, d_sigma, reinterpret_cast<const cplx<R>*>(d_theta),
                                                      part);
    YQ_LAUNCH_CHECK();
    oloc_finish_noalloc_kernel<<<cdiv_u(cnt, 256), 256, 0, st>>>(n, m, q->use_bias, nsplit, 1.0 / ns, part, d_oloc);
    YQ_LAUNCH_CHECK();
}
}  // namespace
}  // namespace yq

using namespace yq;

extern "C" int yq_rbm_oloc_noalloc(yq_rbm q, int ns, const int8_t* d_sigma, const void* d_theta, double* d_oloc) {
    try {
        if (!q || !d_sigma || !d_theta || !d_oloc) throw Error(YQ_E_ARG, "oloc_noalloc: null argument");
        if (ns < 1) throw Error(YQ_E_ARG, "oloc_noalloc: ns must be >= 1");
        const size_t cnt = size_t(q->n + 1) * (q->m + 1);
        if (cnt * sizeof(c128) > NOALLOC_SCRATCH_BYTES)
            throw Error(YQ_E_ARG, "oloc_noalloc: (n + 1) (m + 1) = " + std::to_string(cnt) +
                                      " exceeds the static scratch of 4 MiB (at most 262144 complex partial sums)");
        YQ_CUDA(cudaSetDevice(q->ctx->device));
        c128* part = static_cast<c128*>(scratch_address(q->ctx->device));
        rbm_prepare(q);  // refreshes derived arrays allocated when the RBM was created
        if (q->dtype == YQ_C64)
            oloc_noalloc_t<float>(q, ns, d_sigma, d_theta, reinterpret_cast<c128*>(d_oloc), part);
        else
            oloc_noalloc_t<double>(q, ns, d_sigma, d_theta, reinterpret_cast<c128*>(d_oloc), part);
        return YQ_OK;
    } catch (const Error& e) {
        record_error(e.what());
        return e.code;
    } catch (const std::exception& e) {
        record_error(e.what());
        return YQ_E_ARG;
    }
}
