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

#include "internal.hpp"

namespace yq {

constexpr size_t NOALLOC_SCRATCH_BYTES = size_t(4) << 20;
static __device__ __align__(256) unsigned char g_noalloc_scratch[NOALLOC_SCRATCH_BYTES];

void record_error(const std::string& msg);  // capi.cu

namespace {
constexpr int TS = 8;  // samples staged per step

// Partial sums over a chunk of samples of s_i t_j, t_j = tanh(theta_j), for rows
// i in [0, n] and columns j in [0, m]: row i = n (s := 1) sums t_j, the gradient of
// the hidden bias b_j; column j = m (t := 1) sums s_i, the gradient of the visible
// bias a_i; the others are the W_ji entries.  A block covers 32 columns x 32 rows
// (a thread keeps four rows of one column) and stages, for TS samples at a time,
// tanh(theta) of its 32 columns and sigma of its 32 rows in shared memory, so each
// tanh is evaluated once per block rather than once per row.
template <typename R>
__global__ void __launch_bounds__(256) oloc_partial_noalloc_kernel(int n, int m, int ns, int chunk,
                                                                   const int8_t* __restrict__ sigma,
                                                                   const cplx<R>* __restrict__ theta,
                                                                   c128* __restrict__ part) {
    __shared__ double t_re[TS][32], t_im[TS][32];
    __shared__ double s_v[TS][32];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int jb = blockIdx.x * 32, ib = blockIdx.y * 32;
    const int j = jb + lane;
    const int split = blockIdx.z;
    const int s0 = split * chunk, s1 = min(ns, s0 + chunk);
    double ar[4] = {0., 0., 0., 0.}, ai[4] = {0., 0., 0., 0.};
    for (int sb = s0; sb < s1; sb += TS) {
        // one (sample, column) tanh and one (sample, row) spin per thread
        {
            const int ss = threadIdx.x >> 5, c = threadIdx.x & 31;
            const int s = sb + ss;
            double tr = 0., ti = 0., sv = 0.;
            if (s < s1) {
                const int jj = jb + c, ii = ib + c;
                if (jj < m) {
                    const cplx<R> tv = ctanh(theta[size_t(s) * m + jj]);
                    tr = double(tv.re);
                    ti = double(tv.im);
                } else if (jj == m) {
                    tr = 1.0;
                }
                if (ii < n)
                    sv = double(sigma[size_t(s) * n + ii]);
                else if (ii == n)
                    sv = 1.0;
            }
            t_re[ss][c] = tr;
            t_im[ss][c] = ti;
            s_v[ss][c] = sv;
        }
        __syncthreads();
#pragma unroll
        for (int ss = 0; ss < TS; ++ss) {
            const double tr = t_re[ss][lane], ti = t_im[ss][lane];
#pragma unroll
            for (int k = 0; k < 4; ++k) {
                const double sv = s_v[ss][warp * 4 + k];
                ar[k] += sv * tr;
                ai[k] += sv * ti;
            }
        }
        __syncthreads();
    }
    if (j > m) return;
#pragma unroll
    for (int k = 0; k < 4; ++k) {
        const int i = ib + warp * 4 + k;
        if (i <= n) part[size_t(split) * (n + 1) * (m + 1) + size_t(i) * (m + 1) + j] = mk(ar[k], ai[k]);
    }
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

// Device address of the scratch array for this context's device, looked up at the
// context's first call of the entry point with that device current.  It is kept
// with the context: a device reset, which ends every context's stream and buffers,
// cannot leave a stale address behind for a new context.
void* scratch_address(yq_ctx_s* ctx) {
    if (!ctx->noalloc_scratch) {
        void* p = nullptr;
        cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
        if (e != cudaSuccess || !p)
            throw Error(YQ_E_CUDA, std::string("oloc_noalloc: cudaGetSymbolAddress failed: ") + cudaGetErrorString(e));
        ctx->noalloc_scratch = p;
    }
    return ctx->noalloc_scratch;
}

template <typename R>
void oloc_noalloc_t(yq_rbm_s* q, int ns, const int8_t* d_sigma, const void* d_theta, c128* d_oloc, c128* part) {
    const int n = q->n, m = q->m;
    const size_t cnt = size_t(n + 1) * (m + 1);
    const size_t cap = NOALLOC_SCRATCH_BYTES / sizeof(c128);
    dim3 g(cdiv_u(m + 1, 32), cdiv_u(n + 1, 32), 1);
    int nsplit = int(std::min<size_t>(64, cap / cnt));
    nsplit = std::max(1, std::min({nsplit, ns, std::max(1, int((8 * 148) / std::max(1u, g.x * g.y)))}));
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
        c128* part = static_cast<c128*>(scratch_address(q->ctx));
        // only sigma and theta are read: the machine's parameters play no part
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
