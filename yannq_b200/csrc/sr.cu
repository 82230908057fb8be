// Stochastic reconfiguration on the device (GroundState/SRMat.hpp):
//   E_loc -> FP64 statistics -> structured column mean of O -> centred O writer
//   -> F = O~^H (E - <E>) / Ns -> S = O~^H O~ / Ns (P x P) or its sample-space dual
//   T = O~ O~^H / Ns (Ns x Ns) -> blocked FP64 Cholesky -> triangular solves ->
//   v (= O~^H y in T-mode) -> SGD update of the FP64 master parameters.
#include <algorithm>
#include <cmath>
#include <vector>

#include "chol.hpp"
#include "gemm64.cuh"
#include "gram_tc.hpp"
#include "internal.hpp"

namespace yq {

static constexpr int NB = CHOL_NB;  // Cholesky block size

// ---------------------------------------------------------------------------
template <typename R>
__global__ void tanh_kernel(size_t count, const cplx<R>* __restrict__ th, cplx<R>* __restrict__ t) {
    for (size_t i = size_t(blockIdx.x) * blockDim.x + threadIdx.x; i < count; i += size_t(gridDim.x) * blockDim.x)
        t[i] = ctanh(th[i]);
}

// Observables/Energy.hpp:53-58 with compensated (Kahan) FP64 sums:
// stats = {E = <Re E_loc>, Var = <Re E_loc^2> - E^2, <E_loc>.re, <E_loc>.im}
__global__ void energy_stats_kernel(int ns, const c128* __restrict__ e, double* __restrict__ stats,
                                    int* __restrict__ status) {
    __shared__ double sh[4][256];
    double s[4] = {0, 0, 0, 0}, c[4] = {0, 0, 0, 0};
    for (int i = threadIdx.x; i < ns; i += blockDim.x) {
        double v[4] = {e[i].re, e[i].re * e[i].re, e[i].re, e[i].im};
#pragma unroll
        for (int q = 0; q < 4; ++q) {
            double y = v[q] - c[q];
            double t = s[q] + y;
            c[q] = (t - s[q]) - y;
            s[q] = t;
        }
    }
#pragma unroll
    for (int q = 0; q < 4; ++q) sh[q][threadIdx.x] = s[q];
    __syncthreads();
    if (threadIdx.x == 0) {
        double tot[4];
        for (int q = 0; q < 4; ++q) {
            double ss = 0., cc = 0.;
            for (int k = 0; k < blockDim.x; ++k) {
                double y = sh[q][k] - cc;
                double t = ss + y;
                cc = (t - ss) - y;
                ss = t;
            }
            tot[q] = ss / ns;
        }
        stats[0] = tot[0];
        stats[1] = tot[1] - tot[0] * tot[0];
        stats[2] = tot[2];
        stats[3] = tot[3];
        if (!isfinite(tot[0]) || !isfinite(tot[3])) atomicOr(status, DS_NONFINITE);
    }
}

// Column mean of O without forming O (the RBM's O row is [s_i t_j | s | t]):
// part[split][i][j] = sum over the split's samples of s_i t_j for i in [0, n]
// (i = n: s := 1, the b block) and j in [0, m] (j = m: t := 1, the a block).  A
// thread keeps four rows i for one column j, so one load of t_j feeds eight FP64
// FMAs; a block covers 32 columns x 32 rows.
template <typename R>
__global__ void __launch_bounds__(256) oloc_partial_kernel(int n, int m, int ns, int chunk,
                                                           const int8_t* __restrict__ sigma,
                                                           const cplx<R>* __restrict__ t, c128* __restrict__ part) {
    const int j = blockIdx.x * 32 + (threadIdx.x & 31);
    const int i0 = blockIdx.y * 32 + (threadIdx.x >> 5) * 4;
    const int split = blockIdx.z;
    if (i0 > n || j > m) return;
    const int s0 = split * chunk, s1 = min(ns, s0 + chunk);
    double ar[4] = {0., 0., 0., 0.}, ai[4] = {0., 0., 0., 0.};
    // the four spins of a thread as one 4-byte load when the rows allow it (n a
    // multiple of 4, all four inside the row); the spin row is the same for the
    // warp's 32 threads
    const bool packed = (n & 3) == 0 && i0 + 4 <= n;
    for (int s = s0; s < s1; ++s) {
        const cplx<R> tv = (j < m) ? t[size_t(s) * m + j] : mk(R(1), R(0));
        const double tr = double(tv.re), ti = double(tv.im);
        const int8_t* sg = sigma + size_t(s) * n;
        double sv[4];
        if (packed) {
            const uint32_t w = *reinterpret_cast<const uint32_t*>(sg + i0);
#pragma unroll
            for (int k = 0; k < 4; ++k) sv[k] = double(int8_t((w >> (8 * k)) & 0xffu));
        } else {
#pragma unroll
            for (int k = 0; k < 4; ++k) sv[k] = (i0 + k < n) ? double(sg[i0 + k]) : 1.0;
        }
#pragma unroll
        for (int k = 0; k < 4; ++k) {
            ar[k] += sv[k] * tr;
            ai[k] += sv[k] * ti;
        }
    }
#pragma unroll
    for (int k = 0; k < 4; ++k) {
        const int i = i0 + k;
        if (i <= n) part[size_t(split) * (n + 1) * (m + 1) + size_t(i) * (m + 1) + j] = mk(ar[k], ai[k]);
    }
}

__global__ void oloc_reduce_kernel(int n, int m, bool bias, int nsplit, double inv_ns, const c128* __restrict__ part,
                                   c128* __restrict__ oloc) {
    const size_t cnt = size_t(n + 1) * (m + 1);
    for (size_t q = size_t(blockIdx.x) * blockDim.x + threadIdx.x; q < cnt; q += size_t(gridDim.x) * blockDim.x) {
        c128 acc = mk(0., 0.);
        for (int sp = 0; sp < nsplit; ++sp) acc = acc + part[size_t(sp) * cnt + q];
        acc = inv_ns * acc;
        int i = int(q / (m + 1)), j = int(q % (m + 1));
        const size_t nm = size_t(n) * m;
        if (i < n && j < m)
            oloc[size_t(i) * m + j] = acc;
        else if (bias && i < n && j == m)
            oloc[nm + i] = acc;
        else if (bias && i == n && j < m)
            oloc[nm + n + j] = acc;
    }
}

// Centred log-derivative rows O~[s, p] = O[s, p] - oloc[p] (GroundState/utils.hpp:12-51 and
// SRMat.hpp:99-100).  Row-major, P contiguous.  A thread owns two adjacent columns:
// their place in [s_i t_j | s | t] and their means are resolved once, then the
// thread walks O_ROWS rows, reading sigma and t from L1/L2 and storing both values
// at once (one 16-byte store for complex64 rows of even P, two for complex128).
// For complex64 the per-row arithmetic is branch-free (s := 1 or t := 1 by a
// select) and four rows' loads are issued before their stores: 0.63 -> 0.86 of the
// copy peak on the XXZ workload, where the complex128 rows (32 bytes a thread)
// measured best one row at a time.
constexpr int O_ROWS = 16;
template <typename R>
__global__ void __launch_bounds__(256) o_writer_kernel(int n, int m, bool bias, size_t P, int ns,
                                                       const int8_t* __restrict__ sigma,
                                                       const cplx<R>* __restrict__ t, const c128* __restrict__ oloc,
                                                       cplx<R>* __restrict__ O) {
    const size_t p0 = (size_t(blockIdx.x) * blockDim.x + threadIdx.x) * 2;
    if (p0 >= P) return;
    const size_t nm = size_t(n) * m;
    int kind[2], ci[2], cj[2];  // kind 0: s_i t_j, 1: s_i, 2: t_j, 3: past the row
    R olr[2], oli[2];
#pragma unroll
    for (int e = 0; e < 2; ++e) {
        const size_t p = p0 + e;
        kind[e] = 3;
        ci[e] = cj[e] = 0;
        olr[e] = oli[e] = R(0);
        if (p < P) {
            if (p < nm) {
                kind[e] = 0;
                ci[e] = int(p / m);
                cj[e] = int(p - size_t(ci[e]) * m);
            } else if (p < nm + n) {
                kind[e] = 1;
                ci[e] = int(p - nm);
            } else {
                kind[e] = 2;
                cj[e] = int(p - nm - n);
            }
            const c128 o = oloc[p];
            olr[e] = R(o.re);
            oli[e] = R(o.im);
        }
    }
    const int groups = (ns + O_ROWS - 1) / O_ROWS;
    if constexpr (sizeof(R) == 4) {
        constexpr int RU = 4;  // rows whose loads are in flight together
        const bool pair16 = (P % 2) == 0 && kind[1] != 3;
        bool use_s[2], use_t[2];
#pragma unroll
        for (int e = 0; e < 2; ++e) {
            use_s[e] = kind[e] == 0 || kind[e] == 1;
            use_t[e] = kind[e] == 0 || kind[e] == 2;
        }
        for (int gi = blockIdx.y; gi < groups; gi += gridDim.y)
            for (int s = gi * O_ROWS, s1 = min(ns, s + O_ROWS); s < s1; s += RU) {
                cplx<R> v[RU][2];
#pragma unroll
                for (int u = 0; u < RU; ++u) {
                    const int su = min(s + u, s1 - 1);  // a short last group repeats its last row, not stored
                    const int8_t* sg = sigma + size_t(su) * n;
                    const cplx<R>* ts = t + size_t(su) * m;
#pragma unroll
                    for (int e = 0; e < 2; ++e) {
                        const R sraw = R(sg[ci[e]]);
                        const cplx<R> traw = ts[cj[e]];
                        const R sv = use_s[e] ? sraw : R(1);
                        const R tr = use_t[e] ? traw.re : R(1), ti = use_t[e] ? traw.im : R(0);
                        v[u][e] = mk(sv * tr - olr[e], sv * ti - oli[e]);
                    }
                }
#pragma unroll
                for (int u = 0; u < RU; ++u) {
                    if (s + u >= s1) break;
                    cplx<R>* row = O + size_t(s + u) * P;
                    if (pair16) {
                        *reinterpret_cast<float4*>(row + p0) =
                            make_float4(v[u][0].re, v[u][0].im, v[u][1].re, v[u][1].im);
                    } else {
                        row[p0] = v[u][0];
                        if (kind[1] != 3) row[p0 + 1] = v[u][1];
                    }
                }
            }
    } else {
        for (int gi = blockIdx.y; gi < groups; gi += gridDim.y)
            for (int s = gi * O_ROWS, s1 = min(ns, s + O_ROWS); s < s1; ++s) {
                const int8_t* sg = sigma + size_t(s) * n;
                const cplx<R>* ts = t + size_t(s) * m;
                cplx<R> v[2];
#pragma unroll
                for (int e = 0; e < 2; ++e) {
                    cplx<R> x = mk(R(0), R(0));
                    if (kind[e] == 0) {
                        const R sv = R(sg[ci[e]]);
                        const cplx<R> tv = ts[cj[e]];
                        x = mk(sv * tv.re, sv * tv.im);
                    } else if (kind[e] == 1) {
                        x = mk(R(sg[ci[e]]), R(0));
                    } else if (kind[e] == 2) {
                        x = ts[cj[e]];
                    }
                    v[e] = mk(x.re - olr[e], x.im - oli[e]);
                }
                cplx<R>* row = O + size_t(s) * P;
                row[p0] = v[0];
                if (kind[1] != 3) row[p0 + 1] = v[1];
            }
    }
}

// out_p (partials) = sum_s conj(O~[s, p]) y_s over sample chunks.
template <typename R>
__global__ void ohy_partial_kernel(size_t P, int ns, int chunk, const cplx<R>* __restrict__ O,
                                   const c128* __restrict__ yv, c128* __restrict__ part) {
    const size_t p = size_t(blockIdx.x) * blockDim.x + threadIdx.x;
    const int split = blockIdx.y;
    if (p >= P) return;
    const int s0 = split * chunk, s1 = min(ns, s0 + chunk);
    double ar = 0., ai = 0.;
    int s = s0;
    // eight independent row loads in flight per thread
    for (; s + 8 <= s1; s += 8) {
        cplx<R> o[8];
#pragma unroll
        for (int u = 0; u < 8; ++u) o[u] = O[size_t(s + u) * P + p];
#pragma unroll
        for (int u = 0; u < 8; ++u) {
            const c128 y = yv[s + u];
            // conj(o) * y
            ar += double(o[u].re) * y.re + double(o[u].im) * y.im;
            ai += double(o[u].re) * y.im - double(o[u].im) * y.re;
        }
    }
    for (; s < s1; ++s) {
        const cplx<R> o = O[size_t(s) * P + p];
        const c128 y = yv[s];
        ar += double(o.re) * y.re + double(o.im) * y.im;
        ai += double(o.re) * y.im - double(o.im) * y.re;
    }
    part[size_t(split) * P + p] = mk(ar, ai);
}

// The same for complex64 O~ with an even P: two columns per thread, one 16-byte
// load per row (eight rows in flight).  At most 40 registers, so that twelve
// 128-thread blocks share an SM.
constexpr int OHY_BLOCKS_PER_SM = 12;
__global__ void __launch_bounds__(128, OHY_BLOCKS_PER_SM) ohy_pair_kernel(size_t P, int ns, int chunk, const c64* __restrict__ O, const c128* __restrict__ yv,
                                c128* __restrict__ part) {
    const size_t p2 = size_t(blockIdx.x) * blockDim.x + threadIdx.x;
    const int split = blockIdx.y;
    const size_t P2 = P / 2;
    if (p2 >= P2) return;
    const int s0 = split * chunk, s1 = min(ns, s0 + chunk);
    const float4* O4 = reinterpret_cast<const float4*>(O);
    double a0r = 0., a0i = 0., a1r = 0., a1i = 0.;
    int s = s0;
    for (; s + 8 <= s1; s += 8) {
        float4 o[8];
#pragma unroll
        for (int u = 0; u < 8; ++u) o[u] = O4[size_t(s + u) * P2 + p2];
#pragma unroll
        for (int u = 0; u < 8; ++u) {
            const c128 y = yv[s + u];
            a0r += double(o[u].x) * y.re + double(o[u].y) * y.im;
            a0i += double(o[u].x) * y.im - double(o[u].y) * y.re;
            a1r += double(o[u].z) * y.re + double(o[u].w) * y.im;
            a1i += double(o[u].z) * y.im - double(o[u].w) * y.re;
        }
    }
    for (; s < s1; ++s) {
        const float4 o = O4[size_t(s) * P2 + p2];
        const c128 y = yv[s];
        a0r += double(o.x) * y.re + double(o.y) * y.im;
        a0i += double(o.x) * y.im - double(o.y) * y.re;
        a1r += double(o.z) * y.re + double(o.w) * y.im;
        a1i += double(o.z) * y.im - double(o.w) * y.re;
    }
    part[size_t(split) * P + 2 * p2] = mk(a0r, a0i);
    part[size_t(split) * P + 2 * p2 + 1] = mk(a1r, a1i);
}

// part[split][p] = sum over the split's sample chunk of conj(O~[s, p]) y_s; returns
// the number of splits (at most 64; part holds 64 P entries).  The complex64 pair
// kernel's blocks all do the same work, so its split count fills whole waves: as
// many as fit in four waves of the resident blocks (a partial last wave cost ~20 %
// at Ns = 8192, P = 41,904).
template <typename R>
static int launch_ohy(size_t P, int ns, const cplx<R>* O, const c128* y, c128* part, int sm_count,
                      cudaStream_t st) {
    if constexpr (sizeof(R) == 4) {
        if (P % 2 == 0) {
            static const int per_sm = [] {
                int b = 0;
                YQ_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&b, ohy_pair_kernel, 128, 0));
                return std::max(1, b);
            }();
            const unsigned gx = cdiv_u(P / 2, 128);
            const long long slots = 4LL * per_sm * sm_count;
            const int nsplit = int(std::max(1LL, std::min<long long>(std::min(64, ns), slots / gx)));
            const int chunk = (ns + nsplit - 1) / nsplit;
            ohy_pair_kernel<<<dim3(gx, nsplit), 128, 0, st>>>(P, ns, chunk, O, y, part);
            YQ_LAUNCH_CHECK();
            return nsplit;
        }
    }
    const unsigned gx = cdiv_u(P, 256);
    const int nsplit = std::max(1, std::min({64, ns, int(8 * 148 / gx)}));
    const int chunk = (ns + nsplit - 1) / nsplit;
    ohy_partial_kernel<R><<<dim3(gx, nsplit), 256, 0, st>>>(P, ns, chunk, O, y, part);
    YQ_LAUNCH_CHECK();
    return nsplit;
}

__global__ void reduce_parts_kernel(size_t P, int nsplit, double alpha, const c128* __restrict__ part,
                                    const c128* __restrict__ addv, double beta, c128* __restrict__ out) {
    for (size_t p = size_t(blockIdx.x) * blockDim.x + threadIdx.x; p < P; p += size_t(gridDim.x) * blockDim.x) {
        c128 acc = mk(0., 0.);
        for (int sp = 0; sp < nsplit; ++sp) acc = acc + part[size_t(sp) * P + p];
        acc = alpha * acc;
        if (addv) acc = acc + beta * addv[p];
        out[p] = acc;
    }
}

// out_s = alpha * sum_p O~[s, p] x_p  (one block streams one sample row; four
// loads of the row in flight per thread)
// The same for complex64 O~ with an even P: two rows per block, so that each pair
// of FP64 x entries read from L2 serves both, and two columns per 16-byte load
// (two loads per row in flight).  The row index is clamped for the second row of
// an odd last block, whose result is not written.
__global__ void __launch_bounds__(256) ox_pair_kernel(size_t P, int ns, const float4* __restrict__ O4,
                                                      const c128* __restrict__ x, double alpha,
                                                      c128* __restrict__ out) {
    constexpr int RB = 2, U = 2;
    __shared__ c128 red[RB][8];
    const int s0 = blockIdx.x * RB;
    const size_t P2 = P / 2;
    const float4* rows[RB];
#pragma unroll
    for (int r = 0; r < RB; ++r) rows[r] = O4 + size_t(min(s0 + r, ns - 1)) * P2;
    double ar[RB], ai[RB];
#pragma unroll
    for (int r = 0; r < RB; ++r) ar[r] = ai[r] = 0.;
    const size_t step = blockDim.x;
    size_t q = threadIdx.x;
    for (; q + (U - 1) * step < P2; q += U * step) {
        float4 o[U][RB];
        c128 x0[U], x1[U];
#pragma unroll
        for (int u = 0; u < U; ++u) {
            x0[u] = x[2 * (q + u * step)];
            x1[u] = x[2 * (q + u * step) + 1];
#pragma unroll
            for (int r = 0; r < RB; ++r) o[u][r] = rows[r][q + u * step];
        }
#pragma unroll
        for (int u = 0; u < U; ++u)
#pragma unroll
            for (int r = 0; r < RB; ++r) {
                ar[r] += double(o[u][r].x) * x0[u].re - double(o[u][r].y) * x0[u].im + double(o[u][r].z) * x1[u].re -
                         double(o[u][r].w) * x1[u].im;
                ai[r] += double(o[u][r].x) * x0[u].im + double(o[u][r].y) * x0[u].re + double(o[u][r].z) * x1[u].im +
                         double(o[u][r].w) * x1[u].re;
            }
    }
    for (; q < P2; q += step) {
        const c128 a = x[2 * q], b = x[2 * q + 1];
#pragma unroll
        for (int r = 0; r < RB; ++r) {
            const float4 o = rows[r][q];
            ar[r] += double(o.x) * a.re - double(o.y) * a.im + double(o.z) * b.re - double(o.w) * b.im;
            ai[r] += double(o.x) * a.im + double(o.y) * a.re + double(o.z) * b.im + double(o.w) * b.re;
        }
    }
#pragma unroll
    for (int r = 0; r < RB; ++r) {
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) {
            ar[r] += __shfl_xor_sync(0xffffffffu, ar[r], o);
            ai[r] += __shfl_xor_sync(0xffffffffu, ai[r], o);
        }
        if ((threadIdx.x & 31) == 0) red[r][threadIdx.x >> 5] = mk(ar[r], ai[r]);
    }
    __syncthreads();
    if (threadIdx.x < RB && s0 + int(threadIdx.x) < ns) {
        c128 t = red[threadIdx.x][0];
        for (int w = 1; w < int(blockDim.x >> 5); ++w) t = t + red[threadIdx.x][w];
        out[s0 + threadIdx.x] = alpha * t;
    }
}

template <typename R>
__global__ void ox_kernel(size_t P, int ns, const cplx<R>* __restrict__ O, const c128* __restrict__ x, double alpha,
                          c128* __restrict__ out) {
    __shared__ c128 red[8];
    const int s = blockIdx.x;
    const cplx<R>* row = O + size_t(s) * P;
    double ar = 0., ai = 0.;
    const size_t step = blockDim.x;
    size_t p = threadIdx.x;
    for (; p + 3 * step < P; p += 4 * step) {
        cplx<R> o[4];
        c128 xv[4];
#pragma unroll
        for (int u = 0; u < 4; ++u) {
            o[u] = row[p + u * step];
            xv[u] = x[p + u * step];
        }
#pragma unroll
        for (int u = 0; u < 4; ++u) {
            ar += double(o[u].re) * xv[u].re - double(o[u].im) * xv[u].im;
            ai += double(o[u].re) * xv[u].im + double(o[u].im) * xv[u].re;
        }
    }
    for (; p < P; p += step) {
        const cplx<R> o = row[p];
        const c128 xv = x[p];
        ar += double(o.re) * xv.re - double(o.im) * xv.im;
        ai += double(o.re) * xv.im + double(o.im) * xv.re;
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        ar += __shfl_xor_sync(0xffffffffu, ar, o);
        ai += __shfl_xor_sync(0xffffffffu, ai, o);
    }
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = mk(ar, ai);
    __syncthreads();
    if (threadIdx.x == 0) {
        c128 r = red[0];
        for (int w = 1; w < int(blockDim.x >> 5); ++w) r = r + red[w];
        out[s] = alpha * r;
    }
}

// y_s = (E_s - <E>) / Ns  (centred right-hand side of the T-mode solve)
__global__ void centred_rhs_kernel(int ns, int ns_pad, const c128* __restrict__ e, const double* __restrict__ stats,
                                   c128* __restrict__ y) {
    int s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= ns_pad) return;
    if (s >= ns) {
        y[s] = mk(0., 0.);
        return;
    }
    y[s] = (1.0 / ns) * (e[s] - mk(stats[2], stats[3]));
}

// ---------------------------------------------------------------------------
// Padding of the SR matrix to a multiple of NB: zero off-diagonal, unit diagonal.
__global__ void pad_identity_kernel(c128* G, int dim, int dim_pad) {
    size_t total = size_t(dim_pad) * dim_pad;
    for (size_t q = size_t(blockIdx.x) * blockDim.x + threadIdx.x; q < total; q += size_t(gridDim.x) * blockDim.x) {
        int r = int(q / dim_pad), c = int(q % dim_pad);
        if (r >= dim || c >= dim) G[q] = mk(r == c ? 1.0 : 0.0, 0.0);
    }
}

// ---------------------------------------------------------------------------
__global__ void update_kernel(size_t P, double lr, const c128* __restrict__ v, c128* __restrict__ p64,
                              double* __restrict__ part) {
    __shared__ double red[8];
    double acc = 0.;
    for (size_t p = size_t(blockIdx.x) * blockDim.x + threadIdx.x; p < P; p += size_t(gridDim.x) * blockDim.x) {
        c128 vv = v[p];
        acc += vv.re * vv.re + vv.im * vv.im;
        p64[p] = p64[p] - lr * vv;
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, o);
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = acc;
    __syncthreads();
    if (threadIdx.x == 0) {
        double r = 0.;
        for (int w = 0; w < int(blockDim.x >> 5); ++w) r += red[w];
        part[blockIdx.x] = r;
    }
}

__global__ void finish_norm_kernel(int nb, const double* __restrict__ part, double* __restrict__ stats,
                                   int* __restrict__ status) {
    double r = 0.;
    for (int i = 0; i < nb; ++i) r += part[i];
    stats[4] = sqrt(r);
    if (!isfinite(r)) atomicOr(status, DS_NONFINITE);
}

// ---------------------------------------------------------------------------
template <typename R>
static void construct_t(yq_sr_s* sr) {
    yq_rbm_s* q = sr->q;
    yq_ctx_s* ctx = q->ctx;
    cudaStream_t st = ctx->stream;
    const int ns = sr->ns, n = q->n, m = q->m;
    const size_t P = q->P;
    const cplx<R>* theta = sr->S->theta.as<cplx<R>>();
    const int8_t* sigma = sr->S->sigma.as<int8_t>();

    ctx->stage_begin(ST_ELOC);
    ham_eloc(sr->H, q, ns, sigma, theta, sr->eloc.as<c128>());
    energy_stats_kernel<<<1, 256, 0, st>>>(ns, sr->eloc.as<c128>(), sr->stats.as<double>(), ctx->status.as<int>());
    YQ_LAUNCH_CHECK();
    ctx->stage_end(ST_ELOC);

    ctx->stage_begin(ST_MEAN);
    const size_t cnt = size_t(ns) * m;
    tanh_kernel<R><<<std::min<size_t>(cdiv_u(cnt, 256), 148 * 16), 256, 0, st>>>(cnt, theta, sr->tanhs.as<cplx<R>>());
    YQ_LAUNCH_CHECK();
    // column mean of O, split over sample chunks (deterministic two-stage sum)
    {
        dim3 g(cdiv_u(m + 1, 32), cdiv_u(n + 1, 32), 1);
        int nsplit = std::max(1, std::min(64, int((8 * 148) / std::max(1u, g.x * g.y))));
        nsplit = std::min(nsplit, ns);
        int chunk = (ns + nsplit - 1) / nsplit;
        g.z = nsplit;
        sr->part.ensure(std::max(size_t(nsplit) * (n + 1) * (m + 1), size_t(64) * P) * sizeof(c128));
        oloc_partial_kernel<R><<<g, 256, 0, st>>>(n, m, ns, chunk, sigma, sr->tanhs.as<cplx<R>>(), sr->part.as<c128>());
        YQ_LAUNCH_CHECK();
        oloc_reduce_kernel<<<cdiv_u(size_t(n + 1) * (m + 1), 256), 256, 0, st>>>(
            n, m, q->use_bias, nsplit, 1.0 / ns, sr->part.as<c128>(), sr->oloc.as<c128>());
        YQ_LAUNCH_CHECK();
    }
    ctx->stage_end(ST_MEAN);

    ctx->stage_begin(ST_O);
    bool fused = false;
    if constexpr (sizeof(R) == 4) {
        if (sr->precision == YQ_PREC_MIXED && sr->mode == YQ_SR_T) {
            // centred rows and their BF16 planes in one pass
            gram_tc_write_o_and_operands(n, m, q->use_bias, P, ns, sigma, sr->tanhs.as<c64>(), sr->oloc.as<c128>(),
                                         sr->O.as<c64>(), sr->xh.as<uint16_t>(), sr->xl.as<uint16_t>(),
                                         sr->yh.as<uint16_t>(), sr->yl.as<uint16_t>(), st);
            fused = true;
        }
    }
    if (!fused) {
        const dim3 g(cdiv_u(P, 512), std::min(65535u, cdiv_u(size_t(ns), O_ROWS)));
        o_writer_kernel<R><<<g, 256, 0, st>>>(n, m, q->use_bias, P, ns, sigma, sr->tanhs.as<cplx<R>>(),
                                              sr->oloc.as<c128>(), sr->O.as<cplx<R>>());
        YQ_LAUNCH_CHECK();
    }
    ctx->stage_end(ST_O);

    // F = O~^H (E - <E>) / Ns (SRMat.hpp:101-102; equal to O~^H E / Ns since O~^H 1 = 0)
    const int vlen = std::max(ns, sr->dim_pad);
    centred_rhs_kernel<<<cdiv_u(vlen, 256), 256, 0, st>>>(ns, vlen, sr->eloc.as<c128>(), sr->stats.as<double>(),
                                                          sr->y.as<c128>());
    YQ_LAUNCH_CHECK();
    {
        const int nsplit = launch_ohy<R>(P, ns, sr->O.as<cplx<R>>(), sr->y.as<c128>(), sr->part.as<c128>(),
                                         sr->q->ctx->sm_count, st);
        reduce_parts_kernel<<<cdiv_u(P, 256), 256, 0, st>>>(P, nsplit, 1.0, sr->part.as<c128>(), nullptr, 0.0,
                                                            sr->grad.as<c128>());
        YQ_LAUNCH_CHECK();
    }
}

void sr_construct(yq_sr_s* sr) {
    yq_rbm_s* q = sr->q;
    yq_sampler_s* S = sr->S;
    YQ_CHECK_ARG(S->ns > 0, "construct: the sampler holds no samples");
    if (sr->precision == YQ_PREC_MIXED)
        YQ_CHECK_ARG(q->dtype == YQ_C64, "construct: mixed precision needs a complex64 RBM");
    else
        YQ_CHECK_ARG(q->dtype == YQ_C128, "construct: FP64 precision needs a complex128 RBM");
    rbm_prepare(q);
    const int ns = S->ns;
    const size_t P = q->P;
    sr->ns = ns;
    // AUTO takes the sample-space form when Ns < P, unless the runner averages the
    // Fisher matrix over iterations (beta2 != 0), which only the S-form can hold
    sr->mode = sr->mode_req == YQ_SR_AUTO ? ((size_t(ns) < P && sr->beta2 == 0.0) ? YQ_SR_T : YQ_SR_S)
                                          : sr->mode_req;
    // mixed precision: T-form on the tensor cores; S-form (Ns >= P) with FP32 O~ and FP64 sums
    sr->dim = sr->mode == YQ_SR_T ? ns : int(P);
    sr->dim_pad = ((sr->dim + NB - 1) / NB) * NB;
    const size_t cs = q->csize();
    sr->eloc.ensure(size_t(ns) * sizeof(c128));
    sr->tanhs.ensure(size_t(ns) * q->m * cs);
    sr->O.ensure(size_t(ns) * P * cs);
    sr->oloc.ensure(P * sizeof(c128));
    sr->grad.ensure(P * sizeof(c128));
    sr->v.ensure(P * sizeof(c128));
    sr->work_p.ensure(P * sizeof(c128));
    const size_t vec = size_t(std::max(ns, sr->dim_pad));
    sr->y.ensure(vec * sizeof(c128));
    sr->rhs.ensure(vec * sizeof(c128));
    sr->work_s.ensure(vec * sizeof(c128));
    sr->s1.ensure(vec * sizeof(c128));
    sr->s2.ensure(vec * sizeof(c128));
    sr->s3.ensure(vec * sizeof(c128));
    sr->s4.ensure(vec * sizeof(c128));
    sr->stats.ensure(64 * sizeof(double));
    if (sr->precision == YQ_PREC_MIXED && sr->mode == YQ_SR_T) {
        const size_t kpad = gram_tc_kpad(P);
        const size_t rows = gram_tc_rows(ns);
        sr->xh.ensure(rows * kpad * 2);
        sr->xl.ensure(rows * kpad * 2);
        sr->yh.ensure(rows * kpad * 2);
        sr->yl.ensure(rows * kpad * 2);
    }
    if (q->dtype == YQ_C64)
        construct_t<float>(sr);
    else
        construct_t<double>(sr);
    sr->constructed = true;
    sr->solved = false;
}

// Form the shifted SR matrix (S or T) into G (lower, padded).
template <typename R>
static void form_matrix_t(yq_sr_s* sr, double shift) {
    cudaStream_t st = sr->q->ctx->stream;
    const size_t P = sr->q->P;
    const int ns = sr->ns;
    sr->G.ensure(size_t(sr->dim_pad) * sr->dim_pad * sizeof(c128));
    sr->Linv.ensure(size_t(sr->dim_pad / NB) * NB * NB * sizeof(c128));
    sr->LinvH.ensure(size_t(sr->dim_pad / NB) * NB * NB * sizeof(c128));
    c128* G = sr->G.as<c128>();
    if (sr->dim_pad != sr->dim) {
        pad_identity_kernel<<<148 * 8, 256, 0, st>>>(G, sr->dim, sr->dim_pad);
        YQ_LAUNCH_CHECK();
    }
    if (sr->mode == YQ_SR_T) {
        if (sr->precision == YQ_PREC_MIXED)
            gram_tc_run(sr->xh.as<uint16_t>(), sr->xl.as<uint16_t>(), sr->yh.as<uint16_t>(), sr->yl.as<uint16_t>(),
                        ns, P, G, size_t(sr->dim_pad), 1.0 / ns, shift, sr->q->ctx->status.as<int>(),
                        sr->q->ctx->sm_count, sr->gram_ws, st);
        else
            gram_fp64<R>(sr->O.as<cplx<R>>(), P, 0, ns, int(P), G, size_t(sr->dim_pad), 1.0 / ns, 0, shift, st);
    } else {
        gram_fp64<R>(sr->O.as<cplx<R>>(), P, 1, int(P), ns, G, size_t(sr->dim_pad), 1.0 / ns, 0, shift, st);
    }
}

static void form_matrix(yq_sr_s* sr, double shift) {
    if (sr->q->dtype == YQ_C64)
        form_matrix_t<float>(sr, shift);
    else
        form_matrix_t<double>(sr, shift);
}

// y <- O~^H x * alpha  (P-vector out), x: ns-vector
template <typename R>
static void op_ohy(yq_sr_s* sr, const c128* x, double alpha, c128* out, const c128* addv, double beta) {
    cudaStream_t st = sr->q->ctx->stream;
    const size_t P = sr->q->P;
    const int ns = sr->ns;
    const int nsplit = launch_ohy<R>(P, ns, sr->O.as<cplx<R>>(), x, sr->part.as<c128>(), sr->q->ctx->sm_count, st);
    reduce_parts_kernel<<<cdiv_u(P, 256), 256, 0, st>>>(P, nsplit, alpha, sr->part.as<c128>(), addv, beta, out);
    YQ_LAUNCH_CHECK();
}
template <typename R>
static void op_ox(yq_sr_s* sr, const c128* x, double alpha, c128* out) {
    if constexpr (sizeof(R) == 4) {
        if (sr->q->P % 2 == 0) {
            ox_pair_kernel<<<cdiv_u(size_t(sr->ns), 2), 256, 0, sr->q->ctx->stream>>>(
                sr->q->P, sr->ns, reinterpret_cast<const float4*>(sr->O.as<cplx<R>>()), x, alpha, out);
            YQ_LAUNCH_CHECK();
            return;
        }
    }
    ox_kernel<R><<<sr->ns, 256, 0, sr->q->ctx->stream>>>(sr->q->P, sr->ns, sr->O.as<cplx<R>>(), x, alpha, out);
    YQ_LAUNCH_CHECK();
}

// apply(x) = O~^H (O~ x) / Ns + shift x  (SRMat.hpp:170-189)
template <typename R>
static void sr_apply(yq_sr_s* sr, const c128* x, double shift, c128* out) {
    op_ox<R>(sr, x, 1.0 / sr->ns, sr->work_s.as<c128>());
    op_ohy<R>(sr, sr->work_s.as<c128>(), 1.0, out, x, shift);
}

// ---------------------------------------------------------------------------
// Device-side vector helpers for CG (host-driven loop, FP64).
__global__ void dotc_kernel(size_t n, const c128* __restrict__ a, const c128* __restrict__ b, double* __restrict__ out) {
    __shared__ c128 red[8];
    c128 acc = mk(0., 0.);
    for (size_t i = size_t(blockIdx.x) * blockDim.x + threadIdx.x; i < n; i += size_t(gridDim.x) * blockDim.x)
        acc = acc + conj(a[i]) * b[i];
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        acc.re += __shfl_xor_sync(0xffffffffu, acc.re, o);
        acc.im += __shfl_xor_sync(0xffffffffu, acc.im, o);
    }
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = acc;
    __syncthreads();
    if (threadIdx.x == 0) {
        c128 r = red[0];
        for (int w = 1; w < int(blockDim.x >> 5); ++w) r = r + red[w];
        out[2 * blockIdx.x] = r.re;
        out[2 * blockIdx.x + 1] = r.im;
    }
}
__global__ void axpy_kernel(size_t n, c128 alpha, const c128* __restrict__ x, c128* __restrict__ y) {
    for (size_t i = size_t(blockIdx.x) * blockDim.x + threadIdx.x; i < n; i += size_t(gridDim.x) * blockDim.x)
        y[i] = y[i] + alpha * x[i];
}
__global__ void xpby_kernel(size_t n, const c128* __restrict__ x, double beta, c128* __restrict__ y) {
    for (size_t i = size_t(blockIdx.x) * blockDim.x + threadIdx.x; i < n; i += size_t(gridDim.x) * blockDim.x)
        y[i] = x[i] + beta * y[i];
}

static c128 dotc(yq_sr_s* sr, size_t n, const c128* a, const c128* b) {
    cudaStream_t st = sr->q->ctx->stream;
    const int blocks = 128;
    double* buf = sr->q->ctx->scratch.as<double>();
    dotc_kernel<<<blocks, 256, 0, st>>>(n, a, b, buf);
    YQ_LAUNCH_CHECK();
    double h[2 * blocks];
    YQ_CUDA(cudaMemcpyAsync(h, buf, sizeof(h), cudaMemcpyDeviceToHost, st));
    YQ_CUDA(cudaStreamSynchronize(st));
    c128 r = mk(0., 0.);
    for (int i = 0; i < blocks; ++i) r = r + mk(h[2 * i], h[2 * i + 1]);
    return r;
}

// Eigen::ConjugateGradient<..., Lower|Upper, IdentityPreconditioner> semantics,
// solving (S + shift) x = b into sr->v.
template <typename R>
static void solve_cg_t(yq_sr_s* sr, const c128* b, double shift, double tol, int* iters, double* relres) {
    cudaStream_t st = sr->q->ctx->stream;
    const size_t P = sr->q->P;
    DevBuf rb, pb, tb;
    rb.ensure(P * sizeof(c128));
    pb.ensure(P * sizeof(c128));
    tb.ensure(P * sizeof(c128));
    c128 *x = sr->v.as<c128>(), *r = rb.as<c128>(), *p = pb.as<c128>(), *tmp = tb.as<c128>();
    YQ_CUDA(cudaMemsetAsync(x, 0, P * sizeof(c128), st));
    YQ_CUDA(cudaMemcpyAsync(r, b, P * sizeof(c128), cudaMemcpyDeviceToDevice, st));
    const unsigned g = std::min(148u * 8, cdiv_u(P, 256));
    double rhsNorm2 = dotc(sr, P, r, r).re;
    int it = 0;
    double res2 = rhsNorm2;
    if (rhsNorm2 > 0.) {
        const double threshold = tol * tol * rhsNorm2;
        YQ_CUDA(cudaMemcpyAsync(p, r, P * sizeof(c128), cudaMemcpyDeviceToDevice, st));
        double absNew = dotc(sr, P, r, p).re;
        const int maxit = int(2 * P);
        while (it < maxit) {
            sr_apply<R>(sr, p, shift, tmp);
            c128 pt = dotc(sr, P, p, tmp);
            c128 alpha = cdiv(mk(absNew, 0.0), pt);
            axpy_kernel<<<g, 256, 0, st>>>(P, alpha, p, x);
            axpy_kernel<<<g, 256, 0, st>>>(P, mk(-alpha.re, -alpha.im), tmp, r);
            YQ_LAUNCH_CHECK();
            res2 = dotc(sr, P, r, r).re;
            if (res2 < threshold) break;
            double absOld = absNew;
            absNew = res2;
            xpby_kernel<<<g, 256, 0, st>>>(P, r, absNew / absOld, p);
            YQ_LAUNCH_CHECK();
            ++it;
        }
    }
    if (iters) *iters = it;
    if (relres) *relres = rhsNorm2 > 0. ? std::sqrt(res2 / rhsNorm2) : 0.;
}

__global__ void residual_kernel(size_t n, const c128* __restrict__ b, const c128* __restrict__ ax, c128* __restrict__ r) {
    for (size_t i = size_t(blockIdx.x) * blockDim.x + threadIdx.x; i < n; i += size_t(gridDim.x) * blockDim.x)
        r[i] = b[i] - ax[i];
}

// v = (g - w) / shift: the Woodbury form of (S + shift)^{-1} g in T-mode, with
// w = O~^H (T + shift)^{-1} O~ g / Ns (S = O~^H O~ / Ns, T = O~ O~^H / Ns).
__global__ void woodbury_kernel(size_t P, double inv_shift, const c128* __restrict__ g, const c128* __restrict__ w,
                                c128* __restrict__ v) {
    for (size_t i = size_t(blockIdx.x) * blockDim.x + threadIdx.x; i < P; i += size_t(gridDim.x) * blockDim.x)
        v[i] = inv_shift * (g[i] - w[i]);
}

// ObsAvg::update (Runners/RunRBM.hpp:26-30): avg = beta avg + (1 - beta) x.
__global__ void ema_kernel(size_t n, double beta, const c128* __restrict__ x, c128* __restrict__ avg) {
    for (size_t i = size_t(blockIdx.x) * blockDim.x + threadIdx.x; i < n; i += size_t(gridDim.x) * blockDim.x)
        avg[i] = beta * avg[i] + (1.0 - beta) * x[i];
}

// ObsAvg::getAvg (RunRBM.hpp:32-35): out = avg / denom, denom = 1 - beta^t.
__global__ void avg_div_kernel(size_t n, double denom, const c128* __restrict__ avg, c128* __restrict__ out) {
    for (size_t i = size_t(blockIdx.x) * blockDim.x + threadIdx.x; i < n; i += size_t(gridDim.x) * blockDim.x)
        out[i] = mk(avg[i].re / denom, avg[i].im / denom);
}

// fisherAvg.update(corrMat()) and fisher = getAvg() + lambda I (RunRBM.hpp:187-190)
// on the lower triangle of the padded S-form matrix G (formed without shift; the
// padding's unit diagonal averages to itself).
__global__ void fisher_avg_kernel(int dim, int dim_pad, double beta, double denom, double shift, c128* __restrict__ G,
                                  c128* __restrict__ favg) {
    const size_t total = size_t(dim_pad) * dim_pad;
    for (size_t q = size_t(blockIdx.x) * blockDim.x + threadIdx.x; q < total; q += size_t(gridDim.x) * blockDim.x) {
        const int r = int(q / dim_pad), c = int(q % dim_pad);
        if (c > r) continue;
        const c128 f = beta * favg[q] + (1.0 - beta) * G[q];
        favg[q] = f;
        G[q] = mk(f.re / denom + ((r == c && r < dim) ? shift : 0.0), f.im / denom);
    }
}

// The factorisation used for the LLT solves of one SR object.  The mixed-precision
// T-form (whose matrix comes from BF16x3 products) uses the panel form with
// tensor-core trailing updates; everything else the persistent FP64 tile kernel.
// YQ_CHOLESKY=tiled|recursive overrides (the recursive launch-per-step variant is
// kept for comparison).
struct LltPlan {
    bool recursive = false, panels = false;
};

static LltPlan llt_plan(const yq_sr_s* sr) {
    static const int forced = [] {
        const char* e = std::getenv("YQ_CHOLESKY");
        if (!e) return 0;
        if (std::string(e) == "recursive") return 1;
        if (std::string(e) == "tiled") return 2;
        return 0;
    }();
    LltPlan pl;
    pl.recursive = forced == 1;
    pl.panels = forced == 0 && sr->precision == YQ_PREC_MIXED && sr->mode == YQ_SR_T;
    return pl;
}

static void llt_factor(yq_sr_s* sr, const LltPlan& pl) {
    yq_ctx_s* ctx = sr->q->ctx;
    cudaStream_t st = ctx->stream;
    sr->chol_work.ensure(chol_tile_scratch_bytes(sr->dim_pad));
    if (pl.recursive) {
        chol_factor(sr->G.as<c128>(), sr->dim_pad, size_t(sr->dim_pad), sr->Linv.as<c128>(), sr->LinvH.as<c128>(),
                    ctx->status.as<int>(), st);
    } else if (pl.panels) {
        sr->chol_planes.ensure(chol_panel_planes_bytes(sr->dim_pad));
        chol_factor_panels(sr->G.as<c128>(), sr->dim_pad, size_t(sr->dim_pad), sr->Linv.as<c128>(),
                           sr->LinvH.as<c128>(), ctx->status.as<int>(), sr->chol_work.p, sr->chol_planes.p,
                           ctx->sm_count, st);
    } else {
        chol_factor_tiled(sr->G.as<c128>(), sr->dim_pad, size_t(sr->dim_pad), sr->Linv.as<c128>(),
                          sr->LinvH.as<c128>(), ctx->status.as<int>(), sr->chol_work.p, ctx->sm_count, st);
    }
}

// out = (L L^H)^{-1} b (b may be overwritten; tmp is scratch for the recursive form).
static void llt_apply(yq_sr_s* sr, const LltPlan& pl, c128* b, c128* tmp, c128* out) {
    yq_ctx_s* ctx = sr->q->ctx;
    const size_t dp = size_t(sr->dim_pad);
    if (pl.recursive)
        yq::chol_solve(sr->G.as<c128>(), sr->dim_pad, dp, sr->Linv.as<c128>(), sr->LinvH.as<c128>(), b, tmp, out,
                       ctx->stream);
    else
        chol_solve_tiled(sr->G.as<c128>(), sr->dim_pad, dp, sr->Linv.as<c128>(), sr->LinvH.as<c128>(), b, out,
                         ctx->status.as<int>(), sr->chol_work.p, ctx->sm_count, ctx->stream);
}

// Hermitian inner product Re <a, b> = Re sum conj(a_i) b_i of two device vectors
// into *out, one block (the T-form vectors hold at most a few hundred thousand
// entries), FP64 sums in a fixed order.
__global__ void __launch_bounds__(1024) dot_re_kernel(size_t n, const c128* __restrict__ a,
                                                      const c128* __restrict__ b, double* __restrict__ out) {
    __shared__ double red[32];
    double acc = 0.;
    for (size_t i = threadIdx.x; i < n; i += blockDim.x) acc += a[i].re * b[i].re + a[i].im * b[i].im;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, o);
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = acc;
    __syncthreads();
    if (threadIdx.x == 0) {
        double t = 0.;
        for (int w = 0; w < int(blockDim.x >> 5); ++w) t += red[w];
        *out = t;
    }
}

// PCG step scalars on the device (sc: [0] <r, z>, [1] <p, q>, [2] <r', z'>):
// x += a p, r -= a q with a = <r, z> / <p, q>.
__global__ void pcg_xr_kernel(size_t n, const double* __restrict__ sc, const c128* __restrict__ p,
                              const c128* __restrict__ q, c128* __restrict__ x, c128* __restrict__ r) {
    const double a = sc[1] != 0.0 ? sc[0] / sc[1] : 0.0;
    for (size_t i = size_t(blockIdx.x) * blockDim.x + threadIdx.x; i < n; i += size_t(gridDim.x) * blockDim.x) {
        x[i] = x[i] + a * p[i];
        r[i] = r[i] - a * q[i];
    }
}
// p = z + b p with b = <r', z'> / <r, z>; afterwards <r', z'> becomes <r, z> (one
// block does the swap after every block has read the old value: a separate launch).
__global__ void pcg_p_kernel(size_t n, const double* __restrict__ sc, const c128* __restrict__ z,
                             c128* __restrict__ p) {
    const double b = sc[0] != 0.0 ? sc[2] / sc[0] : 0.0;
    for (size_t i = size_t(blockIdx.x) * blockDim.x + threadIdx.x; i < n; i += size_t(gridDim.x) * blockDim.x)
        p[i] = z[i] + b * p[i];
}
__global__ void pcg_swap_kernel(double* sc) { sc[0] = sc[2]; }

// ohy += a w over the P parameters, a = <r, z> / <p, q> as in pcg_xr_kernel (read
// before the scalars move on).
__global__ void pcg_w_kernel(size_t n, const double* __restrict__ sc, const c128* __restrict__ w,
                             c128* __restrict__ ohy) {
    const double a = sc[1] != 0.0 ? sc[0] / sc[1] : 0.0;
    for (size_t i = size_t(blockIdx.x) * blockDim.x + threadIdx.x; i < n; i += size_t(gridDim.x) * blockDim.x)
        ohy[i] = ohy[i] + a * w[i];
}

// T-form: sol = (T + shift)^{-1} rhs (dim_pad entries, zero beyond ns) and
// ohy = O~^H sol (P entries).  steps = 0: one application of the Cholesky factor.
// steps = s > 0: s + 1 iterations of conjugate gradients from zero, preconditioned
// by the factor, on the exact operator T y = O~ (O~^H y) / Ns + shift y with FP64
// sums and residuals; each iteration applies the factor once and T once, and
// O~^H sol is accumulated from the O~^H p of those products (x = sum a_k p_k), so
// no product over O~ is spent on the solution itself.  (Plain iterative
// refinement x += M^{-1} (b - T x) diverges where the BF16x3 factor is a poor
// approximation of an ill-conditioned T -- at converged parameters of the 12 x 12
// workload its second step already moved the solution away -- while CG
// preconditioned by the same Hermitian positive definite factor converges for any
// such preconditioner.)  The step scalars stay on the device, so the sequence has
// no host round trip and can be captured in a graph.
template <typename R>
static void t_solve(yq_sr_s* sr, const LltPlan& pl, double shift, const c128* rhs, c128* sol, c128* ohy,
                    int steps) {
    cudaStream_t st = sr->q->ctx->stream;
    const size_t dp = size_t(sr->dim_pad);
    const size_t P = sr->q->P;
    const int ns = sr->ns;
    c128* b = sr->rhs.as<c128>();
    c128* tmp = sr->s2.as<c128>();
    if (steps <= 0) {
        YQ_CUDA(cudaMemcpyAsync(b, rhs, dp * sizeof(c128), cudaMemcpyDeviceToDevice, st));
        llt_apply(sr, pl, b, tmp, sol);
        op_ohy<R>(sr, sol, 1.0, ohy, nullptr, 0.0);
        return;
    }
    sr->pcg.ensure(4 * dp * sizeof(c128) + 8 * sizeof(double));
    c128* r = sr->pcg.as<c128>();
    c128* z = r + dp;
    c128* p = z + dp;
    c128* q = p + dp;
    double* sc = reinterpret_cast<double*>(q + dp);
    c128* w = sr->work_p.as<c128>();
    const unsigned g = std::min(148u * 8, cdiv_u(dp, 256));
    const unsigned gp = std::min(148u * 8, cdiv_u(P, 256));
    auto precond = [&](const c128* in, c128* out) {  // out = M^{-1} in (in kept)
        YQ_CUDA(cudaMemcpyAsync(out, in, dp * sizeof(c128), cudaMemcpyDeviceToDevice, st));
        llt_apply(sr, pl, out, tmp, out);
    };
    YQ_CUDA(cudaMemcpyAsync(r, rhs, dp * sizeof(c128), cudaMemcpyDeviceToDevice, st));
    YQ_CUDA(cudaMemsetAsync(sol, 0, dp * sizeof(c128), st));
    YQ_CUDA(cudaMemsetAsync(ohy, 0, P * sizeof(c128), st));
    precond(r, z);
    YQ_CUDA(cudaMemcpyAsync(p, z, dp * sizeof(c128), cudaMemcpyDeviceToDevice, st));
    dot_re_kernel<<<1, 1024, 0, st>>>(dp, r, z, sc + 0);
    YQ_LAUNCH_CHECK();
    const int iters = steps + 1;
    for (int k = 0; k < iters; ++k) {
        // w = O~^H p ; q = T p = O~ w / Ns + shift p (zero beyond ns)
        op_ohy<R>(sr, p, 1.0, w, nullptr, 0.0);
        YQ_CUDA(cudaMemsetAsync(q, 0, dp * sizeof(c128), st));
        op_ox<R>(sr, w, 1.0 / ns, q);
        axpy_kernel<<<cdiv_u(ns, 256), 256, 0, st>>>(size_t(ns), mk(shift, 0.0), p, q);
        dot_re_kernel<<<1, 1024, 0, st>>>(dp, p, q, sc + 1);
        pcg_xr_kernel<<<g, 256, 0, st>>>(dp, sc, p, q, sol, r);
        pcg_w_kernel<<<gp, 256, 0, st>>>(P, sc, w, ohy);
        YQ_LAUNCH_CHECK();
        if (k + 1 < iters) {
            precond(r, z);
            dot_re_kernel<<<1, 1024, 0, st>>>(dp, r, z, sc + 2);
            pcg_p_kernel<<<g, 256, 0, st>>>(dp, sc, z, p);
            pcg_swap_kernel<<<1, 1, 0, st>>>(sc);
            YQ_LAUNCH_CHECK();
        }
    }
}

// solveExact (SRMat.hpp:231-237) or its T-form dual into sr->v.  rhs (P entries)
// replaces energyGrad() when given; in T-mode it is solved through the Woodbury
// form (needs shift > 0).  fisher_beta >= 0 averages the S-form matrix into
// sr->favg before the shift is added (RunRBM.hpp:187-190).
template <typename R>
static void solve_llt_t(yq_sr_s* sr, double shift, int ir_steps, const c128* rhs = nullptr,
                        double fisher_beta = -1.0) {
    yq_ctx_s* ctx = sr->q->ctx;
    cudaStream_t st = ctx->stream;
    const size_t P = sr->q->P;
    const int ns = sr->ns;
    const bool avg = fisher_beta >= 0.0;
    ctx->stage_begin(ST_GRAM);
    form_matrix_t<R>(sr, avg ? 0.0 : shift);
    if (avg) {
        const size_t cnt = size_t(sr->dim_pad) * sr->dim_pad;
        if (sr->t_fisher == 0) {
            sr->favg.ensure(cnt * sizeof(c128));
            YQ_CUDA(cudaMemsetAsync(sr->favg.p, 0, cnt * sizeof(c128), st));
        }
        ++sr->t_fisher;
        const double denom = 1.0 - std::pow(fisher_beta, double(sr->t_fisher));
        fisher_avg_kernel<<<std::min(148u * 16, cdiv_u(cnt, 256)), 256, 0, st>>>(
            sr->dim, sr->dim_pad, fisher_beta, denom, shift, sr->G.as<c128>(), sr->favg.as<c128>());
        YQ_LAUNCH_CHECK();
    }
    ctx->stage_end(ST_GRAM);
    ctx->stage_begin(ST_SOLVE);
    const LltPlan pl = llt_plan(sr);
    llt_factor(sr, pl);
    const size_t dp = size_t(sr->dim_pad);
    if (sr->mode == YQ_SR_T) {
        c128* sol = sr->s1.as<c128>();
        if (!rhs) {
            // y = (T + shift)^{-1} (E - <E>) / Ns ; v = O~^H y   (push-through identity)
            t_solve<R>(sr, pl, shift, sr->y.as<c128>(), sol, sr->v.as<c128>(), ir_steps);
        } else {
            // v = (g - O~^H (T + shift)^{-1} O~ g / Ns) / shift
            sr->trhs.ensure(dp * sizeof(c128));
            c128* b = sr->trhs.as<c128>();
            YQ_CUDA(cudaMemsetAsync(b, 0, dp * sizeof(c128), st));
            op_ox<R>(sr, rhs, 1.0 / ns, b);
            sr->ohy_sol.ensure(P * sizeof(c128));
            t_solve<R>(sr, pl, shift, b, sol, sr->ohy_sol.as<c128>(), ir_steps);
            woodbury_kernel<<<cdiv_u(P, 256), 256, 0, st>>>(P, 1.0 / shift, rhs, sr->ohy_sol.as<c128>(),
                                                           sr->v.as<c128>());
            YQ_LAUNCH_CHECK();
        }
    } else {
        c128* b = sr->rhs.as<c128>();
        YQ_CUDA(cudaMemsetAsync(b, 0, dp * sizeof(c128), st));
        YQ_CUDA(cudaMemcpyAsync(b, rhs ? rhs : sr->grad.as<c128>(), P * sizeof(c128), cudaMemcpyDeviceToDevice, st));
        llt_apply(sr, pl, b, sr->s2.as<c128>(), sr->s1.as<c128>());
        YQ_CUDA(cudaMemcpyAsync(sr->v.as<c128>(), sr->s1.p, P * sizeof(c128), cudaMemcpyDeviceToDevice, st));
    }
    ctx->stage_end(ST_SOLVE);
}

void sr_solve(yq_sr_s* sr, double shift, int solver, double cg_tol, int ir_steps, int* iters, double* relres) {
    if (!sr->constructed) throw Error(YQ_E_STATE, "solve: call construct first");
    YQ_CHECK_ARG(shift >= 0.0, "solve: shift must be >= 0");
    YQ_CHECK_ARG(ir_steps <= 64, "solve: at most 64 CG steps");
    if (solver == YQ_SOLVE_CG) {
        sr->q->ctx->stage_begin(ST_SOLVE);
        if (sr->q->dtype == YQ_C64)
            solve_cg_t<float>(sr, sr->grad.as<c128>(), shift, cg_tol, iters, relres);
        else
            solve_cg_t<double>(sr, sr->grad.as<c128>(), shift, cg_tol, iters, relres);
        sr->q->ctx->stage_end(ST_SOLVE);
    } else {
        if (sr->q->dtype == YQ_C64)
            solve_llt_t<float>(sr, shift, ir_steps);
        else
            solve_llt_t<double>(sr, shift, ir_steps);
        if (iters) *iters = 0;
        if (relres) *relres = 0.;
    }
    sr->solved = true;
}

// |apply(v) - b| (RunRBM.hpp:190: cgErr = (srm.apply(v) - grad).norm()).
template <typename R>
static double cg_residual_norm(yq_sr_s* sr, const c128* b, double shift) {
    cudaStream_t st = sr->q->ctx->stream;
    const size_t P = sr->q->P;
    DevBuf rb;
    rb.ensure(P * sizeof(c128));
    c128* ax = sr->work_p.as<c128>();
    c128* r = rb.as<c128>();
    sr_apply<R>(sr, sr->v.as<c128>(), shift, ax);
    residual_kernel<<<std::min(148u * 8, cdiv_u(P, 256)), 256, 0, st>>>(P, b, ax, r);
    YQ_LAUNCH_CHECK();
    return std::sqrt(dotc(sr, P, r, r).re);
}

void sr_solve_runner(yq_sr_s* sr, double shift, int solver, double cg_tol, int ir_steps, int* iters, double* relres,
                     double* cg_err) {
    if (!sr->constructed) throw Error(YQ_E_STATE, "solve: call construct first");
    YQ_CHECK_ARG(shift >= 0.0, "solve: shift must be >= 0");
    YQ_CHECK_ARG(ir_steps <= 64, "solve: at most 64 CG steps");
    *cg_err = 0.;
    const bool c64 = sr->q->dtype == YQ_C64;
    const bool use_cg = solver == YQ_SOLVE_CG && sr->beta2 == 0.0;  // RunRBM.hpp:184
    if (sr->beta2 != 0.0 && sr->mode != YQ_SR_S)
        throw Error(YQ_E_UNSUPPORTED, "iteration: averaging the Fisher matrix (beta2 != 0) needs the S-form");
    if (sr->beta1 != 0.0 && sr->mode == YQ_SR_T && !use_cg && !(shift > 0.0))
        throw Error(YQ_E_ARG, "iteration: gradient momentum in the T-form needs shift > 0");
    cudaStream_t st = sr->q->ctx->stream;
    const size_t P = sr->q->P;
    const unsigned g = std::min(148u * 8, cdiv_u(P, 256));
    // gradAvg.update(energyGrad()); grad = gradAvg.getAvg()  (RunRBM.hpp:180-181)
    const c128* rhs = nullptr;
    auto grad_update = [&] {
        if (sr->t_grad == 0) {
            sr->gavg.ensure(P * sizeof(c128));
            YQ_CUDA(cudaMemsetAsync(sr->gavg.p, 0, P * sizeof(c128), st));
        }
        ema_kernel<<<g, 256, 0, st>>>(P, sr->beta1, sr->grad.as<c128>(), sr->gavg.as<c128>());
        YQ_LAUNCH_CHECK();
        ++sr->t_grad;
    };
    if (sr->beta1 != 0.0) {
        grad_update();
        sr->gused.ensure(P * sizeof(c128));
        avg_div_kernel<<<g, 256, 0, st>>>(P, 1.0 - std::pow(sr->beta1, double(sr->t_grad)), sr->gavg.as<c128>(),
                                          sr->gused.as<c128>());
        YQ_LAUNCH_CHECK();
        rhs = sr->gused.as<c128>();
    }
    if (use_cg) {
        const c128* b = rhs ? rhs : sr->grad.as<c128>();
        sr->q->ctx->stage_begin(ST_SOLVE);
        if (c64)
            solve_cg_t<float>(sr, b, shift, cg_tol, iters, relres);
        else
            solve_cg_t<double>(sr, b, shift, cg_tol, iters, relres);
        *cg_err = c64 ? cg_residual_norm<float>(sr, b, shift) : cg_residual_norm<double>(sr, b, shift);
        sr->q->ctx->stage_end(ST_SOLVE);
    } else {
        if (sr->beta1 != 0.0) grad_update();  // the second gradAvg.update of RunRBM.hpp:186
        const double fb = sr->beta2 != 0.0 ? sr->beta2 : -1.0;
        if (c64)
            solve_llt_t<float>(sr, shift, ir_steps, rhs, fb);
        else
            solve_llt_t<double>(sr, shift, ir_steps, rhs, fb);
        if (iters) *iters = 0;
        if (relres) *relres = 0.;
    }
    sr->solved = true;
}

void sr_form_matrix_public(yq_sr_s* sr, double shift) { form_matrix(sr, shift); }

// |v| into stats[4] and the clip factor min(1, clip / |v|) into stats[5]
// (RunRBM.hpp:205-209; clip 0 disables it).
__global__ void norm_clip_kernel(int nb, double clip, const double* __restrict__ part, double* __restrict__ stats,
                                 int* __restrict__ status) {
    double r = 0.;
    for (int i = 0; i < nb; ++i) r += part[i];
    const double nv = sqrt(r);
    stats[4] = nv;
    stats[5] = (clip != 0.0 && nv > clip) ? clip / nv : 1.0;
    if (!isfinite(r)) atomicOr(status, DS_NONFINITE);
}

__global__ void norm_parts_kernel(size_t P, const c128* __restrict__ v, double* __restrict__ part) {
    __shared__ double red[8];
    double acc = 0.;
    for (size_t p = size_t(blockIdx.x) * blockDim.x + threadIdx.x; p < P; p += size_t(gridDim.x) * blockDim.x)
        acc += v[p].re * v[p].re + v[p].im * v[p].im;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, o);
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = acc;
    __syncthreads();
    if (threadIdx.x == 0) {
        double s = 0.;
        for (int w = 0; w < int(blockDim.x >> 5); ++w) s += red[w];
        part[blockIdx.x] = s;
    }
}

__global__ void clipped_update_kernel(size_t P, double lr, const double* __restrict__ stats,
                                      const c128* __restrict__ v, c128* __restrict__ p64) {
    const double s = lr * stats[5];
    for (size_t p = size_t(blockIdx.x) * blockDim.x + threadIdx.x; p < P; p += size_t(gridDim.x) * blockDim.x)
        p64[p] = p64[p] - s * v[p];
}

void sr_update_params(yq_sr_s* sr, double lr) {
    if (!sr->solved) throw Error(YQ_E_STATE, "update: call solve first");
    yq_ctx_s* ctx = sr->q->ctx;
    cudaStream_t st = ctx->stream;
    ctx->stage_begin(ST_UPDATE);
    const int blocks = 148;
    if (sr->grad_clip == 0.0) {
        update_kernel<<<blocks, 256, 0, st>>>(sr->q->P, lr, sr->v.as<c128>(), sr->q->p64.as<c128>(),
                                              ctx->scratch.as<double>());
        finish_norm_kernel<<<1, 1, 0, st>>>(blocks, ctx->scratch.as<double>(), sr->stats.as<double>(),
                                            ctx->status.as<int>());
        YQ_LAUNCH_CHECK();
    } else {
        // |v| first, then the update scaled by the clip factor (device-side, no host round trip)
        norm_parts_kernel<<<blocks, 256, 0, st>>>(sr->q->P, sr->v.as<c128>(), ctx->scratch.as<double>());
        norm_clip_kernel<<<1, 1, 0, st>>>(blocks, sr->grad_clip, ctx->scratch.as<double>(), sr->stats.as<double>(),
                                          ctx->status.as<int>());
        clipped_update_kernel<<<blocks, 256, 0, st>>>(sr->q->P, lr, sr->stats.as<double>(), sr->v.as<c128>(),
                                                      sr->q->p64.as<c128>());
        YQ_LAUNCH_CHECK();
    }
    sr->q->version++;
    ctx->stage_end(ST_UPDATE);
}

}  // namespace yq
