// FP64-accumulating complex GEMM / HERK used by the SR matrix of the plain FP64
// path and by the recursive Cholesky and TRSM:
//
//   C(r, c) = [C(r, c) +] alpha * sum_k A(r, k) conj(B(c, k))  [+ shift if r == c]
//
// A(r, k) = A[r lda + k] (KMODE 0: rows K-contiguous) or conj(A[k lda + r])
// (KMODE 1: columns K-contiguous, S = O~^H O~ from row-major O~); the same for B.
// `lower` restricts the work to the lower-triangle 64 x 64 tiles of a square C
// (elements r >= c written).  64 x 64 tiles, 128 threads with an 8 x 4 register
// tile each, 16-deep K chunks double-buffered in shared memory by cp.async.
#pragma once
#include "common.cuh"

namespace yq {

namespace gemm_detail {
constexpr int TM = 64, TK = 16, LDS = TM + 1;

template <int BYTES>
__device__ __forceinline__ void cp_async(void* smem, const void* gmem, bool valid) {
    const unsigned s = static_cast<unsigned>(__cvta_generic_to_shared(smem));
    const int src = valid ? BYTES : 0;  // zero-fill when out of range
    if (BYTES == 16)
        asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;" ::"r"(s), "l"(gmem), "r"(src) : "memory");
    else
        asm volatile("cp.async.ca.shared.global [%0], [%1], 8, %2;" ::"r"(s), "l"(gmem), "r"(src) : "memory");
}
__device__ __forceinline__ void cp_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
template <int N>
__device__ __forceinline__ void cp_wait() {
    asm volatile("cp.async.wait_group %0;" ::"n"(N) : "memory");
}
}  // namespace gemm_detail

template <typename R>
struct GemmArgs {
    const cplx<R>* A;
    size_t lda;
    const cplx<R>* B;
    size_t ldb;
    int M, N, K;
    c128* C;
    size_t ldc;
    double alpha;
    int accumulate;
    double shift;
    int lower;
};

template <typename R, int KMODE>
__global__ void __launch_bounds__(128) gemm_c64acc_kernel(GemmArgs<R> g) {
    using namespace gemm_detail;
    extern __shared__ __align__(16) unsigned char gsm[];
    typedef cplx<R> Tile[TK][LDS];
    Tile* As = reinterpret_cast<Tile*>(gsm);
    Tile* Bs = reinterpret_cast<Tile*>(gsm + 2 * sizeof(Tile));
    long long bi, bj;
    if (g.lower) {
        const long long t = blockIdx.x;
        bi = (long long)((sqrt(8.0 * double(t) + 1.0) - 1.0) * 0.5);
        while (bi * (bi + 1) / 2 > t) --bi;
        while ((bi + 1) * (bi + 2) / 2 <= t) ++bi;
        bj = t - bi * (bi + 1) / 2;
    } else {
        bi = blockIdx.y;
        bj = blockIdx.x;
    }
    const int r0 = int(bi) * TM, c0 = int(bj) * TM;
    const int tid = threadIdx.x, tr = tid >> 4, tc = tid & 15;
    const int nch = (g.K + TK - 1) / TK;

    auto load = [&](int buf, int ch) {
        const int k0 = ch * TK;
#pragma unroll
        for (int q = 0; q < 8; ++q) {
            const int e = tid + 128 * q;
            int row, kk;
            if (KMODE == 0) {
                row = e >> 4;
                kk = e & 15;
            } else {
                kk = e >> 6;
                row = e & 63;
            }
            const int k = k0 + kk, ra = r0 + row, rb = c0 + row;
            const bool va = k < g.K && ra < g.M, vb = k < g.K && rb < g.N;
            const cplx<R>* pa = KMODE == 0 ? g.A + (va ? size_t(ra) * g.lda + k : 0) : g.A + (va ? size_t(k) * g.lda + ra : 0);
            const cplx<R>* pb = KMODE == 0 ? g.B + (vb ? size_t(rb) * g.ldb + k : 0) : g.B + (vb ? size_t(k) * g.ldb + rb : 0);
            cp_async<sizeof(cplx<R>)>(&As[buf][kk][row], pa, va);
            cp_async<sizeof(cplx<R>)>(&Bs[buf][kk][row], pb, vb);
        }
        cp_commit();
    };

    double acc[8][4][2];
#pragma unroll
    for (int i = 0; i < 8; ++i)
#pragma unroll
        for (int j = 0; j < 4; ++j) acc[i][j][0] = acc[i][j][1] = 0.0;

    if (nch > 0) load(0, 0);
    for (int ch = 0; ch < nch; ++ch) {
        const int buf = ch & 1;
        if (ch + 1 < nch) {
            load(buf ^ 1, ch + 1);
            cp_wait<1>();
        } else {
            cp_wait<0>();
        }
        __syncthreads();
#pragma unroll 4
        for (int kk = 0; kk < TK; ++kk) {
            double ar[8], ai[8], br[4], bim[4];
#pragma unroll
            for (int i = 0; i < 8; ++i) {
                cplx<R> v = As[buf][kk][tr + 8 * i];
                ar[i] = double(v.re);
                ai[i] = KMODE == 0 ? double(v.im) : -double(v.im);
            }
#pragma unroll
            for (int j = 0; j < 4; ++j) {
                cplx<R> v = Bs[buf][kk][tc + 16 * j];
                br[j] = double(v.re);
                bim[j] = KMODE == 0 ? double(v.im) : -double(v.im);
            }
#pragma unroll
            for (int i = 0; i < 8; ++i)
#pragma unroll
                for (int j = 0; j < 4; ++j) {
                    // a * conj(b)
                    acc[i][j][0] = fma(ar[i], br[j], fma(ai[i], bim[j], acc[i][j][0]));
                    acc[i][j][1] = fma(ai[i], br[j], fma(-ar[i], bim[j], acc[i][j][1]));
                }
        }
        __syncthreads();
    }
#pragma unroll
    for (int i = 0; i < 8; ++i)
#pragma unroll
        for (int j = 0; j < 4; ++j) {
            const int r = r0 + tr + 8 * i, c = c0 + tc + 16 * j;
            if (r < g.M && c < g.N && (!g.lower || r >= c)) {
                c128* dst = g.C + size_t(r) * g.ldc + c;
                c128 v = mk(g.alpha * acc[i][j][0], g.alpha * acc[i][j][1]);
                if (g.accumulate) v = v + *dst;
                if (r == c) v.re += g.shift;
                *dst = v;
            }
        }
}

// ---------------------------------------------------------------------------
// FP64 tensor-core (DMMA, mma.sync m8n8k4 .f64) variant for complex128 operands.
// 128 threads = 2 x 2 warps, warp tile 32 x 32 = 4 x 4 sub-tiles of 8 x 8.  For each
// sub-tile two accumulators: Re += Ar Br + Ai Bi, Im += Ai Br + Ar (-Bi)
// (a conj(b) with the -Bi fragment negated on load).  Shared tiles are
// [row][k] with a 20-element row stride so that the 8-lane phases of the
// 16-byte fragment loads hit distinct banks.
namespace gemm_detail {
constexpr int DK = 16, DLS = 20;
}

__device__ __forceinline__ void dmma_m8n8k4(double (&d)[2], double a, double b) {
    asm volatile("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0,%1}, {%2}, {%3}, {%0,%1};"
                 : "+d"(d[0]), "+d"(d[1])
                 : "d"(a), "d"(b));
}

template <int KMODE>
__global__ void __launch_bounds__(128) gemm_z_dmma_kernel(GemmArgs<double> g) {
    using namespace gemm_detail;
    extern __shared__ __align__(16) unsigned char gsm[];
    typedef c128 Tile[64][DLS];
    Tile* As = reinterpret_cast<Tile*>(gsm);
    Tile* Bs = reinterpret_cast<Tile*>(gsm + 2 * sizeof(Tile));
    long long bi, bj;
    if (g.lower) {
        const long long t = blockIdx.x;
        bi = (long long)((sqrt(8.0 * double(t) + 1.0) - 1.0) * 0.5);
        while (bi * (bi + 1) / 2 > t) --bi;
        while ((bi + 1) * (bi + 2) / 2 <= t) ++bi;
        bj = t - bi * (bi + 1) / 2;
    } else {
        bi = blockIdx.y;
        bj = blockIdx.x;
    }
    const int r0 = int(bi) * 64, c0 = int(bj) * 64;
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const int wm = warp >> 1, wn = warp & 1;
    const int fr = lane >> 2, fk = lane & 3;  // fragment row / k of this lane
    const int nch = (g.K + DK - 1) / DK;

    auto load = [&](int buf, int ch) {
        const int k0 = ch * DK;
#pragma unroll
        for (int q = 0; q < 8; ++q) {
            const int e = tid + 128 * q;
            int row, kk;
            if (KMODE == 0) {
                row = e >> 4;
                kk = e & 15;
            } else {
                kk = e >> 6;
                row = e & 63;
            }
            const int k = k0 + kk, ra = r0 + row, rb = c0 + row;
            const bool va = k < g.K && ra < g.M, vb = k < g.K && rb < g.N;
            const c128* pa = KMODE == 0 ? g.A + (va ? size_t(ra) * g.lda + k : 0) : g.A + (va ? size_t(k) * g.lda + ra : 0);
            const c128* pb = KMODE == 0 ? g.B + (vb ? size_t(rb) * g.ldb + k : 0) : g.B + (vb ? size_t(k) * g.ldb + rb : 0);
            cp_async<16>(&As[buf][row][kk], pa, va);
            cp_async<16>(&Bs[buf][row][kk], pb, vb);
        }
        cp_commit();
    };

    double cre[4][4][2], cim[4][4][2];
#pragma unroll
    for (int i = 0; i < 4; ++i)
#pragma unroll
        for (int j = 0; j < 4; ++j) cre[i][j][0] = cre[i][j][1] = cim[i][j][0] = cim[i][j][1] = 0.0;

    if (nch > 0) load(0, 0);
    for (int ch = 0; ch < nch; ++ch) {
        const int buf = ch & 1;
        if (ch + 1 < nch) {
            load(buf ^ 1, ch + 1);
            cp_wait<1>();
        } else {
            cp_wait<0>();
        }
        __syncthreads();
#pragma unroll
        for (int ks = 0; ks < DK / 4; ++ks) {
            const int k = ks * 4 + fk;
            double ar[4], ai[4], br[4], bi_[4], bn[4];
#pragma unroll
            for (int i = 0; i < 4; ++i) {
                c128 v = As[buf][wm * 32 + i * 8 + fr][k];
                ar[i] = v.re;
                ai[i] = KMODE == 0 ? v.im : -v.im;
            }
#pragma unroll
            for (int j = 0; j < 4; ++j) {
                c128 v = Bs[buf][wn * 32 + j * 8 + fr][k];
                br[j] = v.re;
                bi_[j] = KMODE == 0 ? v.im : -v.im;
                bn[j] = -bi_[j];
            }
#pragma unroll
            for (int i = 0; i < 4; ++i)
#pragma unroll
                for (int j = 0; j < 4; ++j) {
                    dmma_m8n8k4(cre[i][j], ar[i], br[j]);
                    dmma_m8n8k4(cre[i][j], ai[i], bi_[j]);
                    dmma_m8n8k4(cim[i][j], ai[i], br[j]);
                    dmma_m8n8k4(cim[i][j], ar[i], bn[j]);
                }
        }
        __syncthreads();
    }
#pragma unroll
    for (int i = 0; i < 4; ++i)
#pragma unroll
        for (int j = 0; j < 4; ++j)
#pragma unroll
            for (int h = 0; h < 2; ++h) {
                const int r = r0 + wm * 32 + i * 8 + fr, c = c0 + wn * 32 + j * 8 + 2 * fk + h;
                if (r < g.M && c < g.N && (!g.lower || r >= c)) {
                    c128* dst = g.C + size_t(r) * g.ldc + c;
                    c128 v = mk(g.alpha * cre[i][j][h], g.alpha * cim[i][j][h]);
                    if (g.accumulate) v = v + *dst;
                    if (r == c) v.re += g.shift;
                    *dst = v;
                }
            }
}

// Launch helper.  lower != 0 requires M == N.
template <typename R>
static void gemm_c64acc(const cplx<R>* A, size_t lda, const cplx<R>* B, size_t ldb, int kmode, int M, int N, int K,
                        c128* C, size_t ldc, double alpha, int accumulate, double shift, int lower, cudaStream_t st);

template <>
void gemm_c64acc<double>(const c128* A, size_t lda, const c128* B, size_t ldb, int kmode, int M, int N, int K, c128* C,
                         size_t ldc, double alpha, int accumulate, double shift, int lower, cudaStream_t st) {
    if (M <= 0 || N <= 0) return;
    GemmArgs<double> g{A, lda, B, ldb, M, N, K, C, ldc, alpha, accumulate, shift, lower};
    dim3 grid;
    if (lower) {
        const long long nt = (M + 63) / 64;
        grid = dim3(unsigned(nt * (nt + 1) / 2));
    } else {
        grid = dim3(cdiv_u(N, 64), cdiv_u(M, 64));
    }
    const size_t smem = 4 * size_t(64) * gemm_detail::DLS * sizeof(c128);
    static bool attr = false;
    if (!attr) {
        YQ_CUDA(cudaFuncSetAttribute(gemm_z_dmma_kernel<0>, cudaFuncAttributeMaxDynamicSharedMemorySize, int(smem)));
        YQ_CUDA(cudaFuncSetAttribute(gemm_z_dmma_kernel<1>, cudaFuncAttributeMaxDynamicSharedMemorySize, int(smem)));
        attr = true;
    }
    if (kmode == 0)
        gemm_z_dmma_kernel<0><<<grid, 128, smem, st>>>(g);
    else
        gemm_z_dmma_kernel<1><<<grid, 128, smem, st>>>(g);
    YQ_LAUNCH_CHECK();
}

template <typename R>
static void gemm_c64acc(const cplx<R>* A, size_t lda, const cplx<R>* B, size_t ldb, int kmode, int M, int N, int K,
                        c128* C, size_t ldc, double alpha, int accumulate, double shift, int lower, cudaStream_t st) {
    if (M <= 0 || N <= 0) return;
    GemmArgs<R> g{A, lda, B, ldb, M, N, K, C, ldc, alpha, accumulate, shift, lower};
    dim3 grid;
    if (lower) {
        const long long nt = (M + 63) / 64;
        grid = dim3(unsigned(nt * (nt + 1) / 2));
    } else {
        grid = dim3(cdiv_u(N, 64), cdiv_u(M, 64));
    }
    const size_t smem = 4 * size_t(gemm_detail::TK) * gemm_detail::LDS * sizeof(cplx<R>);
    static bool attr = false;  // per template instantiation
    if (!attr) {
        YQ_CUDA(cudaFuncSetAttribute(gemm_c64acc_kernel<R, 0>, cudaFuncAttributeMaxDynamicSharedMemorySize, int(smem)));
        YQ_CUDA(cudaFuncSetAttribute(gemm_c64acc_kernel<R, 1>, cudaFuncAttributeMaxDynamicSharedMemorySize, int(smem)));
        attr = true;
    }
    if (kmode == 0)
        gemm_c64acc_kernel<R, 0><<<grid, 128, smem, st>>>(g);
    else
        gemm_c64acc_kernel<R, 1><<<grid, 128, smem, st>>>(g);
    YQ_LAUNCH_CHECK();
}

// Gram matrix of the rows of Z: C = alpha Z Z^H (lower tiles) [+ C] [+ shift I].
template <typename R>
static void gram_fp64(const cplx<R>* Z, size_t ldz, int kmode, int nrows, int K, c128* C, size_t ldc, double alpha,
                      int accumulate, double shift, cudaStream_t st) {
    gemm_c64acc<R>(Z, ldz, Z, ldz, kmode, nrows, nrows, K, C, ldc, alpha, accumulate, shift, 1, st);
}

}  // namespace yq
