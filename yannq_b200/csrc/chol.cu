// Recursive FP64 Cholesky (lower, row-major, in place) and triangular solves of
// the SR step (the Eigen::LLT of GroundState/SRMat.hpp:231-237).
//
//   chol(A):  L11 = chol(A11);  L21 = A21 L11^{-H} (recursive TRSM);
//             A22 -= L21 L21^H (HERK, K = n/2);  L22 = chol(A22)
//   trsm:     X [La 0; Lb Lc]^H = [Ba Bb]:  Xa = Ba La^{-H};  Bb -= Xa Lb^H;  Xb = Bb Lc^{-H}
//
// Almost all flops land in large-K complex GEMMs (gemm64.cuh).  The recursion
// bottoms out in 64-wide blocks:
//   chol_diag_kernel   one CTA: unblocked factorisation of a 64 x 64 diagonal block
//                      in shared memory, then its inverse by the blocked recursion
//                      X21 = -X22 (L21 X11) over 8 -> 16 -> 32 -> 64 (log depth);
//   chol_panel_kernel  X = B L_kk^{-H} for 64 columns (product with the stored inverse).
// The solves recurse the same way; their base cases multiply by the stored
// inverses and their off-diagonal steps are coalesced matrix-vector products.
#include <algorithm>

#include "chol.hpp"
#include "gemm64.cuh"
#include "internal.hpp"

namespace yq {

namespace {
constexpr int NB = CHOL_NB;
constexpr int LDS = NB + 1;  // padded shared-memory row stride (complex elements)
constexpr size_t SM_DIAG = size_t(3) * NB * LDS * sizeof(c128);
constexpr size_t SM_PANEL = (size_t(NB) * NB + size_t(32) * LDS) * sizeof(c128);

__device__ __forceinline__ c128 warp_sum_c(c128 v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        v.re += __shfl_xor_sync(0xffffffffu, v.re, o);
        v.im += __shfl_xor_sync(0xffffffffu, v.im, o);
    }
    return v;
}

inline int split_half(int size) { return ((size / NB) / 2) * NB; }
}  // namespace

__global__ void __launch_bounds__(256) chol_diag_kernel(c128* __restrict__ G, size_t ld, int k0,
                                                        c128* __restrict__ Linv, c128* __restrict__ LinvH,
                                                        int* __restrict__ status) {
    extern __shared__ c128 sm[];
    c128* A = sm;
    c128* X = A + NB * LDS;
    c128* T = X + NB * LDS;
    const int tid = threadIdx.x;
    for (int e = tid; e < NB * NB; e += blockDim.x) {
        const int r = e / NB, c = e % NB;
        A[r * LDS + c] = (c <= r) ? G[size_t(k0 + r) * ld + k0 + c] : mk(0., 0.);
        X[r * LDS + c] = mk(0., 0.);
    }
    __syncthreads();
    for (int c = 0; c < NB; ++c) {
        if (tid == 0) {
            double d = A[c * LDS + c].re;
            if (!(d > 0.0)) {
                atomicOr(status, DS_NOT_PD);
                d = 1.0;
            }
            A[c * LDS + c] = mk(sqrt(d), 0.0);
        }
        __syncthreads();
        const double inv = 1.0 / A[c * LDS + c].re;
        for (int r = c + 1 + tid; r < NB; r += blockDim.x) A[r * LDS + c] = inv * A[r * LDS + c];
        __syncthreads();
        const int w = NB - c - 1;
        const int tri = w * (w + 1) / 2;  // lower triangle of the trailing block, row by row
        for (int e = tid; e < tri; e += blockDim.x) {
            int r = int((sqrtf(8.0f * float(e) + 1.0f) - 1.0f) * 0.5f);
            while (r * (r + 1) / 2 > e) --r;
            while ((r + 1) * (r + 2) / 2 <= e) ++r;
            const int q = e - r * (r + 1) / 2;
            const int rr = c + 1 + r, qq = c + 1 + q;
            A[rr * LDS + qq] = A[rr * LDS + qq] - A[rr * LDS + c] * conj(A[qq * LDS + c]);
        }
        __syncthreads();
    }
    // inverse of the 8 x 8 diagonal blocks: one column per thread
    if (tid < NB) {
        const int o = (tid >> 3) * 8, col = tid & 7;
        for (int r = col; r < 8; ++r) {
            c128 acc = mk(r == col ? 1.0 : 0.0, 0.0);
            for (int q = col; q < r; ++q) acc = acc - A[(o + r) * LDS + o + q] * X[(o + q) * LDS + o + col];
            X[(o + r) * LDS + o + col] = (1.0 / A[(o + r) * LDS + o + r].re) * acc;
        }
    }
    __syncthreads();
    // [[L11, 0], [L21, L22]]^{-1} = [[X11, 0], [-X22 L21 X11, X22]], block sizes 8, 16, 32
    for (int s = 8; s < NB; s *= 2) {
        const int cnt = (NB / (2 * s)) * s * s;
        for (int e = tid; e < cnt; e += blockDim.x) {
            const int p = e / (s * s), i = (e / s) % s, j = e % s, o = 2 * s * p;
            c128 acc = mk(0., 0.);
            for (int q = j; q < s; ++q) acc = acc + A[(o + s + i) * LDS + o + q] * X[(o + q) * LDS + o + j];
            T[(o + i) * LDS + o + j] = acc;
        }
        __syncthreads();
        for (int e = tid; e < cnt; e += blockDim.x) {
            const int p = e / (s * s), i = (e / s) % s, j = e % s, o = 2 * s * p;
            c128 acc = mk(0., 0.);
            for (int q = 0; q <= i; ++q) acc = acc + X[(o + s + i) * LDS + o + s + q] * T[(o + q) * LDS + o + j];
            X[(o + s + i) * LDS + o + j] = mk(-acc.re, -acc.im);
        }
        __syncthreads();
    }
    for (int e = tid; e < NB * NB; e += blockDim.x) {
        const int r = e / NB, c = e % NB;
        if (c <= r) G[size_t(k0 + r) * ld + k0 + c] = A[r * LDS + c];
        Linv[e] = X[r * LDS + c];
        LinvH[e] = conj(X[c * LDS + r]);
    }
}

// X[r, k0:k0+64] = B[r, k0:k0+64] (L_kk^{-1})^H for rows r in [r_begin, r_end), 32 per CTA.
__global__ void __launch_bounds__(256) chol_panel_kernel(c128* __restrict__ G, size_t ld, int k0, int r_begin,
                                                         int r_end, const c128* __restrict__ LinvH) {
    extern __shared__ c128 sm[];
    c128* LH = sm;            // [64][64]
    c128* Ar = sm + NB * NB;  // [32][LDS]
    const int tid = threadIdx.x;
    const int rbase = r_begin + blockIdx.x * 32;
    for (int e = tid; e < NB * NB; e += blockDim.x) LH[e] = LinvH[e];
    for (int e = tid; e < 32 * NB; e += blockDim.x) {
        const int rr = e / NB, c = e % NB, r = rbase + rr;
        Ar[rr * LDS + c] = (r < r_end) ? G[size_t(r) * ld + k0 + c] : mk(0., 0.);
    }
    __syncthreads();
    const int rr = tid >> 3, cg = tid & 7, r = rbase + rr;
    if (r >= r_end) return;
#pragma unroll
    for (int q = 0; q < 8; ++q) {
        const int c = cg + 8 * q;
        c128 acc = mk(0., 0.);
        for (int qq = 0; qq <= c; ++qq) acc = acc + Ar[rr * LDS + qq] * LH[qq * NB + c];
        G[size_t(r) * ld + k0 + c] = acc;
    }
}

// In-place x_k = M x_k for one 64-block with M = L_kk^{-1} (forward) or L_kk^{-H} (backward).
__global__ void __launch_bounds__(256) chol_block_apply_kernel(const c128* __restrict__ Mk, c128* __restrict__ x) {
    __shared__ c128 xb[NB];
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    if (tid < NB) xb[tid] = x[tid];
    __syncthreads();
#pragma unroll
    for (int i = 0; i < NB / 8; ++i) {
        const int r = warp * (NB / 8) + i;
        const c128* Mr = Mk + r * NB;
        c128 v = warp_sum_c(Mr[lane] * xb[lane] + Mr[lane + 32] * xb[lane + 32]);
        if (lane == 0) x[r] = v;
    }
}

// y[r] -= sum_k A[r, k] x[k], r < m, k < kk  (warp per row)
__global__ void __launch_bounds__(256) gemv_sub_kernel(const c128* __restrict__ A, size_t ld, int m, int kk,
                                                       const c128* __restrict__ x, c128* __restrict__ y) {
    const int warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5, lane = threadIdx.x & 31;
    if (warp >= m) return;
    const c128* row = A + size_t(warp) * ld;
    c128 acc = mk(0., 0.);
    for (int k = lane; k < kk; k += 32) acc = acc + row[k] * x[k];
    acc = warp_sum_c(acc);
    if (lane == 0) y[warp] = y[warp] - acc;
}

// y[c] -= sum_r conj(A[r, c]) x[r], c < kk, r < m  (32 columns per CTA, 8 warps split the rows)
__global__ void __launch_bounds__(256) gemv_h_sub_kernel(const c128* __restrict__ A, size_t ld, int m, int kk,
                                                         const c128* __restrict__ x, c128* __restrict__ y) {
    __shared__ c128 part[8][32];
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int c = blockIdx.x * 32 + lane;
    c128 acc = mk(0., 0.);
    if (c < kk)
        for (int r = warp; r < m; r += 8) acc = acc + conj(A[size_t(r) * ld + c]) * x[r];
    part[warp][lane] = acc;
    __syncthreads();
    if (warp == 0 && c < kk) {
        c128 s = part[0][lane];
        for (int w = 1; w < 8; ++w) s = s + part[w][lane];
        y[c] = y[c] - s;
    }
}

// ---------------------------------------------------------------------------
namespace {
struct CholCtx {
    c128* G;
    size_t ld;
    c128* Linv;
    c128* LinvH;
    int* status;
    cudaStream_t st;
};

void trsm_rec(const CholCtx& C, int row0, int nrows, int col0, int width) {
    if (nrows <= 0) return;
    if (width == NB) {
        chol_panel_kernel<<<cdiv_u(nrows, 32), 256, SM_PANEL, C.st>>>(C.G, C.ld, col0, row0, row0 + nrows,
                                                                      C.LinvH + size_t(col0 / NB) * NB * NB);
        YQ_LAUNCH_CHECK();
        return;
    }
    const int h = split_half(width);
    trsm_rec(C, row0, nrows, col0, h);
    // Bb -= Xa Lb^H:  Xa = G[row0.., col0..col0+h), Lb = G[col0+h.., col0..col0+h)
    gemm_c64acc<double>(C.G + size_t(row0) * C.ld + col0, C.ld, C.G + size_t(col0 + h) * C.ld + col0, C.ld, 0, nrows,
                        width - h, h, C.G + size_t(row0) * C.ld + col0 + h, C.ld, -1.0, 1, 0.0, 0, C.st);
    trsm_rec(C, row0, nrows, col0 + h, width - h);
}

void chol_rec(const CholCtx& C, int off, int size) {
    if (size == NB) {
        chol_diag_kernel<<<1, 256, SM_DIAG, C.st>>>(C.G, C.ld, off, C.Linv + size_t(off / NB) * NB * NB,
                                                    C.LinvH + size_t(off / NB) * NB * NB, C.status);
        YQ_LAUNCH_CHECK();
        return;
    }
    const int h = split_half(size);
    chol_rec(C, off, h);
    trsm_rec(C, off + h, size - h, off, h);
    gram_fp64<double>(C.G + size_t(off + h) * C.ld + off, C.ld, 0, size - h, h, C.G + size_t(off + h) * C.ld + off + h,
                      C.ld, -1.0, 1, 0.0, C.st);
    chol_rec(C, off + h, size - h);
}

void fwd_rec(const CholCtx& C, int off, int size, c128* b) {
    if (size == NB) {
        chol_block_apply_kernel<<<1, 256, 0, C.st>>>(C.Linv + size_t(off / NB) * NB * NB, b + off);
        YQ_LAUNCH_CHECK();
        return;
    }
    const int h = split_half(size);
    fwd_rec(C, off, h, b);
    gemv_sub_kernel<<<cdiv_u(size_t(size - h) * 32, 256), 256, 0, C.st>>>(C.G + size_t(off + h) * C.ld + off, C.ld,
                                                                          size - h, h, b + off, b + off + h);
    YQ_LAUNCH_CHECK();
    fwd_rec(C, off + h, size - h, b);
}

void bwd_rec(const CholCtx& C, int off, int size, c128* b) {
    if (size == NB) {
        chol_block_apply_kernel<<<1, 256, 0, C.st>>>(C.LinvH + size_t(off / NB) * NB * NB, b + off);
        YQ_LAUNCH_CHECK();
        return;
    }
    const int h = split_half(size);
    bwd_rec(C, off + h, size - h, b);
    gemv_h_sub_kernel<<<cdiv_u(h, 32), 256, 0, C.st>>>(C.G + size_t(off + h) * C.ld + off, C.ld, size - h, h,
                                                       b + off + h, b + off);
    YQ_LAUNCH_CHECK();
    bwd_rec(C, off, h, b);
}
}  // namespace

void chol_factor(c128* G, int n, size_t ld, c128* Linv, c128* LinvH, int* status, cudaStream_t st) {
    YQ_CHECK_ARG(n % NB == 0 && n > 0, "cholesky: dimension must be a positive multiple of 64");
    static bool attrs = false;
    if (!attrs) {
        YQ_CUDA(cudaFuncSetAttribute(chol_diag_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, int(SM_DIAG)));
        YQ_CUDA(cudaFuncSetAttribute(chol_panel_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, int(SM_PANEL)));
        attrs = true;
    }
    chol_rec(CholCtx{G, ld, Linv, LinvH, status, st}, 0, n);
}

void chol_solve(const c128* G, int n, size_t ld, const c128* Linv, const c128* LinvH, c128* b, c128* work,
                c128* out, cudaStream_t st) {
    CholCtx C{const_cast<c128*>(G), ld, const_cast<c128*>(Linv), const_cast<c128*>(LinvH), nullptr, st};
    (void)work;
    fwd_rec(C, 0, n, b);
    bwd_rec(C, 0, n, b);
    YQ_CUDA(cudaMemcpyAsync(out, b, size_t(n) * sizeof(c128), cudaMemcpyDeviceToDevice, st));
}

}  // namespace yq
