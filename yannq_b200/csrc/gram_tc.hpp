// Tensor-core (tcgen05) Hermitian rank-k kernels of the mixed-precision SR path.
//
// For a complex matrix A (rows x K) the product A A^H is one real GEMM pair
//   Re(A A^H) = X X^T,  Im(A A^H) = Y X^T,   X = [Re A | Im A],  Y = [Im A | -Re A],
// with every operand split into BF16 hi + lo parts and the three products
// hi.hi + hi.lo + lo.hi accumulated in FP32 in TMEM.  The same kernel forms the
// Gram matrix T = O~ O~^H / Ns + shift I and applies the trailing updates
// C -= L21 L21^H of the panel Cholesky.
#pragma once
#include <cuda_bf16.h>

#include <cstddef>
#include <cstdint>

#include "common.cuh"

namespace yq {

// Operand split: X = [Re | Im], Y = [Im | -Re]; x = hi + lo with hi = bf16(x),
// lo = bf16(x - hi).
__device__ __forceinline__ void split_bf16(float v, uint16_t& hi, uint16_t& lo) {
    __nv_bfloat16 h = __float2bfloat16_rn(v);
    __nv_bfloat16 l = __float2bfloat16_rn(v - __bfloat162float(h));
    hi = __bfloat16_as_ushort(h);
    lo = __bfloat16_as_ushort(l);
}

constexpr int TC_BM = 128;  // rows of a tile (TMEM lanes)
constexpr int TC_BK = 64;   // K per stage: 64 BF16 = one 128-byte swizzle atom row

// K extent (2P) padded to the stage depth, and the padded row count of the operands.
inline size_t gram_tc_kpad(size_t P) { return ((2 * P + TC_BK - 1) / TC_BK) * TC_BK; }
inline size_t gram_tc_rows(int ns) { return ((size_t(ns) + TC_BM - 1) / TC_BM) * TC_BM; }

// The centred complex64 rows O~[s, p] = [s_i t_j | s | t] - oloc (row-major, P per
// row) of the mixed T path and, from the same stored values, the four BF16 planes
// X = [Re | Im], Y = [Im | -Re] split into hi and lo (rows padded with zeros to
// gram_tc_rows(ns), K padded with zeros to gram_tc_kpad(P)), in one pass.
void gram_tc_write_o_and_operands(int n, int m, bool bias, size_t P, int ns, const int8_t* sigma, const c64* t,
                                  const c128* oloc, c64* O, uint16_t* xh, uint16_t* xl, uint16_t* yh, uint16_t* yl,
                                  cudaStream_t st);

// G[r, c] (r >= c, r, c < ns) = alpha * T_(r,c) + shift * [r == c], complex FP64, row stride ldg.
// The tiles left after the last full wave of sm_count CTAs (one CTA per SM) are
// split along K into chunks whose FP32 partials go to `ws` (grown as needed, at
// most sm_count x 256 KiB) and are summed in a fixed order in FP64.
void gram_tc_run(const uint16_t* xh, const uint16_t* xl, const uint16_t* yh, const uint16_t* yl, int ns, size_t P,
                 c128* G, size_t ldg, double alpha, double shift, int* d_status, int sm_count, DevBuf& ws,
                 cudaStream_t st);

// General form over planes of `rows_pad` rows (a multiple of 128) and `kpad` BF16
// columns (a multiple of 64):  for r >= c, r, c < n
//   C[r, c] = (accumulate ? C[r, c] : 0) + alpha (A A^H)_(r,c) + shift [r == c].
void herk_tc_run(const uint16_t* xh, const uint16_t* xl, const uint16_t* yh, const uint16_t* yl, int n,
                 size_t rows_pad, size_t kpad, c128* C, size_t ldc, double alpha, double shift, bool accumulate,
                 int* d_status, cudaStream_t st);
// False when YQ_TC_SPLIT=0: the K-splits below then keep whole tiles.
bool tc_split_enabled();

// The same with the K-split of the tiles after the last full wave of sm_count CTAs:
// the partials go to `ws` (grown as needed) or, when ws is null, to `ws_fixed` if the
// split fits in ws_fixed_bytes (at most sm_count x 256 KiB); otherwise whole tiles.
void herk_tc_launch(const uint16_t* xh, const uint16_t* xl, const uint16_t* yh, const uint16_t* yl, int n,
                    size_t rows_pad, size_t kpad, c128* C, size_t ldc, double alpha, double shift, bool accumulate,
                    int* d_status, int sm_count, DevBuf* ws, float2* ws_fixed, size_t ws_fixed_bytes,
                    cudaStream_t st);

}  // namespace yq
