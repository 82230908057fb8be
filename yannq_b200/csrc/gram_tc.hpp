// Tensor-core (tcgen05) Gram matrix of the mixed-precision SR path:
//   T = O~ O~^H / Ns + shift I   from complex64 O~ (Ns x P, row-major),
// as one real GEMM  [X; Y] X^T  with X = [Re O~ | Im O~], Y = [Im O~ | -Re O~]
// (T_re = X X^T, T_im = Y X^T), each operand split into BF16 hi + lo parts and
// the three products hi.hi + hi.lo + lo.hi accumulated in FP32 in TMEM.
#pragma once
#include <cstddef>
#include <cstdint>

#include "common.cuh"

namespace yq {

constexpr int TC_BM = 128;  // rows of a tile (TMEM lanes)
constexpr int TC_BN = 128;  // columns of a tile (TMEM columns, FP32)
constexpr int TC_BK = 64;   // K per stage: 64 BF16 = one 128-byte swizzle atom row

// K extent (2P) padded to the stage depth, and the padded row count of the operands.
inline size_t gram_tc_kpad(size_t P) { return ((2 * P + TC_BK - 1) / TC_BK) * TC_BK; }
inline size_t gram_tc_rows(int ns) { return ((size_t(ns) + TC_BM - 1) / TC_BM) * TC_BM; }

// Split O~ into the four BF16 planes (rows padded with zeros to gram_tc_rows(ns),
// K padded with zeros to gram_tc_kpad(P)).
void gram_tc_prepare_operands(const c64* O, int ns, size_t P, uint16_t* xh, uint16_t* xl, uint16_t* yh, uint16_t* yl,
                              cudaStream_t st);

// G[r, c] (r >= c, r, c < ns) = alpha * T_(r,c) + shift * [r == c], complex FP64, row stride ldg.
void gram_tc_run(const uint16_t* xh, const uint16_t* xl, const uint16_t* yh, const uint16_t* yl, int ns, size_t P,
                 c128* G, size_t ldg, double alpha, double shift, int* d_status, cudaStream_t st);

}  // namespace yq
