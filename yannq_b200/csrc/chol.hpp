// Blocked FP64 Cholesky of the shifted SR matrix and the triangular solves
// (the Eigen::LLT of GroundState/SRMat.hpp:231-237 and Runners/RunRBM.hpp:196-201).
#pragma once
#include "common.cuh"

namespace yq {

constexpr int CHOL_NB = 64;

// In-place lower Cholesky of the Hermitian matrix G (row-major, n x n, n a multiple
// of CHOL_NB, lower triangle used).  Linv / LinvH receive, per diagonal block, the
// inverse of L_kk and its conjugate transpose (n / CHOL_NB blocks of 64 x 64).
// A non-positive pivot sets DS_NOT_PD in *status (the factorisation continues with
// a unit pivot so that every launch stays well defined).
void chol_factor(c128* G, int n, size_t ld, c128* Linv, c128* LinvH, int* status, cudaStream_t st);

// out = (L L^H)^{-1} b.  b is overwritten (forward sweep), work holds L^{-1} b.
void chol_solve(const c128* G, int n, size_t ld, const c128* Linv, const c128* LinvH, c128* b, c128* work,
                c128* out, cudaStream_t st);

// Persistent tile variants (chol_tile.cu): one cooperative launch each for the
// factorisation and for each sweep of the solve.  `scratch` holds the tile
// flags, the work counter and the tile order (chol_tile_scratch_bytes(n) bytes).
size_t chol_tile_scratch_bytes(int n);
void chol_factor_tiled(c128* G, int n, size_t ld, c128* Linv, c128* LinvH, int* status, void* scratch,
                       int sm_count, cudaStream_t st);
// Panel form for matrices whose accuracy is that of the BF16x3 products: the
// persistent FP64 tile kernel factors each CHOL_PANEL-wide block column (tiles
// updated only by the columns of their own panel), and the trailing matrix is
// updated once per panel on the tensor cores (C -= L21 L21^H, BF16x3, FP32
// accumulation).  `planes` holds chol_panel_planes_bytes(n) bytes of split operands.
constexpr int CHOL_PANEL = 512;
size_t chol_panel_planes_bytes(int n);
void chol_factor_panels(c128* G, int n, size_t ld, c128* Linv, c128* LinvH, int* status, void* scratch,
                        void* planes, int sm_count, cudaStream_t st);
// out = (L L^H)^{-1} b; out may be b.  `scratch` also holds the forward result.
void chol_solve_tiled(const c128* G, int n, size_t ld, const c128* Linv, const c128* LinvH, c128* b, c128* out,
                      int* status, void* scratch, int sm_count, cudaStream_t st);

// Failure injection for the bounded flag waits (tests only): which = 0 the tile
// factorisation, 1 the forward solve, each with the flag of its first work item
// never published and a wait limit of `cap` polls.  Returns the flags published.
int chol_debug_unpublished_flag(int which, unsigned cap, int* status, int sm_count, cudaStream_t st);

}  // namespace yq
