// Persistent tile Cholesky and triangular solves (FP64, complex, lower, in place).
//
// One launch with at most one CTA per SM factors the whole matrix.  Tiles of
// 64 x 64 are numbered column by column (diagonal tile first in each column) and
// handed out in that order by an atomic counter; tile (i, j) computes
//   F = A_ij - sum_{k<j} L_ik L_jk^H          (DMMA m8n8k4, operands staged by cp.async)
//   i == j:  L_jj = chol(F) in shared memory, plus L_jj^{-1} and L_jj^{-H}
//   i >  j:  L_ij = F L_jj^{-H}
// and publishes a flag.  A tile waits only on tiles with smaller numbers (left
// columns, or the diagonal of its own column), which were handed out earlier to
// running CTAs, so the schedule cannot deadlock.  Every wait is bounded: a
// timeout sets DS_TIMEOUT and an abort word that makes every CTA stop.
//
// The solves use the same scheme with 64-row blocks: the forward sweep of block
// row r accumulates L[r, k] x_k as each x_k is published (its L tiles streamed
// into shared memory ahead of the flags), then applies L_rr^{-1}; the backward
// sweep runs the block rows in reverse with L^H.
#include <algorithm>
#include <vector>

#include "chol.hpp"
#include "gram_tc.hpp"
#include "internal.hpp"

namespace yq {

namespace {
constexpr int TB = 64;        // tile size
constexpr int KC = 16;        // K chunk of the staged operands
constexpr int SLS = 20;       // staged row stride (complex)
constexpr int FLS = TB + 1;   // factor-tile row stride (complex)
constexpr size_t SM_STAGE = size_t(4) * TB * SLS * sizeof(c128);   // 2 stages x {A, B}
constexpr size_t SM_FACTOR = size_t(3) * TB * FLS * sizeof(c128);  // F, X, T
constexpr size_t SM_TILE = SM_FACTOR > SM_STAGE ? SM_FACTOR : SM_STAGE;

__device__ __forceinline__ void cpa16(void* smem, const void* gmem) {
    const unsigned s = static_cast<unsigned>(__cvta_generic_to_shared(smem));
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"(s), "l"(gmem) : "memory");
}
__device__ __forceinline__ void cpa_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
__device__ __forceinline__ void cpa_wait_all() { asm volatile("cp.async.wait_group 0;" ::: "memory"); }
__device__ __forceinline__ void cpa_wait_one() { asm volatile("cp.async.wait_group 1;" ::: "memory"); }

__device__ __forceinline__ int ld_acquire(const int* p) {
    int v;
    asm volatile("ld.acquire.gpu.global.b32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
    return v;
}
__device__ __forceinline__ void st_release(int* p, int v) {
    asm volatile("st.release.gpu.global.b32 [%0], %1;" ::"l"(p), "r"(v) : "memory");
}
__device__ __forceinline__ int ld_relaxed(const int* p) {
    int v;
    asm volatile("ld.relaxed.gpu.global.b32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
    return v;
}
__device__ __forceinline__ void fence_acq_rel() { asm volatile("fence.acq_rel.gpu;" ::: "memory"); }

__device__ __forceinline__ void dmma(double (&d)[2], double a, double b) {
    asm volatile("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0,%1}, {%2}, {%3}, {%0,%1};"
                 : "+d"(d[0]), "+d"(d[1])
                 : "d"(a), "d"(b));
}

struct Sync {
    int* status;
    int* abort_word;
    unsigned cap;
};

// Thread 0 waits for *flag != 0 (bounded), then the CTA synchronises.  Returns
// false when this or another CTA gave up.
__device__ bool wait_flag(const int* flag, const Sync& S, int* s_ok) {
    if (threadIdx.x == 0) {
        int ok = 1;
        unsigned it = 0;
        while (ld_relaxed(flag) == 0) {
            // the abort word every 32 polls: one outstanding load per poll
            if ((++it & 31u) == 0 && (ld_acquire(S.abort_word) != 0 || it > S.cap)) {
                ok = 0;
                break;
            }
            __nanosleep(32);
        }
        if (ok) fence_acq_rel();  // with the relaxed read of the flag: an acquire pattern
        if (!ok && it > S.cap) {
            atomicOr(S.status, DS_TIMEOUT);
            atomicExch(S.abort_word, 1);
        }
        *s_ok = ok;
    }
    __syncthreads();
    return *s_ok != 0;
}

// Publishes a flag after every thread's global writes of the tile: the CTA
// barrier orders them before thread 0's gpu-scope fence, which is cumulative over
// what the barrier made it observe, and the release store then publishes them.
__device__ void publish(int* flag) {
    __syncthreads();
    if (threadIdx.x == 0) {
        __threadfence();
        st_release(flag, 1);
    }
}

// c += A B^H over K = 4 * nk for the warp's sub-tiles p < 4, q < NQ: rows
// 8 (rb + p) .. + 7 and columns 8 (cb + q) .. + 7 of the 64 x 64 product; with
// LOWER only the sub-tiles on or below the diagonal (p >= q, for rb == cb).  A and
// B are read from shared memory rows (row stride lda / ldb complex).
template <int NQ, bool LOWER>
__device__ __forceinline__ void warp_mma(const c128* A, int lda, const c128* B, int ldb, int nk, int rb, int cb, int fr,
                                         int fk, double (&cre)[4][4][2], double (&cim)[4][4][2]) {
    for (int ks = 0; ks < nk; ++ks) {
        const int k = ks * 4 + fk;
        double ar[4], ai[4], br[NQ], bi[NQ], bn[NQ];
#pragma unroll
        for (int i = 0; i < 4; ++i) {
            const c128 v = A[((rb + i) * 8 + fr) * lda + k];
            ar[i] = v.re;
            ai[i] = v.im;
        }
#pragma unroll
        for (int j = 0; j < NQ; ++j) {
            const c128 v = B[((cb + j) * 8 + fr) * ldb + k];
            br[j] = v.re;
            bi[j] = v.im;
            bn[j] = -v.im;
        }
#pragma unroll
        for (int i = 0; i < 4; ++i)
#pragma unroll
            for (int j = 0; j < NQ; ++j) {
                if (!LOWER || i >= j) {
                    dmma(cre[i][j], ar[i], br[j]);
                    dmma(cre[i][j], ai[i], bi[j]);
                    dmma(cim[i][j], ai[i], br[j]);
                    dmma(cim[i][j], ar[i], bn[j]);
                }
            }
    }
}

// Sub-tiles of a warp in the sums F = A_ij - sum_k L_ik L_jk^H.  Off-diagonal
// tiles: warp (wm, wn) owns the 32 x 32 block (wm, wn) (kind 0).  Diagonal tiles
// need only the lower triangle, 36 of the 64 sub-tiles, spread 10 / 10 / 8 / 8
// over the warps: the two diagonal 32 x 32 blocks' lower halves (kind 1) and the
// lower-left block as two 32 x 16 halves (kind 2), so the critical diagonal update
// costs 10 sub-tile products per warp instead of 16.
struct WarpTiles {
    int rb, cb, kind;
    __device__ __forceinline__ int nq() const { return kind == 2 ? 2 : 4; }
    __device__ __forceinline__ bool has(int p, int q) const { return q < nq() && (kind != 1 || p >= q); }
};
__device__ __forceinline__ WarpTiles warp_tiles(int warp, bool diag) {
    if (!diag) return WarpTiles{4 * (warp >> 1), 4 * (warp & 1), 0};
    if (warp < 2) return WarpTiles{4 * warp, 4 * warp, 1};
    return WarpTiles{4, 2 * (warp - 2), 2};
}
__device__ __forceinline__ void warp_mma_tiles(const WarpTiles& wt, const c128* A, int lda, const c128* B, int ldb,
                                               int nk, int fr, int fk, double (&cre)[4][4][2],
                                               double (&cim)[4][4][2]) {
    if (wt.kind == 0) warp_mma<4, false>(A, lda, B, ldb, nk, wt.rb, wt.cb, fr, fk, cre, cim);
    else if (wt.kind == 1) warp_mma<4, true>(A, lda, B, ldb, nk, wt.rb, wt.cb, fr, fk, cre, cim);
    else warp_mma<2, false>(A, lda, B, ldb, nk, wt.rb, wt.cb, fr, fk, cre, cim);
}

// L_ij = F X^H with X = L_jj^{-1} lower triangular: column block cb (columns
// 8 cb .. 8 cb + 7) sums over k < 8 (cb + 1) only.  Warp w owns the column blocks
// 7 - w and w over all 64 rows, 9 blocks of K work for every warp, 576 DMMA per
// warp instead of 1024 for the full product.
__device__ __forceinline__ void trsm_mma(const c128* F, const c128* X, int warp, int fr, int fk,
                                         double (&cre)[8][2][2], double (&cim)[8][2][2]) {
    const int cbs[2] = {7 - warp, warp};
    const int nk0 = 2 * (8 - warp), nk1 = 2 * (warp + 1);
    for (int ks = 0; ks < nk0; ++ks) {
        const int k = ks * 4 + fk;
        const bool two = ks < nk1;
        double ar[8], ai[8], br[2], bi[2], bn[2];
#pragma unroll
        for (int i = 0; i < 8; ++i) {
            const c128 v = F[(i * 8 + fr) * FLS + k];
            ar[i] = v.re;
            ai[i] = v.im;
        }
#pragma unroll
        for (int j = 0; j < 2; ++j) {
            const c128 v = (j == 0 || two) ? X[(cbs[j] * 8 + fr) * FLS + k] : mk(0., 0.);
            br[j] = v.re;
            bi[j] = v.im;
            bn[j] = -v.im;
        }
#pragma unroll
        for (int i = 0; i < 8; ++i)
#pragma unroll
            for (int j = 0; j < 2; ++j) {
                if (j == 0 || two) {
                    dmma(cre[i][j], ar[i], br[j]);
                    dmma(cre[i][j], ai[i], bi[j]);
                    dmma(cim[i][j], ai[i], br[j]);
                    dmma(cim[i][j], ar[i], bn[j]);
                }
            }
    }
}

// Factorisation of the 64 x 64 tile F (lower part) in shared memory and its
// inverse X = L^{-1}, by recursive halving (128 threads):
//   chol(A11) -> L11, X11;   L21 = A21 X11^H;   A22 -= L21 L21^H;
//   chol(A22) -> L22, X22;   X21 = -X22 (L21 X11),
// with the products on DMMA (m8n8k4, one 8 x 8 output tile per warp at a time)
// and 8 x 8 leaves factored and inverted by one warp in registers (two elements
// per lane; pivots and columns move by shuffles).  Levels of size 16 and below run
// in warp 0 alone (warp barriers), the levels above use all four warps.  T is
// scratch.  On exit F holds L in its lower triangle (the caller reads only that)
// and X holds L^{-1} with zeros above the diagonal.

// Warp 0: the 8 x 8 diagonal block at o, element-parallel.  Lane l holds row
// r = l >> 2 and columns q0 = l & 3, q1 = q0 + 4.  Right-looking factorisation:
// per column one pivot broadcast and three complex shuffles (the column entries of
// this lane's row and of its two columns), then the rank-1 update of the lane's
// elements, e -= a_rc conj(a_qc) / d with the product formed before the pivot's
// reciprocal square root is known; the inverse by right-looking substitution from
// the identity (row k is final after its scaling by 1 / L_kk, then rows below
// subtract L_rk X_k).  Every lane takes the same instruction stream (selects, no
// divergent branches), and the function is not inlined, so the leaves of one
// factorisation run one copy of the code that stays in the instruction cache:
// single-warp timings on a B200, 4.8k cycles per leaf with branches and inlined
// at each call site, 3.1k in this form once its code is cached.
__device__ __noinline__ void leaf8(c128* F, c128* X, int o, int* status) {
    const int lane = threadIdx.x & 31, r = lane >> 2, q0 = lane & 3;
    const int qq[2] = {q0, q0 + 4};
    c128 e[2];
#pragma unroll
    for (int h = 0; h < 2; ++h) e[h] = qq[h] <= r ? F[(o + r) * FLS + o + qq[h]] : mk(0., 0.);
    double sc[8];  // 1 / L_cc
    bool bad = false;
#pragma unroll
    for (int c = 0; c < 8; ++c) {
        const int hc = c >> 2, lc = c & 3;
        double d = __shfl_sync(0xffffffffu, e[hc].re, 4 * c + lc);
        bad |= !(d > 0.0);
        d = d > 0.0 ? d : 1.0;  // unit pivot keeps the launch well defined
        const double s = rsqrt(d);
        sc[c] = s;
        const double are = __shfl_sync(0xffffffffu, e[hc].re, 4 * r + lc);
        const double aim = __shfl_sync(0xffffffffu, e[hc].im, 4 * r + lc);
        double pre[2], pim[2];  // a_rc conj(a_qc)
#pragma unroll
        for (int h = 0; h < 2; ++h) {
            const double bre = __shfl_sync(0xffffffffu, e[hc].re, 4 * qq[h] + lc);
            const double bim = __shfl_sync(0xffffffffu, e[hc].im, 4 * qq[h] + lc);
            pre[h] = are * bre + aim * bim;
            pim[h] = aim * bre - are * bim;
        }
        const double s2 = s * s;
#pragma unroll
        for (int h = 0; h < 2; ++h) {
            const int q = qq[h];
            const c128 upd = mk(fma(-s2, pre[h], e[h].re), fma(-s2, pim[h], e[h].im));
            const c128 col = r == c ? mk(d * s, 0.0) : (r > c ? mk(s * are, s * aim) : e[h]);
            e[h] = (q > c && r >= q) ? upd : (q == c ? col : e[h]);
        }
    }
    if (bad && lane == 0) atomicOr(status, DS_NOT_PD);
    c128 y[2];
#pragma unroll
    for (int h = 0; h < 2; ++h) y[h] = mk(qq[h] == r ? 1.0 : 0.0, 0.0);
#pragma unroll
    for (int k = 0; k < 8; ++k) {
        const int hk = k >> 2, lk = k & 3;
        const double f = r == k ? sc[k] : 1.0;
#pragma unroll
        for (int h = 0; h < 2; ++h) y[h] = f * y[h];
        c128 lrk, xk[2];
        lrk.re = __shfl_sync(0xffffffffu, e[hk].re, 4 * r + lk);
        lrk.im = __shfl_sync(0xffffffffu, e[hk].im, 4 * r + lk);
#pragma unroll
        for (int h = 0; h < 2; ++h) {
            xk[h].re = __shfl_sync(0xffffffffu, y[h].re, 4 * k + q0);
            xk[h].im = __shfl_sync(0xffffffffu, y[h].im, 4 * k + q0);
        }
#pragma unroll
        for (int h = 0; h < 2; ++h) {
            const c128 nv = y[h] - lrk * xk[h];
            y[h] = r > k ? nv : y[h];
        }
    }
#pragma unroll
    for (int h = 0; h < 2; ++h) {
        const bool low = qq[h] <= r;
        F[(o + r) * FLS + o + qq[h]] = low ? e[h] : mk(0., 0.);
        X[(o + r) * FLS + o + qq[h]] = low ? y[h] : mk(0., 0.);
    }
}

enum { OP_BH = 0, OP_B = 1 };  // op(B) = B^H (B stored by output columns) or B (stored K x n)

// out (h x h, row stride FLS) = (acc ? out : 0) + alpha A op(B), K = h; A row-major
// (stride FLS).  Output 8 x 8 tiles are spread over `nw` warps starting at warp 0.
template <int H, int OP>
__device__ __forceinline__ void tile_prod(c128* out, const c128* A, const c128* B, double alpha, bool acc, int nw) {
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31, fr = lane >> 2, fk = lane & 3;
    constexpr int NT = H / 8;
    for (int t = warp; t < NT * NT; t += nw) {
        const int ti = t / NT, tj = t % NT;
        double cre[2] = {0., 0.}, cim[2] = {0., 0.};
#pragma unroll
        for (int ks = 0; ks < H / 4; ++ks) {
            const int k = ks * 4 + fk;
            const c128 a = A[(ti * 8 + fr) * FLS + k];
            c128 b;
            if (OP == OP_BH) b = conj(B[(tj * 8 + fr) * FLS + k]);
            else b = B[k * FLS + tj * 8 + fr];
            dmma(cre, a.re, b.re);
            dmma(cre, -a.im, b.im);
            dmma(cim, a.re, b.im);
            dmma(cim, a.im, b.re);
        }
#pragma unroll
        for (int h = 0; h < 2; ++h) {
            c128* po = out + (ti * 8 + fr) * FLS + tj * 8 + 2 * fk + h;
            const c128 v = mk(alpha * cre[h], alpha * cim[h]);
            *po = acc ? *po + v : v;
        }
    }
}

// The four products of the top level (H = 32, four warps) with their triangular
// shapes: the zero halves of L11^{-1} and L22^{-1} are skipped and the Hermitian
// update forms only its lower 8 x 8 tiles, so each warp issues at most 24 of the
// 32 tile k-steps of a full product (a full 32^3 product took 2.7k cycles on one
// SM).  Work per 8 x 8 output tile (ti, tj), in k-steps of 4:
//   P_UPPER_BH  out = A X^H, X lower:  k < 8 (tj + 1)   warp w owns row ti = w
//   P_LOWER_B   out = A X,   X lower:  k >= 8 tj         warp w owns row ti = w
//   P_LLOWER_B  out = X B,   X lower:  k < 8 (ti + 1)    warp w owns column tj = w
// (each warp 20 k-steps), and P_HERM out += alpha A A^H for ti >= tj (3 / 3 / 2 / 2
// tiles per warp of 8 k-steps each).
enum { P_UPPER_BH = 0, P_HERM = 1, P_LOWER_B = 2, P_LLOWER_B = 3 };
template <int MODE>
__device__ __forceinline__ void tile_prod32(c128* out, const c128* A, const c128* B, double alpha, bool acc) {
    constexpr int H = 32;
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31, fr = lane >> 2, fk = lane & 3;
    // P_HERM tile lists, 4 ti + tj in 4 bits per tile, 12 bits per warp: warp 0
    // (0,0) (1,0) (1,1); warp 1 (2,0) (2,1) (2,2); warp 2 (3,0) (3,1); warp 3 (3,2) (3,3)
    constexpr unsigned long long herm_tiles = 0xfe0dca98540ull;
    int ti[4], tj[4], lo[4], hi[4];
#pragma unroll
    for (int u = 0; u < 4; ++u) {
        if (MODE == P_UPPER_BH) { ti[u] = warp; tj[u] = u; lo[u] = 0; hi[u] = 2 * (u + 1); }
        else if (MODE == P_LOWER_B) { ti[u] = warp; tj[u] = u; lo[u] = 2 * u; hi[u] = H / 4; }
        else if (MODE == P_LLOWER_B) { ti[u] = u; tj[u] = warp; lo[u] = 0; hi[u] = 2 * (u + 1); }
        else {
            const bool on = u < (warp < 2 ? 3 : 2);
            const int code = on ? int((herm_tiles >> (12 * warp + 4 * u)) & 15u) : 0;
            ti[u] = code >> 2;
            tj[u] = code & 3;
            lo[u] = 0;
            hi[u] = on ? H / 4 : 0;
        }
    }
    double cre[4][2], cim[4][2];
#pragma unroll
    for (int u = 0; u < 4; ++u) cre[u][0] = cre[u][1] = cim[u][0] = cim[u][1] = 0.;
#pragma unroll
    for (int ks = 0; ks < H / 4; ++ks) {
        const int k = ks * 4 + fk;
#pragma unroll
        for (int u = 0; u < 4; ++u) {
            if (ks >= lo[u] && ks < hi[u]) {
                const c128 a = A[(ti[u] * 8 + fr) * FLS + k];
                const c128 b = (MODE == P_UPPER_BH || MODE == P_HERM) ? conj(B[(tj[u] * 8 + fr) * FLS + k])
                                                                     : B[k * FLS + tj[u] * 8 + fr];
                dmma(cre[u], a.re, b.re);
                dmma(cre[u], -a.im, b.im);
                dmma(cim[u], a.re, b.im);
                dmma(cim[u], a.im, b.re);
            }
        }
    }
#pragma unroll
    for (int u = 0; u < 4; ++u) {
        if (hi[u] > lo[u]) {
#pragma unroll
            for (int h = 0; h < 2; ++h) {
                c128* po = out + (ti[u] * 8 + fr) * FLS + tj[u] * 8 + 2 * fk + h;
                const c128 v = mk(alpha * cre[u][h], alpha * cim[u][h]);
                *po = acc ? *po + v : v;
            }
        }
    }
}

template <int N>
__device__ __forceinline__ void level_sync() {
    if (N <= 16) __syncwarp();
    else __syncthreads();
}

template <int N>
__device__ void chol_rec(c128* F, c128* X, c128* T, int o, int* status) {
    if constexpr (N == 8) {
        if ((threadIdx.x >> 5) == 0) leaf8(F, X, o, status);
    } else {
        constexpr int H = N / 2;
        const int nw = N <= 16 ? 1 : 4;
        const bool active = N > 16 || (threadIdx.x >> 5) == 0;
        c128* A21 = F + (o + H) * FLS + o;
        c128* A22 = F + (o + H) * FLS + o + H;
        c128* X11 = X + o * FLS + o;
        c128* X21 = X + (o + H) * FLS + o;
        c128* X22 = X + (o + H) * FLS + o + H;
        c128* L21 = T + (o + H) * FLS + o;   // lower scratch
        c128* W = T + o * FLS + o + H;       // upper scratch: L21 X11
        chol_rec<H>(F, X, T, o, status);
        level_sync<N>();
        if constexpr (H == 32) tile_prod32<P_UPPER_BH>(L21, A21, X11, 1.0, false);
        else if (active) tile_prod<H, OP_BH>(L21, A21, X11, 1.0, false, nw);
        level_sync<N>();
        if (active) {
            for (int e = threadIdx.x; e < H * H; e += 32 * nw) A21[(e / H) * FLS + e % H] = L21[(e / H) * FLS + e % H];
            if constexpr (H == 32) tile_prod32<P_HERM>(A22, L21, L21, -1.0, true);
            else tile_prod<H, OP_BH>(A22, L21, L21, -1.0, true, nw);
        }
        level_sync<N>();
        chol_rec<H>(F, X, T, o + H, status);
        level_sync<N>();
        if constexpr (H == 32) tile_prod32<P_LOWER_B>(W, L21, X11, 1.0, false);
        else if (active) tile_prod<H, OP_B>(W, L21, X11, 1.0, false, nw);
        level_sync<N>();
        if constexpr (H == 32) tile_prod32<P_LLOWER_B>(X21, X22, W, -1.0, false);
        else if (active) tile_prod<H, OP_B>(X21, X22, W, -1.0, false, nw);
        level_sync<N>();
    }
}

__device__ void factor_tile(c128* F, c128* X, c128* T, int* status) {
    for (int e = threadIdx.x; e < TB * TB; e += blockDim.x) X[(e / TB) * FLS + e % TB] = mk(0., 0.);
    __syncthreads();
    chol_rec<TB>(F, X, T, 0, status);
    __syncthreads();
}

struct TileArgs {
    c128* G;
    size_t ld;
    int nt;
    int kbeg;  // first tile column that contributes to the updates (0: the whole factorisation)
    c128* Linv;
    c128* LinvH;
    const int2* items;
    int nitems;
    int* counter;
    int* flags;  // nt x nt
    Sync S;
    // BF16 planes of the panel's rows below it for the trailing update (null: none):
    // row i TB + r - r0, K index (j - kbeg) TB + c and kp / 2 + that (kp = 2 x panel width)
    uint16_t *xh, *xl, *yh, *yl;
    int r0, kp;
};

__global__ void __launch_bounds__(128, 1) chol_tile_kernel(TileArgs a) {
    extern __shared__ __align__(16) unsigned char sm[];
    typedef c128 Stage[TB][SLS];
    Stage* As = reinterpret_cast<Stage*>(sm);
    Stage* Bs = reinterpret_cast<Stage*>(sm + 2 * sizeof(Stage));
    c128* F = reinterpret_cast<c128*>(sm);
    c128* X = F + TB * FLS;
    c128* T = X + TB * FLS;
    __shared__ int s_item, s_ok;
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const int fr = lane >> 2, fk = lane & 3;
    for (;;) {
        if (tid == 0) s_item = ld_acquire(a.S.abort_word) ? a.nitems : atomicAdd(a.counter, 1);
        __syncthreads();
        const int w = s_item;
        __syncthreads();
        if (w >= a.nitems) break;
        const int i = a.items[w].x, j = a.items[w].y;
        const WarpTiles wt = warp_tiles(warp, i == j);
        // A_ij is read once the sum over k is done: start bringing it into L2 now
        // (64 rows of 1 KiB, one 128-byte line per thread and step).
        for (int e = tid; e < TB * 8; e += blockDim.x)
            asm volatile("prefetch.global.L2 [%0];" ::"l"(a.G + size_t(i * TB + (e >> 3)) * a.ld + j * TB + (e & 7) * 8));
        double cre[4][4][2], cim[4][4][2];
#pragma unroll
        for (int p = 0; p < 4; ++p)
#pragma unroll
            for (int q = 0; q < 4; ++q) cre[p][q][0] = cre[p][q][1] = cim[p][q][0] = cim[p][q][1] = 0.0;
        // ---- F = A_ij - sum_k L_ik L_jk^H
        const int nchunk = 4 * (j - a.kbeg);
        bool ok = true;
        auto load = [&](int buf, int c) {
            const int kb = a.kbeg + (c >> 2), k0 = kb * TB + (c & 3) * KC;
#pragma unroll
            for (int q = 0; q < 8; ++q) {
                const int e = tid + 128 * q, row = e >> 4, kk = e & 15;
                cpa16(&As[buf][row][kk], a.G + size_t(i * TB + row) * a.ld + k0 + kk);
                cpa16(&Bs[buf][row][kk], a.G + size_t(j * TB + row) * a.ld + k0 + kk);
            }
            cpa_commit();
        };
        if (nchunk > 0) {
            ok = wait_flag(&a.flags[i * a.nt + a.kbeg], a.S, &s_ok) &&
                 wait_flag(&a.flags[j * a.nt + a.kbeg], a.S, &s_ok);
            if (ok) load(0, 0);
        }
        for (int c = 0; ok && c < nchunk; ++c) {
            const int buf = c & 1;
            if (c + 1 < nchunk) {
                if (((c + 1) & 3) == 0) {
                    const int kb = a.kbeg + ((c + 1) >> 2);
                    ok = wait_flag(&a.flags[i * a.nt + kb], a.S, &s_ok) &&
                         wait_flag(&a.flags[j * a.nt + kb], a.S, &s_ok);
                    if (!ok) break;
                }
                load(buf ^ 1, c + 1);
                cpa_wait_one();
            } else {
                cpa_wait_all();
            }
            __syncthreads();
            warp_mma_tiles(wt, &As[buf][0][0], SLS, &Bs[buf][0][0], SLS, KC / 4, fr, fk, cre, cim);
            __syncthreads();
        }
        cpa_wait_all();
        __syncthreads();
        if (!ok) break;
        // (a diagonal tile's sub-tiles above its diagonal are left unset: the
        // factorisation reads and writes back only the lower triangle)
#pragma unroll
        for (int p = 0; p < 4; ++p)
#pragma unroll
            for (int q = 0; q < 4; ++q) {
                if (!wt.has(p, q)) continue;
#pragma unroll
                for (int h = 0; h < 2; ++h) {
                    const int r = (wt.rb + p) * 8 + fr, c = (wt.cb + q) * 8 + 2 * fk + h;
                    const c128 g = a.G[size_t(i * TB + r) * a.ld + j * TB + c];
                    F[r * FLS + c] = mk(g.re - cre[p][q][h], g.im - cim[p][q][h]);
                }
            }
        __syncthreads();
        if (i == j) {
            factor_tile(F, X, T, a.S.status);
            c128* Li = a.Linv + size_t(j) * TB * TB;
            c128* LiH = a.LinvH + size_t(j) * TB * TB;
            // The column's other tiles read only L_jj^{-1}: it is published first.
            // L_jj itself and L_jj^{-H} serve the triangular solves, which run
            // after this launch.
            for (int e = tid; e < TB * TB; e += blockDim.x) Li[e] = X[(e / TB) * FLS + e % TB];
            publish(&a.flags[j * a.nt + j]);
            for (int e = tid; e < TB * TB; e += blockDim.x) {
                const int r = e / TB, c = e % TB;
                if (c <= r) a.G[size_t(j * TB + r) * a.ld + j * TB + c] = F[r * FLS + c];
                LiH[e] = conj(X[c * FLS + r]);
            }
        } else {
            if (!wait_flag(&a.flags[j * a.nt + j], a.S, &s_ok)) break;
            // X <- L_jj^{-1} (rows r, K-contiguous): L_ij = F (L_jj^{-1})^H
            const c128* Li = a.Linv + size_t(j) * TB * TB;
            for (int e = tid; e < TB * TB; e += blockDim.x) {
                const int r = e / TB, c = e % TB;
                cpa16(&X[r * FLS + c], Li + e);
            }
            cpa_commit();
            cpa_wait_all();
            __syncthreads();
            double tre[8][2][2], tim[8][2][2];
#pragma unroll
            for (int p = 0; p < 8; ++p)
#pragma unroll
                for (int q = 0; q < 2; ++q) tre[p][q][0] = tre[p][q][1] = tim[p][q][0] = tim[p][q][1] = 0.0;
            trsm_mma(F, X, warp, fr, fk, tre, tim);
#pragma unroll
            for (int p = 0; p < 8; ++p)
#pragma unroll
                for (int q = 0; q < 2; ++q)
#pragma unroll
                    for (int h = 0; h < 2; ++h) {
                        const int r = p * 8 + fr, c = (q == 0 ? 7 - warp : warp) * 8 + 2 * fk + h;
                        a.G[size_t(i * TB + r) * a.ld + j * TB + c] = mk(tre[p][q][h], tim[p][q][h]);
                    }
            if (a.xh && i * TB >= a.r0) {
                // The trailing update's operands straight from the registers: X = [Re | Im],
                // Y = [Im | -Re] of the FP64 values rounded to FP32, each split into BF16 hi + lo;
                // the two adjacent columns of a lane go out as one 4-byte store per plane.
                const int hk = a.kp >> 1;
#pragma unroll
                for (int p = 0; p < 8; ++p)
#pragma unroll
                    for (int q = 0; q < 2; ++q) {
                        const int r = p * 8 + fr, c = (q == 0 ? 7 - warp : warp) * 8 + 2 * fk;
                        const size_t e = size_t(i * TB + r - a.r0) * a.kp + size_t(j - a.kbeg) * TB + c;
                        uint16_t h0, l0, h1, l1;
                        auto put = [&](uint16_t* hi, uint16_t* lo, size_t at, float v0, float v1) {
                            split_bf16(v0, h0, l0);
                            split_bf16(v1, h1, l1);
                            *reinterpret_cast<uint32_t*>(hi + at) = uint32_t(h0) | (uint32_t(h1) << 16);
                            *reinterpret_cast<uint32_t*>(lo + at) = uint32_t(l0) | (uint32_t(l1) << 16);
                        };
                        const float re0 = float(tre[p][q][0]), re1 = float(tre[p][q][1]);
                        const float im0 = float(tim[p][q][0]), im1 = float(tim[p][q][1]);
                        put(a.xh, a.xl, e, re0, re1);
                        put(a.xh, a.xl, e + hk, im0, im1);
                        put(a.yh, a.yl, e, im0, im1);
                        put(a.yh, a.yl, e + hk, -re0, -re1);
                    }
            }
            publish(&a.flags[i * a.nt + j]);
        }
    }
    cpa_wait_all();
}

// ---------------------------------------------------------------------------
struct SolveArgs {
    const c128* G;
    size_t ld;
    int nt;
    const c128* Linv;
    const c128* LinvH;
    const c128* b;  // right-hand side
    c128* x;        // result, every entry SOLVE_EMPTY until its block is written
    int* flags;     // nt, set after each block (bookkeeping: no sweep waits on them)
    int* counter;  // block rows are claimed in sweep order from this counter
    Sync S;
};

// Next block row of the sweep for this CTA (nt when done or aborted).  Rows are
// claimed in order by running CTAs only, so a row's wait is always on rows held
// by CTAs that are already running: no co-residency is needed.
__device__ __forceinline__ int claim_row(const SolveArgs& a, int* s_row) {
    if (threadIdx.x == 0) *s_row = ld_acquire(a.S.abort_word) ? a.nt : atomicAdd(a.counter, 1);
    __syncthreads();
    const int t = *s_row;
    __syncthreads();
    return t;
}

// Solve sweeps.  One CTA per 64-row block (persistent over blocks r = blockIdx.x,
// + gridDim.x, ...).  The L tiles a block needs do not depend on the sweep, so they
// stream into shared memory (cp.async, two buffers) ahead of the solution; only
// the 64-entry solution block x_k is waited for.  The diagonal inverse is staged
// at the start.  Each chain link is then a shared-memory mat-vec.
//
// The solution vector is its own flag: it starts filled with the bit pattern
// SOLVE_EMPTY (all ones, a NaN that no arithmetic result here has: FP64 operations
// return the positive canonical NaN, and a result that matched would be stored as
// that instead), and a waiting CTA polls the 64 entries of block k until none is
// SOLVE_EMPTY.  Each entry's halves are written and read as single 8-byte strong
// accesses, so a read that sees a value sees the final one.  A link of the chain
// thus costs one trip through L2 (the store, seen by the next poll) instead of a
// fence, a flag store, a flag poll and a load of the block.
constexpr unsigned long long SOLVE_EMPTY = ~0ull;
constexpr int SLD = TB + 1;  // staged tile row stride (complex)
constexpr size_t SM_SOLVE = size_t(3) * TB * SLD * sizeof(c128) + 2 * TB * sizeof(c128);

// Threads 0..63 poll entry k TB + tid of x until it is written (bounded; the abort
// word every 64 polls) and copy it to dst; false when this or another CTA gave up.
__device__ bool poll_block(const c128* x, c128* dst, const Sync& S) {
    int ok = 1;
    if (threadIdx.x < TB) {
        const c128* p = x + threadIdx.x;
        unsigned long long re, im;
        unsigned it = 0;
        while (true) {
            asm volatile("ld.relaxed.gpu.global.v2.b64 {%0, %1}, [%2];" : "=l"(re), "=l"(im) : "l"(p) : "memory");
            if (re != SOLVE_EMPTY && im != SOLVE_EMPTY) break;
            if ((++it & 63u) == 0 && (ld_acquire(S.abort_word) != 0 || it > S.cap)) {
                ok = 0;
                break;
            }
        }
        if (ok) {
            dst[threadIdx.x] = mk(__longlong_as_double(static_cast<long long>(re)),
                                  __longlong_as_double(static_cast<long long>(im)));
        } else if (it > S.cap) {
            atomicOr(S.status, DS_TIMEOUT);
            atomicExch(S.abort_word, 1);
        }
    }
    return __syncthreads_and(ok) != 0;
}

// Writes one solution entry (never the SOLVE_EMPTY pattern) as two strong 8-byte stores.
__device__ __forceinline__ void store_entry(c128* x, c128 v) {
    unsigned long long re = static_cast<unsigned long long>(__double_as_longlong(v.re));
    unsigned long long im = static_cast<unsigned long long>(__double_as_longlong(v.im));
    if (re == SOLVE_EMPTY) re = 0x7fffffffffffffffull;
    if (im == SOLVE_EMPTY) im = 0x7fffffffffffffffull;
    asm volatile("st.relaxed.gpu.global.v2.b64 [%0], {%1, %2};" ::"l"(x), "l"(re), "l"(im) : "memory");
}

// Stage the 64 x 64 tile at `src` (row stride ld) into dst[64][SLD].
__device__ __forceinline__ void stage_tile(c128* dst, const c128* src, size_t ld) {
    for (int e = threadIdx.x; e < TB * TB; e += blockDim.x) {
        const int r = e >> 6, c = e & 63;
        cpa16(&dst[r * SLD + c], src + size_t(r) * ld + c);
    }
}

// sum_{c < 32} op(A[c sa]) x[c] with four independent partial sums: each link of a
// sweep's chain runs two of these, and one running sum would be a chain of 64
// dependent FP64 FMAs.
template <bool CONJ>
__device__ __forceinline__ c128 dot32(const c128* A, int sa, const c128* x) {
    c128 p[4] = {mk(0., 0.), mk(0., 0.), mk(0., 0.), mk(0., 0.)};
#pragma unroll
    for (int c = 0; c < 32; c += 4)
#pragma unroll
        for (int u = 0; u < 4; ++u) {
            const c128 a = A[(c + u) * sa];
            p[u] = p[u] + (CONJ ? conj(a) : a) * x[c + u];
        }
    return (p[0] + p[1]) + (p[2] + p[3]);
}

// Forward: x_r = L_rr^{-1} (b_r - sum_{k<r} L_rk x_k), block rows in increasing order.
__global__ void __launch_bounds__(128, 1) chol_fwd_tile_kernel(SolveArgs a) {
    extern __shared__ __align__(16) unsigned char sm[];
    c128* buf = reinterpret_cast<c128*>(sm);   // 2 tiles
    c128* Li = buf + 2 * TB * SLD;             // diagonal inverse
    c128* xk = Li + TB * SLD;                  // published block
    c128* acc = xk + TB;
    __shared__ int s_row;
    const int tid = threadIdx.x, row = tid >> 1, half = tid & 1;
    for (int r = claim_row(a, &s_row); r < a.nt; r = claim_row(a, &s_row)) {
        stage_tile(Li, a.Linv + size_t(r) * TB * TB, TB);
        cpa_commit();
        if (r > 0) stage_tile(buf, a.G + size_t(r) * TB * a.ld, a.ld);
        cpa_commit();
        if (tid < TB) acc[tid] = a.b[r * TB + tid];
        bool ok = true;
        for (int k = 0; k < r; ++k) {
            if (k + 1 < r) stage_tile(buf + ((k + 1) & 1) * TB * SLD, a.G + size_t(r) * TB * a.ld + (k + 1) * TB, a.ld);
            cpa_commit();
            if (!poll_block(a.x + k * TB, xk, a.S)) {
                ok = false;
                break;
            }
            cpa_wait_one();  // tile k (and everything before it) has landed
            __syncthreads();
            const c128* T = buf + (k & 1) * TB * SLD + row * SLD + half * 32;
            c128 v = dot32<false>(T, 1, xk + half * 32);
            v.re += __shfl_xor_sync(0xffffffffu, v.re, 1);
            v.im += __shfl_xor_sync(0xffffffffu, v.im, 1);
            __syncthreads();
            if (half == 0) acc[row] = acc[row] - v;
        }
        cpa_wait_all();
        __syncthreads();
        if (!ok) return;
        c128 v = dot32<false>(Li + row * SLD + half * 32, 1, acc + half * 32);
        v.re += __shfl_xor_sync(0xffffffffu, v.re, 1);
        v.im += __shfl_xor_sync(0xffffffffu, v.im, 1);
        if (half == 0) store_entry(a.x + r * TB + row, v);
        publish(&a.flags[r]);
    }
}

// Backward: z_r = L_rr^{-H} (x_r - sum_{k>r} L_kr^H z_k), block rows in decreasing order.
__global__ void __launch_bounds__(128, 1) chol_bwd_tile_kernel(SolveArgs a) {
    extern __shared__ __align__(16) unsigned char sm[];
    c128* buf = reinterpret_cast<c128*>(sm);
    c128* Li = buf + 2 * TB * SLD;
    c128* zk = Li + TB * SLD;
    c128* acc = zk + TB;
    __shared__ int s_row;
    const int tid = threadIdx.x, col = tid >> 1, half = tid & 1;
    for (int t = claim_row(a, &s_row); t < a.nt; t = claim_row(a, &s_row)) {
        const int r = a.nt - 1 - t;
        stage_tile(Li, a.LinvH + size_t(r) * TB * TB, TB);
        cpa_commit();
        if (r + 1 < a.nt) stage_tile(buf, a.G + size_t(a.nt - 1) * TB * a.ld + r * TB, a.ld);
        cpa_commit();
        if (tid < TB) acc[tid] = a.b[r * TB + tid];
        bool ok = true;
        for (int k = a.nt - 1, i = 0; k > r; --k, ++i) {
            if (k - 1 > r) stage_tile(buf + ((i + 1) & 1) * TB * SLD, a.G + size_t(k - 1) * TB * a.ld + r * TB, a.ld);
            cpa_commit();
            if (!poll_block(a.x + k * TB, zk, a.S)) {
                ok = false;
                break;
            }
            cpa_wait_one();
            __syncthreads();
            // acc[col] -= sum_row conj(L[k*64 + row][r*64 + col]) z_k[row]
            const c128* T = buf + (i & 1) * TB * SLD + col;
            c128 v = dot32<true>(T + half * 32 * SLD, SLD, zk + half * 32);
            v.re += __shfl_xor_sync(0xffffffffu, v.re, 1);
            v.im += __shfl_xor_sync(0xffffffffu, v.im, 1);
            __syncthreads();
            if (half == 0) acc[col] = acc[col] - v;
        }
        cpa_wait_all();
        __syncthreads();
        if (!ok) return;
        const int rowo = col;
        c128 v = dot32<false>(Li + rowo * SLD + half * 32, 1, acc + half * 32);
        v.re += __shfl_xor_sync(0xffffffffu, v.re, 1);
        v.im += __shfl_xor_sync(0xffffffffu, v.im, 1);
        if (half == 0) store_entry(a.x + r * TB + rowo, v);
        publish(&a.flags[r]);
    }
}

int coresident_blocks(const void* fn, int threads, size_t smem, int sm_count) {
    int per_sm = 0;
    YQ_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, fn, threads, smem));
    if (per_sm < 1) throw Error(YQ_E_UNSUPPORTED, "persistent Cholesky: kernel does not fit on an SM");
    return per_sm * sm_count;
}
}  // namespace

// Scratch layout (ints): [0] tile counter of the full factorisation, [1] abort word
// of the factorisation, [2] abort word of the solves, [3] / [4] block-row counters
// of the forward / backward sweeps, [16 .. 16 + nt) tile counters
// of the panels, then the tile flags (nt x nt), the solve flags (2 nt), the
// 16-byte aligned tile list, and the 16-byte aligned forward-sweep result (n c128).
struct Scratch {
    int* words;
    int* panel_counters;
    int* flags;
    int* sflags;
    int2* items;
    c128* xs;
    Scratch(void* p, int nt) {
        words = static_cast<int*>(p);
        panel_counters = words + 16;
        flags = panel_counters + nt;
        sflags = flags + size_t(nt) * nt;
        items = reinterpret_cast<int2*>((reinterpret_cast<uintptr_t>(sflags + 2 * size_t(nt)) + 15) & ~uintptr_t(15));
        xs = reinterpret_cast<c128*>(
            (reinterpret_cast<uintptr_t>(items + size_t(nt) * (nt + 1) / 2) + 15) & ~uintptr_t(15));
    }
};

size_t chol_tile_scratch_bytes(int n) {
    const size_t nt = size_t(n) / TB;
    return (16 + nt + nt * nt + 2 * nt) * sizeof(int) + nt * (nt + 1) / 2 * sizeof(int2) + 256 +
           size_t(n) * sizeof(c128) + 16;
}

// Column-major tile order, diagonal first: column j starts at j nt - j (j - 1) / 2.
__global__ void tile_items_kernel(int nt, int2* items) {
    const int j = blockIdx.x;
    const size_t off = size_t(j) * nt - size_t(j) * (j - 1) / 2;
    for (int i = j + threadIdx.x; i < nt; i += blockDim.x) items[off + (i - j)] = make_int2(i, j);
}
static void write_items(const Scratch& sc, int nt, cudaStream_t st) {
    tile_items_kernel<<<nt, 128, 0, st>>>(nt, sc.items);
    YQ_LAUNCH_CHECK();
}

static int tile_grid() {
    static int per_sm = -1;
    if (per_sm < 0) {
        YQ_CUDA(cudaFuncSetAttribute(chol_tile_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, int(SM_TILE)));
        YQ_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, chol_tile_kernel, 128, SM_TILE));
        if (per_sm < 1) throw Error(YQ_E_UNSUPPORTED, "persistent Cholesky: kernel does not fit on an SM");
    }
    return per_sm;
}

// Ordinary launch: tiles are handed out by the counter to running CTAs only, so the
// grid needs no co-residency and can share the device with other work.  Small
// matrices get a grid proportional to their tile columns: the factorisation is a
// chain of one diagonal tile per column (~80 us each), and about 1.5 CTAs per tile
// column keep the tiles of the current column ahead of it; every CTA beyond that
// only waits on flags while holding an SM (one CTA per SM) that the kernels of
// other problems sharing the device could use.
static void launch_tiles(const TileArgs& a, int nitems, int sm_count, cudaStream_t st) {
    const int grid = std::min({tile_grid() * sm_count, std::max(1, nitems), std::max(16, a.nt + a.nt / 2)});
    chol_tile_kernel<<<grid, 128, SM_TILE, st>>>(a);
    YQ_LAUNCH_CHECK();
}

void chol_factor_tiled(c128* G, int n, size_t ld, c128* Linv, c128* LinvH, int* status, void* scratch,
                       int sm_count, cudaStream_t st) {
    YQ_CHECK_ARG(n % TB == 0 && n > 0, "cholesky: dimension must be a positive multiple of 64");
    const int nt = n / TB;
    Scratch sc(scratch, nt);
    write_items(sc, nt, st);
    YQ_CUDA(cudaMemsetAsync(sc.words, 0, reinterpret_cast<char*>(sc.sflags) - reinterpret_cast<char*>(sc.words), st));
    const int nitems = nt * (nt + 1) / 2;
    TileArgs a{G, ld, nt, 0, Linv, LinvH, sc.items, nitems, sc.words + 0, sc.flags, Sync{status, sc.words + 1, 1u << 24}};
    launch_tiles(a, nitems, sm_count, st);
}

// BF16 planes of one panel, then the K-split partials of the trailing updates'
// last waves (up to 160 partial tiles of 128 x 256 float2)
static size_t panel_operand_bytes(int n) {
    const size_t rows = ((size_t(n) + TC_BM - 1) / TC_BM) * TC_BM;
    return 4 * rows * size_t(2 * CHOL_PANEL) * sizeof(uint16_t);
}
constexpr size_t TRAIL_SPLIT_BYTES = size_t(160) * 128 * 256 * 8;

size_t chol_panel_planes_bytes(int n) { return panel_operand_bytes(n) + TRAIL_SPLIT_BYTES; }

void chol_factor_panels(c128* G, int n, size_t ld, c128* Linv, c128* LinvH, int* status, void* scratch,
                        void* planes, int sm_count, cudaStream_t st) {
    YQ_CHECK_ARG(n % TB == 0 && n > 0, "cholesky: dimension must be a positive multiple of 64");
    const int nt = n / TB, pw = CHOL_PANEL / TB;
    Scratch sc(scratch, nt);
    write_items(sc, nt, st);
    YQ_CUDA(cudaMemsetAsync(sc.words, 0, reinterpret_cast<char*>(sc.sflags) - reinterpret_cast<char*>(sc.words), st));
    const size_t plane_elems = panel_operand_bytes(n) / (4 * sizeof(uint16_t));
    float2* split_ws = reinterpret_cast<float2*>(static_cast<char*>(planes) + panel_operand_bytes(n));
    uint16_t* xh = static_cast<uint16_t*>(planes);
    uint16_t *xl = xh + plane_elems, *yh = xl + plane_elems, *yl = yh + plane_elems;
    int first = 0;  // index of the panel's first tile in the column-major list
    for (int j0 = 0, p = 0; j0 < nt; j0 += pw, ++p) {
        const int j1 = std::min(nt, j0 + pw);
        int count = 0;
        for (int j = j0; j < j1; ++j) count += nt - j;
        // the panel's rows below it go to the trailing update, whose BF16 planes
        // (K = 2 w) the panel's tiles write as they form those rows; the planes'
        // padding rows (n2 .. rows_pad) are zeroed here
        const int r0 = j1 * TB, n2 = n - r0, w = (j1 - j0) * TB;
        const size_t rows_pad = ((size_t(std::max(n2, 1)) + TC_BM - 1) / TC_BM) * TC_BM;
        const bool trail = j1 < nt;
        if (trail && rows_pad > size_t(n2)) {
            const size_t off = size_t(n2) * 2 * w, cnt = (rows_pad - size_t(n2)) * 2 * w * sizeof(uint16_t);
            for (uint16_t* pl : {xh, xl, yh, yl}) YQ_CUDA(cudaMemsetAsync(pl + off, 0, cnt, st));
        }
        TileArgs a{G, ld, nt, j0, Linv, LinvH, sc.items + first, count, sc.panel_counters + p, sc.flags,
                   Sync{status, sc.words + 1, 1u << 24}, trail ? xh : nullptr, xl, yh, yl, r0, 2 * w};
        launch_tiles(a, count, sm_count, st);
        first += count;
        if (!trail) break;
        // trailing update  G[r0:, r0:] -= L21 L21^H  on the tensor cores
        herk_tc_launch(xh, xl, yh, yl, n2, rows_pad, size_t(2 * w), G + size_t(r0) * ld + r0, ld, -1.0, 0.0, true,
                       status, sm_count, nullptr, tc_split_enabled() ? split_ws : nullptr, TRAIL_SPLIT_BYTES, st);
    }
}

void chol_solve_tiled(const c128* G, int n, size_t ld, const c128* Linv, const c128* LinvH, c128* b, c128* out,
                      int* status, void* scratch, int sm_count, cudaStream_t st) {
    const int nt = n / TB;
    Scratch sc(scratch, nt);
    int* words = sc.words;
    int* sflags = sc.sflags;
    YQ_CUDA(cudaMemsetAsync(sflags, 0, 2 * size_t(nt) * sizeof(int), st));
    YQ_CUDA(cudaMemsetAsync(words + 2, 0, 3 * sizeof(int), st));  // abort word and row counters of the solves
    static bool attr = false;
    if (!attr) {
        YQ_CUDA(cudaFuncSetAttribute(chol_fwd_tile_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, int(SM_SOLVE)));
        YQ_CUDA(cudaFuncSetAttribute(chol_bwd_tile_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, int(SM_SOLVE)));
        attr = true;
    }
    const int grid_f = std::min(nt, coresident_blocks(reinterpret_cast<const void*>(chol_fwd_tile_kernel), 128,
                                                      SM_SOLVE, sm_count));
    const int grid_b = std::min(nt, coresident_blocks(reinterpret_cast<const void*>(chol_bwd_tile_kernel), 128,
                                                      SM_SOLVE, sm_count));
    // forward b -> xs, backward xs -> out (b may be out: it is read by the forward sweep only)
    YQ_CUDA(cudaMemsetAsync(sc.xs, 0xff, size_t(n) * sizeof(c128), st));
    SolveArgs fa{G, ld, nt, Linv, LinvH, b, sc.xs, sflags, words + 3, Sync{status, words + 2, 1u << 24}};
    chol_fwd_tile_kernel<<<grid_f, 128, SM_SOLVE, st>>>(fa);
    YQ_LAUNCH_CHECK();
    YQ_CUDA(cudaMemsetAsync(out, 0xff, size_t(n) * sizeof(c128), st));
    SolveArgs ba{G, ld, nt, Linv, LinvH, sc.xs, out, sflags + nt, words + 4, Sync{status, words + 2, 1u << 24}};
    chol_bwd_tile_kernel<<<grid_b, 128, SM_SOLVE, st>>>(ba);
    YQ_LAUNCH_CHECK();
}

// Failure injection for the bounded waits (tests only): a 4 x 4-tile problem whose
// first work item -- the tile (0, 0) of the factorisation (which = 0) or the block
// row 0 of the forward solve (which = 1) -- is never claimed, because its counter
// starts at 1, so the flag that item would publish is never set.  Every other item
// depends on it; the first wait to pass `cap` polls sets DS_TIMEOUT and the abort
// word, and every CTA returns through its normal exit (pending copies drained).
// Returns the number of flags published (0 when every CTA stopped).
int chol_debug_unpublished_flag(int which, unsigned cap, int* status, int sm_count, cudaStream_t st) {
    constexpr int nt = 4, n = nt * TB;
    DevBuf G, Li, LiH, b, scratch;
    G.ensure(size_t(n) * n * sizeof(c128));
    Li.ensure(size_t(n) * TB * sizeof(c128));
    LiH.ensure(size_t(n) * TB * sizeof(c128));
    b.ensure(size_t(n) * sizeof(c128));
    scratch.ensure(chol_tile_scratch_bytes(n));
    YQ_CUDA(cudaMemsetAsync(G.p, 0, G.bytes, st));
    YQ_CUDA(cudaMemsetAsync(Li.p, 0, Li.bytes, st));
    YQ_CUDA(cudaMemsetAsync(LiH.p, 0, LiH.bytes, st));
    YQ_CUDA(cudaMemsetAsync(b.p, 0, b.bytes, st));
    Scratch sc(scratch.p, nt);
    write_items(sc, nt, st);
    YQ_CUDA(cudaMemsetAsync(sc.words, 0, reinterpret_cast<char*>(sc.items) - reinterpret_cast<char*>(sc.words), st));
    const int one = 1;
    int* published_base = nullptr;
    int nflags = 0;
    if (which == 0) {
        YQ_CUDA(cudaMemcpyAsync(sc.words + 0, &one, sizeof(int), cudaMemcpyHostToDevice, st));
        const int nitems = nt * (nt + 1) / 2;
        TileArgs a{G.as<c128>(), size_t(n), nt, 0, Li.as<c128>(), LiH.as<c128>(), sc.items, nitems, sc.words + 0,
                   sc.flags, Sync{status, sc.words + 1, cap}};
        launch_tiles(a, nitems, sm_count, st);
        published_base = sc.flags;
        nflags = nt * nt;
    } else {
        static bool attr = false;
        if (!attr) {
            YQ_CUDA(cudaFuncSetAttribute(chol_fwd_tile_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         int(SM_SOLVE)));
            attr = true;
        }
        YQ_CUDA(cudaMemcpyAsync(sc.words + 3, &one, sizeof(int), cudaMemcpyHostToDevice, st));
        const int grid = std::min(nt, coresident_blocks(reinterpret_cast<const void*>(chol_fwd_tile_kernel), 128,
                                                        SM_SOLVE, sm_count));
        YQ_CUDA(cudaMemsetAsync(sc.xs, 0xff, size_t(n) * sizeof(c128), st));
        SolveArgs fa{G.as<c128>(), size_t(n), nt, Li.as<c128>(), LiH.as<c128>(), b.as<c128>(), sc.xs, sc.sflags,
                     sc.words + 3, Sync{status, sc.words + 2, cap}};
        chol_fwd_tile_kernel<<<grid, 128, SM_SOLVE, st>>>(fa);
        YQ_LAUNCH_CHECK();
        published_base = sc.sflags;
        nflags = nt;
    }
    std::vector<int> flags(static_cast<size_t>(nflags));
    YQ_CUDA(cudaMemcpyAsync(flags.data(), published_base, size_t(nflags) * sizeof(int), cudaMemcpyDeviceToHost, st));
    YQ_CUDA(cudaStreamSynchronize(st));
    int published = 0;
    for (int f : flags) published += f != 0;
    return published;
}

}  // namespace yq
