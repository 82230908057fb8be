// tcgen05 Hermitian rank-k kernel of the mixed-precision SR path (see gram_tc.hpp).
//
// One CTA per 128 x 256 complex output tile of the lower triangle.  Both parts
// of the tile are accumulated by the same CTA: TMEM columns 0..255 hold Re = X X^T
// and columns 256..511 hold Im = Y X^T, so each staged B tile feeds two MMAs and
// the epilogue writes whole complex numbers.  Warp roles:
//   warp 0       TMA producer: 3-stage ring of {X 128x64, Y 128x64, B 256x64} BF16
//                tiles, 128-byte swizzle, completion counted on "full" mbarriers;
//   warp 1       TMEM allocator and single-thread MMA issuer: 2 x 4
//                tcgen05.mma.cta_group::1.kind::f16 (M128 N256 K16) per stage,
//                tcgen05.commit releases the stage ("empty") and finally "done";
//   warps 2..5   epilogue: tcgen05.ld 32x32b.x32 from TMEM, scale, FP64 store
//                (or read-add-store for the trailing updates of the Cholesky).
// K runs over three segments (hi.hi, hi.lo, lo.hi) of the split operands.
// Every mbarrier wait is bounded: on timeout the kernel sets DS_TIMEOUT in the
// status word, the other roles stop at their next wait, and TMEM is released.
// No cluster launch and no multicast: each CTA fetches its own tiles.
#include <cuda.h>
#include <cudaTypedefs.h>
#include <cuda_bf16.h>

#include <cstdlib>
#include <mutex>
#include <string>

#include "gram_tc.hpp"
#include "internal.hpp"

namespace yq {

// ---------------------------------------------------------------------------
// Row s of O~ (the O writer's centred value, complex64) and its four planes:
// k = p holds (Re, Im), k = P + p holds (Im, -Re); rows >= ns and k >= 2P are zero.
__global__ void o_and_operands_kernel(int n, int m, bool bias, size_t P, int ns, size_t rows_pad, size_t kpad,
                                      const int8_t* __restrict__ sigma, const c64* __restrict__ t,
                                      const c128* __restrict__ oloc, c64* __restrict__ O, uint16_t* __restrict__ xh,
                                      uint16_t* __restrict__ xl, uint16_t* __restrict__ yh,
                                      uint16_t* __restrict__ yl) {
    // column indices fit 32 bits (P < 2^31, checked by the caller): 32-bit division
    const unsigned nm = unsigned(n) * unsigned(m), um = unsigned(m), uP = unsigned(P);
    for (size_t row = blockIdx.y; row < rows_pad; row += gridDim.y) {
        const int8_t* sg = sigma + row * n;
        const c64* ts = t + row * m;
        const size_t base = row * kpad;
        for (unsigned p = blockIdx.x * blockDim.x + threadIdx.x; p < uP; p += gridDim.x * blockDim.x) {
            float re = 0.f, im = 0.f;
            if (row < size_t(ns)) {
                c64 v;
                if (p < nm) {
                    const unsigned i = p / um, j = p - i * um;
                    const float sv = float(sg[i]);
                    v = mk(sv * ts[j].re, sv * ts[j].im);
                } else if (p < nm + n) {
                    v = mk(float(sg[p - nm]), 0.f);
                } else {
                    v = ts[p - nm - n];
                }
                const c128 o = oloc[p];
                re = v.re - float(o.re);
                im = v.im - float(o.im);
                O[row * P + p] = mk(re, im);
            }
            uint16_t a, b;
            split_bf16(re, a, b);
            xh[base + p] = a;
            xl[base + p] = b;
            split_bf16(im, a, b);
            yh[base + p] = a;
            yl[base + p] = b;
            split_bf16(im, a, b);
            xh[base + P + p] = a;
            xl[base + P + p] = b;
            split_bf16(-re, a, b);
            yh[base + P + p] = a;
            yl[base + P + p] = b;
        }
        for (size_t k = 2 * P + size_t(blockIdx.x) * blockDim.x + threadIdx.x; k < kpad;
             k += size_t(gridDim.x) * blockDim.x) {
            xh[base + k] = 0;
            xl[base + k] = 0;
            yh[base + k] = 0;
            yl[base + k] = 0;
        }
    }
}

// The same with two consecutive columns per thread when P is even: one 16-byte store
// of O~ and one 4-byte store per plane and half of K (nine 2- or 8-byte stores per
// element before), each covering a contiguous 512 or 128 bytes per warp.  Row
// offsets row * P (complex) and row * kpad, P + p and 2P (BF16) are then even, so
// every vector store is aligned to its size.  Values and zeros are the same as
// above, bit for bit.  (Four columns per thread, two 16-byte O~ stores per thread
// with each warp store touching every sector half, measured slower than the
// one-column kernel: 1.83 against 1.54 ms at Ns = 8192.)
__global__ void o_and_operands2_kernel(int n, int m, size_t P, int ns, size_t rows_pad, size_t kpad,
                                       const int8_t* __restrict__ sigma, const c64* __restrict__ t,
                                       const c128* __restrict__ oloc, c64* __restrict__ O, uint16_t* __restrict__ xh,
                                       uint16_t* __restrict__ xl, uint16_t* __restrict__ yh,
                                       uint16_t* __restrict__ yl) {
    const unsigned nm = unsigned(n) * unsigned(m), um = unsigned(m), uP2 = unsigned(P / 2);
    for (size_t row = blockIdx.y; row < rows_pad; row += gridDim.y) {
        const int8_t* sg = sigma + row * n;
        const c64* ts = t + row * m;
        const size_t base = row * kpad;
        for (unsigned q = blockIdx.x * blockDim.x + threadIdx.x; q < uP2; q += gridDim.x * blockDim.x) {
            const unsigned p0 = 2 * q;
            float re[2] = {0.f, 0.f}, im[2] = {0.f, 0.f};
            if (row < size_t(ns)) {
#pragma unroll
                for (int e = 0; e < 2; ++e) {
                    const unsigned p = p0 + e;
                    c64 v;
                    if (p < nm) {
                        const unsigned i = p / um, j = p - i * um;
                        const float sv = float(sg[i]);
                        v = mk(sv * ts[j].re, sv * ts[j].im);
                    } else if (p < nm + n) {
                        v = mk(float(sg[p - nm]), 0.f);
                    } else {
                        v = ts[p - nm - n];
                    }
                    const c128 o = oloc[p];
                    re[e] = v.re - float(o.re);
                    im[e] = v.im - float(o.im);
                }
                *reinterpret_cast<float4*>(O + row * P + p0) = make_float4(re[0], im[0], re[1], im[1]);
            }
            uint16_t a0[2], b0[2], a1[2], b1[2], a2[2], b2[2];
#pragma unroll
            for (int e = 0; e < 2; ++e) {
                split_bf16(re[e], a0[e], b0[e]);
                split_bf16(im[e], a1[e], b1[e]);
                split_bf16(-re[e], a2[e], b2[e]);
            }
            auto pk = [](const uint16_t (&v)[2]) { return unsigned(v[0]) | (unsigned(v[1]) << 16); };
            // k = p: X = Re, Y = Im;  k = P + p: X = Im, Y = -Re
            *reinterpret_cast<unsigned*>(xh + base + p0) = pk(a0);
            *reinterpret_cast<unsigned*>(xl + base + p0) = pk(b0);
            *reinterpret_cast<unsigned*>(yh + base + p0) = pk(a1);
            *reinterpret_cast<unsigned*>(yl + base + p0) = pk(b1);
            *reinterpret_cast<unsigned*>(xh + base + P + p0) = pk(a1);
            *reinterpret_cast<unsigned*>(xl + base + P + p0) = pk(b1);
            *reinterpret_cast<unsigned*>(yh + base + P + p0) = pk(a2);
            *reinterpret_cast<unsigned*>(yl + base + P + p0) = pk(b2);
        }
        for (size_t k = 2 * P + 2 * (size_t(blockIdx.x) * blockDim.x + threadIdx.x); k < kpad;
             k += 2 * size_t(gridDim.x) * blockDim.x) {
            *reinterpret_cast<unsigned*>(xh + base + k) = 0u;
            *reinterpret_cast<unsigned*>(xl + base + k) = 0u;
            *reinterpret_cast<unsigned*>(yh + base + k) = 0u;
            *reinterpret_cast<unsigned*>(yl + base + k) = 0u;
        }
    }
}

void gram_tc_write_o_and_operands(int n, int m, bool bias, size_t P, int ns, const int8_t* sigma, const c64* t,
                                  const c128* oloc, c64* O, uint16_t* xh, uint16_t* xl, uint16_t* yh, uint16_t* yl,
                                  cudaStream_t st) {
    YQ_CHECK_ARG(P < (size_t(1) << 31), "O: more than 2^31 parameters");
    const size_t kpad = gram_tc_kpad(P), rows = gram_tc_rows(ns);
    if (P % 2 == 0) {
        dim3 g(std::min<unsigned>(64u, cdiv_u(P / 2, 256)), unsigned(std::min<size_t>(rows, 65535)));
        o_and_operands2_kernel<<<g, 256, 0, st>>>(n, m, P, ns, rows, kpad, sigma, t, oloc, O, xh, xl, yh, yl);
        YQ_LAUNCH_CHECK();
        return;
    }
    dim3 g(std::min<unsigned>(64u, cdiv_u(P, 256)), unsigned(std::min<size_t>(rows, 65535)));
    o_and_operands_kernel<<<g, 256, 0, st>>>(n, m, bias, P, ns, rows, kpad, sigma, t, oloc, O, xh, xl, yh, yl);
    YQ_LAUNCH_CHECK();
}

// ---------------------------------------------------------------------------
constexpr int TC_STAGES = 3;
constexpr int TC_BNW = 256;                                   // output columns per tile
constexpr int TC_A_BYTES = TC_BM * TC_BK * 2;                 // 16 KiB (X or Y rows)
constexpr int TC_B_BYTES = TC_BNW * TC_BK * 2;                // 32 KiB
constexpr int TC_STAGE_BYTES = 2 * TC_A_BYTES + TC_B_BYTES;   // 64 KiB
constexpr int TC_TMEM_COLS = 512;                             // Re: 0..255, Im: 256..511
constexpr int TC_THREADS = 192;
constexpr size_t TC_SMEM = size_t(TC_STAGES) * TC_STAGE_BYTES + 1024 /*align*/ + 256 /*barriers*/;

struct TcParams {
    int n;                 // output rows (= columns) that are written
    int nt;                // 128-row tiles
    int kb_per_seg;        // kpad / 64
    c128* C;
    size_t ldc;
    double alpha, shift;
    int accumulate;
    int* status;
    unsigned wait_cap;
    // K-split of the tiles after the last full wave: CTA index >= full_tiles maps to
    // tile full_tiles + u / split, K-chunk u % split of kb_chunk stages, whose FP32
    // partial goes to ws (128 x 256 float2 per chunk) instead of C
    int full_tiles, split, kb_chunk;
    float2* ws;
};

__device__ __forceinline__ uint32_t smem_u32(const void* p) {
    return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}
__device__ __forceinline__ void mbar_init(uint32_t a, uint32_t count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(a), "r"(count) : "memory");
}
__device__ __forceinline__ void mbar_expect_tx(uint32_t a, uint32_t bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(a), "r"(bytes) : "memory");
}
__device__ __forceinline__ bool mbar_try(uint32_t a, uint32_t parity) {
    uint32_t ok;
    asm volatile(
        "{\n\t.reg .pred P1;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 P1, [%1], %2;\n\t"
        "selp.b32 %0, 1, 0, P1;\n\t}"
        : "=r"(ok)
        : "r"(a), "r"(parity)
        : "memory");
    return ok != 0;
}
// Bounded wait; false on timeout or when another role aborted.
__device__ __forceinline__ bool mbar_wait(uint32_t a, uint32_t parity, volatile int* abort_flag, unsigned cap,
                                          int* status) {
    for (unsigned it = 0; it < cap; ++it) {
        if (mbar_try(a, parity)) return true;
        if (*abort_flag) return false;
    }
    *abort_flag = 1;
    atomicOr(status, DS_TIMEOUT);
    return false;
}
__device__ __forceinline__ void tma_load_2d(uint32_t dst, const CUtensorMap* map, int x, int y, uint32_t mbar) {
    asm volatile(
        "cp.async.bulk.tensor.2d.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3}], [%4];" ::
            "r"(dst),
        "l"(reinterpret_cast<uint64_t>(map)), "r"(x), "r"(y), "r"(mbar)
        : "memory");
}
// K-major operand tile with 128-byte swizzle: rows of 128 B, 8-row groups 1024 B apart.
__device__ __forceinline__ uint64_t sw128_desc(uint32_t saddr) {
    uint64_t d = 0;
    d |= uint64_t((saddr >> 4) & 0x3FFFu);  // start address
    d |= uint64_t(1) << 16;                  // leading byte offset (unused for swizzled K-major)
    d |= uint64_t(1024 >> 4) << 32;          // stride byte offset: 8 rows x 128 B
    d |= uint64_t(1) << 46;                  // descriptor version (sm_100)
    d |= uint64_t(2) << 61;                  // SWIZZLE_128B
    return d;
}
// kind::f16 instruction descriptor: FP32 accumulate, BF16 A and B, K-major, M = 128, N = 256.
constexpr uint32_t TC_IDESC = (1u << 4) | (1u << 7) | (1u << 10) | (uint32_t(TC_BNW >> 3) << 17) |
                              (uint32_t(TC_BM >> 4) << 24);

__device__ __forceinline__ void umma_bf16(uint32_t tmem_d, uint64_t da, uint64_t db, uint32_t accumulate) {
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "setp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}" ::"r"(tmem_d),
        "l"(da), "l"(db), "r"(TC_IDESC), "r"(accumulate)
        : "memory");
}
__device__ __forceinline__ void umma_commit(uint32_t mbar) {
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(mbar)
                 : "memory");
}

#define YQ_TMEM_LD_X32(taddr, v)                                                                                   \
    asm volatile(                                                                                                  \
        "tcgen05.ld.sync.aligned.32x32b.x32.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15,%16,%17,%18," \
        "%19,%20,%21,%22,%23,%24,%25,%26,%27,%28,%29,%30,%31}, [%32];"                                            \
        : "=r"(v[0]), "=r"(v[1]), "=r"(v[2]), "=r"(v[3]), "=r"(v[4]), "=r"(v[5]), "=r"(v[6]), "=r"(v[7]),        \
          "=r"(v[8]), "=r"(v[9]), "=r"(v[10]), "=r"(v[11]), "=r"(v[12]), "=r"(v[13]), "=r"(v[14]), "=r"(v[15]),  \
          "=r"(v[16]), "=r"(v[17]), "=r"(v[18]), "=r"(v[19]), "=r"(v[20]), "=r"(v[21]), "=r"(v[22]),            \
          "=r"(v[23]), "=r"(v[24]), "=r"(v[25]), "=r"(v[26]), "=r"(v[27]), "=r"(v[28]), "=r"(v[29]),            \
          "=r"(v[30]), "=r"(v[31])                                                                                 \
        : "r"(taddr))

__global__ void __launch_bounds__(TC_THREADS, 1)
    herk_tc_kernel(const __grid_constant__ CUtensorMap mXh, const __grid_constant__ CUtensorMap mXl,
                   const __grid_constant__ CUtensorMap mYh, const __grid_constant__ CUtensorMap mYl,
                   const __grid_constant__ CUtensorMap mBh, const __grid_constant__ CUtensorMap mBl, TcParams p) {
    extern __shared__ uint8_t smem_raw[];
    // 1024-byte aligned stage buffers, barriers after them
    const uint32_t raw = smem_u32(smem_raw);
    const uint32_t base = (raw + 1023u) & ~1023u;
    uint8_t* gbase = smem_raw + (base - raw);
    uint8_t* bar_area = gbase + size_t(TC_STAGES) * TC_STAGE_BYTES;
    uint64_t* full = reinterpret_cast<uint64_t*>(bar_area);
    uint64_t* empty = full + TC_STAGES;
    uint64_t* done = empty + TC_STAGES;
    uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(done + 1);
    volatile int* abort_flag = reinterpret_cast<volatile int*>(tmem_slot + 1);

    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;

    // tile of this CTA: 128-row block bi, 256-column block bj <= bi / 2
    int t = blockIdx.x;
    int s_idx = -1;  // K-chunk of a split tile
    if (t >= p.full_tiles) {
        const int u = t - p.full_tiles;
        t = p.full_tiles + u / p.split;
        s_idx = u - (u / p.split) * p.split;
    }
    const int tile = t;
    int bi = 0;
    while (bi < p.nt && t >= (bi >> 1) + 1) {
        t -= (bi >> 1) + 1;
        ++bi;
    }
    const int bj = t;

    if (threadIdx.x == 0) {
        for (int s = 0; s < TC_STAGES; ++s) {
            mbar_init(smem_u32(&full[s]), 1);
            mbar_init(smem_u32(&empty[s]), 1);
        }
        mbar_init(smem_u32(done), 1);
        *abort_flag = 0;
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
        asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
    }
    if (warp == 1) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(tmem_slot)),
                     "r"(TC_TMEM_COLS)
                     : "memory");
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
    }
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    const uint32_t tmem = *tmem_slot;
    const int total_kb = 3 * p.kb_per_seg;
    const int kb0 = s_idx < 0 ? 0 : s_idx * p.kb_chunk;
    const int kb1 = s_idx < 0 ? total_kb : min(total_kb, kb0 + p.kb_chunk);

    if (warp == 0) {
        if (lane == 0) {
            for (int kb = kb0; kb < kb1; ++kb) {
                const int stage = (kb - kb0) % TC_STAGES, round = (kb - kb0) / TC_STAGES;
                if (round > 0 && !mbar_wait(smem_u32(&empty[stage]), uint32_t((round - 1) & 1), abort_flag,
                                            p.wait_cap, p.status))
                    break;
                const uint32_t fb = smem_u32(&full[stage]);
                mbar_expect_tx(fb, TC_STAGE_BYTES);
                const int seg = kb / p.kb_per_seg;
                const int kx = (kb - seg * p.kb_per_seg) * TC_BK;
                const uint32_t sx = smem_u32(gbase + size_t(stage) * TC_STAGE_BYTES);
                tma_load_2d(sx, seg == 2 ? &mXl : &mXh, kx, bi * TC_BM, fb);
                tma_load_2d(sx + TC_A_BYTES, seg == 2 ? &mYl : &mYh, kx, bi * TC_BM, fb);
                tma_load_2d(sx + 2 * TC_A_BYTES, seg == 1 ? &mBl : &mBh, kx, bj * TC_BNW, fb);
            }
        }
    } else if (warp == 1) {
        if (lane == 0) {
            for (int kb = kb0; kb < kb1; ++kb) {
                const int stage = (kb - kb0) % TC_STAGES, round = (kb - kb0) / TC_STAGES;
                if (!mbar_wait(smem_u32(&full[stage]), uint32_t(round & 1), abort_flag, p.wait_cap, p.status)) break;
                asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
                const uint32_t sx = smem_u32(gbase + size_t(stage) * TC_STAGE_BYTES);
                const uint32_t sy = sx + TC_A_BYTES, sb = sx + 2 * TC_A_BYTES;
#pragma unroll
                for (int k = 0; k < TC_BK / 16; ++k) {
                    const uint32_t acc = ((kb - kb0) | k) != 0 ? 1u : 0u;
                    const uint64_t db = sw128_desc(sb + k * 32);
                    umma_bf16(tmem, sw128_desc(sx + k * 32), db, acc);
                    umma_bf16(tmem + TC_BNW, sw128_desc(sy + k * 32), db, acc);
                }
                umma_commit(smem_u32(&empty[stage]));
            }
            umma_commit(smem_u32(done));  // tracks every MMA issued above
        }
        __syncwarp();
    } else {
        // epilogue: warp w reads TMEM lanes 32 (w % 4) .. +31 (rows rbase .. rbase + 31).
        // Each 32 x 32 chunk is transposed through shared memory (the stage ring is
        // idle once "done" has fired) so that a warp reads and writes 512 contiguous
        // bytes of one row per instruction.
        const int lg = warp & 3;
        const int rbase = bi * TC_BM + lg * 32;
        const int cbase = bj * TC_BNW;
        if (p.accumulate) {
            // bring this warp's rows of C into L2 while the main loop runs: one
            // 128-byte line per lane, a row segment (256 x 16 B) per instruction
            for (int rr = 0; rr < 32; ++rr) {
                const int r = rbase + rr;
                if (r < p.n && cbase + 8 * lane <= r)
                    asm volatile("prefetch.global.L2 [%0];" ::"l"(p.C + size_t(r) * p.ldc + cbase + 8 * lane));
            }
        }
        const bool ok = mbar_wait(smem_u32(done), 0u, abort_flag, p.wait_cap, p.status);
        asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
        asm volatile("fence.proxy.async.shared::cta;" ::: "memory");  // stage ring reused by generic stores
        constexpr int SLD = 33;  // staged row stride (float2), conflict-light in both directions
        float2* stg = reinterpret_cast<float2*>(gbase) + (warp - 2) * (32 * SLD);
#pragma unroll 1
        for (int chunk = 0; chunk < TC_BNW / 32; ++chunk) {
            uint32_t vr[32], vi[32];
            const uint32_t taddr = tmem + (uint32_t(lg * 32) << 16) + uint32_t(chunk * 32);
            YQ_TMEM_LD_X32(taddr, vr);
            YQ_TMEM_LD_X32(taddr + TC_BNW, vi);
            asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
            const int c0 = cbase + chunk * 32;
            if (!ok || rbase >= p.n || c0 > rbase + 31) continue;  // warp-uniform
#pragma unroll
            for (int i = 0; i < 32; ++i) stg[lane * SLD + i] = make_float2(__uint_as_float(vr[i]), __uint_as_float(vi[i]));
            __syncwarp();
            if (s_idx >= 0) {  // partial of a split tile: rows lg * 32 + rr, columns chunk * 32 + lane
                float2* wt = p.ws + (size_t(tile - p.full_tiles) * p.split + s_idx) * (TC_BM * TC_BNW);
#pragma unroll 4
                for (int rr = 0; rr < 32; ++rr) wt[(lg * 32 + rr) * TC_BNW + chunk * 32 + lane] = stg[rr * SLD + lane];
                __syncwarp();
                continue;
            }
            const int c = c0 + lane;
            if (p.accumulate) {
#pragma unroll
                for (int h = 0; h < 2; ++h) {
                    double2 o[16];
#pragma unroll
                    for (int k = 0; k < 16; ++k) {
                        const int r = rbase + 16 * h + k;
                        o[k] = (r < p.n && c <= r) ? reinterpret_cast<const double2*>(p.C + size_t(r) * p.ldc)[c]
                                                   : make_double2(0.0, 0.0);
                    }
#pragma unroll
                    for (int k = 0; k < 16; ++k) {
                        const int rr = 16 * h + k, r = rbase + rr;
                        if (r < p.n && c <= r) {
                            const float2 v = stg[rr * SLD + lane];
                            o[k].x += p.alpha * double(v.x);
                            o[k].y += p.alpha * double(v.y);
                            reinterpret_cast<double2*>(p.C + size_t(r) * p.ldc)[c] = o[k];
                        }
                    }
                }
            } else {
#pragma unroll 4
                for (int rr = 0; rr < 32; ++rr) {
                    const int r = rbase + rr;
                    if (r < p.n && c <= r) {
                        const float2 v = stg[rr * SLD + lane];
                        double re = p.alpha * double(v.x);
                        if (c == r) re += p.shift;
                        reinterpret_cast<double2*>(p.C + size_t(r) * p.ldc)[c] = make_double2(re, p.alpha * double(v.y));
                    }
                }
            }
            __syncwarp();
        }
    }
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    if (warp == 1) {
        asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(TC_TMEM_COLS)
                     : "memory");
    }
}

// C (lower part, r < n) of the split tiles: [C +] alpha * (sum of the K-chunk
// partials in chunk order, in FP64) + shift on the diagonal.  blockIdx.y: split tile.
__global__ void split_reduce_kernel(TcParams p) {
    int t = p.full_tiles + int(blockIdx.y), bi = 0;
    while (bi < p.nt && t >= (bi >> 1) + 1) {
        t -= (bi >> 1) + 1;
        ++bi;
    }
    const int bj = t;
    const float2* w = p.ws + size_t(blockIdx.y) * p.split * (TC_BM * TC_BNW);
    for (int e = blockIdx.x * blockDim.x + threadIdx.x; e < TC_BM * TC_BNW; e += gridDim.x * blockDim.x) {
        const int r = bi * TC_BM + e / TC_BNW, c = bj * TC_BNW + e % TC_BNW;
        if (r >= p.n || c > r) continue;
        double re = 0.0, im = 0.0;
        for (int k = 0; k < p.split; ++k) {
            const float2 v = w[size_t(k) * (TC_BM * TC_BNW) + e];
            re += double(v.x);
            im += double(v.y);
        }
        re *= p.alpha;
        im *= p.alpha;
        if (c == r) re += p.shift;
        double2* out = reinterpret_cast<double2*>(p.C + size_t(r) * p.ldc) + c;
        if (p.accumulate) {
            const double2 o = *out;
            re += o.x;
            im += o.y;
        }
        *out = make_double2(re, im);
    }
}

// ---------------------------------------------------------------------------
static PFN_cuTensorMapEncodeTiled_v12000 get_encode() {
    static PFN_cuTensorMapEncodeTiled_v12000 fn = nullptr;
    static std::once_flag once;
    std::call_once(once, [] {
        void* ptr = nullptr;
        cudaDriverEntryPointQueryResult q;
        if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &ptr, cudaEnableDefault, &q) == cudaSuccess &&
            q == cudaDriverEntryPointSuccess)
            fn = reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(ptr);
    });
    if (!fn) throw Error(YQ_E_CUDA, "cuTensorMapEncodeTiled is unavailable");
    return fn;
}

static CUtensorMap make_map(const uint16_t* base, size_t rows, size_t kpad, uint32_t box_rows) {
    CUtensorMap m;
    cuuint64_t dims[2] = {cuuint64_t(kpad), cuuint64_t(rows)};
    cuuint64_t strides[1] = {cuuint64_t(kpad * 2)};
    cuuint32_t box[2] = {cuuint32_t(TC_BK), box_rows};
    cuuint32_t estr[2] = {1, 1};
    CUresult r = get_encode()(&m, CU_TENSOR_MAP_DATA_TYPE_BFLOAT16, 2, const_cast<uint16_t*>(base), dims, strides, box,
                              estr, CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_128B,
                              CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    if (r != CUDA_SUCCESS) throw Error(YQ_E_CUDA, "cuTensorMapEncodeTiled failed: " + std::to_string(int(r)));
    return m;
}

// YQ_TC_SPLIT=0 keeps whole tiles in the last partial wave (Gram and trailing updates)
bool tc_split_enabled() {
    static const bool on = [] {
        const char* e = std::getenv("YQ_TC_SPLIT");
        return !(e && std::string(e) == "0");
    }();
    return on;
}

namespace {
// Tiles of the lower triangle of an n x n output, and the K-split of the tiles
// after the last full wave of sm_count CTAs (split <= 1: none).
struct TcSplit {
    int tiles, full, split, kb_chunk;
};
TcSplit plan_split(int n, size_t kpad, int sm_count) {
    TcSplit q{};
    const int nt = int((size_t(n) + TC_BM - 1) / TC_BM);
    for (int b = 0; b < nt; ++b) q.tiles += (b >> 1) + 1;
    q.full = q.tiles;
    q.split = 1;
    q.kb_chunk = 0;
    const int W = std::max(1, sm_count);
    const int R = q.tiles % W;
    const int total_kb = 3 * int(kpad / TC_BK);
    if (R == 0) return q;
    const int want = W / R;
    if (want < 2 || total_kb < 2 * TC_STAGES) return q;
    const int chunk = (total_kb + want - 1) / want;
    q.kb_chunk = chunk;
    q.split = (total_kb + chunk - 1) / chunk;  // every chunk non-empty
    q.full = q.tiles - R;
    return q;
}
}  // namespace

void herk_tc_run(const uint16_t* xh, const uint16_t* xl, const uint16_t* yh, const uint16_t* yl, int n,
                 size_t rows_pad, size_t kpad, c128* C, size_t ldc, double alpha, double shift, bool accumulate,
                 int* d_status, cudaStream_t st) {
    herk_tc_launch(xh, xl, yh, yl, n, rows_pad, kpad, C, ldc, alpha, shift, accumulate, d_status, 0, nullptr, nullptr,
                   0, st);
}

void herk_tc_launch(const uint16_t* xh, const uint16_t* xl, const uint16_t* yh, const uint16_t* yl, int n,
                    size_t rows_pad, size_t kpad, c128* C, size_t ldc, double alpha, double shift, bool accumulate,
                    int* d_status, int sm_count, DevBuf* ws, float2* ws_fixed, size_t ws_fixed_bytes,
                    cudaStream_t st) {
    YQ_CHECK_ARG(n > 0 && kpad % TC_BK == 0 && kpad > 0 && rows_pad % TC_BM == 0 && size_t(n) <= rows_pad,
                 "herk_tc: operand padding");
    YQ_CHECK_ARG(reinterpret_cast<uintptr_t>(xh) % 16 == 0 && reinterpret_cast<uintptr_t>(xl) % 16 == 0 &&
                     reinterpret_cast<uintptr_t>(yh) % 16 == 0 && reinterpret_cast<uintptr_t>(yl) % 16 == 0,
                 "herk_tc: operand base addresses must be 16-byte aligned");
    YQ_CHECK_ARG(reinterpret_cast<uintptr_t>(C) % 16 == 0, "herk_tc: output must be 16-byte aligned");
    CUtensorMap mXh = make_map(xh, rows_pad, kpad, TC_BM), mXl = make_map(xl, rows_pad, kpad, TC_BM);
    CUtensorMap mYh = make_map(yh, rows_pad, kpad, TC_BM), mYl = make_map(yl, rows_pad, kpad, TC_BM);
    CUtensorMap mBh = make_map(xh, rows_pad, kpad, TC_BNW), mBl = make_map(xl, rows_pad, kpad, TC_BNW);
    TcParams p;
    p.n = n;
    p.nt = int((size_t(n) + TC_BM - 1) / TC_BM);
    TcSplit sp = plan_split(n, kpad, sm_count);
    p.ws = nullptr;
    if (sp.tiles > sp.full) {
        const size_t need = size_t(sp.tiles - sp.full) * sp.split * TC_BM * TC_BNW * sizeof(float2);
        if (ws) {
            ws->ensure(need);
            p.ws = ws->as<float2>();
        } else if (ws_fixed && need <= ws_fixed_bytes) {
            p.ws = ws_fixed;
        } else {  // no workspace: whole tiles
            sp.full = sp.tiles;
            sp.split = 1;
        }
    }
    const int tiles = sp.tiles;
    p.full_tiles = sp.full;
    p.split = sp.split;
    p.kb_chunk = sp.kb_chunk;
    const int R = tiles - sp.full;
    p.kb_per_seg = int(kpad / TC_BK);
    p.C = C;
    p.ldc = ldc;
    p.alpha = alpha;
    p.shift = shift;
    p.accumulate = accumulate ? 1 : 0;
    p.status = d_status;
    p.wait_cap = 1u << 24;
    static bool attr = false;
    if (!attr) {
        YQ_CUDA(cudaFuncSetAttribute(herk_tc_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, int(TC_SMEM)));
        attr = true;
    }
    herk_tc_kernel<<<sp.full + R * sp.split, TC_THREADS, TC_SMEM, st>>>(mXh, mXl, mYh, mYl, mBh, mBl, p);
    YQ_LAUNCH_CHECK();
    if (R > 0) {
        split_reduce_kernel<<<dim3(32, unsigned(R)), 256, 0, st>>>(p);
        YQ_LAUNCH_CHECK();
    }
}

void gram_tc_run(const uint16_t* xh, const uint16_t* xl, const uint16_t* yh, const uint16_t* yl, int ns, size_t P,
                 c128* G, size_t ldg, double alpha, double shift, int* d_status, int sm_count, DevBuf& ws,
                 cudaStream_t st) {
    herk_tc_launch(xh, xl, yh, yl, ns, gram_tc_rows(ns), gram_tc_kpad(P), G, ldg, alpha, shift, false, d_status,
                   sm_count, tc_split_enabled() ? &ws : nullptr, nullptr, 0, st);
}

}  // namespace yq
