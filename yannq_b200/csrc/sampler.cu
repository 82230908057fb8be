// Persistent Metropolis sampler: one warp per chain.
//
// Restates Samplers/SamplerMT.hpp (nTmps = 1) driving LocalSweeper
// (Samplers/LocalSweeper.hpp:32-53), SwapSweeper (Samplers/SwapSweeper.hpp:28-57,
// plus a neighbour-pair variant) or HamiltonianSweeper
// (Samplers/HamiltonianSweeper.hpp:22-50: proposals from the Hamiltonian's
// offDiagonals list, counted and selected with warp ballots).  Per chain the warp holds
//   sigma           int8 in shared memory (one row per warp),
//   theta_j, t_j    = theta and tanh(theta) for j = lane + 32 r in registers,
// and evaluates the reference's acceptance min(1, exp(2 beta Re logRatio)) with
// the product form of ratio.cuh: per proposal one column of tau = tanh(2W)
// (coalesced, L2-resident), one log per lane and a butterfly warp sum.  On an
// accepted move theta follows the reference's incremental update exactly
// (States/RBMState.hpp:248-266) and t follows tanh's addition formula; t is
// recomputed from theta at the end of every sweep, theta itself from sigma in
// FP64 every `resync` sweeps when requested.
//
// Random numbers: Philox4x32-10 with counter (proposal, epoch, chain, tag); the
// next proposal's columns are prefetched into L1 while the current one is scored.
#include <cstdlib>
#include <map>
#include <mutex>
#include <string>
#include <vector>

#include "internal.hpp"
#include "ratio.cuh"

namespace yq {

template <typename R>
struct SampArgs {
    int n, m, n_chains, L, n_total, n_discard, resync, reinit, nup, nstride;
    bool bias;
    uint64_t seed;
    uint32_t epoch;
    const uint32_t* epoch_dev;  // optional device-side epoch offset (graph replays)
    // parallel tempering (one launch per sweep): per-chain beta, theta carried over
    // between launches, recording of the slot-0 chain of each group, Re log psi out
    const double* beta;
    const cplx<R>* theta_in;
    cplx<R>* theta_out;
    double* lp_out;
    const int* slot;
    int ntemps, groups, rec_index, sw0, acc_add;
    const c128* p64;
    const cplx<R>* W;
    const cplx<R>* tau;
    const c128* Lk;
    int8_t* chains;
    int8_t* out_sigma;
    cplx<R>* out_theta;
    unsigned long long* acc;
    const HamMove* moves;  // HamiltonianSweeper proposals
    int n_moves;
};

// Is offDiagonals entry e present in s, with sites fa, fb (fb may be -1) flipped?
__device__ __forceinline__ bool move_present(const HamMove& e, const int8_t* s, int fa, int fb) {
    if (e.b < 0) return (e.on & 1) != 0;
    int zz = s[e.a] * s[e.b];
    const int flips = (e.a == fa || e.a == fb) + (e.b == fa || e.b == fb);
    if (flips == 1) zz = -zz;
    return ((e.on >> (zz > 0 ? 0 : 1)) & 1) != 0;
}

// Size of offDiagonals(s with fa, fb flipped), the same in every lane.
__device__ __forceinline__ int count_moves(const HamMove* __restrict__ mv, int K, const int8_t* s, int fa, int fb,
                                           int lane) {
    int cnt = 0;
    for (int e = lane; e < K; e += 32) cnt += move_present(mv[e], s, fa, fb) ? 1 : 0;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) cnt += __shfl_xor_sync(0xffffffffu, cnt, o);
    return cnt;
}

// Index of the r-th present entry of offDiagonals(s) (0 <= r < count), in list order.
__device__ __forceinline__ int select_move(const HamMove* __restrict__ mv, int K, const int8_t* s, int r, int lane) {
    for (int base = 0; base < K; base += 32) {
        const int e = base + lane;
        const bool on = e < K && move_present(mv[e], s, -1, -1);
        const unsigned bal = __ballot_sync(0xffffffffu, on);
        const int cnt = __popc(bal);
        if (r < cnt) {
            const bool mine = on && __popc(bal & ((1u << lane) - 1u)) == r;
            const unsigned who = __ballot_sync(0xffffffffu, mine);
            return base + (__ffs(who) - 1);
        }
        r -= cnt;
    }
    return -1;
}

__device__ __forceinline__ void prefetch_l1(const void* p) {
    asm volatile("prefetch.global.L1 [%0];" ::"l"(p));
}

template <typename R>
__device__ __forceinline__ R warp_allsum(R v) {
    // xor butterfly: every lane ends with the bitwise identical sum
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}

// The proposal draws of one chain, 32 at a time: lane l evaluates the Philox
// block of proposal 32 b + l once, and proposal g reads its four words from lane
// g mod 32 -- the same values as one draw(seed, g, ...) per proposal, at 1/32 of
// the Philox rounds.  The block index only changes with g, so it is warp-uniform.
struct DrawCache {
    uint32_t blk = 0xffffffffu;
    U4 mine;
    __device__ __forceinline__ U4 get(uint64_t seed, uint32_t g, uint32_t epoch, uint32_t chain, int lane) {
        const uint32_t b = g >> 5;
        if (b != blk) {
            blk = b;
            mine = draw(seed, (b << 5) + uint32_t(lane), epoch, chain, TAG_SWEEP);
        }
        const int src = int(g & 31u);
        U4 r;
        r.x = __shfl_sync(0xffffffffu, mine.x, src);
        r.y = __shfl_sync(0xffffffffu, mine.y, src);
        r.z = __shfl_sync(0xffffffffu, mine.z, src);
        r.w = __shfl_sync(0xffffffffu, mine.w, src);
        return r;
    }
};

// Per-unit arithmetic of the complex64 sampler.  Its products, logs and the
// acceptance exponential feed only the Metropolis comparison u < p and the
// incremental tanh update, so the single-precision hardware approximations
// (MUFU log2 / exp2, correctly rounded reciprocal) replace the accurate library
// forms; the complex128 path keeps the accurate ones (draw-for-draw parity with the
// FP64 reference restatement).
template <typename R>
__device__ __forceinline__ R sampler_log(R x) {
    return log(x);
}
template <>
__device__ __forceinline__ float sampler_log<float>(float x) {
    return __logf(x);
}
template <typename R>
__device__ __forceinline__ R sampler_exp(R x) {
    return exp(x);
}
template <>
__device__ __forceinline__ float sampler_exp<float>(float x) {
    return __expf(x);
}
// a / b for the tanh update (b = the unit's factor, away from 0 by the cancellation guard)
template <typename R>
__device__ __forceinline__ cplx<R> sampler_div(cplx<R> a, cplx<R> b) {
    return cdiv(a, b);
}
template <>
__device__ __forceinline__ cplx<float> sampler_div<float>(cplx<float> a, cplx<float> b) {
    const float r = __frcp_rn(b.re * b.re + b.im * b.im);
    return mk((a.re * b.re + a.im * b.im) * r, (a.im * b.re - a.re * b.im) * r);
}

// Sum of the chain's WPC warp partials (each already a warp butterfly sum), in
// warp order, through the chain's double-buffered slots at a named barrier of the
// WPC warps (barrier 0 stays __syncthreads).  A slot pair is rewritten two
// proposals later, after every warp of the chain has passed the barrier that
// follows its reads.
template <typename R, int WPC>
__device__ __forceinline__ R chain_sum(R v, R* part, int& pbuf, int wchain, int sub, int lane) {
    if constexpr (WPC == 1) {
        return v;
    } else {
        R* b = part + pbuf * WPC;
        if (lane == 0) b[sub] = v;
        asm volatile("bar.sync %0, %1;" ::"r"(1 + wchain), "r"(32 * WPC) : "memory");
        R t = b[0];
#pragma unroll
        for (int w = 1; w < WPC; ++w) t += b[w];
        pbuf ^= 1;
        return t;
    }
}

template <typename R>
struct LogGroup {
    static constexpr int G = 8;
};
template <>
struct LogGroup<float> {
    static constexpr int G = 2;
};

template <typename R, int JPL>
__device__ __forceinline__ void theta_fp64(const SampArgs<R>& A, const int8_t* s, int lane, cplx<R> (&th)[JPL],
                                           int sub = 0, int wpc = 1) {
    const size_t nm = size_t(A.n) * A.m;
#pragma unroll
    for (int r = 0; r < JPL; ++r) {
        const int j = lane + 32 * (sub + wpc * r);
        if (j < A.m) {
            double ar = 0., ai = 0.;
            for (int i = 0; i < A.n; ++i) {
                c128 w = A.p64[size_t(i) * A.m + j];
                double sv = double(s[i]);
                ar += w.re * sv;
                ai += w.im * sv;
            }
            if (A.bias) {
                c128 b = A.p64[nm + A.n + j];
                ar += b.re;
                ai += b.im;
            }
            th[r] = mk(R(ar), R(ai));
        } else {
            th[r] = mk(R(0), R(0));
        }
    }
}

// WPC warps per chain: hidden unit j = lane + 32 (sub + WPC r) of the chain's warp
// `sub`.  With WPC = 2 the two warps draw the same proposals, keep their own copy
// of sigma, and combine their partial log-sums through shared memory at a named
// barrier of the pair (one per proposal, double-buffered), adding the two halves
// in the same order so that both take the same decision.  Only plain chains
// (no tempering) of local or exchange moves use it.
template <typename R, int MOVE, int JPL, int WPC>
__global__ void __launch_bounds__(128, WPC == 2 ? 4 : 1) metropolis_kernel(SampArgs<R> A) {
    extern __shared__ int8_t smem_sig[];
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int wchain = warp / WPC, sub = warp - wchain * WPC;
    const int c = blockIdx.x * ((blockDim.x >> 5) / WPC) + wchain;
    if (c >= A.n_chains) return;  // uniform over the chain's warps
    const int n = A.n, m = A.m;
    const uint32_t epoch = A.epoch_dev ? A.epoch + *A.epoch_dev : A.epoch;
    int8_t* s = smem_sig + warp * A.nstride;
    int8_t* cs = A.chains + size_t(c) * n;
    // partial log-sums of the chain's warps: [2 buffers][WPC], after every warp's sigma row
    R* part = reinterpret_cast<R*>(smem_sig + ((size_t((blockDim.x >> 5)) * A.nstride + 15) & ~size_t(15))) +
              size_t(wchain) * 2 * WPC;
    int pbuf = 0;

    // ---- chain initialisation (SamplerMT::randomize, Utilities/Utility.hpp:63-88)
    if (A.reinit) {
        if (A.nup < 0) {
            for (int i = lane; i < n; i += 32) {
                U4 x = draw(A.seed, uint32_t(i), epoch, uint32_t(c), TAG_INIT);
                s[i] = (x.x & 1u) ? int8_t(-1) : int8_t(1);
            }
        } else {
            if (lane == 0) {
                for (int i = 0; i < n; ++i) s[i] = (i < A.nup) ? int8_t(-1) : int8_t(1);
                for (int i = n - 1; i >= 1; --i) {
                    U4 x = draw(A.seed, uint32_t(i), epoch, uint32_t(c), TAG_SHUF);
                    int j = int(draw_site(x.x, uint32_t(i + 1)));
                    int8_t tmp = s[i];
                    s[i] = s[j];
                    s[j] = tmp;
                }
            }
        }
    } else {
        for (int i = lane; i < n; i += 32) s[i] = cs[i];
    }
    __syncwarp();

    const R beta = A.beta ? R(A.beta[c]) : R(1);
    cplx<R> th[JPL], t[JPL];
    if (A.theta_in) {
#pragma unroll
        for (int r = 0; r < JPL; ++r) {
            const int j = lane + 32 * (sub + WPC * r);
            th[r] = j < m ? A.theta_in[size_t(c) * m + j] : mk(R(0), R(0));
        }
    } else {
        theta_fp64<R, JPL>(A, s, lane, th, sub, WPC);
    }
#pragma unroll
    for (int r = 0; r < JPL; ++r) t[r] = ctanh(th[r]);

    unsigned long long nacc = 0;
    const uint32_t L = uint32_t(A.L);
    const R two = R(2);
    constexpr int G = LogGroup<R>::G;

    // The proposal sites do not depend on acceptance, so the next proposal's draw
    // and (local moves) its tau and W columns and L_k, a_k are loaded into
    // registers one proposal ahead; exchange moves prefetch their two columns
    // into L1.
    // (register pipelining for complex64 only: complex128 would spill)
    constexpr bool REGPIPE = MOVE == YQ_MOVE_LOCAL && sizeof(R) == 4;
    constexpr bool HAMMOVE = MOVE == YQ_MOVE_HAMILTONIAN;  // proposals depend on the state: nothing ahead
    DrawCache dc;
    U4 xcur = dc.get(A.seed, uint32_t(A.sw0) * L, epoch, uint32_t(c), lane);
    cplx<R> tvn[JPL], wvn[JPL];
    double lkn = 0., abn = 0.;
    auto load_cols = [&](int kq) {
#pragma unroll
        for (int r = 0; r < JPL; ++r) {
            const int j = lane + 32 * (sub + WPC * r);
            tvn[r] = j < m ? A.tau[size_t(kq) * m + j] : mk(R(0), R(0));
            wvn[r] = j < m ? A.W[size_t(kq) * m + j] : mk(R(0), R(0));
        }
        lkn = A.Lk[kq].re;
        abn = A.bias ? A.p64[size_t(n) * m + kq].re : 0.0;
    };
    if (REGPIPE) {
        load_cols(int(draw_site(xcur.x, uint32_t(n))));
    } else if (!HAMMOVE) {
        const int k0 = int(draw_site(xcur.x, uint32_t(n)));
#pragma unroll
        for (int r = 0; r < JPL; ++r) {
            int j = lane + 32 * (sub + WPC * r);
            if (j < m) {
                prefetch_l1(A.tau + size_t(k0) * m + j);
                prefetch_l1(A.W + size_t(k0) * m + j);
            }
        }
    }

    for (int sw = 0; sw < A.n_total; ++sw) {
        for (uint32_t p = 0; p < L; ++p) {
            const uint32_t g = uint32_t(A.sw0 + sw) * L + p;
            const U4 x = xcur;
            const U4 xn = dc.get(A.seed, g + 1u, epoch, uint32_t(c), lane);
            xcur = xn;
            if (!REGPIPE && !HAMMOVE) {
                // prefetch the next proposal's columns into L1
                int kn = int(draw_site(xn.x, uint32_t(n)));
                int ln = (MOVE == YQ_MOVE_EXCHANGE_ANY) ? int(draw_site(xn.y, uint32_t(n))) : (kn + 1) % n;
#pragma unroll
                for (int r = 0; r < JPL; ++r) {
                    int j = lane + 32 * (sub + WPC * r);
                    if (j < m) {
                        prefetch_l1(A.tau + size_t(kn) * m + j);
                        prefetch_l1(A.W + size_t(kn) * m + j);
                        if (MOVE != YQ_MOVE_LOCAL) {
                            prefetch_l1(A.tau + size_t(ln) * m + j);
                            prefetch_l1(A.W + size_t(ln) * m + j);
                        }
                    }
                }
            }
            const R u = draw_uniform<R>(x);
            int k, l = -1;
            R wfac = R(1);  // HamiltonianSweeper.hpp:39-42: w1 / w2
            if (HAMMOVE) {
                const int w1 = count_moves(A.moves, A.n_moves, s, -1, -1, lane);
                if (w1 == 0) continue;  // empty list: the slot is consumed
                const int e = select_move(A.moves, A.n_moves, s, int(draw_site(x.x, uint32_t(w1))), lane);
                if (e < 0) continue;  // not reached: r < w1 entries are present
                k = A.moves[e].a;
                l = A.moves[e].b;
                const int w2 = count_moves(A.moves, A.n_moves, s, k, l, lane);
                wfac = R(w1) / R(w2);
            } else {
                k = int(draw_site(x.x, uint32_t(n)));
                if (MOVE != YQ_MOVE_LOCAL) l = (MOVE == YQ_MOVE_EXCHANGE_ANY) ? int(draw_site(x.y, uint32_t(n))) : (k + 1) % n;
            }
            // HamiltonianSweeper.hpp:42 has no beta
            const R bexp = HAMMOVE ? R(1) : beta;
            if (MOVE == YQ_MOVE_LOCAL || (HAMMOVE && l < 0)) {
                const R sk = R(s[k]);
                const cplx<R>* wk = A.W + size_t(k) * m;
                cplx<R> tv[JPL], wv[JPL], d[JPL];
                double lk, ab;
                if (REGPIPE) {
#pragma unroll
                    for (int r = 0; r < JPL; ++r) {
                        tv[r] = tvn[r];
                        wv[r] = wvn[r];
                    }
                    lk = lkn;
                    ab = abn;
                    load_cols(int(draw_site(xn.x, uint32_t(n))));  // next proposal, in flight meanwhile
                } else {
#pragma unroll
                    for (int r = 0; r < JPL; ++r) {
                        const int j = lane + 32 * (sub + WPC * r);
                        tv[r] = j < m ? A.tau[size_t(k) * m + j] : mk(R(0), R(0));
                    }
                    lk = A.Lk[k].re;
                    ab = A.bias ? A.p64[size_t(n) * m + k].re : 0.0;
                }
                unsigned exact = 0u;  // bit r: factor r re-evaluated in logcosh form (ratio.cuh)
#pragma unroll
                for (int r = 0; r < JPL; ++r) {
                    int j = lane + 32 * (sub + WPC * r);
                    if (j < m) {
                        bool ex;
                        d[r] = factor1<R>(t[r], tv[r], sk, th[r], REGPIPE ? &wv[r] : wk + j, ex);
                        exact |= unsigned(ex) << r;
                    } else {
                        d[r] = one<R>();
                    }
                }
                R ls = R(0);
                cplx<R> pr = mk(R(1), R(0));
#pragma unroll
                for (int r = 0; r < JPL; ++r) {
                    pr = pr * d[r];
                    if ((r % G) == G - 1 || r == JPL - 1) {
                        ls += sampler_log<R>(norm2(pr));
                        pr = mk(R(1), R(0));
                    }
                }
                ls = chain_sum<R, WPC>(warp_allsum(ls), part, pbuf, wchain, sub, lane);
                const double base = lk - 2.0 * double(sk) * ab;
                const R logr = R(0.5) * ls + R(base);
                // LocalSweeper.hpp:45-47: p = min(1, exp(beta * 2 * Re logRatio)); accept if u < p
                if (u < sampler_exp<R>(two * bexp * logr) * wfac) {
#pragma unroll
                    for (int r = 0; r < JPL; ++r) {
                        int j = lane + 32 * (sub + WPC * r);
                        if (j < m) {
                            const cplx<R> w = REGPIPE ? wv[r] : wk[j];
                            th[r] = th[r] - (two * sk) * w;
                            t[r] = ((exact >> r) & 1u) ? ctanh(th[r]) : sampler_div<R>(t[r] - sk * tv[r], d[r]);
                        }
                    }
                    __syncwarp();
                    if (lane == 0) s[k] = int8_t(-s[k]);
                    __syncwarp();
                    ++nacc;
                }
            } else {
                const int8_t sk8 = s[k], sl8 = s[l];
                if (!HAMMOVE && sk8 == sl8) continue;  // SwapSweeper.hpp:43-46: the slot is consumed
                const R sk = R(sk8), sl = R(sl8);
                const cplx<R>* tk = A.tau + size_t(k) * m;
                const cplx<R>* tl = A.tau + size_t(l) * m;
                const cplx<R>* wk = A.W + size_t(k) * m;
                const cplx<R>* wl = A.W + size_t(l) * m;
                cplx<R> tx[JPL], ty[JPL], d[JPL];
                unsigned exact = 0u;
#pragma unroll
                for (int r = 0; r < JPL; ++r) {
                    int j = lane + 32 * (sub + WPC * r);
                    if (j < m) {
                        tx[r] = sk * tk[j];
                        ty[r] = sl * tl[j];
                        bool ex;
                        d[r] = factor2<R>(t[r], tx[r], ty[r], sk, sl, th[r], wk + j, wl + j, ex);
                        exact |= unsigned(ex) << r;
                    } else {
                        tx[r] = mk(R(0), R(0));
                        ty[r] = mk(R(0), R(0));
                        d[r] = one<R>();
                    }
                }
                R ls = R(0);
                cplx<R> pr = mk(R(1), R(0));
#pragma unroll
                for (int r = 0; r < JPL; ++r) {
                    pr = pr * d[r];
                    if ((r % G) == G - 1 || r == JPL - 1) {
                        ls += sampler_log<R>(norm2(pr));
                        pr = mk(R(1), R(0));
                    }
                }
                ls = chain_sum<R, WPC>(warp_allsum(ls), part, pbuf, wchain, sub, lane);
                double base = A.Lk[k].re + A.Lk[l].re;
                if (A.bias)
                    base -= 2.0 * double(sk) * A.p64[size_t(n) * m + k].re +
                            2.0 * double(sl) * A.p64[size_t(n) * m + l].re;
                const R logr = R(0.5) * ls + R(base);
                if (u < sampler_exp<R>(two * bexp * logr) * wfac) {
#pragma unroll
                    for (int r = 0; r < JPL; ++r) {
                        int j = lane + 32 * (sub + WPC * r);
                        if (j < m) {
                            cplx<R> a = wk[j], b = wl[j];
                            // States/RBMState.hpp:261-262: theta += -2 s_k W_k - 2 s_l W_l
                            cplx<R> dd = mk(-(two * sk) * a.re - (two * sl) * b.re, -(two * sk) * a.im - (two * sl) * b.im);
                            th[r] = th[r] + dd;
                            cplx<R> sxy = tx[r] + ty[r];
                            t[r] = ((exact >> r) & 1u) ? ctanh(th[r])
                                                       : sampler_div<R>(t[r] * (one<R>() + tx[r] * ty[r]) - sxy, d[r]);
                        }
                    }
                    __syncwarp();
                    if (lane == 0) {
                        s[k] = int8_t(-sk8);
                        s[l] = int8_t(-sl8);
                    }
                    __syncwarp();
                    ++nacc;
                }
            }
        }
        // ---- end of sweep: record (SamplerMT.hpp:196-201), resync
        // tempered sampling records after mixChains, in pt_mix_kernel
        if (sw >= A.n_discard && !A.slot) {
            const size_t idx = size_t(sw - A.n_discard) * A.n_chains + c;
            if (sub == 0)
                for (int i = lane; i < n; i += 32) A.out_sigma[idx * n + i] = s[i];
#pragma unroll
            for (int r = 0; r < JPL; ++r) {
                int j = lane + 32 * (sub + WPC * r);
                if (j < m) A.out_theta[idx * m + j] = th[r];
            }
        }
        if (A.resync > 0 && ((A.sw0 + sw + 1) % A.resync) == 0) theta_fp64<R, JPL>(A, s, lane, th, sub, WPC);
#pragma unroll
        for (int r = 0; r < JPL; ++r) t[r] = ctanh(th[r]);
    }
    __syncwarp();
    if (sub == 0)
        for (int i = lane; i < n; i += 32) cs[i] = s[i];
    if (A.theta_out) {
#pragma unroll
        for (int r = 0; r < JPL; ++r) {
            const int j = lane + 32 * (sub + WPC * r);
            if (j < m) A.theta_out[size_t(c) * m + j] = th[r];
        }
    }
    if (A.lp_out) {
        // Re log psi = Re(a) . sigma + sum_j Re logcosh(theta_j)   (RBM.hpp:367-378)
        double lp = 0.;
#pragma unroll
        for (int r = 0; r < JPL; ++r) {
            const int j = lane + 32 * (sub + WPC * r);
            if (j < m) lp += clogcosh(cast<double>(th[r])).re;
        }
        if (A.bias)
            for (int i = lane; i < n; i += 32) lp += double(s[i]) * A.p64[size_t(n) * m + i].re;
        lp = warp_allsum(lp);
        if (lane == 0) A.lp_out[c] = lp;
    }
    if (lane == 0 && sub == 0) A.acc[c] = (A.acc_add ? A.acc[c] : 0ull) + nacc;
}

// mixChains (SamplerMT.hpp:120-153) for one group per thread: even slot pairs
// (0,1),(2,3),..., then odd pairs (1,2),...,(ntemps-3, ntemps-2); a swap exchanges
// the chains' slots (temperatures).  p = exp((beta_{t+1} - beta_t) 2 (lp(slot t) -
// lp(slot t+1))), u from counter (64 sweep + t, epoch, group, TAG_PT).
// A recorded sweep then appends the slot-0 chain of the group (SamplerMT.hpp:196-201,
// after mixChains): sigma from the chains, theta (tbytes per chain) from the
// carried-over theta, into output row rec_index * groups + group.
__global__ void pt_mix_kernel(int groups, int ntemps, const double* __restrict__ lp, int* __restrict__ slot,
                              double* __restrict__ beta, uint64_t seed, uint32_t epoch, const uint32_t* epoch_dev,
                              uint32_t sweep, int record, int rec_index, int n, const int8_t* __restrict__ chains,
                              int tbytes, const uint8_t* __restrict__ theta, int8_t* __restrict__ out_sigma,
                              uint8_t* __restrict__ out_theta) {
    const int gr = blockIdx.x * blockDim.x + threadIdx.x;
    if (gr >= groups) return;
    const uint32_t ep = epoch_dev ? epoch + *epoch_dev : epoch;
    int at[64];
    for (int k = 0; k < ntemps; ++k) at[slot[gr * ntemps + k]] = gr * ntemps + k;
    auto bt = [&](int t) { return double(ntemps - t) / double(ntemps); };
    auto attempt = [&](int t) {
        const int a = at[t], b = at[t + 1];
        const double pr = exp((bt(t + 1) - bt(t)) * 2.0 * (lp[a] - lp[b]));
        const U4 x = draw(seed, sweep * 64u + uint32_t(t), ep, uint32_t(gr), TAG_PT);
        if (draw_u53(x.z, x.w) < pr) {
            at[t] = b;
            at[t + 1] = a;
        }
    };
    for (int t = 0; t + 1 < ntemps; t += 2) attempt(t);
    for (int t = 1; t + 1 < ntemps - 1; t += 2) attempt(t);
    for (int t = 0; t < ntemps; ++t) {
        slot[at[t]] = t;
        beta[at[t]] = bt(t);
    }
    if (record) {
        const size_t row = size_t(rec_index) * groups + gr;
        const int c0 = at[0];
        for (int i = 0; i < n; ++i) out_sigma[row * n + i] = chains[size_t(c0) * n + i];
        for (int b = 0; b < tbytes; ++b) out_theta[row * tbytes + b] = theta[size_t(c0) * tbytes + b];
    }
}

__global__ void pt_reset_kernel(int n_chains, int ntemps, int* __restrict__ slot, double* __restrict__ beta) {
    const int c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= n_chains) return;
    slot[c] = c % ntemps;
    beta[c] = double(ntemps - c % ntemps) / double(ntemps);
}

template <typename R, int MOVE, int JPL, int WPC>
static void launch_w(const SampArgs<R>& A, int warps, cudaStream_t st) {
    const int chains_per_cta = warps / WPC;
    dim3 grid(cdiv_u(A.n_chains, chains_per_cta));
    const size_t smem = ((size_t(warps) * A.nstride + 15) & ~size_t(15)) + size_t(chains_per_cta) * 2 * WPC * sizeof(R);
    metropolis_kernel<R, MOVE, JPL, WPC><<<grid, warps * 32, smem, st>>>(A);
    YQ_LAUNCH_CHECK();
}

// Units per lane for WPC warps per chain: the smallest instantiated count that covers m.
template <typename R, int MOVE, int WPC>
static void launch_jpl(const SampArgs<R>& A, int warps, cudaStream_t st) {
    const int need = (A.m + 32 * WPC - 1) / (32 * WPC);
#define YQ_JPL(J)                                   \
    if (need <= J) {                                \
        launch_w<R, MOVE, J, WPC>(A, warps, st);    \
        return;                                     \
    }
    if constexpr (WPC == 1) {
        YQ_JPL(1) YQ_JPL(2) YQ_JPL(4) YQ_JPL(8) YQ_JPL(9) YQ_JPL(12) YQ_JPL(16) YQ_JPL(32)
    } else {
        YQ_JPL(1) YQ_JPL(2) YQ_JPL(3) YQ_JPL(4) YQ_JPL(5) YQ_JPL(6) YQ_JPL(8) YQ_JPL(16)
    }
#undef YQ_JPL
    throw Error(YQ_E_UNSUPPORTED, "sampler: m > 1024 hidden units is not built");
}

// Launch shape: warps per chain (1, or 2 for complex64 plain chains of local and
// exchange moves) and warps per block (at most 4, the kernel's launch bound).
struct Shape {
    int wpc, warps;
};

template <typename R, int MOVE>
static constexpr bool split_ok() {
    return sizeof(R) == 4 && MOVE != YQ_MOVE_HAMILTONIAN;
}

template <typename R, int MOVE>
static void launch_shape(const SampArgs<R>& A, Shape sh, cudaStream_t st) {
    if constexpr (split_ok<R, MOVE>()) {
        if (sh.wpc == 2) {
            launch_jpl<R, MOVE, 2>(A, sh.warps, st);
            return;
        }
    }
    launch_jpl<R, MOVE, 1>(A, sh.warps, st);
}

// Autotuned launch shape.  On the first call of a configuration (type, move, n, m,
// chains, sweep length, tempering) the kernel runs two sweeps from a scratch copy
// of the chains into scratch outputs in every candidate shape -- 1, 2 and 4 chains
// per CTA with one warp per chain, and for complex64 plain chains 1 and 2 chains
// per CTA with two warps per chain -- timed with CUDA events on the library stream
// after one untimed launch, the candidates taken in turn over two rounds so that a
// clock still ramping up weighs on all of them alike; the fastest (least of its two
// times) is kept for the process.  With one warp per chain the chains evolve
// identically whatever the block shape (each warp owns one chain and its own
// Philox counters); two warps per chain draw the same proposals and add the two
// halves of each log-ratio sum, a different rounding of the same sum.  Calls made
// while the stream is being captured, and YQ_AUTOTUNE=0, use 4 chains per CTA and
// one warp per chain; YQ_CHAINS_PER_CTA=1, 2 or 4 fixes the chains per CTA (one
// warp per chain unless YQ_WARPS_PER_CHAIN=2), YQ_WARPS_PER_CHAIN=1 or 2 restricts
// the candidates to that split.
constexpr int N_TUNE = 5;
struct TuneEntry {
    Shape shape;
    float ms[N_TUNE];
};
static std::mutex g_tune_mu;
static std::map<std::vector<long long>, TuneEntry> g_tune;

static int env_int(const char* name) {
    const char* e = std::getenv(name);
    return e ? std::atoi(e) : 0;
}

template <typename R, int MOVE>
static Shape tuned_shape(const SampArgs<R>& A, cudaStream_t st) {
    static const bool enabled = [] {
        const char* e = std::getenv("YQ_AUTOTUNE");
        return !(e && std::string(e) == "0");
    }();
    static const int forced_cpc = [] {
        const int v = env_int("YQ_CHAINS_PER_CTA");
        return (v == 1 || v == 2 || v == 4) ? v : 0;
    }();
    static const int forced_wpc = [] {
        const int v = env_int("YQ_WARPS_PER_CHAIN");
        return (v == 1 || v == 2) ? v : 0;
    }();
    const bool plain = A.slot == nullptr && A.theta_in == nullptr && A.theta_out == nullptr && A.lp_out == nullptr;
    const bool can_split = split_ok<R, MOVE>() && plain;
    Shape cand[N_TUNE];
    int nc = 0;
    for (int wpc = 1; wpc <= 2; ++wpc) {
        if (wpc == 2 && !can_split) continue;
        if (forced_wpc && wpc != forced_wpc) continue;
        for (int cpc = 1; cpc <= 4; cpc *= 2) {
            if (cpc * wpc > 4) continue;
            if (forced_cpc && cpc != forced_cpc) continue;
            cand[nc++] = Shape{wpc, cpc * wpc};
        }
    }
    if (nc == 0) cand[nc++] = Shape{1, forced_cpc ? forced_cpc : 4};  // a split the configuration does not take
    if (nc == 1) return cand[0];
    cudaStreamCaptureStatus cap = cudaStreamCaptureStatusNone;
    YQ_CUDA(cudaStreamIsCapturing(st, &cap));
    const std::vector<long long> key = {static_cast<long long>(sizeof(R)), MOVE, A.n, A.m, A.n_chains, A.L,
                                        plain ? 1 : 0};
    {
        std::lock_guard<std::mutex> lk(g_tune_mu);
        auto it = g_tune.find(key);
        if (it != g_tune.end()) return it->second.shape;
    }
    if (!enabled || cap != cudaStreamCaptureStatusNone) return Shape{1, 4};
    // Two sweeps, the last one recorded: the kernel writes recorded sweep sw to
    // rows (sw - n_discard) * n_chains + chain, so the scratch outputs hold
    // (n_total - n_discard) x n_chains rows.
    constexpr int trial_sweeps = 2, trial_recorded = 1, rounds = 2;
    DevBuf ch, sg, th, acc;
    ch.ensure(size_t(A.n_chains) * A.n);
    sg.ensure(size_t(trial_recorded) * A.n_chains * A.n);
    th.ensure(size_t(trial_recorded) * A.n_chains * A.m * sizeof(cplx<R>));
    acc.ensure(size_t(A.n_chains) * sizeof(unsigned long long));
    SampArgs<R> T = A;
    T.chains = ch.as<int8_t>();
    T.out_sigma = sg.as<int8_t>();
    T.out_theta = th.as<cplx<R>>();
    T.acc = acc.as<unsigned long long>();
    T.n_total = trial_sweeps;
    T.n_discard = trial_sweeps - trial_recorded;
    T.epoch_dev = nullptr;
    T.theta_in = nullptr;  // nothing of the real chain state is read or written
    T.theta_out = nullptr;
    T.lp_out = nullptr;
    T.slot = nullptr;
    T.acc_add = 0;
    T.sw0 = 0;
    if (!A.reinit)
        YQ_CUDA(cudaMemcpyAsync(ch.p, A.chains, size_t(A.n_chains) * A.n, cudaMemcpyDeviceToDevice, st));
    cudaEvent_t e0, e1;
    YQ_CUDA(cudaEventCreate(&e0));
    YQ_CUDA(cudaEventCreate(&e1));
    TuneEntry best{cand[0], {1e30f, 1e30f, 1e30f, 1e30f, 1e30f}};
    launch_shape<R, MOVE>(T, cand[0], st);  // untimed: caches and clocks
    for (int round = 0; round < rounds; ++round) {
        for (int c = 0; c < nc; ++c) {
            YQ_CUDA(cudaEventRecord(e0, st));
            launch_shape<R, MOVE>(T, cand[c], st);
            YQ_CUDA(cudaEventRecord(e1, st));
            YQ_CUDA(cudaEventSynchronize(e1));
            float t = 0.f;
            YQ_CUDA(cudaEventElapsedTime(&t, e0, e1));
            best.ms[c] = std::min(best.ms[c], t);
        }
    }
    float best_ms = 1e30f;
    for (int c = 0; c < nc; ++c) {
        if (best.ms[c] < best_ms) {
            best_ms = best.ms[c];
            best.shape = cand[c];
        }
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    std::lock_guard<std::mutex> lk(g_tune_mu);
    g_tune[key] = best;
    return best.shape;
}

template <typename R, int MOVE>
static void dispatch_shape(const SampArgs<R>& A, cudaStream_t st, int* chains_per_cta, int* warps_per_chain) {
    const Shape sh = tuned_shape<R, MOVE>(A, st);
    if (chains_per_cta) *chains_per_cta = sh.warps / sh.wpc;
    if (warps_per_chain) *warps_per_chain = sh.wpc;
    launch_shape<R, MOVE>(A, sh, st);
}

template <typename R>
static void launch_sweeps(yq_sampler_s* S, const SampArgs<R>& A, cudaStream_t st) {
    int* cpc = &S->chains_per_cta;
    int* wpc = &S->warps_per_chain;
    switch (S->move) {
        case YQ_MOVE_LOCAL: dispatch_shape<R, YQ_MOVE_LOCAL>(A, st, cpc, wpc); break;
        case YQ_MOVE_EXCHANGE_ANY: dispatch_shape<R, YQ_MOVE_EXCHANGE_ANY>(A, st, cpc, wpc); break;
        case YQ_MOVE_HAMILTONIAN: dispatch_shape<R, YQ_MOVE_HAMILTONIAN>(A, st, cpc, wpc); break;
        default: dispatch_shape<R, YQ_MOVE_EXCHANGE_NN>(A, st, cpc, wpc); break;
    }
}

template <typename R>
static void run_t(yq_sampler_s* S, int n_sweeps, int n_discard, uint64_t seed, uint32_t epoch, int reinit) {
    yq_rbm_s* q = S->q;
    SampArgs<R> A;
    A.n = q->n;
    A.m = q->m;
    A.n_chains = S->n_chains;
    A.L = S->sweep_len > 0 ? S->sweep_len : q->n;
    A.n_total = n_discard + n_sweeps;
    A.n_discard = n_discard;
    A.resync = S->resync;
    A.reinit = reinit;
    A.nup = S->nup;
    A.nstride = (q->n + 15) & ~15;
    A.bias = q->use_bias;
    A.seed = seed;
    A.epoch = epoch;
    A.epoch_dev = S->epoch_dev;
    A.beta = nullptr;
    A.theta_in = nullptr;
    A.theta_out = nullptr;
    A.lp_out = nullptr;
    A.slot = nullptr;
    A.ntemps = 1;
    A.groups = S->n_chains;
    A.rec_index = 0;
    A.sw0 = 0;
    A.acc_add = 0;
    A.p64 = q->p64.as<c128>();
    A.W = q->W.as<cplx<R>>();
    A.tau = q->tau.as<cplx<R>>();
    A.Lk = q->Lk.as<c128>();
    A.chains = S->chains.as<int8_t>();
    A.out_sigma = S->sigma.as<int8_t>();
    A.out_theta = S->theta.as<cplx<R>>();
    A.acc = S->acc.as<unsigned long long>();
    A.moves = S->ham ? S->ham->moves.as<HamMove>() : nullptr;
    A.n_moves = S->ham ? S->ham->n_moves : 0;
    cudaStream_t st = q->ctx->stream;
    if (S->ntemps <= 1) {
        launch_sweeps<R>(S, A, st);
        return;
    }
    // parallel tempering: one launch per sweep, then mixChains per group
    const int nt = S->ntemps, groups = S->n_chains / nt;
    S->pt_theta.ensure(size_t(S->n_chains) * q->m * sizeof(cplx<R>));
    S->pt_lp.ensure(size_t(S->n_chains) * sizeof(double));
    if (reinit || !S->pt_ready) {
        pt_reset_kernel<<<cdiv_u(S->n_chains, 128), 128, 0, st>>>(S->n_chains, nt, S->pt_slot.as<int>(),
                                                                 S->pt_beta.as<double>());
        YQ_LAUNCH_CHECK();
        S->pt_ready = true;
    }
    A.beta = S->pt_beta.as<double>();
    A.slot = S->pt_slot.as<int>();
    A.theta_out = S->pt_theta.as<cplx<R>>();
    A.lp_out = S->pt_lp.as<double>();
    A.ntemps = nt;
    A.groups = groups;
    A.n_total = 1;
    for (int sw = 0; sw < n_discard + n_sweeps; ++sw) {
        A.sw0 = sw;
        A.reinit = sw == 0 ? reinit : 0;
        A.theta_in = sw == 0 ? nullptr : S->pt_theta.as<cplx<R>>();
        A.n_discard = sw < n_discard ? 1 : 0;
        A.rec_index = sw - n_discard;
        A.acc_add = sw > 0;
        launch_sweeps<R>(S, A, st);
        pt_mix_kernel<<<cdiv_u(groups, 128), 128, 0, st>>>(
            groups, nt, S->pt_lp.as<double>(), S->pt_slot.as<int>(), S->pt_beta.as<double>(), seed, epoch,
            S->epoch_dev, uint32_t(sw), sw >= n_discard ? 1 : 0, sw - n_discard, q->n, S->chains.as<int8_t>(),
            int(q->m * sizeof(cplx<R>)), S->pt_theta.as<uint8_t>(), S->sigma.as<int8_t>(), S->theta.as<uint8_t>());
        YQ_LAUNCH_CHECK();
    }
}

void sampler_run(yq_sampler_s* S, int n_sweeps, int n_discard, uint64_t seed, uint32_t epoch, int reinit) {
    yq_rbm_s* q = S->q;
    YQ_CHECK_ARG(n_sweeps > 0 && n_discard >= 0, "sample: n_sweeps must be > 0 and n_discard >= 0");
    YQ_CHECK_ARG(reinit || S->have_chains, "sample: reinit = 0 needs chains (set_chains or an earlier sample)");
    if (S->move == YQ_MOVE_HAMILTONIAN && !S->ham)
        throw Error(YQ_E_STATE, "sample: a HamiltonianSweeper sampler needs yq_sampler_set_hamiltonian");
    const long long L = S->sweep_len > 0 ? S->sweep_len : q->n;
    YQ_CHECK_ARG((long long)(n_sweeps + n_discard) * L < (1LL << 32) - 1, "sample: too many proposals per call");
    rbm_prepare(q);
    const size_t ns = size_t(S->n_chains / std::max(1, S->ntemps)) * n_sweeps;
    S->sigma.ensure(ns * q->n);
    S->theta.ensure(ns * q->m * q->csize());
    if (q->dtype == YQ_C64)
        run_t<float>(S, n_sweeps, n_discard, seed, epoch, reinit);
    else
        run_t<double>(S, n_sweeps, n_discard, seed, epoch, reinit);
    S->have_chains = true;
    S->ns = int(ns);
    S->proposals = uint64_t(n_sweeps + n_discard) * uint64_t(L);
}

}  // namespace yq
