// Exact summation over a basis and exact sampling from |psi|^2 on the device.
//
//   exact_summation  GroundState/SRMatExact.hpp:97-132 (constructExact, eloc,
//                    energyGrad, corrMat): with w_s = |psi_s|^2 / Z over the basis,
//                      E = sum_s w_s E_loc(s),  Var = sum_s w_s |E_loc(s)|^2 - E^2,
//                      o = sum_s w_s O_s,       Z_s = sqrt(w_s) (O_s - o),
//                      F = sum_s conj(Z_s) sqrt(w_s) E_loc(s),   S = Z^H Z,
//                    which equal the reference's (diag psi O)^H k - E conj(o) and
//                    O^H diag|psi|^2 O - conj(o) o^T for normalised psi, k = H psi.
//   sample_exact     Samplers/ExactSampler.hpp:49-79: inclusive CDF of |psi|^2 over
//                    the basis, r = u * total, lower_bound, with u drawn from the
//                    exact-sampler Philox stream (counter (i, epoch, 0, TAG_EXACT)).
//
// The basis is either every configuration of n spins (Basis/BasisFull.hpp) or the
// configurations with nup spins down in increasing order (Basis/BasisJz.hpp),
// unranked on the device by the combinatorial number system.  Everything is FP64
// apart from E_loc of a complex64 machine, which runs the machine's own product
// form.  Weights are formed as exp(2 Re log psi - max) so no |psi|^2 overflows.
#include <algorithm>
#include <cmath>
#include <vector>

#include "basis.cuh"
#include "chol.hpp"
#include "gemm64.cuh"
#include "internal.hpp"

namespace yq {

namespace {

// ---------------------------------------------------------------------------
// Deterministic FP64 reductions (fixed grid, fixed order).
constexpr int RED_BLOCKS = 256;

__device__ __forceinline__ double block_sum(double v, double* red) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    __syncthreads();
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = v;
    __syncthreads();
    double t = 0.;
    if (threadIdx.x == 0)
        for (int w = 0; w < int(blockDim.x >> 5); ++w) t += red[w];
    return t;  // valid in thread 0
}
__device__ __forceinline__ double block_max(double v, double* red) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v = fmax(v, __shfl_xor_sync(0xffffffffu, v, o));
    __syncthreads();
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = v;
    __syncthreads();
    double t = -INFINITY;
    if (threadIdx.x == 0)
        for (int w = 0; w < int(blockDim.x >> 5); ++w) t = fmax(t, red[w]);
    return t;
}

// part[b] = max over this block's share of 2 Re log psi
__global__ void lmax_partial_kernel(uint64_t dim, const c128* __restrict__ logpsi, double* __restrict__ part) {
    __shared__ double red[32];
    double m = -INFINITY;
    for (uint64_t s = uint64_t(blockIdx.x) * blockDim.x + threadIdx.x; s < dim; s += uint64_t(gridDim.x) * blockDim.x)
        m = fmax(m, 2.0 * logpsi[s].re);
    m = block_max(m, red);
    if (threadIdx.x == 0) part[blockIdx.x] = m;
}
// p_s = exp(2 Re log psi_s - max); part[b] = block share of sum p
__global__ void prob_kernel(uint64_t dim, const c128* __restrict__ logpsi, const double* __restrict__ pmax, int nparts,
                            double* __restrict__ p, double* __restrict__ part) {
    __shared__ double red[32];
    double mx = -INFINITY;
    for (int b = 0; b < nparts; ++b) mx = fmax(mx, pmax[b]);
    double acc = 0.;
    for (uint64_t s = uint64_t(blockIdx.x) * blockDim.x + threadIdx.x; s < dim; s += uint64_t(gridDim.x) * blockDim.x) {
        const double v = exp(2.0 * logpsi[s].re - mx);
        p[s] = v;
        acc += v;
    }
    acc = block_sum(acc, red);
    if (threadIdx.x == 0) part[blockIdx.x] = acc;
}
// w_s = p_s / Z; per-block partial sums of w E_loc (re, im) and w |E_loc|^2
__global__ void weight_stats_kernel(uint64_t dim, const double* __restrict__ zpart, int nparts, double* __restrict__ w,
                                    const c128* __restrict__ eloc, double* __restrict__ part) {
    __shared__ double red[32];
    double z = 0.;
    for (int b = 0; b < nparts; ++b) z += zpart[b];
    const double iz = 1.0 / z;
    double er = 0., ei = 0., e2 = 0.;
    for (uint64_t s = uint64_t(blockIdx.x) * blockDim.x + threadIdx.x; s < dim; s += uint64_t(gridDim.x) * blockDim.x) {
        const double ws = w[s] * iz;
        w[s] = ws;
        const c128 e = eloc[s];
        er += ws * e.re;
        ei += ws * e.im;
        e2 += ws * norm2(e);
    }
    er = block_sum(er, red);
    ei = block_sum(ei, red);
    e2 = block_sum(e2, red);
    if (threadIdx.x == 0) {
        part[3 * blockIdx.x] = er;
        part[3 * blockIdx.x + 1] = ei;
        part[3 * blockIdx.x + 2] = e2;
    }
}
__global__ void stats_final_kernel(const double* __restrict__ part, int nparts, double* __restrict__ out) {
    if (threadIdx.x != 0) return;
    double er = 0., ei = 0., e2 = 0.;
    for (int b = 0; b < nparts; ++b) {
        er += part[3 * b];
        ei += part[3 * b + 1];
        e2 += part[3 * b + 2];
    }
    out[0] = er;
    out[1] = e2 - er * er;
    out[2] = er;
    out[3] = ei;
}

// ---------------------------------------------------------------------------
// O rows (RBM.hpp:390-406): [sigma_i tanh(theta_j) (index i m + j) | sigma_i | tanh(theta_j)], FP64.
__global__ void tanh_kernel(size_t cnt, const c128* __restrict__ theta, c128* __restrict__ t) {
    for (size_t q = size_t(blockIdx.x) * blockDim.x + threadIdx.x; q < cnt; q += size_t(gridDim.x) * blockDim.x)
        t[q] = ctanh(theta[q]);
}
__global__ void o_rows_kernel(uint64_t dim, int n, int m, bool bias, size_t P, const int8_t* __restrict__ sigma,
                              const c128* __restrict__ t, c128* __restrict__ O) {
    for (uint64_t s = blockIdx.y; s < dim; s += gridDim.y) {
        const int8_t* sg = sigma + s * n;
        const c128* ts = t + s * m;
        c128* row = O + s * P;
        for (size_t p = size_t(blockIdx.x) * blockDim.x + threadIdx.x; p < P; p += size_t(gridDim.x) * blockDim.x) {
            c128 v;
            if (p < size_t(n) * m) {
                const int i = int(p / m), j = int(p % m);
                v = double(sg[i]) * ts[j];
            } else if (bias && p < size_t(n) * m + n) {
                v = mk(double(sg[p - size_t(n) * m]), 0.0);
            } else {
                v = ts[p - size_t(n) * m - n];
            }
            row[p] = v;
        }
    }
}

// part[split][p] = sum over a chunk of rows of y_s * (conj ? conj(O_sp) : O_sp)
template <bool CONJ>
__global__ void colsum_partial_kernel(size_t P, uint64_t dim, uint64_t chunk, const c128* __restrict__ O,
                                      const c128* __restrict__ y, c128* __restrict__ part) {
    const size_t p = size_t(blockIdx.x) * blockDim.x + threadIdx.x;
    if (p >= P) return;
    const uint64_t s0 = blockIdx.y * chunk, s1 = min(dim, s0 + chunk);
    double ar = 0., ai = 0.;
    for (uint64_t s = s0; s < s1; ++s) {
        c128 o = O[s * P + p];
        if (CONJ) o = conj(o);
        const c128 v = o * y[s];
        ar += v.re;
        ai += v.im;
    }
    part[size_t(blockIdx.y) * P + p] = mk(ar, ai);
}
__global__ void colsum_final_kernel(size_t P, int nsplit, const c128* __restrict__ part, c128* __restrict__ out) {
    for (size_t p = size_t(blockIdx.x) * blockDim.x + threadIdx.x; p < P; p += size_t(gridDim.x) * blockDim.x) {
        c128 acc = mk(0., 0.);
        for (int k = 0; k < nsplit; ++k) acc = acc + part[size_t(k) * P + p];
        out[p] = acc;
    }
}
// y_s = w_s (as complex), or sqrt(w_s) E_loc(s)
__global__ void weight_vec_kernel(uint64_t dim, const double* __restrict__ w, const c128* __restrict__ eloc,
                                  c128* __restrict__ y) {
    for (uint64_t s = uint64_t(blockIdx.x) * blockDim.x + threadIdx.x; s < dim; s += uint64_t(gridDim.x) * blockDim.x)
        y[s] = eloc ? sqrt(w[s]) * eloc[s] : mk(w[s], 0.0);
}
// Z_s = sqrt(w_s) (O_s - o)
__global__ void centre_scale_kernel(uint64_t dim, size_t P, const double* __restrict__ w, const c128* __restrict__ o,
                                    c128* __restrict__ O) {
    for (uint64_t s = blockIdx.y; s < dim; s += gridDim.y) {
        const double sw = sqrt(w[s]);
        for (size_t p = size_t(blockIdx.x) * blockDim.x + threadIdx.x; p < P; p += size_t(gridDim.x) * blockDim.x)
            O[s * P + p] = sw * (O[s * P + p] - o[p]);
    }
}

// sum_s y_s op(O_sp) into out (P entries), split over row chunks.
template <bool CONJ>
void colsum(const c128* O, uint64_t dim, size_t P, const c128* y, c128* part, int nsplit, c128* out, cudaStream_t st) {
    const uint64_t chunk = (dim + nsplit - 1) / nsplit;
    dim3 g(cdiv_u(P, 256), unsigned(nsplit));
    colsum_partial_kernel<CONJ><<<g, 256, 0, st>>>(P, dim, chunk, O, y, part);
    YQ_LAUNCH_CHECK();
    colsum_final_kernel<<<cdiv_u(P, 256), 256, 0, st>>>(P, nsplit, part, out);
    YQ_LAUNCH_CHECK();
}

// ---------------------------------------------------------------------------
// Inclusive FP64 prefix sum: per-block scans of SCAN_PER elements, a scan of the
// block totals, then the block offsets added.
constexpr int SCAN_THREADS = 1024, SCAN_ITEMS = 8, SCAN_PER = SCAN_THREADS * SCAN_ITEMS;

__device__ double block_inclusive_scan(double v, double* sh) {
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const double t = __shfl_up_sync(0xffffffffu, v, o);
        if (lane >= o) v += t;
    }
    if (lane == 31) sh[warp] = v;
    __syncthreads();
    if (warp == 0) {
        double x = lane < int(blockDim.x >> 5) ? sh[lane] : 0.;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const double t = __shfl_up_sync(0xffffffffu, x, o);
            if (lane >= o) x += t;
        }
        sh[lane] = x;
    }
    __syncthreads();
    if (warp > 0) v += sh[warp - 1];
    __syncthreads();
    return v;
}
__global__ void __launch_bounds__(SCAN_THREADS) scan_block_kernel(uint64_t dim, const double* __restrict__ in,
                                                                  double* __restrict__ out,
                                                                  double* __restrict__ totals) {
    __shared__ double sh[32];
    const uint64_t base = uint64_t(blockIdx.x) * SCAN_PER + uint64_t(threadIdx.x) * SCAN_ITEMS;
    double v[SCAN_ITEMS];
    double run = 0.;
#pragma unroll
    for (int k = 0; k < SCAN_ITEMS; ++k) {
        run += base + k < dim ? in[base + k] : 0.;
        v[k] = run;
    }
    const double incl = block_inclusive_scan(run, sh);
    const double excl = incl - run;
#pragma unroll
    for (int k = 0; k < SCAN_ITEMS; ++k)
        if (base + k < dim) out[base + k] = excl + v[k];
    if (threadIdx.x == blockDim.x - 1) totals[blockIdx.x] = incl;
}
__global__ void __launch_bounds__(SCAN_THREADS) scan_totals_kernel(int nb, double* __restrict__ totals) {
    __shared__ double sh[32];
    double carry = 0.;
    for (int b0 = 0; b0 < nb; b0 += SCAN_THREADS) {
        const int b = b0 + int(threadIdx.x);
        const double x = b < nb ? totals[b] : 0.;
        const double incl = block_inclusive_scan(x, sh);
        if (b < nb) totals[b] = carry + incl - x;  // exclusive offsets
        __shared__ double last;
        if (threadIdx.x == blockDim.x - 1) last = incl;
        __syncthreads();
        carry += last;
        __syncthreads();
    }
}
__global__ void scan_add_kernel(uint64_t dim, const double* __restrict__ offsets, double* __restrict__ out) {
    for (uint64_t k = uint64_t(blockIdx.x) * blockDim.x + threadIdx.x; k < dim; k += uint64_t(gridDim.x) * blockDim.x)
        out[k] += offsets[k / SCAN_PER];
}

// Sample i: u from the exact-sampler stream, r = u * total, first cdf >= r.
__global__ void exact_draw_kernel(int ns, uint64_t dim, int n, const double* __restrict__ cdf, uint64_t seed,
                                  uint32_t epoch, const int8_t* __restrict__ bsigma, int8_t* __restrict__ sigma,
                                  uint64_t* __restrict__ pos) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= ns) return;
    const U4 x = draw(seed, uint32_t(i), epoch, 0u, TAG_EXACT);
    const double r = draw_u53(x.z, x.w) * cdf[dim - 1];
    uint64_t lo = 0, hi = dim;  // lower_bound
    while (lo < hi) {
        const uint64_t mid = (lo + hi) >> 1;
        if (cdf[mid] < r) lo = mid + 1;
        else hi = mid;
    }
    if (lo >= dim) lo = dim - 1;  // the reference pads the last entry by 1e-8
    if (pos) pos[i] = lo;
    for (int k = 0; k < n; ++k) sigma[size_t(i) * n + k] = bsigma[lo * n + k];
}

// theta of `rows` configurations in launches of at most 32768 rows (grid.y limit).
void theta_rows(yq_rbm_s* q, uint64_t rows, const int8_t* sigma, void* theta, bool c128_out) {
    const size_t es = c128_out || q->dtype == YQ_C128 ? sizeof(c128) : sizeof(c64);
    for (uint64_t r0 = 0; r0 < rows; r0 += 32768) {
        const int nr = int(std::min<uint64_t>(32768, rows - r0));
        rbm_theta(q, nr, sigma + r0 * q->n, static_cast<char*>(theta) + r0 * q->m * es, c128_out);
    }
}

// Basis configurations, theta (FP64), log psi and weights p_s = exp(2 Re log psi - max).
struct BasisState {
    Basis b;
    DevBuf binom, index, sigma, theta, logpsi, part;
};
void basis_state(yq_rbm_s* q, int kind, int nup, BasisState& bs) {
    cudaStream_t st = q->ctx->stream;
    bs.b = make_basis(q->n, kind, nup);
    const uint64_t dim = bs.b.dim;
    bs.index.ensure(dim * sizeof(uint64_t));
    bs.sigma.ensure(dim * q->n);
    const uint64_t* d_binom = nullptr;
    if (kind == YQ_BASIS_JZ) {
        bs.binom.ensure(bs.b.binom.size() * sizeof(uint64_t));
        YQ_CUDA(cudaMemcpyAsync(bs.binom.p, bs.b.binom.data(), bs.b.binom.size() * sizeof(uint64_t),
                                cudaMemcpyHostToDevice, st));
        d_binom = bs.binom.as<uint64_t>();
    }
    basis_kernel<<<std::max(1u, std::min(148u * 16, cdiv_u(dim, 256))), 256, 0, st>>>(
        dim, q->n, kind, nup, d_binom, bs.index.as<uint64_t>(), bs.sigma.as<int8_t>());
    YQ_LAUNCH_CHECK();
    bs.theta.ensure(dim * q->m * sizeof(c128));
    theta_rows(q, dim, bs.sigma.as<int8_t>(), bs.theta.p, true);
    bs.logpsi.ensure(dim * sizeof(c128));
    rbm_log_psi(q, int(dim), bs.sigma.as<int8_t>(), bs.logpsi.as<c128>());
}

}  // namespace

void exact_summation(yq_rbm_s* q, yq_ham_s* H, int kind, int nup, double* stats, c128* d_oloc, c128* d_grad,
                     c128* d_S, size_t ldS, double shift) {
    YQ_CHECK_ARG(H->n == q->n, "exact: Hamiltonian and RBM sizes differ");
    YQ_CHECK_ARG(kind != YQ_BASIS_JZ || H->conserves_sz,
                 "exact: the Jz basis needs a Hamiltonian that conserves Sz (XXZ, XXX, J1J2)");
    cudaStream_t st = q->ctx->stream;
    rbm_prepare(q);
    BasisState bs;
    basis_state(q, kind, nup, bs);
    const uint64_t dim = bs.b.dim;
    const size_t P = q->P;
    // E_loc with the machine's own compute type
    DevBuf eloc, thc;
    eloc.ensure(dim * sizeof(c128));
    const void* th = bs.theta.p;
    if (q->dtype == YQ_C64) {
        thc.ensure(dim * q->m * sizeof(c64));
        theta_rows(q, dim, bs.sigma.as<int8_t>(), thc.p, false);
        th = thc.p;
    }
    ham_eloc(H, q, int(dim), bs.sigma.as<int8_t>(), th, eloc.as<c128>());
    // weights and energy statistics
    DevBuf w, part, out;
    w.ensure(dim * sizeof(double));
    part.ensure(4 * RED_BLOCKS * sizeof(double));
    out.ensure(8 * sizeof(double));
    double* pmax = part.as<double>();
    double* pz = pmax + RED_BLOCKS;
    double* pst = pz + RED_BLOCKS;
    lmax_partial_kernel<<<RED_BLOCKS, 256, 0, st>>>(dim, bs.logpsi.as<c128>(), pmax);
    prob_kernel<<<RED_BLOCKS, 256, 0, st>>>(dim, bs.logpsi.as<c128>(), pmax, RED_BLOCKS, w.as<double>(), pz);
    weight_stats_kernel<<<RED_BLOCKS, 256, 0, st>>>(dim, pz, RED_BLOCKS, w.as<double>(), eloc.as<c128>(), pst);
    stats_final_kernel<<<1, 32, 0, st>>>(pst, RED_BLOCKS, out.as<double>());
    YQ_LAUNCH_CHECK();
    // O rows, weighted mean, centred and scaled rows
    DevBuf t, O, y, cpart;
    t.ensure(dim * q->m * sizeof(c128));
    O.ensure(dim * P * sizeof(c128));
    y.ensure(dim * sizeof(c128));
    const uint64_t want = uint64_t(8 * 148) / std::max(1u, cdiv_u(P, 256));
    const int nsplit = int(std::max<uint64_t>(1, std::min<uint64_t>(std::min<uint64_t>(64, dim), want)));
    cpart.ensure(size_t(nsplit) * P * sizeof(c128));
    const size_t tcnt = dim * q->m;
    tanh_kernel<<<std::max(1u, std::min(148u * 16, cdiv_u(tcnt, 256))), 256, 0, st>>>(tcnt, bs.theta.as<c128>(),
                                                                                    t.as<c128>());
    dim3 og(std::max(1u, std::min(16u, cdiv_u(P, 256))), unsigned(std::min<uint64_t>(dim, 65535)));
    o_rows_kernel<<<og, 256, 0, st>>>(dim, q->n, q->m, q->use_bias, P, bs.sigma.as<int8_t>(), t.as<c128>(),
                                      O.as<c128>());
    YQ_LAUNCH_CHECK();
    weight_vec_kernel<<<std::max(1u, std::min(148u * 8, cdiv_u(dim, 256))), 256, 0, st>>>(dim, w.as<double>(),
                                                                                        nullptr, y.as<c128>());
    YQ_LAUNCH_CHECK();
    colsum<false>(O.as<c128>(), dim, P, y.as<c128>(), cpart.as<c128>(), nsplit, d_oloc, st);
    centre_scale_kernel<<<og, 256, 0, st>>>(dim, P, w.as<double>(), d_oloc, O.as<c128>());
    weight_vec_kernel<<<std::max(1u, std::min(148u * 8, cdiv_u(dim, 256))), 256, 0, st>>>(dim, w.as<double>(),
                                                                                        eloc.as<c128>(), y.as<c128>());
    YQ_LAUNCH_CHECK();
    colsum<true>(O.as<c128>(), dim, P, y.as<c128>(), cpart.as<c128>(), nsplit, d_grad, st);
    if (d_S) gram_fp64<double>(O.as<c128>(), P, 1, int(P), int(dim), d_S, ldS ? ldS : P, 1.0, 0, shift, st);
    double h[4];
    YQ_CUDA(cudaMemcpyAsync(h, out.p, sizeof(h), cudaMemcpyDeviceToHost, st));
    YQ_CUDA(cudaStreamSynchronize(st));
    stats[0] = h[0];
    stats[1] = h[1];
}

namespace {
// unit diagonal and zeros outside the leading dim x dim block of the padded matrix
__global__ void exact_pad_kernel(c128* G, int dim, int dim_pad) {
    const size_t total = size_t(dim_pad) * dim_pad;
    for (size_t q = size_t(blockIdx.x) * blockDim.x + threadIdx.x; q < total; q += size_t(gridDim.x) * blockDim.x) {
        const int r = int(q / dim_pad), c = int(q % dim_pad);
        if (r >= dim || c >= dim) G[q] = mk(r == c ? 1.0 : 0.0, 0.0);
    }
}

// params -= lr v; |v|^2 accumulated by one block (P is at most a few tens of thousands)
__global__ void exact_update_kernel(size_t P, double lr, const c128* __restrict__ v, c128* __restrict__ p64,
                                    double* __restrict__ out) {
    __shared__ double red[32];
    double acc = 0.;
    for (size_t p = threadIdx.x; p < P; p += blockDim.x) {
        const c128 x = v[p];
        acc += x.re * x.re + x.im * x.im;
        p64[p] = p64[p] - lr * x;
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, o);
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = acc;
    __syncthreads();
    if (threadIdx.x == 0) {
        double r = 0.;
        for (int w = 0; w < int(blockDim.x >> 5); ++w) r += red[w];
        out[0] = sqrt(r);
    }
}
}  // namespace

// One epoch of RunRBMExact::run (Runners/RunRBMExact.hpp:46-80): constructExact,
// corrMat + lambda I by LLT (tile Cholesky on the device), v = LLT.solve(energyGrad),
// params -= lr v.  out = {E, Var, |v|}.
void exact_iteration(yq_rbm_s* q, yq_ham_s* H, int kind, int nup, double shift, double lr, double* out) {
    yq_ctx_s* ctx = q->ctx;
    cudaStream_t st = ctx->stream;
    const size_t P = q->P;
    const int dim_pad = int((P + CHOL_NB - 1) / CHOL_NB) * CHOL_NB;
    const size_t dp = size_t(dim_pad);
    DevBuf G, Li, LiH, oloc, grad, b, x, work, nv;
    G.ensure(dp * dp * sizeof(c128));
    Li.ensure(dp * CHOL_NB * sizeof(c128));
    LiH.ensure(dp * CHOL_NB * sizeof(c128));
    oloc.ensure(P * sizeof(c128));
    grad.ensure(P * sizeof(c128));
    b.ensure(dp * sizeof(c128));
    x.ensure(dp * sizeof(c128));
    work.ensure(chol_tile_scratch_bytes(dim_pad));
    nv.ensure(sizeof(double));
    if (dim_pad != int(P)) {
        exact_pad_kernel<<<std::min(148u * 8, cdiv_u(dp * dp, 256)), 256, 0, st>>>(G.as<c128>(), int(P), dim_pad);
        YQ_LAUNCH_CHECK();
    }
    double stats[2];
    exact_summation(q, H, kind, nup, stats, oloc.as<c128>(), grad.as<c128>(), G.as<c128>(), dp, shift);
    chol_factor_tiled(G.as<c128>(), dim_pad, dp, Li.as<c128>(), LiH.as<c128>(), ctx->status.as<int>(), work.p,
                      ctx->sm_count, st);
    YQ_CUDA(cudaMemsetAsync(b.p, 0, dp * sizeof(c128), st));
    YQ_CUDA(cudaMemcpyAsync(b.p, grad.p, P * sizeof(c128), cudaMemcpyDeviceToDevice, st));
    chol_solve_tiled(G.as<c128>(), dim_pad, dp, Li.as<c128>(), LiH.as<c128>(), b.as<c128>(), x.as<c128>(),
                     ctx->status.as<int>(), work.p, ctx->sm_count, st);
    exact_update_kernel<<<1, 1024, 0, st>>>(P, lr, x.as<c128>(), q->p64.as<c128>(), nv.as<double>());
    YQ_LAUNCH_CHECK();
    q->version++;
    double h = 0.;
    YQ_CUDA(cudaMemcpyAsync(&h, nv.p, sizeof(double), cudaMemcpyDeviceToHost, st));
    YQ_CUDA(cudaStreamSynchronize(st));
    out[0] = stats[0];
    out[1] = stats[1];
    out[2] = h;
}

void sampler_sample_exact(yq_sampler_s* S, int ns, uint64_t seed, uint32_t epoch, uint64_t* d_pos) {
    yq_rbm_s* q = S->q;
    cudaStream_t st = q->ctx->stream;
    YQ_CHECK_ARG(ns >= 1, "sample_exact: the number of samples must be >= 1");
    rbm_prepare(q);
    BasisState bs;
    basis_state(q, S->nup >= 0 ? YQ_BASIS_JZ : YQ_BASIS_FULL, S->nup, bs);
    const uint64_t dim = bs.b.dim;
    DevBuf p, cdf, part, totals;
    p.ensure(dim * sizeof(double));
    cdf.ensure(dim * sizeof(double));
    part.ensure(2 * RED_BLOCKS * sizeof(double));
    lmax_partial_kernel<<<RED_BLOCKS, 256, 0, st>>>(dim, bs.logpsi.as<c128>(), part.as<double>());
    prob_kernel<<<RED_BLOCKS, 256, 0, st>>>(dim, bs.logpsi.as<c128>(), part.as<double>(), RED_BLOCKS, p.as<double>(),
                                            part.as<double>() + RED_BLOCKS);
    YQ_LAUNCH_CHECK();
    const int nb = int((dim + SCAN_PER - 1) / SCAN_PER);
    totals.ensure(size_t(nb) * sizeof(double));
    scan_block_kernel<<<nb, SCAN_THREADS, 0, st>>>(dim, p.as<double>(), cdf.as<double>(), totals.as<double>());
    scan_totals_kernel<<<1, SCAN_THREADS, 0, st>>>(nb, totals.as<double>());
    scan_add_kernel<<<std::max(1u, std::min(148u * 16, cdiv_u(dim, 256))), 256, 0, st>>>(dim, totals.as<double>(),
                                                                                       cdf.as<double>());
    YQ_LAUNCH_CHECK();
    S->sigma.ensure(size_t(ns) * q->n);
    S->theta.ensure(size_t(ns) * q->m * q->csize());
    exact_draw_kernel<<<cdiv_u(ns, 128), 128, 0, st>>>(ns, dim, q->n, cdf.as<double>(), seed, epoch,
                                                       bs.sigma.as<int8_t>(), S->sigma.as<int8_t>(), d_pos);
    YQ_LAUNCH_CHECK();
    theta_rows(q, uint64_t(ns), S->sigma.as<int8_t>(), S->theta.p, q->dtype == YQ_C128);
    S->ns = ns;
    S->proposals = 0;
    YQ_CUDA(cudaStreamSynchronize(st));  // the basis buffers are released on return
}

}  // namespace yq
