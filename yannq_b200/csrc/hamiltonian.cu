// Hamiltonians on the device: off-diagonal flip enumeration and the local energy
// E_loc(sigma) = sum_terms coeff * psi(sigma')/psi(sigma) + diagonal
// (Hamiltonians/TFIsing.hpp:28-39, Hamiltonians/XXZ.hpp:37-49, and the 2D TFI
// model built on the same concept), reusing the sample's theta cache.
//
// TFI, XXZ and TFI2D are evaluated from closed-form site rules.  XXX, J1J2,
// XYZNNN and KitaevHex are term tables (HamTerm) built on the host in the
// reference's evaluation order (XXX.hpp:11-22, J1J2.hpp:35-56,
// XYZNNN.hpp:33-53, KitaevHex.hpp:119-146); the kernels walk the table.
#include <algorithm>
#include <vector>

#include "ap.hpp"
#include "basis.cuh"
#include "internal.hpp"
#include "ratio.cuh"

namespace yq {

struct HamDesc {
    int kind, n, lx, ly;
    double J, h, sign;
    const HamTerm* terms;  // term-table kinds, else null
    int nterms;
};

// Diagonal addend and off-diagonal request of term T in state s: request flips
// of a (and b >= 0) with coefficient c, or none when a < 0.
__device__ __forceinline__ void table_term(const HamTerm& T, const int8_t* s, double& d, int& a, int& b,
                                           double& c) {
    const int zz = T.b >= 0 ? s[T.a] * s[T.b] : 1;
    d = T.has_diag ? (zz > 0 ? T.dp : T.dm) : 0.0;
    if (T.nflip == 0) {
        a = -1;
        b = -1;
        c = 0.0;
        return;
    }
    a = T.a;
    b = T.nflip == 2 ? T.b : -1;
    c = zz > 0 ? T.cp : T.cm;
}

__device__ __forceinline__ int right_of(const HamDesc& H, int i) {
    if (H.kind == YQ_HAM_TFI2D) {
        int x = i % H.lx, y = i / H.lx;
        return (x + 1) % H.lx + H.lx * y;
    }
    return (i + 1) % H.n;
}
__device__ __forceinline__ int down_of(const HamDesc& H, int i) {
    int x = i % H.lx, y = i / H.lx;
    return x + H.lx * ((y + 1) % H.ly);
}

// Contribution of site i to the diagonal, in the reference's evaluation order.
__device__ __forceinline__ double diag_term(const HamDesc& H, const int8_t* s, int i) {
    if (H.kind == YQ_HAM_TFI) return H.J * s[i] * s[(i + 1) % H.n];
    if (H.kind == YQ_HAM_XXZ) {
        int zz = s[i] * s[(i + 1) % H.n];
        return H.J * H.h * zz;
    }
    double d = H.J * s[i] * s[right_of(H, i)];
    return d + H.J * s[i] * s[down_of(H, i)];
}
// The i-th off-diagonal request: flip site a (and b >= 0) with coefficient c.
__device__ __forceinline__ void offdiag_term(const HamDesc& H, const int8_t* s, int i, int& a, int& b, double& c) {
    a = i;
    if (H.kind == YQ_HAM_XXZ) {
        b = (i + 1) % H.n;
        int zz = s[i] * s[b];
        c = H.sign * H.J * (1 - zz);
    } else {
        b = -1;
        c = H.h;
    }
}

__global__ void enumerate_kernel(HamDesc H, int ns, const int8_t* __restrict__ sigma, int* __restrict__ oa,
                                 int* __restrict__ ob, double* __restrict__ oc, double* __restrict__ od) {
    int smp = blockIdx.x * blockDim.x + threadIdx.x;
    if (smp >= ns) return;
    const int8_t* s = sigma + size_t(smp) * H.n;
    double diag = 0.;
    for (int i = 0; i < H.n; ++i) {
        if (H.kind == YQ_HAM_TFI2D) {
            diag += H.J * s[i] * s[right_of(H, i)];
            diag += H.J * s[i] * s[down_of(H, i)];
        } else {
            diag += diag_term(H, s, i);
        }
        int a, b;
        double c;
        offdiag_term(H, s, i, a, b, c);
        oa[size_t(smp) * H.n + i] = a;
        ob[size_t(smp) * H.n + i] = b;
        oc[size_t(smp) * H.n + i] = c;
    }
    od[smp] = diag;
}

// Term-table form: one thread per sample walks the table in order, so the
// diagonal is summed in the reference's order and the requests come out in it.
__global__ void enumerate_table_kernel(HamDesc H, int n_off, int ns, const int8_t* __restrict__ sigma,
                                       int* __restrict__ oa, int* __restrict__ ob, double* __restrict__ oc,
                                       double* __restrict__ od) {
    int smp = blockIdx.x * blockDim.x + threadIdx.x;
    if (smp >= ns) return;
    const int8_t* s = sigma + size_t(smp) * H.n;
    double diag = 0.;
    int k = 0;
    for (int t = 0; t < H.nterms; ++t) {
        double d, c;
        int a, b;
        table_term(H.terms[t], s, d, a, b, c);
        if (H.terms[t].has_diag) diag += d;
        if (a < 0) continue;
        const size_t o = size_t(smp) * n_off + k++;
        oa[o] = a;
        ob[o] = b;
        oc[o] = c;
    }
    od[smp] = diag;
}

static HamDesc desc(const yq_ham_s* H) {
    return HamDesc{H->kind, H->n, H->lx, H->ly, H->J, H->h, H->sign, H->terms.as<HamTerm>(), H->nterms};
}

int ham_num_offdiag(const yq_ham_s* H) { return H->nterms > 0 ? H->n_off : H->n; }

void ham_enumerate(yq_ham_s* H, int ns, const int8_t* d_sigma, int* d_a, int* d_b, double* d_c, double* d_diag) {
    if (ns <= 0) return;
    if (H->nterms > 0)
        enumerate_table_kernel<<<cdiv_u(ns, 128), 128, 0, H->ctx->stream>>>(desc(H), H->n_off, ns, d_sigma, d_a, d_b,
                                                                            d_c, d_diag);
    else
        enumerate_kernel<<<cdiv_u(ns, 128), 128, 0, H->ctx->stream>>>(desc(H), ns, d_sigma, d_a, d_b, d_c, d_diag);
    YQ_LAUNCH_CHECK();
}

// ---------------------------------------------------------------------------
// H psi over a basis (NGDExact's sparse product, matrix-free): one thread per
// configuration walks the state form and gathers psi at the flipped
// configurations by their basis rank.
__global__ void apply_basis_kernel(HamDesc H, uint64_t dim, int kind, int nup, const uint64_t* __restrict__ binom,
                                   const uint64_t* __restrict__ index, const int8_t* __restrict__ sigma,
                                   const c128* __restrict__ psi, c128* __restrict__ out) {
    for (uint64_t k = uint64_t(blockIdx.x) * blockDim.x + threadIdx.x; k < dim; k += uint64_t(gridDim.x) * blockDim.x) {
        const int8_t* s = sigma + k * H.n;
        const uint64_t v = index[k];
        double diag = 0.;
        c128 acc = mk(0., 0.);
        const bool table = H.nterms > 0;
        const int nterm = table ? H.nterms : H.n;
        for (int t = 0; t < nterm; ++t) {
            int a, b;
            double c;
            if (table) {
                double d;
                table_term(H.terms[t], s, d, a, b, c);
                diag += d;
                if (a < 0) continue;
            } else {
                diag += diag_term(H, s, t);
                offdiag_term(H, s, t, a, b, c);
            }
            if (c == 0.0) continue;
            const uint64_t w = v ^ (uint64_t(1) << a) ^ (b >= 0 ? uint64_t(1) << b : uint64_t(0));
            const long long j = basis_rank(w, H.n, kind, nup, binom);
            if (j < 0) continue;
            const c128 pj = psi[j];
            acc.re += c * pj.re;
            acc.im += c * pj.im;
        }
        const c128 pk = psi[k];
        out[k] = mk(acc.re + diag * pk.re, acc.im + diag * pk.im);
    }
}

void ham_apply_basis(yq_ham_s* H, uint64_t dim, int kind, int nup, const uint64_t* d_binom, const uint64_t* d_index,
                     const int8_t* d_sigma, const c128* d_psi, c128* d_out, cudaStream_t st) {
    if (dim == 0) return;
    apply_basis_kernel<<<std::max(1u, std::min(148u * 16, cdiv_u(dim, 128))), 128, 0, st>>>(
        desc(H), dim, kind, nup, d_binom, d_index, d_sigma, d_psi, d_out);
    YQ_LAUNCH_CHECK();
}

// ---------------------------------------------------------------------------
// Term tables.  The coefficients are formed with the reference's expressions,
// once for zz = s_a s_b = +1 and once for zz = -1.
namespace {

HamTerm pair_term(int a, int b, bool diag, double dp, double dm, bool flip, double cp, double cm) {
    return HamTerm{a, b, flip ? 2 : 0, diag ? 1 : 0, dp, dm, cp, cm};
}

// KitaevHex.hpp:33-103: row r holds ncol/2 black sites r*ncol + c, then ncol/2
// white sites r*ncol + ncol/2 + c; rows and columns are periodic.
std::vector<std::pair<int, int>> honeycomb_links(int ncol, int nrow, int axis) {
    const int half = ncol / 2;
    auto per = [](int v, int p) { return ((v % p) + p) % p; };
    auto site = [&](int r, int c, bool white) { return per(r, nrow) * ncol + per(c, half) + (white ? half : 0); };
    std::vector<std::pair<int, int>> links;
    if (axis == 2) {  // z: white (r, c) -- black (r + 1, c)
        for (int r = 0; r < nrow; ++r)
            for (int c = 0; c < half; ++c) links.emplace_back(site(r, c, true), site(r + 1, c, false));
        return links;
    }
    // x: black (r, c) -- white (r, c - 1) on even rows, white (r, c) on odd rows;
    // y: black (r, c) -- white (r, c) on even rows, white (r, c + 1) on odd rows.
    for (int odd = 0; odd < 2; ++odd)
        for (int r = odd; r < nrow; r += 2)
            for (int c = 0; c < half; ++c)
                links.emplace_back(site(r, c, false), site(r, c + (axis == 0 ? odd - 1 : odd), true));
    return links;
}

}  // namespace

void ham_build_terms(yq_ham_s* H, double jy, double jz) {
    std::vector<HamTerm> T;
    const int n = H->n;
    if (H->kind == YQ_HAM_XXX) {
        // XXX.hpp:15-19: yysign = s_i s_{i+1}; s += yysign + (1 - yysign) ratio(i, i+1)
        auto off = [](double yy) { return 1.0 - yy; };
        for (int i = 0; i < n; ++i) T.push_back(pair_term(i, (i + 1) % n, true, 1.0, -1.0, true, off(1.0), off(-1.0)));
    } else if (H->kind == YQ_HAM_J1J2 || H->kind == YQ_HAM_XYZNNN) {
        // J1J2.hpp:40-53 / XYZNNN.hpp:38-51: yysign = -s_i s_j; s += -J yysign + c(yysign) ratio(i, j),
        // nearest neighbours (j = i + 1) first, then next-nearest (j = i + 2)
        const bool j1j2 = H->kind == YQ_HAM_J1J2;
        const double J1 = j1j2 ? H->J : -1.0, J2 = j1j2 ? H->h : -1.0;
        const double a = H->J, b = H->h, sign = H->sign;
        for (int d = 1; d <= 2; ++d) {
            const double Jd = d == 1 ? J1 : J2;
            auto off = [&](double yy) {
                if (j1j2) return d == 1 ? J1 * sign * (1.0 + yy) : J2 * (1.0 + yy);
                return d == 1 ? J1 * (a + yy * b) : J2 * (b + yy * a);
            };
            // zz = +1 means yysign = -1
            for (int i = 0; i < n; ++i)
                T.push_back(pair_term(i, (i + d) % n, true, -Jd * -1.0, -Jd * 1.0, true, off(-1.0), off(1.0)));
        }
    } else if (H->kind == YQ_HAM_KITAEV_HEX) {
        // KitaevHex.hpp:125-144: h ratio(i) for every site, Jx ratio(x-link),
        // -Jy zz ratio(y-link), Jz zz for every z-link
        const double Jx = H->J, h = H->h;
        for (int i = 0; i < n; ++i) T.push_back(HamTerm{i, -1, 1, 0, 0.0, 0.0, h, h});
        for (auto& e : honeycomb_links(H->lx, H->ly, 0))
            T.push_back(pair_term(e.first, e.second, false, 0.0, 0.0, true, Jx, Jx));
        for (auto& e : honeycomb_links(H->lx, H->ly, 1))
            T.push_back(pair_term(e.first, e.second, false, 0.0, 0.0, true, -jy * 1, -jy * -1));
        for (auto& e : honeycomb_links(H->lx, H->ly, 2))
            T.push_back(pair_term(e.first, e.second, true, jz * 1, jz * -1, false, 0.0, 0.0));
    } else {
        throw Error(YQ_E_ARG, "ham: not a term-table kind");
    }
    int n_off = 0;
    bool cons = true;
    for (const HamTerm& t : T) {
        if (t.nflip == 0) continue;
        ++n_off;
        // one flip changes Sz; two flips of parallel spins (zz = +1) change it by 2
        if (t.cp != 0.0 || (t.nflip == 1 && t.cm != 0.0)) cons = false;
    }
    H->nterms = int(T.size());
    H->n_off = n_off;
    H->conserves_sz = cons;
    H->terms.ensure(T.size() * sizeof(HamTerm));
    YQ_CUDA(cudaMemcpy(H->terms.p, T.data(), T.size() * sizeof(HamTerm), cudaMemcpyHostToDevice));
}

// offDiagonals (Hamiltonians/TFIsing.hpp:41-50: every site, whatever the state;
// the 2D model likewise).  Other kinds: the off-diagonal requests in order,
// present where their coefficient for the state's zz is non-zero.
void ham_build_moves(yq_ham_s* H) {
    std::vector<HamMove> M;
    const int n = H->n;
    auto bits = [](double cp, double cm) { return (cp != 0.0 ? 1 : 0) | (cm != 0.0 ? 2 : 0); };
    if (H->kind == YQ_HAM_TFI || H->kind == YQ_HAM_TFI2D) {
        for (int i = 0; i < n; ++i) M.push_back(HamMove{i, -1, 3, 0});
    } else if (H->kind == YQ_HAM_XXZ) {
        // XXZ.hpp:40-47: sign J (1 - zz) ratio(i, i+1)
        for (int i = 0; i < n; ++i)
            M.push_back(HamMove{i, (i + 1) % n, bits(H->sign * H->J * (1 - 1), H->sign * H->J * (1 - (-1))), 0});
    } else {
        std::vector<HamTerm> T(size_t(H->nterms));
        YQ_CUDA(cudaMemcpy(T.data(), H->terms.p, T.size() * sizeof(HamTerm), cudaMemcpyDeviceToHost));
        for (const HamTerm& t : T) {
            if (t.nflip == 0) continue;
            if (t.nflip == 1)
                M.push_back(HamMove{t.a, -1, t.cp != 0.0 ? 3 : 0, 0});
            else
                M.push_back(HamMove{t.a, t.b, bits(t.cp, t.cm), 0});
        }
    }
    H->n_moves = int(M.size());
    H->moves.ensure(M.size() * sizeof(HamMove));
    YQ_CUDA(cudaMemcpy(H->moves.p, M.data(), M.size() * sizeof(HamMove), cudaMemcpyHostToDevice));
}

// ---------------------------------------------------------------------------
template <typename R>
struct ElocArgs {
    HamDesc H;
    int m, ns, nstride;
    const int8_t* sigma;
    const cplx<R>* theta;
    const cplx<R>* tauT;
    const cplx<R>* W;
    const c128* Lk;
    const c128* a;  // visible bias (FP64) or null
    c128* out;
    int* status;
};

template <typename R>
__global__ void __launch_bounds__(256) eloc_kernel(ElocArgs<R> A) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    cplx<R>* t = reinterpret_cast<cplx<R>*>(smem_raw);
    cplx<R>* th = t + A.m;
    int8_t* s = reinterpret_cast<int8_t*>(smem_raw + 2 * sizeof(cplx<R>) * A.m);
    __shared__ c128 red[8];
    const int n = A.H.n, m = A.m;
    const int tid = threadIdx.x, nt = blockDim.x;
    for (int smp = blockIdx.x; smp < A.ns; smp += gridDim.x) {
        for (int i = tid; i < n; i += nt) s[i] = A.sigma[size_t(smp) * n + i];
        for (int j = tid; j < m; j += nt) {
            cplx<R> v = A.theta[size_t(smp) * m + j];
            th[j] = v;
            t[j] = ctanh(v);
        }
        __syncthreads();
        c128 acc = mk(0., 0.);
        const bool table = A.H.nterms > 0;
        const int nterm = table ? A.H.nterms : n;
        for (int i = tid; i < nterm; i += nt) {
            int ka, kb;
            double c;
            if (table) {
                double d;
                table_term(A.H.terms[i], s, d, ka, kb, c);
                acc.re += d;
                if (ka < 0) continue;
            } else {
                acc.re += diag_term(A.H, s, i);
                offdiag_term(A.H, s, i, ka, kb, c);
            }
            if (c == 0.0) continue;  // zero coefficient: the reference multiplies the ratio by 0
            c128 val;
            if (kb < 0) {
                ScaledProd<R> P = prod1<R>(ka, R(s[ka]), n, m, t, th, 1, A.tauT, A.W);
                val = value_scaled(base1(A.Lk, A.a, ka, double(s[ka])), P);
            } else {
                ScaledProd<R> P = prod2<R>(ka, R(s[ka]), kb, R(s[kb]), n, m, t, th, 1, A.tauT, A.W);
                val = value_scaled(base1(A.Lk, A.a, ka, double(s[ka])) + base1(A.Lk, A.a, kb, double(s[kb])), P);
            }
            acc = acc + c * val;
        }
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) {
            acc.re += __shfl_xor_sync(0xffffffffu, acc.re, o);
            acc.im += __shfl_xor_sync(0xffffffffu, acc.im, o);
        }
        if ((tid & 31) == 0) red[tid >> 5] = acc;
        __syncthreads();
        if (tid == 0) {
            c128 r = red[0];
            for (int w = 1; w < (nt >> 5); ++w) r = r + red[w];
            A.out[smp] = r;
            if (!isfinite(r.re) || !isfinite(r.im)) atomicOr(A.status, DS_NONFINITE);
        }
        __syncthreads();
    }
}

template <typename R>
static void eloc_t(yq_ham_s* H, yq_rbm_s* q, int ns, const int8_t* d_sigma, const void* d_theta, c128* d_out) {
    ElocArgs<R> A;
    A.H = desc(H);
    A.m = q->m;
    A.ns = ns;
    A.nstride = (H->n + 15) & ~15;
    A.sigma = d_sigma;
    A.theta = reinterpret_cast<const cplx<R>*>(d_theta);
    A.tauT = q->tauT.as<cplx<R>>();
    A.W = q->W.as<cplx<R>>();
    A.Lk = q->Lk.as<c128>();
    A.a = q->use_bias ? q->p64.as<c128>() + size_t(q->n) * q->m : nullptr;
    A.out = d_out;
    A.status = H->ctx->status.as<int>();
    int threads = ((H->n + 31) / 32) * 32;
    if (threads > 256) threads = 256;
    if (threads < 64) threads = 64;
    size_t smem = 2 * sizeof(cplx<R>) * q->m + A.nstride;
    if (smem > 48 * 1024)
        YQ_CUDA(cudaFuncSetAttribute(eloc_kernel<R>, cudaFuncAttributeMaxDynamicSharedMemorySize, int(smem)));
    int blocks = ns < 148 * 16 ? ns : 148 * 16;
    eloc_kernel<R><<<blocks, threads, smem, H->ctx->stream>>>(A);
    YQ_LAUNCH_CHECK();
}

void ham_eloc(yq_ham_s* H, yq_rbm_s* q, int ns, const int8_t* d_sigma, const void* d_theta, c128* d_out) {
    YQ_CHECK_ARG(H->n == q->n, "eloc: Hamiltonian and RBM sizes differ");
    if (ns <= 0) return;
    rbm_prepare(q);
    if (q->dtype == YQ_C64)
        eloc_t<float>(H, q, ns, d_sigma, d_theta, d_out);
    else
        eloc_t<double>(H, q, ns, d_sigma, d_theta, d_out);
}

}  // namespace yq
