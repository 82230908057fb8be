// Internal object model of libyannq_b200 (host side).  The C ABI in capi.cu maps
// each opaque handle of include/yannq_b200.h onto one of these structs.
#pragma once
#include <memory>
#include <string>
#include <vector>

#include "common.cuh"

namespace yq {

enum Stage { ST_SAMPLE = 0, ST_ELOC = 1, ST_O = 2, ST_GRAM = 3, ST_SOLVE = 4, ST_UPDATE = 5, ST_TOTAL = 6, ST_MEAN = 7,
             ST_FF_FORWARD = 8, ST_FF_ADJOINT = 9, ST_FF_ELOC = 10, ST_COUNT = 11 };

// Device-side status word bits (set by kernels, read once per call by the host).
enum : int { DS_NONFINITE = 1, DS_NOT_PD = 2, DS_TIMEOUT = 4 };

}  // namespace yq

struct yq_ctx_s {
    int device = 0;
    int sm_count = 0;
    cudaStream_t stream = nullptr;
    cudaEvent_t ev_start[yq::ST_COUNT] = {};
    cudaEvent_t ev_stop[yq::ST_COUNT] = {};
    bool ev_used[yq::ST_COUNT] = {};
    yq::DevBuf status;  // int device status word
    yq::DevBuf scratch; // small reduction scratch (doubles)
    bool timing = true; // stage events recorded (off while a batch graph is captured)
    void* noalloc_scratch = nullptr;  // device address of the no-allocation entry point's array

    void stage_begin(int s);
    void stage_end(int s);
    int read_status_and_clear();
};

struct yq_rbm_s {
    yq_ctx_s* ctx = nullptr;
    int n = 0, m = 0;
    bool use_bias = true;
    int dtype = YQ_C128;
    size_t P = 0;
    yq::DevBuf p64;  // master parameters, c128 [W col-major | a | b]
    // derived, in the compute type (c64 or c128): W (m x n col-major), a (n), b (m),
    // tau = tanh(2W) (m x n col-major), tauT (n x m), and Lk = sum_j logcosh(2 W_jk) (c128)
    yq::DevBuf W, a, b, tau, tauT, Lk;
    uint64_t version = 1, prepared = 0;
    void prepare();  // refresh derived arrays after a parameter change
    size_t csize() const { return dtype == YQ_C64 ? sizeof(yq::c64) : sizeof(yq::c128); }
};

// One entry of a term-table Hamiltonian (kinds XXX, J1J2, XYZNNN, KitaevHex):
// for zz = s_a s_b (1 when b < 0) the diagonal gains (zz > 0 ? dp : dm) when
// has_diag, and flipping a (and b when nflip == 2) is requested with
// coefficient (zz > 0 ? cp : cm) when nflip > 0.  The four values are formed on
// the host with the reference's own expressions for zz = +1 and zz = -1.
struct HamTerm {
    int a, b, nflip, has_diag;
    double dp, dm, cp, cm;
};

// One entry of a Hamiltonian's offDiagonals list (the HamiltonianSweeper's
// proposals): flip a (and b >= 0); present in state s when bit 0 (zz = s_a s_b
// = +1, or a single flip) or bit 1 (zz = -1) of `on` is set.
struct HamMove {
    int a, b, on, pad;
};

struct yq_ham_s {
    yq_ctx_s* ctx = nullptr;
    int kind = 0, n = 0, lx = 0, ly = 0;
    double J = 0., h = 0., sign = 1.;
    // term-table kinds: terms in the reference's evaluation order
    int nterms = 0, n_off = 0;  // n_off: off-diagonal requests per sample
    bool conserves_sz = false;  // every request keeps the number of down spins
    yq::DevBuf terms;           // nterms HamTerm
    int n_moves = 0;
    yq::DevBuf moves;           // n_moves HamMove (every kind)
};

struct yq_sampler_s {
    yq_rbm_s* q = nullptr;
    int n_chains = 0, move = 0, nup = -1, sweep_len = 0, resync = 0;
    bool have_chains = false;
    yq::DevBuf chains;   // n_chains x n int8
    yq::DevBuf sigma;    // ns x n int8
    yq::DevBuf theta;    // ns x m compute type
    yq::DevBuf acc;      // n_chains u64
    int ns = 0;
    uint64_t proposals = 0;  // per chain, last call
    const uint32_t* epoch_dev = nullptr;  // device epoch offset added to the call's epoch (batched graphs)
    int chains_per_cta = 0;               // autotuned launch shape of the last sample call:
    int warps_per_chain = 0;              //   chains per CTA and warps per chain
    const yq_ham_s* ham = nullptr;        // proposals of YQ_MOVE_HAMILTONIAN
    // parallel tempering (SamplerMT nTmps > 1): chains c = ntemps group + k
    int ntemps = 1;
    bool pt_ready = false;
    yq::DevBuf pt_slot, pt_beta;  // per chain: ladder slot (int), beta (double)
    yq::DevBuf pt_theta, pt_lp;   // theta carried between sweep launches, Re log psi
};

// FeedForward machine Conv1D(1 -> C, kernel K, periodic, no bias) -> LnCosh ->
// FullyConnected(L C -> F, no bias) -> LnCosh -> Sum, FP32 parameters.
struct yq_ff_s {
    yq_ctx_s* ctx = nullptr;
    int L = 0, C = 0, K = 0, F = 0;
    size_t P = 0;                 // K C + L C F
    yq::DevBuf params;            // float [conv kernel (K x C col-major) | fc weight ((L C) x F col-major)]
    int batch = 0;
    yq::DevBuf sigma;             // batch x L int8
    yq::DevBuf logpsi;            // batch double
    yq::DevBuf acts;              // batch x (L C + F) float, when stored
    bool acts_valid = false;
    yq::DevBuf O;                 // batch x P float
    yq::DevBuf eloc;              // batch c128
};

struct yq_sr_s {
    yq_rbm_s* q = nullptr;
    yq_ham_s* H = nullptr;
    yq_sampler_s* S = nullptr;
    int mode_req = YQ_SR_AUTO, precision = YQ_PREC_FP64;
    int mode = YQ_SR_T;  // resolved at construct
    int ns = 0;
    bool constructed = false, solved = false;
    // per-sample data
    yq::DevBuf eloc;    // ns c128
    yq::DevBuf tanhs;   // ns x m compute type
    yq::DevBuf O;       // ns x P compute type, centred (row per sample)
    yq::DevBuf part;    // split-reduction partials (c128)
    yq::DevBuf oloc, grad, v, work_p;   // P c128
    yq::DevBuf y, rhs, work_s;          // max(ns, dim_pad) c128
    yq::DevBuf s1, s2, s3, s4;          // solver scratch vectors
    yq::DevBuf stats;   // double[8]: E, var, mean.re, mean.im, |v|, acc...
    // dense SR matrix and Cholesky factor (lower, row-major, dim_pad x dim_pad)
    int dim = 0, dim_pad = 0;
    yq::DevBuf G, Linv, LinvH;
    yq::DevBuf chol_work;    // persistent Cholesky flags, counters and tile order
    yq::DevBuf chol_planes;  // BF16 split panels of the mixed-precision Cholesky
    // mixed precision operands (BF16 hi/lo planes of [Re|Im] and [Im|-Re])
    yq::DevBuf xh, xl, yh, yl;
    yq::DevBuf gram_ws;  // FP32 partials of the Gram's K-split tiles
    double host_stats[8] = {};
    // RunRBM's exponential averages of the gradient (beta1) and of the Fisher
    // matrix (beta2) and its update clip (Runners/RunRBM.hpp:13-37, 73-82, 181-209),
    // applied by yq_vmc_iteration only; t_* count the ObsAvg updates
    double beta1 = 0., beta2 = 0., grad_clip = 0.;
    long t_grad = 0, t_fisher = 0;
    yq::DevBuf gavg, gused;  // P c128: running average and the bias-corrected gradient
    yq::DevBuf favg;         // dim_pad x dim_pad c128 running Fisher average (S-form)
    yq::DevBuf trhs;         // ns c128: right-hand side of a T-form solve with a given gradient
    yq::DevBuf pcg;          // T-form PCG vectors r, z, p, q (dim_pad c128 each) and step scalars
    yq::DevBuf ohy_sol;      // P c128: O~^H of a T-form solution (the Woodbury form)
    int solve_steps = -1;    // T-form CG steps of yq_sr_solve (-1: the precision's default)
};

// A batch of SR problems advanced together (batch.cu).
struct yq_batch_s {
    yq_ctx_s* ctx = nullptr;
    std::vector<yq_sr_s*> srs;
    yq::DevBuf epoch;  // uint32 device epoch offset
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t exec = nullptr;
    cudaEvent_t fork = nullptr;
    std::vector<cudaEvent_t> joins;
    yq_iter_params captured{};
    bool have_graph = false;
    std::vector<double> host_stats;
    std::vector<unsigned long long> host_acc;
    yq::DevBuf dev_acc_sum;  // per problem accepted proposals (u64)

    ~yq_batch_s() {
        if (exec) cudaGraphExecDestroy(exec);
        if (graph) cudaGraphDestroy(graph);
        if (fork) cudaEventDestroy(fork);
        for (auto e : joins)
            if (e) cudaEventDestroy(e);
    }
};

namespace yq {
// kernels launched from the objects (defined in the .cu files)
void rbm_prepare(yq_rbm_s* q);
void rbm_theta(yq_rbm_s* q, int ns, const int8_t* d_sigma, void* d_theta, bool out_c128);
void rbm_log_psi(yq_rbm_s* q, int ns, const int8_t* d_sigma, c128* d_out);
void rbm_log_ratio(yq_rbm_s* q, int ns, const int8_t* d_sigma, const void* d_theta, int nflip, const int* d_flips,
                   c128* d_out);
void rbm_log_deriv(yq_rbm_s* q, int ns, const int8_t* d_sigma, const void* d_theta, c128* d_out);
void rbm_log_ratio_k(yq_rbm_s* q, int ns, const int8_t* d_sigma, const c128* d_theta, int k, const int* d_flips,
                     c128* d_out);
void rbm_log_ratio_states(yq_rbm_s* q, int ns, const int8_t* d_sa, const c128* d_tha, const int8_t* d_sb,
                          const c128* d_thb, c128* d_out);
void rbm_init_params_host(int n, int m, bool bias, uint64_t seed, double sd, c128* p);

void sampler_run(yq_sampler_s* S, int n_sweeps, int n_discard, uint64_t seed, uint32_t epoch, int reinit);

// RBM checkpoints (cereal binary image of unique_ptr<RBM<T>>)
size_t rbm_archive_size(int n, int m, bool bias, int elem);
void rbm_archive_shape(const uint8_t* buf, size_t size, int* n, int* m, int* use_bias);
void rbm_archive_write(yq_rbm_s* q, int elem, std::vector<uint8_t>& out);
void rbm_archive_read(yq_rbm_s* q, int elem, const uint8_t* buf, size_t size);
std::vector<uint8_t> read_file(const char* path);
void write_file(const char* path, const std::vector<uint8_t>& buf);
void ham_build_terms(yq_ham_s* H, double jy, double jz);  // term-table kinds
void ham_build_moves(yq_ham_s* H);                        // offDiagonals list, every kind
int ham_num_offdiag(const yq_ham_s* H);
void ham_enumerate(yq_ham_s* H, int ns, const int8_t* d_sigma, int* d_a, int* d_b, double* d_c, double* d_diag);
void ham_eloc(yq_ham_s* H, yq_rbm_s* q, int ns, const int8_t* d_sigma, const void* d_theta, c128* d_out);

void sr_construct(yq_sr_s* sr);
// d_S (optional) receives the lower triangle of S + shift I with leading dimension ldS (0: P)
void exact_summation(yq_rbm_s* q, yq_ham_s* H, int kind, int nup, double* stats, c128* d_oloc, c128* d_grad,
                     c128* d_S, size_t ldS = 0, double shift = 0.0);
void exact_iteration(yq_rbm_s* q, yq_ham_s* H, int kind, int nup, double shift, double lr, double* out);
void sampler_sample_exact(yq_sampler_s* S, int ns, uint64_t seed, uint32_t epoch, uint64_t* d_pos);
void batch_create(yq_ctx_s* ctx, int np, yq_sr_s* const* srs, yq_batch_s** out);
void batch_destroy(yq_batch_s* B);
void batch_iteration(yq_batch_s* B, const yq_iter_params& p, yq_iter_result* res);
void sr_solve(yq_sr_s* sr, double shift, int solver, double cg_tol, int ir_steps, int* iters, double* relres);
// RunRBM.hpp:181-203: the solve of one runner epoch with the ObsAvg momentum of
// the gradient and the Fisher matrix; cg_err = |apply(v) - grad| for the CG branch
void sr_solve_runner(yq_sr_s* sr, double shift, int solver, double cg_tol, int ir_steps, int* iters, double* relres,
                     double* cg_err);
void sr_update_params(yq_sr_s* sr, double lr);
void sr_form_matrix_public(yq_sr_s* sr, double shift);
}  // namespace yq
