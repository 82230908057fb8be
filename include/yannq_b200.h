/*
 * yannq_b200.h -- C ABI of libyannq_b200.so, the B200 (sm_100a) backend of the
 * variational Monte Carlo step of yannq (sample -> E_loc -> O -> SR solve -> update).
 *
 * Every entry point returns an int status (YQ_OK = 0 or a YQ_E_* code); the
 * message of the last failure on the calling thread is available through
 * yq_last_error().  Handles are opaque.  One context owns one CUDA stream; calls
 * on one context are not reentrant, distinct contexts may be used from distinct
 * threads.  Complex arrays are interleaved (re, im) doubles on the host side.
 *
 * Each declaration names the reference interface it replaces (paths are relative
 * to the yannq project root).  The reference binds these through its own
 * header-only templates; the headers under include/yannq_gpu are the C++ adapters that let
 * an existing RunRBM-style driver call them.
 */
#ifndef YANNQ_B200_H
#define YANNQ_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ---- status codes ---------------------------------------------------------- */
enum {
    YQ_OK = 0,
    YQ_E_ARG = 1,         /* bad argument (shape, kind, null pointer)             */
    YQ_E_CUDA = 2,        /* CUDA runtime error                                    */
    YQ_E_NOMEM = 3,       /* device allocation failed                              */
    YQ_E_NOT_PD = 4,      /* Cholesky met a non-positive pivot (LLT failure)       */
    YQ_E_NONFINITE = 5,   /* NaN/Inf detected in E_loc, O, S/T or the update      */
    YQ_E_TIMEOUT = 6,     /* a bounded device-side wait gave up                    */
    YQ_E_STATE = 7,       /* call order violated (e.g. solve before construct)    */
    YQ_E_UNSUPPORTED = 8  /* configuration not built into this library            */
};

enum { YQ_C64 = 0, YQ_C128 = 1 };                             /* RBM<complex<float|double>> */
enum { YQ_ARCHIVE_C64 = 0, YQ_ARCHIVE_C128 = 1, YQ_ARCHIVE_F64 = 2, YQ_ARCHIVE_F32 = 3 }; /* archive element T */
enum { YQ_HAM_TFI = 0, YQ_HAM_XXZ = 1, YQ_HAM_TFI2D = 2,       /* Hamiltonian kinds          */
       YQ_HAM_XXX = 3, YQ_HAM_J1J2 = 4, YQ_HAM_XYZNNN = 5, YQ_HAM_KITAEV_HEX = 6 };
enum { YQ_MOVE_LOCAL = 0, YQ_MOVE_EXCHANGE_ANY = 1, YQ_MOVE_EXCHANGE_NN = 2, YQ_MOVE_HAMILTONIAN = 3 };
enum { YQ_SR_AUTO = 0, YQ_SR_S = 1, YQ_SR_T = 2 };             /* S = <O^H O>, T = O O^H dual */
enum { YQ_PREC_FP64 = 0, YQ_PREC_MIXED = 1 };
enum { YQ_SOLVE_LLT = 0, YQ_SOLVE_CG = 1 };
enum { YQ_BASIS_FULL = 0, YQ_BASIS_JZ = 1 };                   /* Basis/BasisFull.hpp, Basis/BasisJz.hpp */

typedef struct yq_ctx_s* yq_ctx;
typedef struct yq_rbm_s* yq_rbm;
typedef struct yq_ham_s* yq_ham;
typedef struct yq_sampler_s* yq_sampler;
typedef struct yq_sr_s* yq_sr;
typedef struct yq_ap_s* yq_ap;
typedef struct yq_ngd_s* yq_ngd;

/* Message of the last failed call on this thread (always NUL-terminated). */
int yq_last_error(char* buf, size_t len);
/* Library version string, e.g. "yannq_b200 0.1 sm_100a". */
const char* yq_version(void);
/* Number of kernels this library has launched in the process so far (no
 * reference counterpart; used to report launches per VMC step). */
int yq_launch_count(uint64_t* out);
/* Number of device allocations (cudaMalloc calls) this library has made in the
 * process so far (no reference counterpart; shows which calls allocate). */
int yq_alloc_count(uint64_t* out);
/* Page-locked host buffers for the host<->device copies of parameters and
 * samples (no reference counterpart: the reference is host-only). */
int yq_host_alloc(size_t bytes, void** out);
int yq_host_free(void* p);

/* ---- context --------------------------------------------------------------- */
/* No reference counterpart (the reference is host-only); owns the device and stream. */
int yq_ctx_create(int device, yq_ctx* out);
int yq_ctx_destroy(yq_ctx ctx);
int yq_ctx_synchronize(yq_ctx ctx);
/* Device time (ms) of the named stage of the last yq_vmc_iteration / yq_sample /
 * yq_sr_construct / yq_sr_solve call, measured with CUDA events on the context's
 * stream.  stage: 0 sample, 1 E_loc, 2 O, 3 S/T, 4 Cholesky+solve, 5 update,
 * 6 total, 7 mean + F.  (The reference times sampling and solving with
 * std::chrono: Runners/RunRBM.hpp:169-214.) */
int yq_ctx_stage_ms(yq_ctx ctx, int stage, float* ms);
/* Micro-benchmarked device roofs (no reference counterpart): out[0] FP64 SIMT
 * TFLOP/s, out[1] FP32 SIMT TFLOP/s, out[2] FP64 tensor-core (DMMA) TFLOP/s,
 * out[3] complex128 logcosh evaluations per second in units of 1e9. */
int yq_measure_peaks(yq_ctx ctx, double* out);

/* ---- RBM machine (Machines/RBM.hpp) ---------------------------------------- */
/* RBM<T>(n, m, useBias) -- Machines/RBM.hpp:48-53; dtype YQ_C64 or YQ_C128. */
int yq_rbm_create(yq_ctx ctx, int n, int m, int use_bias, int dtype, yq_rbm* out);
int yq_rbm_destroy(yq_rbm q);
/* getDim() -- Machines/RBM.hpp:120-126 */
int yq_rbm_dim(yq_rbm q, size_t* dim);
/* setParams / getParams / updateParams -- Machines/RBM.hpp:261-291; host vector of
 * getDim() complex values in the layout [W column-major (m x n) | a | b]. */
int yq_rbm_set_params(yq_rbm q, const double* params);
int yq_rbm_get_params(yq_rbm q, double* params);
int yq_rbm_update_params(yq_rbm q, const double* delta);
/* initializeRandom(re, sigma) -- Machines/RBM.hpp:325-349: draw order a, b, W by
 * columns, each entry (re, im) ~ N(0, sd^2); the normal draws are Philox4x32-10
 * keyed by seed (Box-Muller), identical to the oracle's. */
int yq_rbm_init_random(yq_rbm q, uint64_t seed, double sd);
/* Checkpoints in the reference's format: the cereal binary archive of
 * std::unique_ptr<RBM<T>> that RunRBM writes to w%04d.dat (Runners/RunRBM.hpp:
 * 155-164) and AbstractRunner::initializeFrom reads (Runners/AbstractRunner.hpp:
 * 83-94); layout from Serializers/SerializeRBM.hpp:20-82 and SerializeEigen.hpp:
 * 8-35 (u8 valid, u32 class version 1, u8 useBias, u32 N, u32 M, W as i32 rows,
 * i32 cols and M x N column-major values, then a and b likewise when useBias).
 * elem names T (the file does not record it): YQ_ARCHIVE_C128 std::complex<double>,
 * YQ_ARCHIVE_C64 std::complex<float>, YQ_ARCHIVE_F64 double, YQ_ARCHIVE_F32 float
 * (a real archive needs parameters with zero imaginary parts).  Saving converts
 * the FP64 master parameters to T; loading needs a machine of the archive's N, M
 * and useBias (the reference replaces the whole machine) and converts T to the
 * masters.  Buffers are host memory. */
int yq_rbm_archive_size(yq_rbm q, int elem, size_t* size);
int yq_rbm_save_archive(yq_rbm q, int elem, void* buf, size_t cap, size_t* size);
int yq_rbm_load_archive(yq_rbm q, int elem, const void* buf, size_t size);
/* N, M and useBias of an archive (any element type). */
int yq_rbm_archive_shape(const void* buf, size_t size, int* n, int* m, int* use_bias);
int yq_rbm_save(yq_rbm q, int elem, const char* path);
int yq_rbm_load(yq_rbm q, int elem, const char* path);
int yq_rbm_file_shape(const char* path, int* n, int* m, int* use_bias);
/* calcTheta over a batch -- Machines/RBM.hpp:137-141.  sigma: ns x n int8 (+-1). */
int yq_rbm_theta(yq_rbm q, int ns, const int8_t* sigma, double* theta);
/* logCoeff over a batch -- Machines/RBM.hpp:367-378 (ns complex). */
int yq_rbm_log_psi(yq_rbm q, int ns, const int8_t* sigma, double* out);
/* logRatio(k), logRatio(k, l) -- States/RBMState.hpp:48-94: for each sample s
 * flip sites flips[s*nflip .. s*nflip+nflip) (nflip 1 or 2); out: ns complex
 * log psi(sigma') - log psi(sigma) (defined modulo 2 pi i). */
int yq_rbm_log_ratio(yq_rbm q, int ns, const int8_t* sigma, const double* theta, int nflip, const int* flips,
                     double* out);
/* logRatio(const std::vector<int>&) -- States/RBMState.hpp:107-125: k distinct sites
 * flips[s*k .. s*k+k) of each sample flipped together, in the reference's logCosh
 * form (FP64 from the machine's weights); out: ns complex (modulo 2 pi i). */
int yq_rbm_log_ratio_k(yq_rbm q, int ns, const int8_t* sigma, const double* theta, int k, const int* flips,
                       double* out);
/* logRatio(const RBMStateObj& other) -- States/RBMState.hpp:136-149: log psi of
 * (sigma_other, theta_other) minus log psi of (sigma, theta), per sample; ns complex. */
int yq_rbm_log_ratio_states(yq_rbm q, int ns, const int8_t* sigma, const double* theta, const int8_t* sigma_other,
                            const double* theta_other, double* out);
/* logDeriv over a batch -- Machines/RBM.hpp:390-406 / constructDelta
 * (GroundState/utils.hpp:12-51): out ns x getDim() complex, row per sample. */
int yq_rbm_log_deriv(yq_rbm q, int ns, const int8_t* sigma, const double* theta, double* out);
/* Column mean of the log-derivative rows (the oloc vector of the SR step) from
 * samples already on the device, for callers that cannot let the library allocate
 * device memory (for example a host framework that has reserved the device for
 * its own allocator, or a service loop where allocation latency and its implicit
 * synchronisation are not acceptable).  No counterpart in the reference.
 * d_sigma: ns x n int8 (+-1); d_theta: ns x m in the RBM's compute type (complex64
 * or complex128, the layout yq_sampler_get_samples returns on the host);
 * d_oloc: getDim() complex128 output.  All three are device pointers owned by the
 * caller; the call is asynchronous on the context's stream.
 * Allocates nothing: its partial sums live in a fixed 4 MiB array compiled into
 * the library (held by every GPU that loads it), so it rejects machines with
 * (n + 1) (m + 1) > 262144.  Every call shares that array: calls that overlap on
 * the GPU race and must be serialised by the caller.  The first call on a context
 * looks up the array's device address (with the context's device current) and
 * keeps it with the context; make that first call before any stream capture. */
int yq_rbm_oloc_noalloc(yq_rbm q, int ns, const int8_t* d_sigma, const void* d_theta, double* d_oloc);

/* ---- Hamiltonians (Hamiltonians/TFIsing.hpp, XXZ.hpp, XXX.hpp, J1J2.hpp, ------
 * ---- XYZNNN.hpp, KitaevHex.hpp) ------------------------------------------ */
/* kind YQ_HAM_TFI: TFIsing(n, J, h); YQ_HAM_XXZ: XXZ(n, J, Delta = h, signRule);
 * YQ_HAM_TFI2D: periodic lx x ly square lattice (no reference counterpart; same
 * duck-typed concept: E_loc = sum J s_i (s_right + s_down) + h ratio(i));
 * YQ_HAM_XXX: XXX(n) (Hamiltonians/XXX.hpp:11-22; J, h unused);
 * YQ_HAM_J1J2: J1J2(n, J1 = J, J2 = h, signRule) (Hamiltonians/J1J2.hpp:14-56);
 * YQ_HAM_XYZNNN: XYZNNN(n, a = J, b = h) (Hamiltonians/XYZNNN.hpp:16-53).
 * J1J2 and XYZNNN need n >= 3.  lx, ly are read by YQ_HAM_TFI2D only; KitaevHex
 * has its own creator below. */
int yq_ham_create(yq_ctx ctx, int kind, int n, int lx, int ly, double J, double h, int sign_rule, yq_ham* out);
/* KitaevHex(ncol, nrow, Jx, Jy, Jz) with the field term h * ratio(i) of
 * KitaevHex(n, m, J, h) (Hamiltonians/KitaevHex.hpp:19-31, 119-146): ncol and
 * nrow even, sites = ncol * nrow, links as in blackIdx / whiteIdx / xLinks /
 * yLinks / zLinks (KitaevHex.hpp:33-103). */
int yq_ham_create_kitaev_hex(yq_ctx ctx, int ncol, int nrow, double Jx, double Jy, double Jz, double h,
                             yq_ham* out);
int yq_ham_destroy(yq_ham H);
/* Number of off-diagonal requests per sample that yq_ham_enumerate writes
 * (n for TFI, XXZ, TFI2D and XXX; 2n for J1J2 and XYZNNN; 2 * sites for KitaevHex). */
int yq_ham_num_offdiag(yq_ham H, int* count);
/* The state form's off-diagonal flips for each sample, in the order the
 * reference's operator()(State) requests them (Hamiltonians/TFIsing.hpp:28-39,
 * XXZ.hpp:37-49, XXX.hpp:11-22, J1J2.hpp:35-56, XYZNNN.hpp:33-53,
 * KitaevHex.hpp:119-146), zero coefficients included: per sample K =
 * yq_ham_num_offdiag terms of (site_a, site_b or -1, coeff) and the diagonal
 * sum.  Arrays: ns*K ints / doubles, ns doubles. */
int yq_ham_enumerate(yq_ham H, int ns, const int8_t* sigma, int* site_a, int* site_b, double* coeff, double* diag);
/* Energy::eachSample over a batch -- Observables/Energy.hpp:47-51 with
 * State = RBMStateRef(sigma, theta) (GroundState/utils.hpp:108-126). out: ns complex. */
int yq_eloc(yq_ham H, yq_rbm q, int ns, const int8_t* sigma, const double* theta, double* out);

/* ---- sampler (Samplers/SamplerMT.hpp + LocalSweeper / SwapSweeper) ------- */
/* SamplerMT(qs, nTmps = 1, nChainsPer = n_chains, sweeper) -- SamplerMT.hpp:44-60.
 * move: LocalSweeper (LocalSweeper.hpp:32-53), SwapSweeper with two independent
 * sites (SwapSweeper.hpp:28-57) or with a neighbouring pair (i, i+1).  nup >= 0
 * initialises chains with randomSigma(n, nup) (Utilities/Utility.hpp:77-88),
 * otherwise randomSigma(n).  sweep_len 0 means n proposals per sweep. */
int yq_sampler_create(yq_rbm q, int n_chains, int move, int nup, int sweep_len, yq_sampler* out);
int yq_sampler_destroy(yq_sampler S);
/* HamiltonianSweeper(n, ham) -- Samplers/HamiltonianSweeper.hpp:16-50, for a
 * sampler created with move YQ_MOVE_HAMILTONIAN: every proposal picks one entry
 * of offDiagonals(sigma) uniformly, flips it, and accepts with
 * min(1, |psi(sigma')/psi(sigma)|^2 w1 / w2), w1 and w2 the list sizes in sigma
 * and sigma' (no beta, as the reference's sweep ignores it).  offDiagonals is
 * TFIsing's list of all n sites (Hamiltonians/TFIsing.hpp:41-50; the same for
 * the 2D model); for the other kinds it is the state form's off-diagonal requests
 * whose coefficient in sigma is non-zero.  A proposal slot with an empty list is
 * skipped.  H must outlive the sampler's use of it. */
int yq_sampler_set_hamiltonian(yq_sampler S, yq_ham H);
/* Recompute theta from sigma in FP64 every k recorded/discarded sweeps (0 = never
 * inside one call, as the reference: States/RBMState.hpp:248-255). */
int yq_sampler_set_resync(yq_sampler S, int every_sweeps);
int yq_sampler_set_chains(yq_sampler S, const int8_t* sigma);  /* n_chains x n */
int yq_sampler_get_chains(yq_sampler S, int8_t* sigma);
/* randomize + sample(nSweeps, nDiscard) -- SamplerMT.hpp:103-110, :180-204.
 * reinit != 0 draws fresh chains first (RunRBM.hpp:166).  Samples stay on the
 * device, ordered (sweep, chain); n_samples = n_chains * n_sweeps. */
int yq_sample(yq_sampler S, int n_sweeps, int n_discard, uint64_t seed, uint32_t epoch, int reinit);
int yq_sampler_num_samples(yq_sampler S, int* ns);
/* Copy the last samples to the host: sigma ns x n int8, theta ns x m complex (may be null). */
int yq_sampler_get_samples(yq_sampler S, int8_t* sigma, double* theta);
/* SamplerMT(qs, nTmps, nChainsPer, sweeper) with nTmps > 1 -- Samplers/SamplerMT.hpp:
 * 44-60, 120-204: the sampler's n_chains = nTmps x nChainsPer chains form groups of
 * ntemps consecutive chains with betas (nTmps - t) / nTmps; every sweep each chain
 * sweeps at its beta, then mixChains swaps temperatures between neighbouring
 * slots of a group (even pairs, then odd pairs; u from the parallel-tempering
 * Philox stream), and recorded sweeps keep the beta = 1 chain of every group, so a
 * sample call returns nChainsPer x n_sweeps samples.  ntemps = 1 (default) is the
 * plain sampler.  The ladder positions persist across calls (reset by reinit). */
int yq_sampler_set_tempering(yq_sampler S, int ntemps);
/* Ladder slot of every chain (0 = beta 1), n_chains entries. */
int yq_sampler_get_slots(yq_sampler S, int* slots);
/* No reference counterpart: the launch shape that the sampler's autotuner chose
 * for the configuration of the last yq_sample (0 before any): chains per CTA and
 * warps per chain.  The choice is timed once per configuration per process among
 * 1, 2 and 4 chains per CTA with one warp per chain and, for complex64 plain
 * chains of local or exchange moves, 1 and 2 chains per CTA with two warps per
 * chain (each warp holding half of the hidden units); YQ_AUTOTUNE=0 in the
 * environment fixes 4 chains per CTA and one warp per chain, YQ_CHAINS_PER_CTA=1, 2
 * or 4 and YQ_WARPS_PER_CHAIN=1 or 2 restrict the choice. */
int yq_sampler_chains_per_cta(yq_sampler S, int* out);
int yq_sampler_warps_per_chain(yq_sampler S, int* out);
/* Accepted proposals per chain in the last yq_sample (LocalSweeper::sweep's return). */
int yq_sampler_get_accepts(yq_sampler S, uint64_t* acc);
/* Replace the device samples by host ones (for SR on externally supplied samples). */
int yq_sampler_put_samples(yq_sampler S, int ns, const int8_t* sigma, const double* theta);
/* ExactSampler<Machine>(qs, basis).sample(ns, 0) -- Samplers/ExactSampler.hpp:49-79:
 * replaces the sampler's samples by ns draws from |psi|^2 over the full basis
 * (sampler created with nup < 0) or the basis with nup spins down, at most 2^24
 * configurations.  Draw i uses the exact-sampler Philox stream (seed, counter
 * (i, epoch, 0, tag)) in place of the reference's unseeded engine.  positions
 * (optional, ns entries) receives the drawn basis positions. */
int yq_sampler_sample_exact(yq_sampler S, int ns, uint64_t seed, uint32_t epoch, uint64_t* positions);

/* Failure injection for the bounded device waits (no reference counterpart; for
 * tests): runs the persistent tile Cholesky (which = 0) or the forward triangular
 * solve (which = 1) on a 256 x 256 problem whose first work item is never
 * claimed, so the flag it would publish is never set, with every wait limited to
 * `cap` polls.  The first wait to run out records the timeout and raises the
 * abort word; every CTA then returns.  Returns YQ_E_TIMEOUT (the context stays
 * usable); *published receives the number of flags that were published (0). */
int yq_debug_wait_timeout(yq_ctx ctx, int which, unsigned cap, int* published);

/* ---- stochastic reconfiguration (GroundState/SRMat.hpp) ------------------- */
/* SRMat<Machine, Hamiltonian>(qs, ham) -- SRMat.hpp:83-87, bound to a sampler.
 * mode: S = O~^H O~ / Ns (P x P), T = O~ O~^H / Ns (Ns x Ns, push-through dual),
 * AUTO picks T when Ns < P.  precision: FP64 everywhere, or MIXED (c64 sampling
 * and O, BF16x3 tensor-core S/T with FP32 accumulation, a Cholesky factor of the
 * shifted T used as the preconditioner of CG steps with FP64 residuals on the
 * exact operator, FP64 means). */
int yq_sr_create(yq_rbm q, yq_ham H, yq_sampler S, int mode, int precision, yq_sr* out);
int yq_sr_destroy(yq_sr sr);
/* constructFromSamples -- SRMat.hpp:89-103 (E_loc, O, mean, centring, F). */
int yq_sr_construct(yq_sr sr);
/* eloc() / elocVar() -- SRMat.hpp:151-159 */
int yq_sr_energy(yq_sr sr, double* energy, double* energy_var);
/* elocs, oloc(), energyGrad() to host: which 0 elocs (Ns), 1 oloc (P), 2 grad (P), 3 v (P). */
int yq_sr_get(yq_sr sr, int which, double* out);
/* solveExact(shift) (SRMat.hpp:231-237, Eigen::LLT) in S-mode, or its sample-space
 * dual in T-mode; solver YQ_SOLVE_CG uses SRMat::apply (SRMat.hpp:170-208) with
 * relative-residual tolerance cg_tol.  v (P complex, may be null) receives the
 * solution; iterations/relres (may be null) the CG statistics. */
int yq_sr_solve(yq_sr sr, double shift, int solver, double cg_tol, double* v, int* iterations, double* relres);
/* CG steps of the T-form LLT solve of yq_sr_solve (a setting of this library; the
 * reference solves with Eigen::LLT alone, SRMat.hpp:231-237): 0 applies the
 * Cholesky factor once, s > 0 runs s + 1 iterations of CG from zero preconditioned
 * by the factor, on the exact operator with FP64 sums.  -1 (the default) means 2 for
 * YQ_PREC_MIXED and 0 for YQ_PREC_FP64. */
int yq_sr_set_solve_steps(yq_sr sr, int steps);
/* corrMat() -- SRMat.hpp:142-149: the Hermitian matrix the last LLT solve used
 * (S or T, including the shift), lower triangle, dim x dim complex row-major. */
int yq_sr_matrix(yq_sr sr, int* dim, double* out);

/* ---- exact summation (GroundState/SRMatExact.hpp) ------------------------- */
/* SRMatExact<Machine, Hamiltonian>(qs, ham).constructExact() followed by eloc(),
 * elocVar(), oloc(), energyGrad() and corrMat() -- SRMatExact.hpp:97-132 -- over
 * the full basis (YQ_BASIS_FULL, Basis/BasisFull.hpp, n <= 24) or the basis with
 * nup spins down (YQ_BASIS_JZ, Basis/BasisJz.hpp; XXZ only), at most 2^24
 * configurations, FP64 sums.  stats = {E, Var}; oloc, grad: P complex
 * (interleaved re, im); S: P x P complex row-major, or NULL to skip it. */
int yq_exact(yq_rbm q, yq_ham H, int basis_kind, int nup, double* stats, double* oloc, double* grad, double* S);
/* One epoch of RunRBMExact::run (Runners/RunRBMExact.hpp:46-80): constructExact over
 * the basis (as yq_exact), v = LLT(corrMat() + shift I).solve(energyGrad()) on the
 * device, params -= lr v (the SGD step of Optimizers/SGD.hpp:48-54 with the caller's
 * rate).  out = {E, Var, |v|} (E and Var before the update).  A non-positive
 * pivot returns YQ_E_NOT_PD (the reference ignores it). */
int yq_exact_iteration(yq_rbm q, yq_ham H, int basis_kind, int nup, double shift, double lr, double* out);

/* ---- FeedForward machine (Machines/FeedForward.hpp) ------------------------ */
/* FeedForward with addLayer<Conv1D>(1, channels, kernel, stride 1, no bias),
 * LnCosh, addLayer<FullyConnected>(L * channels, fc_out, no bias), LnCosh and a
 * Sum output (fc_out x Mean({fc_out, 1}, 0), layers/Mean.hpp:92-125), FP32
 * parameters [conv kernel (kernel x channels, column-major) | fc weight
 * ((L channels) x fc_out, column-major)] (FeedForward.hpp:76-127). */
typedef struct yq_ff_s* yq_ff;
int yq_ff_create(yq_ctx ctx, int L, int channels, int kernel, int fc_out, yq_ff* out);
int yq_ff_destroy(yq_ff f);
int yq_ff_dim(yq_ff f, size_t* dim);
int yq_ff_set_params(yq_ff f, const double* params);
int yq_ff_get_params(yq_ff f, double* params);
/* initializeRandom(re, Xavier) -- FeedForward.hpp:42-73, Philox-seeded normals. */
int yq_ff_init_random(yq_ff f, uint64_t seed);
/* The batch of configurations the next calls act on (batch x L int8 from the host,
 * or drawn on the device). */
int yq_ff_set_batch(yq_ff f, int batch, const int8_t* sigma);
int yq_ff_random_batch(yq_ff f, int batch, uint64_t seed);
/* forward / makeData -- FeedForward.hpp:152-184: log psi of the batch (host copy if
 * logpsi != null).  Activations are kept for the adjoint when batch x (L channels +
 * fc_out) floats fit act_budget_bytes; otherwise the adjoint recomputes them. */
int yq_ff_forward(yq_ff f, size_t act_budget_bytes, double* logpsi);
/* backward -- FeedForward.hpp:186-205 with dout = 1: the log-derivative rows
 * (batch x getDim(), host copy as doubles if O != null). */
int yq_ff_adjoint(yq_ff f, double* O);
/* TFIsing(L, J, h)'s local energy of the batch (Hamiltonians/TFIsing.hpp:28-39)
 * with psi-ratios from single-flip updates of the activations. */
int yq_ff_eloc_tfi(yq_ff f, double J, double h, double* eloc);

/* ---- one VMC iteration (Runners/RunRBM.hpp:151-221) ----------------------- */
typedef struct {
    int n_sweeps;          /* recorded sweeps (samples = n_chains * n_sweeps)       */
    int n_discard;         /* thermalisation sweeps per iteration                   */
    int reinit;            /* randomize chains every iteration (reference default) */
    uint64_t seed;
    uint32_t epoch;        /* iteration index ll (also the Philox epoch)           */
    double shift;          /* lambda = max(lambda0 decay^ll, lambda_min) by caller */
    double lr;             /* SGD eta = max(alpha / t^p, 1e-4) by caller            */
    int solver;            /* YQ_SOLVE_LLT or YQ_SOLVE_CG                           */
    double cg_tol;
    int ir_steps;          /* T-form: CG steps as in yq_sr_set_solve_steps (>= 0)  */
} yq_iter_params;

typedef struct {
    double energy, energy_var;
    double update_norm;    /* ||v|| before the clip (RunRBM.hpp:205 nv)             */
    double cg_err;         /* CG branch: ||apply(v) - grad|| (RunRBM.hpp:190); 0 for LLT */
    double accept_rate;
    int status;            /* 0 or the YQ_E_* code recorded by the device checks    */
} yq_iter_result;

/* RunRBM::setMomentum(beta1, beta2) -- Runners/RunRBM.hpp:73-77 with ObsAvg
 * (:13-37): yq_vmc_iteration averages energyGrad() with weight beta1 and, in the
 * LLT branch, corrMat() with weight beta2 (bias-corrected by 1 - beta^t), in the
 * order of RunRBM.hpp:180-201 (gradAvg is updated twice per LLT epoch, as there).
 * beta2 != 0 needs the S-form (YQ_SR_AUTO then picks it; YQ_SR_T fails with
 * YQ_E_UNSUPPORTED); beta1 != 0 in the T-form solves (S + lambda) v = grad by the
 * Woodbury identity through T and needs lambda > 0.  Resets both averages.
 * Batches (yq_batch_*) reject objects with momentum. */
int yq_sr_set_momentum(yq_sr sr, double beta1, double beta2);
/* RunRBM::setGradClip(clip) -- RunRBM.hpp:79-82, 205-209: v *= clip / ||v|| when
 * ||v|| > clip (0 disables); applied on the device by yq_vmc_iteration and batches. */
int yq_sr_set_grad_clip(yq_sr sr, double clip);

/* sampler.randomize + sample + constructFromSamples + solve + update params by -lr v
 * (Runners/RunRBM.hpp:166-214 for one epoch ll = p->epoch). */
int yq_vmc_iteration(yq_sr sr, const yq_iter_params* p, yq_iter_result* r);

/* ---- batches of independent problems --------------------------------------- */
/* No reference counterpart (the reference runs one problem per process): advances
 * nprob SR objects -- each with its own machine, Hamiltonian and sampler, normally
 * each on its own context -- by one RunRBM iteration (Runners/RunRBM.hpp:166-214,
 * LLT solver) per yq_batch_iteration.  The first call (and any call whose
 * parameters other than epoch/reinit change) runs eagerly and captures the next
 * iteration of all problems into one CUDA graph on ctx's stream; later calls
 * replay it, advancing the epoch by one per call from the capturing call's epoch
 * and keeping the chains.  Problem k samples with seed + k.  results: nprob
 * entries; the call fails with the first problem's error code if any failed. */
typedef struct yq_batch_s* yq_batch;
int yq_batch_create(yq_ctx ctx, int nprob, const yq_sr* srs, yq_batch* out);
int yq_batch_iteration(yq_batch B, const yq_iter_params* p, yq_iter_result* results);
int yq_batch_destroy(yq_batch B);

/* ---- AmplitudePhase and NGDExact (Machines/AmplitudePhase.hpp, ----------
 * ---- GroundState/NGDExact.hpp, Runners/RunAmplitudePhase.hpp) ----------- */
/* Phase-network layers: 6 ints per layer {type, a, b, k, stride, use_bias} and one
 * double x.  YQ_LAYER_CONV1D: Conv1D(a = inChannels, b = outChannels, k =
 * kernelSize, stride, useBias) (layers/Conv1D.hpp:57-65, periodic); YQ_LAYER_FC:
 * FullyConnected(a = inputDim, b = outputDim, useBias); the activation layers of
 * layers/ActivationLayer.hpp with x = Tanh's constant, LeakyReLU's negative
 * slope, LeakyHardTanh's outside slope or Cos's a (layers/activations.hpp; the
 * Sigmoid forward exp(z) + 1 and Jacobian (1 - a) a are restated as written). */
enum { YQ_LAYER_CONV1D = 0, YQ_LAYER_FC = 1, YQ_ACT_IDENTITY = 10, YQ_ACT_LNCOSH = 11, YQ_ACT_TANH = 12,
       YQ_ACT_WEAKTANH = 13, YQ_ACT_SIGMOID = 14, YQ_ACT_RELU = 15, YQ_ACT_LEAKYRELU = 16, YQ_ACT_HARDTANH = 17,
       YQ_ACT_SOFTSHRINK = 18, YQ_ACT_LEAKYHARDTANH = 19, YQ_ACT_SOFTSIGN = 20, YQ_ACT_COS = 21 };
enum { YQ_INIT_LECUN = 0, YQ_INIT_XAVIER = 1, YQ_INIT_HE = 2 };  /* FeedForward.hpp InitializationMode */
enum { YQ_NGD_GRAD = 0, YQ_NGD_OLOC_AMP = 1, YQ_NGD_OLOC_PHASE = 2, YQ_NGD_CORR_AMP = 3, YQ_NGD_CORR_PHASE = 4 };
enum { YQ_NGD_AMP = 0, YQ_NGD_PHASE = 1, YQ_NGD_ALL = 2 };      /* RunAmplitudePhase.hpp Mode */
/* AmplitudePhase(N = n, M = m, useBias, FeedForward<double>&& phase) --
 * AmplitudePhase.hpp:37-40: psi = sqrt(A) exp(i pi phi), A = exp(a.s + sum_j
 * logCosh(theta_j)) of a real RBM<double>, phi the network's single output.
 * Parameters are real: [amplitude in the RBM layout W (m x n col-major) | a | b,
 * then each layer's parameters in order (Conv1D kernel (in k) x out col-major then
 * bias, FullyConnected weight in x out col-major then bias)]. */
int yq_ap_create(yq_ctx ctx, int n, int m, int use_bias, int nlayers, const int* layers, const double* layer_x,
                 yq_ap* out);
int yq_ap_destroy(yq_ap q);
/* getDimAmp(), getDimPhase() -- AmplitudePhase.hpp:61-74 */
int yq_ap_dims(yq_ap q, size_t* dim_amp, size_t* dim_phase);
int yq_ap_set_params(yq_ap q, const double* params);
int yq_ap_get_params(yq_ap q, double* params);
/* updateParams -- AmplitudePhase.hpp:156-161 */
int yq_ap_update_params(yq_ap q, const double* delta);
/* initializeRandom(re, sigma) -- AmplitudePhase.hpp:92-97: amplitude N(0, sigma^2)
 * in the RBM draw order, then every parameterised layer N(0, s^2) with s from
 * FeedForward.hpp initializeRandom(re, mode) (LeCun sqrt(1/fanIn), Xavier
 * sqrt(2/(fanIn + fanOut)), He sqrt(2/fanIn)); the reference initializes the
 * phase with Xavier.  Normals: the first Box-Muller value of Philox4x32-10 draw
 * (seed; counter e, 0, 0, parameter tag), e counting through both blocks. */
int yq_ap_init_random(yq_ap q, uint64_t seed, double sigma_amp, int phase_mode);
/* log psi = log(A) / 2 + i pi phi over a batch (AmplitudePhase::coeff, :132-143). out: ns complex. */
int yq_ap_log_psi(yq_ap q, int ns, const int8_t* sigma, double* out);
/* logDeriv -- AmplitudePhase.hpp:42-59: rows [RBM logDeriv / 2 | i pi backward]; out ns x dim complex. */
int yq_ap_log_deriv(yq_ap q, int ns, const int8_t* sigma, double* out);
/* NGDExact(qs, basis, col) -- NGDExact.hpp:196-208: the full basis or the Jz basis
 * (nup spins down; needs a Hamiltonian that conserves Sz) and the Hamiltonian's
 * column form, applied matrix-free.  The machine and H must outlive the object. */
int yq_ngd_create(yq_ap q, yq_ham H, int basis_kind, int nup, yq_ngd* out);
int yq_ngd_destroy(yq_ngd g);
int yq_ngd_basis_size(yq_ngd g, uint64_t* dim);
/* constructExact -- NGDExact.hpp:123-150; energy = eloc() (may be null). */
int yq_ngd_construct(yq_ngd g, double* energy);
/* energyGrad (dim), olocAmp (Pa), olocPhase (Pp), corrMatAmp (Pa x Pa), corrMatPhase
 * (Pp x Pp, row-major) of the last construct -- NGDExact.hpp:152-194. */
int yq_ngd_get(yq_ngd g, int what, double* out);
/* One epoch of RunAmplitudePhaseExact::run (Runners/RunAmplitudePhase.hpp:92-119):
 * constructExact, v = (corrMat + lambda I)^{-1} grad by LLT for the amplitude and/or
 * phase block (mode), params += -lr v (SGD.hpp:48-54 with a caller-given rate).
 * Returns E before the update, |grad| and |v|.  A non-positive pivot returns
 * YQ_E_NOT_PD (the reference ignores it). */
int yq_ngd_iteration(yq_ngd g, double lambda, double lr, int mode, double* energy, double* grad_norm, double* v_norm);

#ifdef __cplusplus
}
#endif
#endif /* YANNQ_B200_H */
