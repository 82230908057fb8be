// yannq oracle: a CPU restatement of the reference's VMC hot path.
//
// TEST INFRASTRUCTURE ONLY.  Nothing in the product library (libyannq_b200.so)
// links, includes or calls this code; it is the checker used by tests/, by the
// smoke check and by the CPU-baseline leg of bench.py.
//
// Each routine restates the reference algorithm named beside it (paths are
// relative to the reference project root).  The reference itself cannot be
// built here (it needs Eigen3, TBB, MKL, cereal, nlohmann/json), so this
// restatement stands in for it; its own fidelity is pinned by the reference's
// known-answer and property tests re-expressed in tests/test_oracle_*.py, by
// exact diagonalisation and by the closed-form energy of the periodic
// transverse-field Ising chain.
//
// Conventions (all follow the reference):
//   * spins sigma_i = +-1 stored as int8; bit i of a basis index set <=> sigma_i = -1
//     (Utilities/Utility.hpp:91-110)
//   * RBM parameters p = [W column-major (m x n) | a (n) | b (m)]
//     (Machines/RBM.hpp:271-291)
//   * complex numbers are interleaved (re, im) doubles at the C boundary.
#pragma once
#include <algorithm>
#include <array>
#include <cmath>
#include <complex>
#include <cstdint>
#include <cstring>
#include <map>
#include <vector>

#include "philox.hpp"

namespace orc {

using cd = std::complex<double>;

// ---------------------------------------------------------------------------
// Utilities/Utility.hpp:14-24 -- stable log(cosh(x)) for real x
inline double logCosh(double x) {
    const double xp = std::fabs(x);
    if (xp <= 12.) return std::log(std::cosh(xp));
    return xp - std::log(2.);
}
// Utilities/Utility.hpp:27-37 -- complex: logCosh(Re) + log(cos(Im) + i tanh(Re) sin(Im))
inline cd logCosh(cd x) {
    const double xr = x.real(), xi = x.imag();
    cd res = logCosh(xr);
    res += std::log(cd{std::cos(xi), std::tanh(xr) * std::sin(xi)});
    return res;
}

// ---------------------------------------------------------------------------
// Machines/RBM.hpp -- a read-only view of an RBM<complex<double>>.
struct RBM {
    int n = 0, m = 0;
    bool useBias = true;
    const cd* p = nullptr;  // [W col-major | a | b]

    inline cd W(int j, int i) const { return p[size_t(i) * m + j]; }  // W(j,i), j<m, i<n
    inline cd A(int i) const { return useBias ? p[size_t(n) * m + i] : cd{}; }
    inline cd B(int j) const { return useBias ? p[size_t(n) * m + n + j] : cd{}; }
    inline size_t dim() const { return useBias ? size_t(n) * m + n + m : size_t(n) * m; }

    // RBM.hpp:137-141  theta = W sigma + b.  Summation order (i ascending, then
    // + b) is fixed so that the device sampler can reproduce theta bit for bit.
    void theta(const int8_t* s, cd* th) const {
        for (int j = 0; j < m; ++j) {
            cd acc = 0.;
            for (int i = 0; i < n; ++i) acc += W(j, i) * double(s[i]);
            th[j] = acc + B(j);
        }
    }
    // RBM.hpp:367-378
    cd logCoeff(const int8_t* s, const cd* th) const {
        cd r = 0.;
        for (int i = 0; i < n; ++i) r += A(i) * double(s[i]);
        for (int j = 0; j < m; ++j) r += logCosh(th[j]);
        return r;
    }
    // RBM.hpp:380-388  psi = exp(a.sigma) prod_j cosh(theta_j)
    cd coeff(const int8_t* s, const cd* th) const {
        cd r = 0.;
        for (int i = 0; i < n; ++i) r += A(i) * double(s[i]);
        cd prod = 1.;
        for (int j = 0; j < m; ++j) prod *= std::cosh(th[j]);
        return std::exp(r) * prod;
    }
    // RBM.hpp:390-406  O = [sigma_i tanh(theta_j) (i*m+j) | sigma | tanh(theta)]
    void logDeriv(const int8_t* s, const cd* th, cd* out) const {
        std::vector<cd> t(m);
        for (int j = 0; j < m; ++j) t[j] = std::tanh(th[j]);
        for (int i = 0; i < n; ++i)
            for (int j = 0; j < m; ++j) out[size_t(i) * m + j] = double(s[i]) * t[j];
        if (!useBias) return;
        for (int i = 0; i < n; ++i) out[size_t(n) * m + i] = double(s[i]);
        for (int j = 0; j < m; ++j) out[size_t(n) * m + n + j] = t[j];
    }

    // States/RBMState.hpp:48-63  log psi(sigma^k) - log psi(sigma)
    cd logRatio1(const int8_t* s, const cd* th, int k) const {
        cd res = -2.0 * A(k) * double(s[k]);
        for (int j = 0; j < m; ++j) res += logCosh(th[j] - 2.0 * double(s[k]) * W(j, k)) - logCosh(th[j]);
        return res;
    }
    // States/RBMState.hpp:78-94
    cd logRatio2(const int8_t* s, const cd* th, int k, int l) const {
        cd res = -2.0 * A(k) * double(s[k]) - 2.0 * A(l) * double(s[l]);
        for (int j = 0; j < m; ++j) {
            cd t = th[j] - 2.0 * double(s[k]) * W(j, k) - 2.0 * double(s[l]) * W(j, l);
            res += logCosh(t) - logCosh(th[j]);
        }
        return res;
    }
    // States/RBMState.hpp:108-127
    cd logRatioVec(const int8_t* s, const cd* th, int nf, const int* f) const {
        cd res = 0.;
        for (int e = 0; e < nf; ++e) res -= 2.0 * A(f[e]) * double(s[f[e]]);
        for (int j = 0; j < m; ++j) {
            cd t = th[j];
            for (int e = 0; e < nf; ++e) t -= 2.0 * double(s[f[e]]) * W(j, f[e]);
            res += logCosh(t) - logCosh(th[j]);
        }
        return res;
    }
    // States/RBMState.hpp:248-255  theta first, then sigma
    void flip1(int8_t* s, cd* th, int k) const {
        for (int j = 0; j < m; ++j) th[j] -= 2.0 * double(s[k]) * W(j, k);
        s[k] = int8_t(-s[k]);
    }
    // States/RBMState.hpp:257-266
    void flip2(int8_t* s, cd* th, int k, int l) const {
        for (int j = 0; j < m; ++j) th[j] += -2.0 * double(s[k]) * W(j, k) - 2.0 * double(s[l]) * W(j, l);
        s[k] = int8_t(-s[k]);
        s[l] = int8_t(-s[l]);
    }
    // States/RBMState.hpp:268-281
    void flipVec(int8_t* s, cd* th, int nf, const int* f) const {
        for (int e = 0; e < nf; ++e)
            for (int j = 0; j < m; ++j) th[j] -= 2.0 * double(s[f[e]]) * W(j, f[e]);
        for (int e = 0; e < nf; ++e) s[f[e]] = int8_t(-s[f[e]]);
    }
};

// Machines/RBM.hpp:325-349 -- draw order a[0..n), b[0..m), then W column by column,
// each complex entry (re, im).  The normal draws come from Philox + Box-Muller
// (reference: std::normal_distribution over an unseeded engine).
void init_params(int n, int m, bool useBias, uint64_t seed, double sd, cd* p);
double normal_pair(uint64_t seed, uint32_t idx, double* second);

// ---------------------------------------------------------------------------
// Hamiltonians.  kind: 0 = TFIsing (1D ring, Hamiltonians/TFIsing.hpp),
// 1 = XXZ (1D ring, Hamiltonians/XXZ.hpp), 2 = TFIsing2D (periodic Lx x Ly; no
// reference counterpart, built on the same duck-typed concept), 3 = XXX
// (Hamiltonians/XXX.hpp), 4 = J1J2 (Hamiltonians/J1J2.hpp), 5 = XYZNNN
// (Hamiltonians/XYZNNN.hpp), 6 = KitaevHex (Hamiltonians/KitaevHex.hpp).
enum HamKind { HAM_TFI = 0, HAM_XXZ = 1, HAM_TFI2D = 2, HAM_XXX = 3, HAM_J1J2 = 4, HAM_XYZNNN = 5, HAM_KITAEV = 6 };
struct Ham {
    int kind = 0;
    int n = 0;        // number of sites
    int lx = 0, ly = 0;  // 2D extents (TFI2D); KitaevHex: lx = n_ (even), ly = m_ rows (even)
    // TFI: J zz coupling, h field.  XXZ: J, h = Delta.  J1J2: J = J1, h = J2.
    // XYZNNN: J = a, h = b.  KitaevHex: J = Jx, jy, jz, h = field.
    double J = 0., h = 0.;
    double sign = 1.;       // XXZ / J1J2 sign rule (-1 when signRule)
    double jy = 0., jz = 0.;
};
// KitaevHex link lists (KitaevHex.hpp:33-103), pairs of site indices in the
// reference's order.
std::vector<std::pair<int, int>> kitaev_links(const Ham& H, int axis);  // axis 0 = x, 1 = y, 2 = z
// offDiagonals(s): the flips the HamiltonianSweeper proposes from ({a, -1} or {a, b})
std::vector<std::array<int, 2>> off_diagonals(const Ham& H, const int8_t* s);

// Off-diagonal flip enumeration of the state form (the "mock state" technique of
// Tests/HamiltonianHelper.hpp:44-92): each requested ratio becomes a (mask, coeff)
// entry; the diagonal sum is returned separately.  Entries with coefficient 0 are
// kept, as the reference state form requests them.
struct FlipTerm {
    uint64_t mask;
    double coeff;
};
double ham_enumerate(const Ham& H, const int8_t* s, std::vector<FlipTerm>& terms);
// Column form: Hamiltonians/TFIsing.hpp:53-65, Hamiltonians/XXZ.hpp:51-64 (std::map, zeros kept)
std::map<uint64_t, double> ham_column(const Ham& H, uint64_t col);
// State form: Hamiltonians/TFIsing.hpp:28-39, XXZ.hpp:37-49, with ratio = exp(logRatio)
cd ham_eloc(const Ham& H, const RBM& q, const int8_t* s, const cd* th);

// ---------------------------------------------------------------------------
// Samplers/LocalSweeper.hpp:32-53, Samplers/SwapSweeper.hpp:28-57, Samplers/SamplerMT.hpp:155-204
enum Move { MOVE_LOCAL = 0, MOVE_EXCHANGE_ANY = 1, MOVE_EXCHANGE_NN = 2, MOVE_HAMILTONIAN = 3 };
struct SampleSpec {
    int n_chains = 1;
    int move = MOVE_LOCAL;
    const Ham* ham = nullptr;  // MOVE_HAMILTONIAN: Samplers/HamiltonianSweeper.hpp:22-50
    int nup = -1;          // >=0: reinitialise with fixed magnetisation (randomSigma(n, nup))
    uint64_t seed = 0;
    uint32_t epoch = 0;
    int reinit = 1;        // draw fresh chains (RunRBM.hpp:166 sampler.randomize)
    int n_sweeps = 1;      // recorded sweeps
    int n_discard = 0;     // thermalisation sweeps
    int sweep_len = 0;     // proposals per sweep (0 -> n, LocalSweeper nSweep_=1)
};
void random_sigma(int n, int nup, uint64_t seed, uint32_t epoch, uint32_t chain, int8_t* s);
// SamplerMT with nTmps = ntemps > 1 (Samplers/SamplerMT.hpp:44-60, :120-204): chain c
// belongs to group c / ntemps; slot[c] is its place in the group's ladder, beta =
// (ntemps - slot) / ntemps.  Every sweep: each chain sweeps at its beta (proposal
// draws as in `sample`), then mixChains per group -- even slot pairs (0,1),(2,3),...
// then odd pairs (1,2),...,(ntemps-3, ntemps-2) -- accepts a swap with
// p = exp((beta_{t+1} - beta_t) 2 (Re log psi(slot t) - Re log psi(slot t+1))) and
// u from counter (64 sweep + t, epoch, group, TAG_PT); swapping exchanges the two
// chains' slots (temperatures) instead of their states.  Recorded sweeps append
// the slot-0 chain of every group: output row (sweep - n_discard) groups + group.
// The chain state (sigma, theta) carries over exactly from sweep to sweep; slot
// is in/out (reset to c % ntemps when sp.reinit).
void sample_pt(const RBM& q, const SampleSpec& sp, int ntemps, int8_t* chain_sigma, int* slot, int8_t* out_sigma,
               cd* out_theta, uint64_t* acc, int nthreads);
// chain_sigma: n_chains x n, in/out.  Outputs sample-major (sweep, chain).
void sample(const RBM& q, const SampleSpec& sp, int8_t* chain_sigma, int8_t* out_sigma, cd* out_theta,
            uint64_t* acc, int nthreads);

// ---------------------------------------------------------------------------
// Dense complex linear algebra restated without Eigen/MKL.
// Lower Cholesky in place (Eigen::LLT semantics): returns 0 on success, k+1 if pivot k <= 0.
int cholesky_lower(int nn, cd* A /* row-major nn x nn, lower used */);
void cholesky_solve(int nn, const cd* L, cd* x);  // x <- (L L^H)^{-1} x
// Eigen::ConjugateGradient<..., Lower|Upper, IdentityPreconditioner>: relative residual
// ||r||/||b|| < tol, at most maxit iterations (Eigen default 2*dim), x0 = 0.

// GroundState/SRMat.hpp:89-237 + GroundState/utils.hpp:12-51 restated.
struct SRResult {
    double energy = 0., energy_var = 0.;
    std::vector<cd> elocs, oloc, grad, v;
    int status = 0;
    int cg_iters = 0;
    double cg_relres = 0.;
};
enum SRMode { SR_S = 0, SR_T = 1 };
enum SRSolver { SOLVE_LLT = 0, SOLVE_CG = 1 };
// Builds O and E_loc from (sigma, theta) samples, centres O, forms F = O~^H E / Ns and
// solves (S + shift) v = F (S-mode, SRMat::solveExact / solveCG) or, in T-mode, the
// sample-space dual v = O~^H (O~ O~^H / Ns + shift)^{-1} (E - <E>) / Ns.
SRResult sr_step(const RBM& q, const Ham& H, int ns, const int8_t* sig, const cd* th, double shift, int mode,
                 int solver, double cgtol, int nthreads);

// GroundState/SRMatExact.hpp:97-132 restated (basis = sorted list of indices).
struct ExactResult {
    double energy = 0., energy_var = 0.;
    std::vector<cd> oloc, grad, S;  // S is P x P row-major
};
ExactResult exact_sr(const RBM& q, const Ham& H, const std::vector<uint64_t>& basis, int nthreads,
                     bool with_S = true);

// Samplers/ExactSampler.hpp:49-79 restated: CDF of the unnormalised |psi|^2 over the
// basis accumulated in long double, r = u * total with u from the exact-sampler
// stream (counter (i, epoch, 0, TAG_EXACT), u53 draw), accum.back() += 1e-8, then
// std::lower_bound.  Returns basis positions, one per sample.
std::vector<uint32_t> exact_sample(const RBM& q, const std::vector<uint64_t>& basis, int nsamples, uint64_t seed,
                                   uint32_t epoch, int nthreads);

// Basis/BasisFull.hpp:126-153, Basis/BasisJz.hpp:25-104
std::vector<uint64_t> basis_full(int n);
std::vector<uint64_t> basis_jz(int n, int nup);
// ED: sparse H over a basis (ED/ConstructSparseMat.hpp:32-57) + Lanczos (the reference has no eigensolver).
double ed_ground_energy(const Ham& H, const std::vector<uint64_t>& basis, int maxit, int nthreads);

// ---------------------------------------------------------------------------
// FeedForward: Conv1D(periodic) -> LnCosh -> FullyConnected -> LnCosh -> Sum
// (Machines/FeedForward.hpp:152-205; layers/Conv1D.hpp:144-225;
//  layers/FullyConnected.hpp:150-179; layers/activations.hpp:74-107; layers/Mean.hpp:92-125)
struct FFNet {
    int L = 0;          // input length (sites)
    int conv_out = 0;   // output channels (input channels = 1)
    int conv_k = 0;     // kernel size
    int fc_out = 0;     // fully connected output width
    // params: [conv kernel (conv_k x conv_out, column-major) | fc weight ((L*conv_out) x fc_out, column-major)]
    const double* p = nullptr;
    size_t dim() const { return size_t(conv_k) * conv_out + size_t(L) * conv_out * fc_out; }
};
double ff_forward(const FFNet& f, const int8_t* s);
void ff_backward(const FFNet& f, const int8_t* s, double* der);

// ---------------------------------------------------------------------------
// AmplitudePhase (Machines/AmplitudePhase.hpp:9-178): a real RBM<double> amplitude
// and a FeedForward<double> phase (Machines/FeedForward.hpp) of layers
// Conv1D (layers/Conv1D.hpp), FullyConnected (layers/FullyConnected.hpp) and the
// activation layers of layers/ActivationLayer.hpp / activations.hpp.
// psi(s) = sqrt(A(s)) exp(i pi phi(s)), A = exp(a.s + sum_j logCosh(theta_j)).
enum LayerType {
    L_CONV1D = 0, L_FC = 1,
    A_IDENTITY = 10, A_LNCOSH = 11, A_TANH = 12, A_WEAKTANH = 13, A_SIGMOID = 14, A_RELU = 15, A_LEAKYRELU = 16,
    A_HARDTANH = 17, A_SOFTSHRINK = 18, A_LEAKYHARDTANH = 19, A_SOFTSIGN = 20, A_COS = 21
};
struct Layer {
    int type = 0;
    int a = 0, b = 0, k = 0, stride = 1, bias = 0;  // Conv1D: in, out channels, kernel; FC: in, out
    double x = 0.;                                   // activation constant / slope
    int in_size = 0, out_size = 0;                   // set by ap_layout
    size_t npar = 0, off = 0;                        // parameters of the layer and their offset
};
struct APNet {
    int n = 0, m = 0;
    bool bias = true;
    std::vector<Layer> layers;
    size_t Pa = 0, Pp = 0;
    const double* p = nullptr;  // [amplitude RBM (reference layout) | phase layers in order]
};
void ap_layout(APNet& q);  // sizes and offsets; throws on a bad stack
std::vector<std::vector<double>> ap_phase_data(const APNet& q, const int8_t* s);   // FeedForward::makeData
void ap_phase_backward(const APNet& q, const std::vector<std::vector<double>>& data, double* der);
double ap_log_amp(const APNet& q, const int8_t* s);  // log A(s) = RBM<double>::logCoeff
void ap_log_deriv_amp(const APNet& q, const int8_t* s, double* out);  // RBM logDeriv / 2
void ap_init(const APNet& q, uint64_t seed, double sigma_amp, int mode, double* p);  // LeCun 0, Xavier 1, He 2
// GroundState/NGDExact.hpp:123-189 over a basis: energy, grad (Pa + Pp), oloc of
// both blocks, the two correlation matrices (row-major) when requested.
struct NGDResult {
    double energy = 0.;
    std::vector<double> grad, oloc_amp, oloc_phase, corr_amp, corr_phase;
};
NGDResult ngd_exact(const APNet& q, const Ham& H, const std::vector<uint64_t>& basis, bool with_corr, int nthreads);

}  // namespace orc
