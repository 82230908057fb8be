// yannq_gpu.hpp -- header-only C++ adapters over the C ABI of libyannq_b200.
//
// They keep the names and call pattern of yannq's template API so that a driver
// written against Yannq/Machines, Yannq/Samplers, Yannq/Hamiltonians,
// Yannq/GroundState and Yannq/Runners switches to the B200 backend by changing
// types, not code:
//
//   yannq::RBM<T>                      -> yannq::gpu::RBM<T>          (Machines/RBM.hpp)
//   TFIsing / XXZ                      -> yannq::gpu::TFIsing / XXZ   (Hamiltonians/*.hpp)
//   LocalSweeper / SwapSweeper         -> same names in yannq::gpu    (Samplers/*Sweeper.hpp)
//   SamplerMT<Machine, State, Sweeper> -> yannq::gpu::SamplerMT<Machine, Sweeper>
//   SRMat<Machine, Hamiltonian>        -> yannq::gpu::SRMat<Machine, Hamiltonian>
//   RunRBM<T>                          -> yannq::gpu::RunRBM<T>        (Runners/RunRBM.hpp)
//
// Parameters, samples and the SR solution stay on the device; vectors cross the
// boundary as std::vector<std::complex<double>> in the reference's layout
// [W column-major (m x n) | a | b].  Errors of the C ABI become yannq::gpu::Error.
#pragma once
#include <algorithm>
#include <chrono>
#include <cmath>
#include <complex>
#include <cstdint>
#include <cstdio>
#include <functional>
#include <random>
#include <stdexcept>
#include <string>
#include <type_traits>
#include <vector>

#include "../yannq_b200.h"

namespace yannq {
namespace gpu {

struct Error : std::runtime_error {
    int code;
    Error(int c, const std::string& m) : std::runtime_error(m), code(c) {}
};

inline void check(int code) {
    if (code != YQ_OK) {
        char buf[1024];
        yq_last_error(buf, sizeof(buf));
        if (code == YQ_E_ARG) throw std::invalid_argument(buf);
        throw Error(code, buf);
    }
}

using cd = std::complex<double>;

// One device and its stream (no reference counterpart: the reference is host-only).
class Context {
    yq_ctx h_ = nullptr;

public:
    explicit Context(int device = 0) { check(yq_ctx_create(device, &h_)); }
    ~Context() { yq_ctx_destroy(h_); }
    Context(const Context&) = delete;
    Context& operator=(const Context&) = delete;
    yq_ctx handle() const { return h_; }
    void synchronize() const { check(yq_ctx_synchronize(h_)); }
    // device milliseconds of the last call's stage: "sample", "eloc", "O", "gram", "solve", "update", "total"
    float stageMs(int stage) const {
        float ms = 0.f;
        check(yq_ctx_stage_ms(h_, stage, &ms));
        return ms;
    }
};

// Machines/RBM.hpp: RBM<T>(n, m, useBias) with T = std::complex<double> (FP64 path)
// or std::complex<float> (mixed-precision path).
template <typename T>
class RBM {
    static_assert(std::is_same<T, std::complex<double>>::value || std::is_same<T, std::complex<float>>::value,
                  "yannq::gpu::RBM supports complex<double> and complex<float>");
    yq_rbm h_ = nullptr;
    uint32_t n_, m_;
    bool useBias_;
    size_t dim_ = 0;

public:
    using Scalar = T;
    using RealScalar = typename T::value_type;
    using Vector = std::vector<cd>;

    RBM(Context& ctx, uint32_t n, uint32_t m, bool useBias = true) : n_(n), m_(m), useBias_(useBias) {
        check(yq_rbm_create(ctx.handle(), int(n), int(m), useBias ? 1 : 0,
                            std::is_same<T, std::complex<double>>::value ? YQ_C128 : YQ_C64, &h_));
        check(yq_rbm_dim(h_, &dim_));
    }
    ~RBM() { yq_rbm_destroy(h_); }
    RBM(const RBM&) = delete;
    RBM& operator=(const RBM&) = delete;

    yq_rbm handle() const { return h_; }
    uint32_t getN() const { return n_; }
    uint32_t getM() const { return m_; }
    uint32_t getDim() const { return uint32_t(dim_); }
    bool useBias() const { return useBias_; }

    // RBM.hpp:271-291
    Vector getParams() const {
        Vector p(dim_);
        check(yq_rbm_get_params(h_, reinterpret_cast<double*>(p.data())));
        return p;
    }
    void setParams(const Vector& p) {
        if (p.size() != dim_) throw std::invalid_argument("setParams: size != getDim()");
        check(yq_rbm_set_params(h_, reinterpret_cast<const double*>(p.data())));
    }
    // RBM.hpp:261-269
    void updateParams(const Vector& d) {
        if (d.size() != dim_) throw std::invalid_argument("updateParams: size != getDim()");
        check(yq_rbm_update_params(h_, reinterpret_cast<const double*>(d.data())));
    }
    // RBM.hpp:325-349 (Philox-seeded normal draws in the reference's order)
    void initializeRandom(uint64_t seed, double sigma = 1e-3) { check(yq_rbm_init_random(h_, seed, sigma)); }

    // cereal image of std::unique_ptr<RBM<T>> (Serializers/SerializeRBM.hpp), as RunRBM writes it
    static constexpr int archiveElem = std::is_same<T, std::complex<double>>::value ? YQ_ARCHIVE_C128 : YQ_ARCHIVE_C64;
    void save(const std::string& path) const { check(yq_rbm_save(h_, archiveElem, path.c_str())); }
    void load(const std::string& path) { check(yq_rbm_load(h_, archiveElem, path.c_str())); }

    // logCoeff over configurations (ns x n, entries +-1), RBM.hpp:367-378
    std::vector<cd> logCoeff(const std::vector<int8_t>& sigma) const {
        const int ns = int(sigma.size() / n_);
        std::vector<cd> out(ns);
        check(yq_rbm_log_psi(h_, ns, sigma.data(), reinterpret_cast<double*>(out.data())));
        return out;
    }
    // calcTheta over configurations, RBM.hpp:137-141
    std::vector<cd> calcTheta(const std::vector<int8_t>& sigma) const {
        const int ns = int(sigma.size() / n_);
        std::vector<cd> out(size_t(ns) * m_);
        check(yq_rbm_theta(h_, ns, sigma.data(), reinterpret_cast<double*>(out.data())));
        return out;
    }
    // logDeriv over (sigma, theta) samples, RBM.hpp:390-406 (row per sample)
    std::vector<cd> logDeriv(const std::vector<int8_t>& sigma, const std::vector<cd>& theta) const {
        const int ns = int(sigma.size() / n_);
        std::vector<cd> out(size_t(ns) * dim_);
        check(yq_rbm_log_deriv(h_, ns, sigma.data(), reinterpret_cast<const double*>(theta.data()),
                               reinterpret_cast<double*>(out.data())));
        return out;
    }
};

// Hamiltonians (duck-typed in the reference; here descriptors of device kernels)
class Hamiltonian {
    yq_ham h_ = nullptr;
    int n_;

protected:
    Hamiltonian(Context& ctx, int kind, int n, int lx, int ly, double J, double h, bool sign) : n_(n) {
        check(yq_ham_create(ctx.handle(), kind, n, lx, ly, J, h, sign ? 1 : 0, &h_));
    }
    Hamiltonian(int n, yq_ham h) : h_(h), n_(n) {}

public:
    virtual ~Hamiltonian() { yq_ham_destroy(h_); }
    Hamiltonian(const Hamiltonian&) = delete;
    Hamiltonian& operator=(const Hamiltonian&) = delete;
    yq_ham handle() const { return h_; }
    int size() const { return n_; }
};
// Hamiltonians/TFIsing.hpp: E_loc = sum_i J s_i s_{i+1} + h ratio(i)
struct TFIsing : Hamiltonian {
    TFIsing(Context& ctx, int n, double J, double h) : Hamiltonian(ctx, YQ_HAM_TFI, n, 0, 0, J, h, false) {}
};
// Hamiltonians/XXZ.hpp
struct XXZ : Hamiltonian {
    XXZ(Context& ctx, int n, double J, double Delta, bool signRule = false)
        : Hamiltonian(ctx, YQ_HAM_XXZ, n, 0, 0, J, Delta, signRule) {}
};
// periodic lx x ly square lattice (no reference counterpart)
struct TFIsing2D : Hamiltonian {
    TFIsing2D(Context& ctx, int lx, int ly, double J, double h)
        : Hamiltonian(ctx, YQ_HAM_TFI2D, lx * ly, lx, ly, J, h, false) {}
};
// Hamiltonians/XXX.hpp
struct XXX : Hamiltonian {
    XXX(Context& ctx, int n) : Hamiltonian(ctx, YQ_HAM_XXX, n, 0, 0, 0.0, 0.0, false) {}
};
// Hamiltonians/J1J2.hpp
struct J1J2 : Hamiltonian {
    J1J2(Context& ctx, int n, double J1, double J2, bool signRule)
        : Hamiltonian(ctx, YQ_HAM_J1J2, n, 0, 0, J1, J2, signRule) {}
};
// Hamiltonians/XYZNNN.hpp
struct XYZNNN : Hamiltonian {
    XYZNNN(Context& ctx, int n, double a, double b) : Hamiltonian(ctx, YQ_HAM_XYZNNN, n, 0, 0, a, b, false) {}
};
// Hamiltonians/KitaevHex.hpp: both reference constructors
struct KitaevHex : Hamiltonian {
    KitaevHex(Context& ctx, int n, int m, double J, double h = 0.0) : Hamiltonian(n * m, make(ctx, n, m, J, J, J, h)) {}
    KitaevHex(Context& ctx, int n, int m, double Jx, double Jy, double Jz)
        : Hamiltonian(n * m, make(ctx, n, m, Jx, Jy, Jz, 0.0)) {}

private:
    static yq_ham make(Context& ctx, int n, int m, double Jx, double Jy, double Jz, double h) {
        yq_ham out = nullptr;
        check(yq_ham_create_kitaev_hex(ctx.handle(), n, m, Jx, Jy, Jz, h, &out));
        return out;
    }
};

// Samplers/LocalSweeper.hpp, Samplers/SwapSweeper.hpp (+ neighbour-pair variant)
struct LocalSweeper {
    static constexpr int move = YQ_MOVE_LOCAL;
    uint32_t n;
    explicit LocalSweeper(uint32_t n_) : n(n_) {}
};
struct SwapSweeper {
    static constexpr int move = YQ_MOVE_EXCHANGE_ANY;
    uint32_t n;
    explicit SwapSweeper(uint32_t n_) : n(n_) {}
};
struct SwapSweeperNN {
    static constexpr int move = YQ_MOVE_EXCHANGE_NN;
    uint32_t n;
    explicit SwapSweeperNN(uint32_t n_) : n(n_) {}
};
// Samplers/HamiltonianSweeper.hpp:16-19: proposals from ham's offDiagonals list
template <class Ham>
struct HamiltonianSweeper {
    static constexpr int move = YQ_MOVE_HAMILTONIAN;
    uint32_t n;
    const Ham& ham;
    HamiltonianSweeper(int n_, const Ham& h) : n(uint32_t(n_)), ham(h) {}
    yq_ham proposals() const { return ham.handle(); }
};

namespace detail {
template <class S>
auto sweeper_ham(const S& s, int) -> decltype(s.proposals()) {
    return s.proposals();
}
template <class S>
yq_ham sweeper_ham(const S&, long) {
    return nullptr;
}
}  // namespace detail

// Utilities/Utility.hpp:61-88: random configurations on the host, for the
// randomizer functors a RunRBM driver passes to run() (entries +-1; nup values of -1).
template <class RandomEngine>
std::vector<int> randomSigma(int n, RandomEngine& re) {
    std::vector<int> sigma(static_cast<size_t>(n));
    std::uniform_int_distribution<> uid(0, 1);
    for (int i = 0; i < n; ++i) sigma[size_t(i)] = -2 * uid(re) + 1;
    return sigma;
}
template <class RandomEngine>
std::vector<int> randomSigma(int n, int nup, RandomEngine& re) {
    std::vector<int> sigma(size_t(n), -1);
    for (int i = nup; i < n; ++i) sigma[size_t(i)] = 1;
    std::shuffle(sigma.begin(), sigma.end(), re);
    return sigma;
}
// A randomizer that draws the chains on the device (the sampler's own Philox
// randomSigma, with its nup) instead of calling a host functor per chain.
struct DeviceRandomSigma {};

// Samples of the last sample() call; they stay on the device.
struct SampleSet {
    yq_sampler sampler;
    int ns;
    std::size_t size() const { return std::size_t(ns); }
};

// Samplers/SamplerMT.hpp: nTmps temperatures x nChainsPer chains (nTmps = 1 or even;
// parallel tempering swaps temperatures between the chains of a group).
template <class Machine, class Sweeper>
class SamplerMT {
    yq_sampler h_ = nullptr;
    uint64_t seed_ = 0;
    uint32_t epoch_ = 0;
    bool reinit_ = true;
    uint32_t nChains_ = 0, n_ = 0;
    std::default_random_engine re_;

public:
    using RandomEngine = std::default_random_engine;
    SamplerMT(const Machine& qs, uint32_t nTmps, uint32_t nChainsPer, const Sweeper& sw, int nup = -1)
        : nChains_(nTmps * nChainsPer), n_(qs.getN()) {
        if (nTmps == 0 || (nTmps != 1 && nTmps % 2 != 0))
            throw std::invalid_argument("SamplerMT: nTmps must be 1 or even");  // SamplerMT.hpp:50
        if (sw.n != qs.getN()) throw std::invalid_argument("SamplerMT: sweeper size differs from the machine");
        check(yq_sampler_create(qs.handle(), int(nTmps * nChainsPer), Sweeper::move, nup, 0, &h_));
        if (yq_ham hm = detail::sweeper_ham(sw, 0)) check(yq_sampler_set_hamiltonian(h_, hm));
        if (nTmps > 1) check(yq_sampler_set_tempering(h_, int(nTmps)));
    }
    ~SamplerMT() { yq_sampler_destroy(h_); }
    SamplerMT(const SamplerMT&) = delete;
    SamplerMT& operator=(const SamplerMT&) = delete;
    yq_sampler handle() const { return h_; }

    // SamplerMT.hpp:72-79, seeded instead of from std::random_device: the device's
    // Philox streams and the host engine handed to randomizers both derive from seed
    void initializeRandomEngine(uint64_t seed = 0) {
        seed_ = seed;
        re_.seed(static_cast<std::default_random_engine::result_type>(seed ^ (seed >> 32)));
    }
    // SamplerMT.hpp:103-110: fresh random chains at the next sample() call
    void randomize() { reinit_ = true; }
    void randomize(DeviceRandomSigma) { reinit_ = true; }
    // SamplerMT.hpp:103-110 with a randomizer functor: chain c starts from
    // randomizer(re) (any container of +-1 with size() and operator[], e.g.
    // std::vector<int> or Eigen::VectorXi), drawn on the host and uploaded.
    template <class Randomizer,
              class = decltype(std::declval<Randomizer&>()(std::declval<std::default_random_engine&>()))>
    void randomize(Randomizer&& randomizer) {
        std::vector<int8_t> chains(size_t(nChains_) * n_);
        for (uint32_t c = 0; c < nChains_; ++c) {
            const auto sigma = randomizer(re_);
            if (size_t(sigma.size()) != size_t(n_))
                throw std::invalid_argument("randomize: the randomizer returned a configuration of the wrong size");
            for (uint32_t i = 0; i < n_; ++i) {
                const int v = int(sigma[i]);
                if (v != 1 && v != -1) throw std::invalid_argument("randomize: configurations must hold +-1");
                chains[size_t(c) * n_ + i] = int8_t(v);
            }
        }
        check(yq_sampler_set_chains(h_, chains.data()));
        reinit_ = false;
    }
    // keep the chains across calls (persistent Markov chains)
    void keepChains() { reinit_ = false; }
    // SamplerMT.hpp:180-204
    SampleSet sample(uint32_t nSweeps, uint32_t nDiscard) {
        check(yq_sample(h_, int(nSweeps), int(nDiscard), seed_, epoch_++, reinit_ ? 1 : 0));
        int ns = 0;
        check(yq_sampler_num_samples(h_, &ns));
        return SampleSet{h_, ns};
    }
    void setEpoch(uint32_t e) { epoch_ = e; }
    bool reinit() const { return reinit_; }
    uint64_t seed() const { return seed_; }
    uint32_t epoch() const { return epoch_; }
};

// GroundState/SRMat.hpp
template <class Machine, class Ham>
class SRMat {
    yq_sr h_ = nullptr;
    const Machine& qs_;

public:
    template <class Sampler>
    SRMat(const Machine& qs, const Ham& ham, const Sampler& sampler, int mode = YQ_SR_AUTO)
        : qs_(qs) {
        const int prec = std::is_same<typename Machine::Scalar, std::complex<float>>::value ? YQ_PREC_MIXED
                                                                                            : YQ_PREC_FP64;
        check(yq_sr_create(qs.handle(), ham.handle(), sampler.handle(), prec == YQ_PREC_MIXED ? YQ_SR_T : mode, prec,
                           &h_));
    }
    ~SRMat() { yq_sr_destroy(h_); }
    SRMat(const SRMat&) = delete;
    SRMat& operator=(const SRMat&) = delete;
    yq_sr handle() const { return h_; }

    // SRMat.hpp:89-103 (the sample set must come from the bound sampler)
    void constructFromSamples(const SampleSet&) { check(yq_sr_construct(h_)); }
    // SRMat.hpp:151-159
    double eloc() const {
        double e, v;
        check(yq_sr_energy(h_, &e, &v));
        return e;
    }
    double elocVar() const {
        double e, v;
        check(yq_sr_energy(h_, &e, &v));
        return v;
    }
    std::vector<cd> energyGrad() const { return get(2, qs_.getDim()); }
    std::vector<cd> oloc() const { return get(1, qs_.getDim()); }
    // SRMat.hpp:231-237
    std::vector<cd> solveExact(double shift) {
        std::vector<cd> v(qs_.getDim());
        check(yq_sr_solve(h_, shift, YQ_SOLVE_LLT, 0.0, reinterpret_cast<double*>(v.data()), nullptr, nullptr));
        return v;
    }
    // SRMat.hpp:197-208
    std::vector<cd> solveCG(double shift, double tol = 1e-4, int* iters = nullptr, double* relres = nullptr) {
        std::vector<cd> v(qs_.getDim());
        check(yq_sr_solve(h_, shift, YQ_SOLVE_CG, tol, reinterpret_cast<double*>(v.data()), iters, relres));
        return v;
    }
    // SRMat.hpp:142-149 (lower triangle of S or of the dual T, without shift)
    std::vector<cd> corrMat(int* dim) {
        check(yq_sr_matrix(h_, dim, nullptr));
        std::vector<cd> out(size_t(*dim) * size_t(*dim));
        check(yq_sr_matrix(h_, dim, reinterpret_cast<double*>(out.data())));
        return out;
    }

private:
    std::vector<cd> get(int which, size_t n) const {
        std::vector<cd> out(n);
        check(yq_sr_get(h_, which, reinterpret_cast<double*>(out.data())));
        return out;
    }
};

// Optimizers/SGD.hpp: update = -max(alpha / t^p, 1e-4) v
struct SGD {
    double alpha = 0.05, p = 0.0;
    int t = 0;
    double eta() {
        ++t;
        return std::max(alpha / std::pow(double(t), p), 1e-4);
    }
};

// Runners/RunRBM.hpp:123-222: the epoch loop on the device.
template <typename T>
class RunRBM {
    Context& ctx_;
    RBM<T> qs_;
    double lambdaIni_ = 1e-3, lambdaDecay_ = 1.0, lambdaMin_ = 1e-4;
    int maxIter_ = 2000, saveWfPer_ = 0;
    bool useCG_ = false;
    double cgTol_ = 1e-4;
    double gradClip_ = 0.0;
    double beta1_ = 0.0, beta2_ = 0.0;
    uint64_t seed_ = 0;
    SGD opt_;
    bool initialized_ = false;

public:
    RunRBM(Context& ctx, unsigned N, unsigned alpha, bool useBias) : ctx_(ctx), qs_(ctx, N, alpha * N, useBias) {}
    // seed of the parameter initialisation and of the sampler's streams used by the
    // reference-shaped run() (the reference seeds from std::random_device)
    void setSeed(uint64_t seed) { seed_ = seed; }
    RBM<T>& getQs() { return qs_; }
    void initializeRandom(uint64_t seed, double wIni = 1e-3) {
        qs_.initializeRandom(seed, wIni);
        initialized_ = true;
    }
    // AbstractRunner.hpp:96-101: N(0, wIni^2) parameters from the runner's seed (setSeed)
    void initializeRandom(double wIni) { initializeRandom(seed_, wIni); }
    void setLambda(double ini, double decay = 1.0, double mn = 0.0) {
        lambdaIni_ = ini;
        lambdaDecay_ = decay;
        lambdaMin_ = mn;
    }
    // AbstractRunner.hpp:83-94: start from a checkpoint written by RunRBM (the
    // file's N, M and useBias must match this runner's machine)
    void initializeFrom(const std::string& path) {
        qs_.load(path);
        initialized_ = true;
    }
    // saveWfPer != 0: the parameters are saved to w%04d.dat (working directory)
    // before every epoch ll with ll % saveWfPer == 0 (RunRBM.hpp:155-164)
    void setIterParams(int maxIter, int saveWfPer) {
        maxIter_ = maxIter;
        saveWfPer_ = saveWfPer;
    }
    void setOptimizer(const SGD& opt) { opt_ = opt; }
    void setSolverParams(bool useCG, double cgTol = 1e-4) {
        useCG_ = useCG;
        cgTol_ = cgTol;
    }
    void setGradClip(double clip) { gradClip_ = clip; }
    // RunRBM.hpp:73-77: ObsAvg weights of the gradient and of the Fisher matrix
    // (beta2 != 0 needs the S-form, i.e. nSweeps x chains >= getDim() on the FP64 path)
    void setMomentum(double beta1 = 0.0, double beta2 = 0.0) {
        beta1_ = beta1;
        beta2_ = beta2;
    }

    // Runners/RunRBM.hpp:123-222 with the reference's signature: every epoch ll
    // (0 .. maxIter) saves w%04d.dat when due, calls sampler.randomize(randomizer)
    // (a host functor randomizer(re) -> configuration, or DeviceRandomSigma{}),
    // samples nSweeps (default getDim()) after nSweepsDiscard (default 0.1 nSweeps)
    // sweeps, and runs constructFromSamples, the momentum-averaged LLT or CG solve,
    // the clip and the SGD step on the device in one yq_vmc_iteration;
    // callback(ll, currE, nv, cgErr, smp_ms, slv_ms).
    template <class Sampler, class Callback, class SweeperRandomizer, class Ham,
              class = typename std::enable_if<std::is_base_of<Hamiltonian, typename std::decay<Ham>::type>::value>::type>
    void run(Sampler& sampler, Callback&& callback, SweeperRandomizer&& randomizer, Ham&& ham, int nSweeps = -1,
             int nSweepsDiscard = -1) {
        if (!initialized_) initializeRandom(seed_, 1e-3);
        SRMat<RBM<T>, typename std::decay<Ham>::type> srm(qs_, ham, sampler);
        check(yq_sr_set_momentum(srm.handle(), beta1_, beta2_));
        check(yq_sr_set_grad_clip(srm.handle(), gradClip_));
        sampler.initializeRandomEngine(seed_);
        const int dim = int(qs_.getDim());
        if (nSweeps == -1) nSweeps = dim;
        if (nSweepsDiscard == -1) nSweepsDiscard = int(0.1 * nSweeps);
        for (int ll = 0; ll <= maxIter_; ++ll) {
            if (saveWfPer_ != 0 && ll % saveWfPer_ == 0) {
                char fileName[30];
                std::snprintf(fileName, sizeof(fileName), "w%04d.dat", ll);
                qs_.save(fileName);
            }
            sampler.randomize(randomizer);
            const double lambda = std::max(lambdaIni_ * std::pow(lambdaDecay_, ll), lambdaMin_);
            yq_iter_params p{nSweeps, nSweepsDiscard, sampler.reinit() ? 1 : 0, sampler.seed(), uint32_t(ll), lambda,
                             opt_.eta(), useCG_ ? YQ_SOLVE_CG : YQ_SOLVE_LLT, cgTol_,
                             std::is_same<T, std::complex<float>>::value ? 2 : 0};
            yq_iter_result r;
            check(yq_vmc_iteration(srm.handle(), &p, &r));
            callback(ll, r.energy, r.update_norm, r.cg_err, ctx_.stageMs(0), ctx_.stageMs(4));
        }
    }

    // The same loop with the chains' randomisation left to the sampler (randomize()
    // for fresh device chains every epoch, keepChains() for persistent chains) and
    // an explicit seed; callback(ll, currE, nv, cgErr, smp_ms, slv_ms) as RunRBM.hpp:219
    template <class Sampler, class Ham, class Callback>
    void run(Sampler& sampler, Callback&& callback, Ham& ham, int nSweeps, int nSweepsDiscard = -1,
             uint64_t seed = 0) {
        if (!initialized_) initializeRandom(seed, 1e-3);
        if (nSweepsDiscard < 0) nSweepsDiscard = int(0.1 * nSweeps);
        SRMat<RBM<T>, Ham> srm(qs_, ham, sampler);
        check(yq_sr_set_momentum(srm.handle(), beta1_, beta2_));
        check(yq_sr_set_grad_clip(srm.handle(), gradClip_));
        sampler.initializeRandomEngine(seed);
        for (int ll = 0; ll <= maxIter_; ++ll) {
            if (saveWfPer_ != 0 && ll % saveWfPer_ == 0) {
                char fileName[30];
                std::snprintf(fileName, sizeof(fileName), "w%04d.dat", ll);
                qs_.save(fileName);
            }
            const double lambda = std::max(lambdaIni_ * std::pow(lambdaDecay_, ll), lambdaMin_);
            yq_iter_params p{nSweeps, nSweepsDiscard, sampler.reinit() ? 1 : 0, seed, uint32_t(ll), lambda,
                             opt_.eta(), useCG_ ? YQ_SOLVE_CG : YQ_SOLVE_LLT, cgTol_,
                             std::is_same<T, std::complex<float>>::value ? 2 : 0};
            yq_iter_result r;
            check(yq_vmc_iteration(srm.handle(), &p, &r));
            callback(ll, r.energy, r.update_norm, r.cg_err, ctx_.stageMs(0), ctx_.stageMs(4));
        }
    }
};

// ---------------------------------------------------------------------------
// Machines/FeedForward.hpp with the layer names of Machines/layers: phase networks
// are built as in the reference, ff.addLayer<Conv1D>(1, 12, 5, 1, false) or
// ff.addLayer<LeakyHardTanh>(0.01), and handed to AmplitudePhase.
struct Conv1D {
    static void encode(std::vector<int>& d, std::vector<double>& x, int in, int out, int kernel, int stride = 1,
                       bool useBias = false) {
        d.insert(d.end(), {YQ_LAYER_CONV1D, in, out, kernel, stride, useBias ? 1 : 0});
        x.push_back(0.0);
    }
};
struct FullyConnected {
    static void encode(std::vector<int>& d, std::vector<double>& x, int in, int out, bool useBias = true) {
        d.insert(d.end(), {YQ_LAYER_FC, in, out, 0, 1, useBias ? 1 : 0});
        x.push_back(0.0);
    }
};
template <int Type>
struct Activation {
    static void encode(std::vector<int>& d, std::vector<double>& x, double c = Type == YQ_ACT_TANH || Type == YQ_ACT_COS ? 1.0
                                                                              : Type == YQ_ACT_LEAKYRELU     ? 0.1
                                                                              : Type == YQ_ACT_LEAKYHARDTANH ? 0.01
                                                                                                             : 0.0) {
        d.insert(d.end(), {Type, 0, 0, 0, 1, 0});
        x.push_back(c);
    }
};
using Identity = Activation<YQ_ACT_IDENTITY>;
using LnCosh = Activation<YQ_ACT_LNCOSH>;
using Tanh = Activation<YQ_ACT_TANH>;
using WeakTanh = Activation<YQ_ACT_WEAKTANH>;
using Sigmoid = Activation<YQ_ACT_SIGMOID>;
using ReLU = Activation<YQ_ACT_RELU>;
using LeakyReLU = Activation<YQ_ACT_LEAKYRELU>;
using HardTanh = Activation<YQ_ACT_HARDTANH>;
using SoftShrink = Activation<YQ_ACT_SOFTSHRINK>;
using LeakyHardTanh = Activation<YQ_ACT_LEAKYHARDTANH>;
using SoftSign = Activation<YQ_ACT_SOFTSIGN>;
using Cos = Activation<YQ_ACT_COS>;

class FeedForward {
    std::vector<int> desc_;
    std::vector<double> x_;

public:
    template <class Layer, typename... Ts>
    void addLayer(Ts&&... args) {
        Layer::encode(desc_, x_, std::forward<Ts>(args)...);
    }
    int numLayers() const { return int(x_.size()); }
    const std::vector<int>& desc() const { return desc_; }
    const std::vector<double>& x() const { return x_; }
};

enum class InitializationMode { LeCun = YQ_INIT_LECUN, Xavier = YQ_INIT_XAVIER, He = YQ_INIT_HE };

// Machines/AmplitudePhase.hpp:9-178: psi = sqrt(A) exp(i pi phi); real parameters
class AmplitudePhase {
    yq_ap h_ = nullptr;
    uint32_t n_;
    size_t dimAmp_ = 0, dimPhase_ = 0;

public:
    using RealVector = std::vector<double>;
    AmplitudePhase(Context& ctx, uint32_t N, uint32_t M, bool useBias, FeedForward&& phase) : n_(N) {
        check(yq_ap_create(ctx.handle(), int(N), int(M), useBias ? 1 : 0, phase.numLayers(), phase.desc().data(),
                           phase.x().data(), &h_));
        check(yq_ap_dims(h_, &dimAmp_, &dimPhase_));
    }
    ~AmplitudePhase() { yq_ap_destroy(h_); }
    AmplitudePhase(const AmplitudePhase&) = delete;
    AmplitudePhase& operator=(const AmplitudePhase&) = delete;
    yq_ap handle() const { return h_; }
    uint32_t getN() const { return n_; }
    uint32_t getDimAmp() const { return uint32_t(dimAmp_); }
    uint32_t getDimPhase() const { return uint32_t(dimPhase_); }
    uint32_t getDim() const { return uint32_t(dimAmp_ + dimPhase_); }
    // AmplitudePhase.hpp:92-97 (amplitude N(0, sigma^2), phase by mode; Xavier in the reference)
    void initializeRandom(uint64_t seed, double sigma, InitializationMode mode = InitializationMode::Xavier) {
        check(yq_ap_init_random(h_, seed, sigma, int(mode)));
    }
    RealVector getParams() const {
        RealVector p(getDim());
        check(yq_ap_get_params(h_, p.data()));
        return p;
    }
    void setParams(const RealVector& p) {
        if (p.size() != getDim()) throw std::invalid_argument("setParams: size != getDim()");
        check(yq_ap_set_params(h_, p.data()));
    }
    void updateParams(const RealVector& d) {
        if (d.size() != getDim()) throw std::invalid_argument("updateParams: size != getDim()");
        check(yq_ap_update_params(h_, d.data()));
    }
};

// Basis/BasisFull.hpp, Basis/BasisJz.hpp
struct BasisFull {
    uint32_t n;
    static constexpr int kind = YQ_BASIS_FULL;
    int nup() const { return 0; }
};
struct BasisJz {
    uint32_t n, nup_;
    static constexpr int kind = YQ_BASIS_JZ;
    BasisJz(uint32_t n_, uint32_t nup) : n(n_), nup_(nup) {}
    int nup() const { return int(nup_); }
};

// GroundState/NGDExact.hpp:18-211 (the Hamiltonian's column form is applied on the device)
class NGDExact {
    yq_ngd h_ = nullptr;
    const AmplitudePhase& qs_;
    double energy_ = 0.;

    std::vector<double> get(int what, size_t count) const {
        std::vector<double> out(count);
        check(yq_ngd_get(h_, what, out.data()));
        return out;
    }

public:
    template <class Basis, class Ham>
    NGDExact(const AmplitudePhase& qs, const Basis& basis, const Ham& ham) : qs_(qs) {
        check(yq_ngd_create(qs.handle(), ham.handle(), Basis::kind, basis.nup(), &h_));
    }
    ~NGDExact() { yq_ngd_destroy(h_); }
    NGDExact(const NGDExact&) = delete;
    NGDExact& operator=(const NGDExact&) = delete;
    yq_ngd handle() const { return h_; }
    void constructExact() { check(yq_ngd_construct(h_, &energy_)); }
    double eloc() const { return energy_; }
    double getEnergy() const { return energy_; }
    std::vector<double> energyGrad() const { return get(YQ_NGD_GRAD, qs_.getDim()); }
    std::vector<double> olocAmp() const { return get(YQ_NGD_OLOC_AMP, qs_.getDimAmp()); }
    std::vector<double> olocPhase() const { return get(YQ_NGD_OLOC_PHASE, qs_.getDimPhase()); }
    std::vector<double> corrMatAmp() const { return get(YQ_NGD_CORR_AMP, size_t(qs_.getDimAmp()) * qs_.getDimAmp()); }
    std::vector<double> corrMatPhase() const {
        return get(YQ_NGD_CORR_PHASE, size_t(qs_.getDimPhase()) * qs_.getDimPhase());
    }
};

enum class Mode { AMP = YQ_NGD_AMP, PHASE = YQ_NGD_PHASE, ALL = YQ_NGD_ALL };

// Runners/RunAmplitudePhase.hpp:12-122
class RunAmplitudePhaseExact {
    AmplitudePhase qs_;
    double lambdaIni_ = 1e-3, lambdaDecay_ = 1.0, lambdaMin_ = 1e-4;
    int maxIter_ = 2000;
    SGD opt_;

public:
    RunAmplitudePhaseExact(Context& ctx, uint32_t N, uint32_t alpha, bool useBias, FeedForward&& phase)
        : qs_(ctx, N, N * alpha, useBias, std::move(phase)) {}
    AmplitudePhase& getQs() { return qs_; }
    void initializeRandom(uint64_t seed, double sigma) { qs_.initializeRandom(seed, sigma); }
    void setLambda(double ini, double decay = 1.0, double mn = 0.0) {
        lambdaIni_ = ini;
        lambdaDecay_ = decay;
        lambdaMin_ = mn;
    }
    // saveWfPer: the reference archives the whole machine; not built for AmplitudePhase
    void setIterParams(int maxIter, int /*saveWfPer*/) { maxIter_ = maxIter; }
    void setOptimizer(const SGD& opt) { opt_ = opt; }

    // callback(ll, currE, |grad|, |v|) as RunAmplitudePhase.hpp:119
    template <class Callback, class Basis, class Ham>
    void run(Callback&& callback, const Basis& basis, const Ham& ham, Mode mode = Mode::ALL) {
        NGDExact ngd(qs_, basis, ham);
        for (int ll = 0; ll <= maxIter_; ++ll) {
            const double lambda = std::max(lambdaIni_ * std::pow(lambdaDecay_, ll), lambdaMin_);
            double e = 0., gn = 0., vn = 0.;
            check(yq_ngd_iteration(ngd.handle(), lambda, opt_.eta(), int(mode), &e, &gn, &vn));
            callback(ll, e, gn, vn);
        }
    }
};

}  // namespace gpu
}  // namespace yannq
