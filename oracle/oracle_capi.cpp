// C entry points of the oracle for the Python test harness (ctypes).
// TEST INFRASTRUCTURE ONLY: see oracle.hpp.  Complex arrays are interleaved doubles.
#include <cstring>

#include "oracle.hpp"

using namespace orc;

namespace {
RBM make_rbm(int n, int m, int use_bias, const double* params) {
    RBM q;
    q.n = n;
    q.m = m;
    q.useBias = use_bias != 0;
    q.p = reinterpret_cast<const cd*>(params);
    return q;
}
// hp = {J, h, sign, jy, jz} (the Ham fields of the same names)
Ham make_ham(int kind, int n, int lx, int ly, const double* hp) {
    Ham H;
    H.kind = kind;
    H.n = n;
    H.lx = lx;
    H.ly = ly;
    H.J = hp[0];
    H.h = hp[1];
    H.sign = hp[2];
    H.jy = hp[3];
    H.jz = hp[4];
    return H;
}
// Phase layers: desc holds 6 ints per layer (type, a, b, k, stride, bias), xs one
// double (activation constant / slope).
APNet make_ap(int n, int m, int use_bias, int nl, const int* desc, const double* xs, const double* p) {
    APNet q;
    q.n = n;
    q.m = m;
    q.bias = use_bias != 0;
    for (int l = 0; l < nl; ++l) {
        Layer L;
        L.type = desc[6 * l];
        L.a = desc[6 * l + 1];
        L.b = desc[6 * l + 2];
        L.k = desc[6 * l + 3];
        L.stride = desc[6 * l + 4];
        L.bias = desc[6 * l + 5];
        L.x = xs[l];
        q.layers.push_back(L);
    }
    ap_layout(q);
    q.p = p;
    return q;
}
}  // namespace

extern "C" {

void orc_philox(const uint32_t* ctr, const uint32_t* key, uint32_t* out) { Philox4x32::generate(ctr, key, out); }

void orc_logcosh(const double* z, double* out) {
    cd r = logCosh(cd{z[0], z[1]});
    out[0] = r.real();
    out[1] = r.imag();
}
double orc_logcosh_real(double x) { return logCosh(x); }

void orc_init_params(int n, int m, int use_bias, uint64_t seed, double sd, double* params) {
    init_params(n, m, use_bias != 0, seed, sd, reinterpret_cast<cd*>(params));
}

void orc_theta(int n, int m, int use_bias, const double* params, const int8_t* s, double* theta) {
    make_rbm(n, m, use_bias, params).theta(s, reinterpret_cast<cd*>(theta));
}

void orc_logpsi(int n, int m, int use_bias, const double* params, const int8_t* s, double* out) {
    RBM q = make_rbm(n, m, use_bias, params);
    std::vector<cd> th(m);
    q.theta(s, th.data());
    cd r = q.logCoeff(s, th.data());
    out[0] = r.real();
    out[1] = r.imag();
}

void orc_psi(int n, int m, int use_bias, const double* params, const int8_t* s, double* out) {
    RBM q = make_rbm(n, m, use_bias, params);
    std::vector<cd> th(m);
    q.theta(s, th.data());
    cd r = q.coeff(s, th.data());
    out[0] = r.real();
    out[1] = r.imag();
}

void orc_logratio(int n, int m, int use_bias, const double* params, const int8_t* s, const double* theta, int nf,
                  const int* f, double* out) {
    RBM q = make_rbm(n, m, use_bias, params);
    const cd* th = reinterpret_cast<const cd*>(theta);
    cd r = nf == 1 ? q.logRatio1(s, th, f[0]) : nf == 2 ? q.logRatio2(s, th, f[0], f[1]) : q.logRatioVec(s, th, nf, f);
    out[0] = r.real();
    out[1] = r.imag();
}

void orc_flip(int n, int m, int use_bias, const double* params, int8_t* s, double* theta, int nf, const int* f) {
    RBM q = make_rbm(n, m, use_bias, params);
    cd* th = reinterpret_cast<cd*>(theta);
    if (nf == 1)
        q.flip1(s, th, f[0]);
    else if (nf == 2)
        q.flip2(s, th, f[0], f[1]);
    else
        q.flipVec(s, th, nf, f);
}

void orc_logderiv(int n, int m, int use_bias, const double* params, const int8_t* s, const double* theta,
                  double* out) {
    make_rbm(n, m, use_bias, params).logDeriv(s, reinterpret_cast<const cd*>(theta), reinterpret_cast<cd*>(out));
}

// constructDelta (GroundState/utils.hpp:12-51): one logDeriv row per sample, OpenMP over samples.
void orc_logderiv_batch(int n, int m, int use_bias, const double* params, int ns, const int8_t* s,
                        const double* theta, double* out, int nthreads) {
    RBM q = make_rbm(n, m, use_bias, params);
    const cd* th = reinterpret_cast<const cd*>(theta);
    cd* o = reinterpret_cast<cd*>(out);
    const size_t P = q.dim();
#pragma omp parallel for schedule(static) num_threads(nthreads > 0 ? nthreads : 1)
    for (int k = 0; k < ns; ++k) q.logDeriv(s + size_t(k) * n, th + size_t(k) * m, o + size_t(k) * P);
}

// Hamiltonian: kind 0 TFI ring, 1 XXZ ring, 2 TFI 2D torus, 3 XXX, 4 J1J2, 5 XYZNNN,
// 6 KitaevHex (oracle.hpp HamKind).
double orc_ham_enumerate(int kind, int n, int lx, int ly, const double* hp, const int8_t* s,
                         uint64_t* masks, double* coeffs, int cap, int* count) {
    Ham H = make_ham(kind, n, lx, ly, hp);
    std::vector<FlipTerm> t;
    double d = ham_enumerate(H, s, t);
    int c = 0;
    for (auto& e : t) {
        if (c < cap) {
            masks[c] = e.mask;
            coeffs[c] = e.coeff;
        }
        ++c;
    }
    *count = c;
    return d;
}

int orc_ham_column(int kind, int n, int lx, int ly, const double* hp, uint64_t col, uint64_t* rows,
                   double* vals, int cap) {
    Ham H = make_ham(kind, n, lx, ly, hp);
    auto mp = ham_column(H, col);
    int c = 0;
    for (auto& kv : mp) {
        if (c < cap) {
            rows[c] = kv.first;
            vals[c] = kv.second;
        }
        ++c;
    }
    return c;
}

void orc_eloc(int kind, int n, int lx, int ly, const double* hp, int m, int use_bias,
              const double* params, int ns, const int8_t* s, const double* theta, double* out, int nthreads) {
    Ham H = make_ham(kind, n, lx, ly, hp);
    RBM q = make_rbm(n, m, use_bias, params);
    const cd* th = reinterpret_cast<const cd*>(theta);
    cd* o = reinterpret_cast<cd*>(out);
#pragma omp parallel for schedule(static) num_threads(nthreads > 0 ? nthreads : 1)
    for (int k = 0; k < ns; ++k) o[k] = ham_eloc(H, q, s + size_t(k) * n, th + size_t(k) * m);
}

void orc_random_sigma(int n, int nup, uint64_t seed, uint32_t epoch, uint32_t chain, int8_t* s) {
    random_sigma(n, nup, seed, epoch, chain, s);
}

void orc_sample(int n, int m, int use_bias, const double* params, int n_chains, int move, int nup, uint64_t seed,
                uint32_t epoch, int reinit, int n_sweeps, int n_discard, int sweep_len, int8_t* chain_sigma,
                int8_t* out_sigma, double* out_theta, uint64_t* acc, int nthreads, int ham_kind, int ham_lx,
                int ham_ly, const double* ham_hp) {
    RBM q = make_rbm(n, m, use_bias, params);
    Ham H;
    if (ham_hp) H = make_ham(ham_kind, n, ham_lx, ham_ly, ham_hp);
    SampleSpec sp;
    sp.ham = ham_hp ? &H : nullptr;
    sp.n_chains = n_chains;
    sp.move = move;
    sp.nup = nup;
    sp.seed = seed;
    sp.epoch = epoch;
    sp.reinit = reinit;
    sp.n_sweeps = n_sweeps;
    sp.n_discard = n_discard;
    sp.sweep_len = sweep_len;
    sample(q, sp, chain_sigma, out_sigma, reinterpret_cast<cd*>(out_theta), acc, nthreads);
}

void orc_sample_pt(int n, int m, int use_bias, const double* params, int n_chains, int ntemps, int move, int nup,
                   uint64_t seed, uint32_t epoch, int reinit, int n_sweeps, int n_discard, int sweep_len,
                   int8_t* chain_sigma, int* slot, int8_t* out_sigma, double* out_theta, uint64_t* acc,
                   int nthreads, int ham_kind, int ham_lx, int ham_ly, const double* ham_hp) {
    RBM q = make_rbm(n, m, use_bias, params);
    Ham H;
    if (ham_hp) H = make_ham(ham_kind, n, ham_lx, ham_ly, ham_hp);
    SampleSpec sp;
    sp.ham = ham_hp ? &H : nullptr;
    sp.n_chains = n_chains;
    sp.move = move;
    sp.nup = nup;
    sp.seed = seed;
    sp.epoch = epoch;
    sp.reinit = reinit;
    sp.n_sweeps = n_sweeps;
    sp.n_discard = n_discard;
    sp.sweep_len = sweep_len;
    sample_pt(q, sp, ntemps, chain_sigma, slot, out_sigma, reinterpret_cast<cd*>(out_theta), acc, nthreads);
}

// One SR step on given samples.  out_v/out_grad/out_oloc: P complex; out_eloc: ns complex;
// out_stats: [energy, energy_var, cg_iters, cg_relres].  Returns the Cholesky status.
int orc_sr_step(int kind, int n, int lx, int ly, const double* hp, int m, int use_bias,
                const double* params, int ns, const int8_t* s, const double* theta, double shift, int mode, int solver,
                double cgtol, double* out_v, double* out_grad, double* out_oloc, double* out_eloc,
                double* out_stats, int nthreads) {
    Ham H = make_ham(kind, n, lx, ly, hp);
    RBM q = make_rbm(n, m, use_bias, params);
    SRResult R = sr_step(q, H, ns, s, reinterpret_cast<const cd*>(theta), shift, mode, solver, cgtol, nthreads);
    const size_t P = q.dim();
    if (out_v) std::memcpy(out_v, R.v.data(), P * sizeof(cd));
    if (out_grad) std::memcpy(out_grad, R.grad.data(), P * sizeof(cd));
    if (out_oloc) std::memcpy(out_oloc, R.oloc.data(), P * sizeof(cd));
    if (out_eloc) std::memcpy(out_eloc, R.elocs.data(), size_t(ns) * sizeof(cd));
    if (out_stats) {
        out_stats[0] = R.energy;
        out_stats[1] = R.energy_var;
        out_stats[2] = R.cg_iters;
        out_stats[3] = R.cg_relres;
    }
    return R.status;
}

// Dense Hermitian Cholesky restatement for cross-checks: A row-major nn x nn (lower used),
// b overwritten by the solution.  Returns 0 or the 1-based failing pivot.
int orc_cholesky_solve(int nn, double* A, double* b) {
    cd* Ac = reinterpret_cast<cd*>(A);
    int st = cholesky_lower(nn, Ac);
    if (st) return st;
    cholesky_solve(nn, Ac, reinterpret_cast<cd*>(b));
    return 0;
}

// basis_kind: 0 full, 1 fixed popcount nup.  out_S may be null.
int orc_exact(int kind, int n, int lx, int ly, const double* hp, int m, int use_bias,
              const double* params, int basis_kind, int nup, double* out_stats, double* out_oloc, double* out_grad,
              double* out_S, int nthreads) {
    Ham H = make_ham(kind, n, lx, ly, hp);
    RBM q = make_rbm(n, m, use_bias, params);
    auto basis = basis_kind == 0 ? basis_full(n) : basis_jz(n, nup);
    ExactResult X = exact_sr(q, H, basis, nthreads, out_S != nullptr);
    const size_t P = q.dim();
    out_stats[0] = X.energy;
    out_stats[1] = X.energy_var;
    if (out_oloc) std::memcpy(out_oloc, X.oloc.data(), P * sizeof(cd));
    if (out_grad) std::memcpy(out_grad, X.grad.data(), P * sizeof(cd));
    if (out_S) std::memcpy(out_S, X.S.data(), P * P * sizeof(cd));
    return int(basis.size());
}

int orc_exact_sample(int n, int m, int use_bias, const double* params, int basis_kind, int nup, int nsamples,
                     uint64_t seed, uint32_t epoch, uint32_t* out_pos, uint64_t* out_index, int nthreads) {
    RBM q = make_rbm(n, m, use_bias, params);
    auto basis = basis_kind == 0 ? basis_full(n) : basis_jz(n, nup);
    auto pos = exact_sample(q, basis, nsamples, seed, epoch, nthreads);
    for (int i = 0; i < nsamples; ++i) {
        out_pos[i] = pos[size_t(i)];
        if (out_index) out_index[i] = basis[pos[size_t(i)]];
    }
    return int(basis.size());
}

int orc_basis(int n, int basis_kind, int nup, uint64_t* out, int cap) {
    auto b = basis_kind == 0 ? basis_full(n) : basis_jz(n, nup);
    for (size_t i = 0; i < b.size() && int(i) < cap; ++i) out[i] = b[i];
    return int(b.size());
}

double orc_ed_ground(int kind, int n, int lx, int ly, const double* hp, int basis_kind, int nup,
                     int maxit, int nthreads) {
    Ham H = make_ham(kind, n, lx, ly, hp);
    auto basis = basis_kind == 0 ? basis_full(n) : basis_jz(n, nup);
    return ed_ground_energy(H, basis, maxit, nthreads);
}

double orc_ff_forward(int L, int conv_out, int conv_k, int fc_out, const double* params, const int8_t* s) {
    FFNet f{L, conv_out, conv_k, fc_out, params};
    return ff_forward(f, s);
}

void orc_ff_backward(int L, int conv_out, int conv_k, int fc_out, const double* params, const int8_t* s,
                     double* der) {
    FFNet f{L, conv_out, conv_k, fc_out, params};
    ff_backward(f, s, der);
}

void orc_ff_batch(int L, int conv_out, int conv_k, int fc_out, const double* params, int batch, const int8_t* s,
                  double* logpsi, double* der, int nthreads) {
    FFNet f{L, conv_out, conv_k, fc_out, params};
    const size_t P = f.dim();
#pragma omp parallel for schedule(static) num_threads(nthreads > 0 ? nthreads : 1)
    for (int b = 0; b < batch; ++b) {
        if (logpsi) logpsi[b] = ff_forward(f, s + size_t(b) * L);
        if (der) ff_backward(f, s + size_t(b) * L, der + size_t(b) * P);
    }
}


// ---- AmplitudePhase / NGDExact ---------------------------------------------
int orc_ap_dims(int n, int m, int use_bias, int nl, const int* desc, const double* xs, uint64_t* dims) {
    try {
        APNet q = make_ap(n, m, use_bias, nl, desc, xs, nullptr);
        dims[0] = q.Pa;
        dims[1] = q.Pp;
        return 0;
    } catch (...) {
        return -1;
    }
}

void orc_ap_init(int n, int m, int use_bias, int nl, const int* desc, const double* xs, uint64_t seed,
                 double sigma_amp, int mode, double* p) {
    APNet q = make_ap(n, m, use_bias, nl, desc, xs, p);
    ap_init(q, seed, sigma_amp, mode, p);
}

// out: ns complex log psi = log A / 2 + i pi phi
void orc_ap_log_psi(int n, int m, int use_bias, int nl, const int* desc, const double* xs, const double* p, int ns,
                    const int8_t* s, double* out) {
    APNet q = make_ap(n, m, use_bias, nl, desc, xs, p);
    for (int k = 0; k < ns; ++k) {
        const int8_t* sk = s + size_t(k) * n;
        auto data = ap_phase_data(q, sk);
        out[2 * k] = 0.5 * ap_log_amp(q, sk);
        out[2 * k + 1] = M_PI * data.back()[0];
    }
}

// out: ns x (Pa + Pp) complex rows [logDerivAmp | i logDerivPhase] (AmplitudePhase.hpp:52-59)
void orc_ap_log_deriv(int n, int m, int use_bias, int nl, const int* desc, const double* xs, const double* p, int ns,
                      const int8_t* s, double* out) {
    APNet q = make_ap(n, m, use_bias, nl, desc, xs, p);
    const size_t P = q.Pa + q.Pp;
    std::vector<double> da(q.Pa), dp(q.Pp);
    for (int k = 0; k < ns; ++k) {
        const int8_t* sk = s + size_t(k) * n;
        ap_log_deriv_amp(q, sk, da.data());
        ap_phase_backward(q, ap_phase_data(q, sk), dp.data());
        double* row = out + 2 * size_t(k) * P;
        for (size_t c = 0; c < q.Pa; ++c) {
            row[2 * c] = da[c];
            row[2 * c + 1] = 0.0;
        }
        for (size_t c = 0; c < q.Pp; ++c) {
            row[2 * (q.Pa + c)] = 0.0;
            row[2 * (q.Pa + c) + 1] = M_PI * dp[c];
        }
    }
}

int orc_ngd_exact(int kind, int n, int lx, int ly, const double* hp, int m, int use_bias, int nl, const int* desc,
                  const double* xs, const double* p, int basis_kind, int nup, int with_corr, double* energy,
                  double* grad, double* oloc_amp, double* oloc_phase, double* corr_amp, double* corr_phase,
                  int nthreads) {
    Ham H = make_ham(kind, n, lx, ly, hp);
    APNet q = make_ap(n, m, use_bias, nl, desc, xs, p);
    auto basis = basis_kind == 0 ? basis_full(n) : basis_jz(n, nup);
    NGDResult R = ngd_exact(q, H, basis, with_corr != 0, nthreads);
    *energy = R.energy;
    std::memcpy(grad, R.grad.data(), R.grad.size() * sizeof(double));
    if (oloc_amp) std::memcpy(oloc_amp, R.oloc_amp.data(), R.oloc_amp.size() * sizeof(double));
    if (oloc_phase) std::memcpy(oloc_phase, R.oloc_phase.data(), R.oloc_phase.size() * sizeof(double));
    if (with_corr && corr_amp) std::memcpy(corr_amp, R.corr_amp.data(), R.corr_amp.size() * sizeof(double));
    if (with_corr && corr_phase) std::memcpy(corr_phase, R.corr_phase.data(), R.corr_phase.size() * sizeof(double));
    return int(basis.size());
}
}  // extern "C"
