// yannq oracle implementation -- TEST INFRASTRUCTURE ONLY (see oracle.hpp).
#include "oracle.hpp"

#include <algorithm>

#include <numeric>
#include <stdexcept>

#ifdef _OPENMP
#include <omp.h>
#endif

namespace orc {

static inline int nthreads_or_default(int nt) {
#ifdef _OPENMP
    return nt > 0 ? nt : omp_get_max_threads();
#else
    (void)nt;
    return 1;
#endif
}

// ---------------------------------------------------------------------------
double normal_pair(uint64_t seed, uint32_t idx, double* second) {
    uint32_t x[4];
    Philox4x32::draw(seed, idx, 0u, 0u, TAG_PARAM, x);
    const double u1 = 1.0 - draw_u53(x[0], x[1]);  // (0, 1]
    const double u2 = draw_u53(x[2], x[3]);
    const double r = std::sqrt(-2.0 * std::log(u1));
    const double ang = 6.283185307179586476925286766559 * u2;
    if (second) *second = r * std::sin(ang);
    return r * std::cos(ang);
}

void init_params(int n, int m, bool useBias, uint64_t seed, double sd, cd* p) {
    // Machines/RBM.hpp:325-349: a, b (if bias) then W(i, j) with i (hidden) fastest.
    uint32_t e = 0;
    auto draw = [&](cd& out) {
        double im;
        double re = normal_pair(seed, e++, &im);
        out = cd{sd * re, sd * im};
    };
    const size_t nm = size_t(n) * m;
    if (useBias) {
        for (int i = 0; i < n; ++i) draw(p[nm + i]);
        for (int j = 0; j < m; ++j) draw(p[nm + n + j]);
    }
    for (int i = 0; i < n; ++i)
        for (int j = 0; j < m; ++j) draw(p[size_t(i) * m + j]);
}

// ---------------------------------------------------------------------------
static inline int right_of(const Ham& H, int i) {
    if (H.kind == 2) {
        int x = i % H.lx, y = i / H.lx;
        return (x + 1) % H.lx + H.lx * y;
    }
    return (i + 1) % H.n;
}
static inline int down_of(const Ham& H, int i) {
    int x = i % H.lx, y = i / H.lx;
    return x + H.lx * ((y + 1) % H.ly);
}

// KitaevHex.hpp:33-103.  Sites of row r: n_/2 black ones (r * n_ + c), then
// n_/2 white ones (r * n_ + n_/2 + c); rows and columns wrap around.
std::vector<std::pair<int, int>> kitaev_links(const Ham& H, int axis) {
    const int nc = H.lx, nr = H.ly, k = nc / 2;
    auto wrap = [](int v, int p) { return ((v % p) + p) % p; };
    auto black = [&](int r, int c) { return wrap(r, nr) * nc + wrap(c, k); };
    auto white = [&](int r, int c) { return wrap(r, nr) * nc + wrap(c, k) + k; };
    std::vector<std::pair<int, int>> out;
    if (axis == 2) {  // zLinks: white (r, c) to black (r + 1, c)
        for (int r = 0; r < nr; ++r)
            for (int c = 0; c < k; ++c) out.emplace_back(white(r, c), black(r + 1, c));
        return out;
    }
    // xLinks: even rows to white (r, c - 1), odd rows to white (r, c);
    // yLinks: even rows to white (r, c), odd rows to white (r, c + 1).  Even rows first.
    for (int parity = 0; parity < 2; ++parity)
        for (int r = parity; r < nr; r += 2)
            for (int c = 0; c < k; ++c) {
                int dc = axis == 0 ? (parity == 0 ? -1 : 0) : (parity == 0 ? 0 : 1);
                out.emplace_back(black(r, c), white(r, c + dc));
            }
    return out;
}

// State forms of XXX (XXX.hpp:11-22), J1J2 (J1J2.hpp:35-56), XYZNNN
// (XYZNNN.hpp:33-53) and KitaevHex (KitaevHex.hpp:119-146) in the reference's
// evaluation order: diag(d) for every real addend, ratio(a, b, c) for every
// c * ratio(a, b) addend (b = -1 for one flip), with the coefficients formed as
// the reference forms them.
template <class Diag, class Ratio>
static void ModelStateForm(const Ham& H, const int8_t* s, Diag diag, Ratio ratio) {
    const int n = H.n;
    if (H.kind == HAM_XXX) {
        for (int i = 0; i < n; ++i) {
            int j = (i + 1) % n;
            double yy = double(s[i] * s[j]);
            diag(yy);
            ratio(i, j, 1.0 - yy);
        }
    } else if (H.kind == HAM_J1J2 || H.kind == HAM_XYZNNN) {
        const bool j1j2 = H.kind == HAM_J1J2;
        const double J1 = j1j2 ? H.J : -1.0, J2 = j1j2 ? H.h : -1.0;
        for (int d = 1; d <= 2; ++d)
            for (int i = 0; i < n; ++i) {
                int j = (i + d) % n;
                double yy = -double(s[i] * s[j]);
                const double Jd = d == 1 ? J1 : J2;
                diag(-Jd * yy);
                double c;
                if (j1j2)
                    c = d == 1 ? J1 * H.sign * (1.0 + yy) : J2 * (1.0 + yy);
                else
                    c = d == 1 ? J1 * (H.J + yy * H.h) : J2 * (H.h + yy * H.J);
                ratio(i, j, c);
            }
    } else if (H.kind == HAM_KITAEV) {
        for (int i = 0; i < n; ++i) ratio(i, -1, H.h);
        for (auto& e : kitaev_links(H, 0)) ratio(e.first, e.second, H.J);
        for (auto& e : kitaev_links(H, 1)) {
            int zz = s[e.first] * s[e.second];
            ratio(e.first, e.second, -H.jy * zz);
        }
        for (auto& e : kitaev_links(H, 2)) {
            int zz = s[e.first] * s[e.second];
            diag(H.jz * zz);
        }
    }
}

double ham_enumerate(const Ham& H, const int8_t* s, std::vector<FlipTerm>& terms) {
    terms.clear();
    double diag = 0.;
    for (int i = 0; i < (H.kind <= HAM_TFI2D ? H.n : 0); ++i) {
        if (H.kind == 0) {  // TFIsing.hpp:31-36
            diag += H.J * s[i] * s[(i + 1) % H.n];
            terms.push_back({uint64_t(1) << i, H.h});
        } else if (H.kind == 1) {  // XXZ.hpp:40-47
            int j = (i + 1) % H.n;
            int zz = s[i] * s[j];
            diag += H.J * H.h * zz;
            terms.push_back({(uint64_t(1) << i) | (uint64_t(1) << j), H.sign * H.J * (1 - zz)});
        } else if (H.kind == 2) {  // TFIsing2D: right and down bonds of every site, then the field
            diag += H.J * s[i] * s[right_of(H, i)];
            diag += H.J * s[i] * s[down_of(H, i)];
            terms.push_back({uint64_t(1) << i, H.h});
        }
    }
    // state forms of the further models, recorded as (mask, coeff) requests
    ModelStateForm(H, s, [&](double d) { diag += d; }, [&](int a, int b, double c) {
        terms.push_back({(uint64_t(1) << a) | (b >= 0 ? uint64_t(1) << b : uint64_t(0)), c});
    });
    return diag;
}

std::map<uint64_t, double> ham_column(const Ham& H, uint64_t col) {
    std::map<uint64_t, double> res;
    auto z = [&](int i) { return 1 - 2 * int((col >> i) & 1u); };
    for (int i = 0; i < (H.kind <= HAM_TFI2D ? H.n : 0); ++i) {
        if (H.kind == 0) {  // TFIsing.hpp:53-65
            res[col ^ (uint64_t(1) << i)] += H.h;
            res[col] += H.J * z(i) * z((i + 1) % H.n);
        } else if (H.kind == 1) {  // XXZ.hpp:51-64
            int j = (i + 1) % H.n;
            int zz = z(i) * z(j);
            uint64_t x = (uint64_t(1) << i) | (uint64_t(1) << j);
            res[col] += H.J * H.h * zz;
            res[col ^ x] += H.sign * H.J * (1 - zz);
        } else if (H.kind == 2) {
            res[col ^ (uint64_t(1) << i)] += H.h;
            res[col] += H.J * z(i) * z(right_of(H, i)) + H.J * z(i) * z(down_of(H, i));
        }
    }
    auto bit = [](int i) { return uint64_t(1) << i; };
    const int n = H.n;
    if (H.kind == HAM_XXX) {  // XXX.hpp:21-34
        for (int i = 0; i < n; ++i) {
            int j = (i + 1) % n, sgn = z(i) * z(j);
            res[col ^ (bit(i) | bit(j))] += 1 - sgn;
            res[col] += sgn;
        }
    } else if (H.kind == HAM_J1J2 || H.kind == HAM_XYZNNN) {  // J1J2.hpp:57-79, XYZNNN.hpp:67-89
        const bool j1j2 = H.kind == HAM_J1J2;
        const double J1 = j1j2 ? H.J : -1.0, J2 = j1j2 ? H.h : -1.0;
        for (int d = 1; d <= 2; ++d)
            for (int i = 0; i < n; ++i) {
                int j = (i + d) % n, zz = z(i) * z(j);
                uint64_t x = bit(i) | bit(j);
                double off;
                if (j1j2)
                    off = d == 1 ? J1 * H.sign * (1.0 - zz * 1.0) : J2 * (1.0 - zz * 1.0);
                else
                    off = d == 1 ? J1 * (H.J - zz * H.h) : J2 * (H.h - zz * H.J);
                res[col ^ x] += off;
                res[col] += (d == 1 ? J1 : J2) * zz;
            }
    } else if (H.kind == HAM_KITAEV) {  // KitaevHex.hpp:148-177
        for (int i = 0; i < n; ++i) res[col ^ bit(i)] += H.h;
        for (auto& e : kitaev_links(H, 0)) res[col ^ (bit(e.first) | bit(e.second))] += H.J;
        for (auto& e : kitaev_links(H, 1)) {
            int zz = z(e.first) * z(e.second);
            res[col ^ (bit(e.first) | bit(e.second))] += -H.jy * zz;
        }
        for (auto& e : kitaev_links(H, 2)) res[col] += H.jz * (z(e.first) * z(e.second));
    }
    return res;
}

cd ham_eloc(const Ham& H, const RBM& q, const int8_t* s, const cd* th) {
    cd acc = 0.;
    for (int i = 0; i < (H.kind <= HAM_TFI2D ? H.n : 0); ++i) {
        if (H.kind == 0) {
            acc += H.J * s[i] * s[(i + 1) % H.n];
            acc += H.h * std::exp(q.logRatio1(s, th, i));
        } else if (H.kind == 1) {
            int j = (i + 1) % H.n;
            int zz = s[i] * s[j];
            acc += H.J * H.h * zz;
            acc += H.sign * H.J * (1 - zz) * std::exp(q.logRatio2(s, th, i, j));
        } else if (H.kind == 2) {
            acc += H.J * s[i] * s[right_of(H, i)];
            acc += H.J * s[i] * s[down_of(H, i)];
            acc += H.h * std::exp(q.logRatio1(s, th, i));
        }
    }
    ModelStateForm(H, s, [&](double d) { acc += d; }, [&](int a, int b, double c) {
        acc += c * std::exp(b < 0 ? q.logRatio1(s, th, a) : q.logRatio2(s, th, a, b));
    });
    return acc;
}

// ---------------------------------------------------------------------------
void random_sigma(int n, int nup, uint64_t seed, uint32_t epoch, uint32_t chain, int8_t* s) {
    uint32_t x[4];
    if (nup < 0) {  // Utilities/Utility.hpp:63-74
        for (int i = 0; i < n; ++i) {
            Philox4x32::draw(seed, uint32_t(i), epoch, chain, TAG_INIT, x);
            s[i] = (x[0] & 1u) ? int8_t(-1) : int8_t(1);
        }
        return;
    }
    // Utilities/Utility.hpp:77-88: nup entries -1, the rest +1, then shuffled
    for (int i = 0; i < n; ++i) s[i] = (i < nup) ? int8_t(-1) : int8_t(1);
    for (int i = n - 1; i >= 1; --i) {
        Philox4x32::draw(seed, uint32_t(i), epoch, chain, TAG_SHUF, x);
        int j = int(draw_site(x[0], uint32_t(i + 1)));
        std::swap(s[i], s[j]);
    }
}

// offDiagonals(s) for the HamiltonianSweeper: TFIsing.hpp:41-50 lists every site
// whatever the state (the 2D model likewise); for the other models, the state
// form's off-diagonal requests whose coefficient in s is non-zero, in order.
std::vector<std::array<int, 2>> off_diagonals(const Ham& H, const int8_t* s) {
    std::vector<std::array<int, 2>> out;
    if (H.kind == HAM_TFI || H.kind == HAM_TFI2D) {
        for (int i = 0; i < H.n; ++i) out.push_back({i, -1});
    } else if (H.kind == HAM_XXZ) {
        for (int i = 0; i < H.n; ++i) {
            int j = (i + 1) % H.n;
            if (H.sign * H.J * (1 - s[i] * s[j]) != 0.0) out.push_back({i, j});
        }
    } else {
        ModelStateForm(H, s, [](double) {}, [&](int a, int b, double c) {
            if (c != 0.0) out.push_back({a, b});
        });
    }
    return out;
}

// One proposal of LocalSweeper (LocalSweeper.hpp:42-52), SwapSweeper
// (SwapSweeper.hpp:39-56, any pair, or its neighbour-pair variant) or
// HamiltonianSweeper (HamiltonianSweeper.hpp:26-49, which takes no beta) from the
// draw x.  Returns whether the move was accepted (and applied).
static bool metropolis_step(const RBM& q, const SampleSpec& sp, int8_t* s, cd* th, const uint32_t x[4],
                            double beta) {
    const int n = q.n;
    const double u = draw_u53(x[2], x[3]);
    if (sp.move == MOVE_LOCAL) {
        int k = int(draw_site(x[0], uint32_t(n)));
        double pr = std::min(1.0, std::exp(beta * 2.0 * q.logRatio1(s, th, k).real()));
        if (u < pr) {
            q.flip1(s, th, k);
            return true;
        }
        return false;
    }
    if (sp.move == MOVE_HAMILTONIAN) {
        auto flips = off_diagonals(*sp.ham, s);
        if (flips.empty()) return false;
        auto f = flips[draw_site(x[0], uint32_t(flips.size()))];
        std::vector<int8_t> sp2(s, s + n);
        sp2[size_t(f[0])] = int8_t(-sp2[size_t(f[0])]);
        if (f[1] >= 0) sp2[size_t(f[1])] = int8_t(-sp2[size_t(f[1])]);
        const double w1 = double(flips.size());
        const double w2 = double(off_diagonals(*sp.ham, sp2.data()).size());
        const cd lr = f[1] < 0 ? q.logRatio1(s, th, f[0]) : q.logRatio2(s, th, f[0], f[1]);
        double pr = std::min(1.0, std::exp(2.0 * lr.real()) * (w1 / w2));
        if (u < pr) {
            if (f[1] < 0)
                q.flip1(s, th, f[0]);
            else
                q.flip2(s, th, f[0], f[1]);
            return true;
        }
        return false;
    }
    int k = int(draw_site(x[0], uint32_t(n)));
    int l = (sp.move == MOVE_EXCHANGE_ANY) ? int(draw_site(x[1], uint32_t(n))) : (k + 1) % n;
    if (s[k] == s[l]) return false;
    double pr = std::min(1.0, std::exp(beta * 2.0 * q.logRatio2(s, th, k, l).real()));
    if (u < pr) {
        q.flip2(s, th, k, l);
        return true;
    }
    return false;
}

void sample(const RBM& q, const SampleSpec& sp, int8_t* chain_sigma, int8_t* out_sigma, cd* out_theta,
            uint64_t* acc, int nthreads) {
    const int n = q.n, m = q.m;
    const int L = sp.sweep_len > 0 ? sp.sweep_len : n;
    const int total = sp.n_discard + sp.n_sweeps;
#pragma omp parallel for schedule(dynamic, 1) num_threads(nthreads_or_default(nthreads))
    for (int c = 0; c < sp.n_chains; ++c) {
        std::vector<int8_t> s(n);
        std::vector<cd> th(m);
        int8_t* cs = chain_sigma + size_t(c) * n;
        if (sp.reinit)
            random_sigma(n, sp.nup, sp.seed, sp.epoch, uint32_t(c), s.data());
        else
            std::copy(cs, cs + n, s.begin());
        q.theta(s.data(), th.data());
        uint64_t nacc = 0;
        uint32_t x[4];
        for (int sw = 0; sw < total; ++sw) {
            for (int p = 0; p < L; ++p) {
                const uint32_t g = uint32_t(sw) * uint32_t(L) + uint32_t(p);
                Philox4x32::draw(sp.seed, g, sp.epoch, uint32_t(c), TAG_SWEEP, x);
                if (metropolis_step(q, sp, s.data(), th.data(), x, 1.0)) ++nacc;
            }
            if (sw >= sp.n_discard) {  // SamplerMT.hpp:165-173 (recorded in (sweep, chain) order)
                size_t idx = size_t(sw - sp.n_discard) * sp.n_chains + c;
                std::copy(s.begin(), s.end(), out_sigma + idx * n);
                std::copy(th.begin(), th.end(), out_theta + idx * m);
            }
        }
        std::copy(s.begin(), s.end(), cs);
        if (acc) acc[c] = nacc;
    }
}

void sample_pt(const RBM& q, const SampleSpec& sp, int ntemps, int8_t* chain_sigma, int* slot, int8_t* out_sigma,
               cd* out_theta, uint64_t* acc, int nthreads) {
    const int n = q.n, m = q.m, nc = sp.n_chains, groups = nc / ntemps;
    const int L = sp.sweep_len > 0 ? sp.sweep_len : n;
    const int total = sp.n_discard + sp.n_sweeps;
    const int nt = nthreads_or_default(nthreads);
    std::vector<int8_t> s(size_t(nc) * n);
    std::vector<cd> th(size_t(nc) * m);
    std::vector<double> lp(nc);
    std::vector<uint64_t> nacc(nc, 0);
    for (int c = 0; c < nc; ++c) {
        int8_t* sc = s.data() + size_t(c) * n;
        if (sp.reinit) {
            random_sigma(n, sp.nup, sp.seed, sp.epoch, uint32_t(c), sc);
            slot[c] = c % ntemps;
        } else {
            std::copy(chain_sigma + size_t(c) * n, chain_sigma + size_t(c + 1) * n, sc);
        }
        q.theta(sc, th.data() + size_t(c) * m);
    }
    auto beta_of = [&](int t) { return double(ntemps - t) / double(ntemps); };
    for (int sw = 0; sw < total; ++sw) {
#pragma omp parallel for schedule(dynamic, 1) num_threads(nt)
        for (int c = 0; c < nc; ++c) {
            int8_t* sc = s.data() + size_t(c) * n;
            cd* tc = th.data() + size_t(c) * m;
            const double beta = beta_of(slot[c]);
            uint32_t x[4];
            for (int p = 0; p < L; ++p) {
                const uint32_t g = uint32_t(sw) * uint32_t(L) + uint32_t(p);
                Philox4x32::draw(sp.seed, g, sp.epoch, uint32_t(c), TAG_SWEEP, x);
                if (metropolis_step(q, sp, sc, tc, x, beta)) ++nacc[c];
            }
            lp[c] = q.logCoeff(sc, tc).real();
        }
        // mixChains (SamplerMT.hpp:120-153)
        for (int gr = 0; gr < groups; ++gr) {
            std::vector<int> at(ntemps);
            for (int k = 0; k < ntemps; ++k) at[size_t(slot[gr * ntemps + k])] = gr * ntemps + k;
            auto attempt = [&](int t) {
                const int a = at[size_t(t)], b = at[size_t(t + 1)];
                const double pr = std::exp((beta_of(t + 1) - beta_of(t)) * 2.0 * (lp[a] - lp[b]));
                uint32_t x[4];
                Philox4x32::draw(sp.seed, uint32_t(sw) * 64u + uint32_t(t), sp.epoch, uint32_t(gr), TAG_PT, x);
                if (draw_u53(x[2], x[3]) < pr) std::swap(at[size_t(t)], at[size_t(t + 1)]);
            };
            for (int t = 0; t + 1 < ntemps; t += 2) attempt(t);
            for (int t = 1; t + 1 < ntemps - 1; t += 2) attempt(t);
            for (int t = 0; t < ntemps; ++t) slot[at[size_t(t)]] = t;
        }
        if (sw >= sp.n_discard) {
            for (int c = 0; c < nc; ++c) {
                if (slot[c] != 0) continue;
                const size_t idx = size_t(sw - sp.n_discard) * groups + c / ntemps;
                std::copy(s.begin() + size_t(c) * n, s.begin() + size_t(c + 1) * n, out_sigma + idx * n);
                std::copy(th.begin() + size_t(c) * m, th.begin() + size_t(c + 1) * m, out_theta + idx * m);
            }
        }
    }
    std::copy(s.begin(), s.end(), chain_sigma);
    if (acc)
        for (int c = 0; c < nc; ++c) acc[c] = nacc[c];
}

// ---------------------------------------------------------------------------
int cholesky_lower(int nn, cd* A) {
    for (int j = 0; j < nn; ++j) {
        cd* rj = A + size_t(j) * nn;
        double d = rj[j].real();
        for (int k = 0; k < j; ++k) d -= std::norm(rj[k]);
        if (!(d > 0.0)) return j + 1;
        const double ljj = std::sqrt(d);
        rj[j] = ljj;
#pragma omp parallel for schedule(static)
        for (int i = j + 1; i < nn; ++i) {
            cd* ri = A + size_t(i) * nn;
            cd acc = ri[j];
            for (int k = 0; k < j; ++k) acc -= ri[k] * std::conj(rj[k]);
            ri[j] = acc / ljj;
        }
    }
    return 0;
}

void cholesky_solve(int nn, const cd* L, cd* x) {
    for (int i = 0; i < nn; ++i) {  // L y = b
        const cd* ri = L + size_t(i) * nn;
        cd acc = x[i];
        for (int k = 0; k < i; ++k) acc -= ri[k] * x[k];
        x[i] = acc / ri[i].real();
    }
    for (int i = nn - 1; i >= 0; --i) {  // L^H x = y
        cd acc = x[i];
        for (int k = i + 1; k < nn; ++k) acc -= std::conj(L[size_t(k) * nn + i]) * x[k];
        x[i] = acc / L[size_t(i) * nn + i].real();
    }
}

template <class ApplyFn>
int conjugate_gradient(size_t dim, ApplyFn&& apply, const cd* b, cd* x, double tol, int maxit, double* relres) {
    std::vector<cd> r(b, b + dim), p(dim), tmp(dim);
    std::fill(x, x + dim, cd{});
    auto dotc = [&](const std::vector<cd>& u, const std::vector<cd>& v) {
        cd s = 0.;
        for (size_t i = 0; i < dim; ++i) s += std::conj(u[i]) * v[i];
        return s;
    };
    double rhsNorm2 = 0.;
    for (size_t i = 0; i < dim; ++i) rhsNorm2 += std::norm(b[i]);
    if (rhsNorm2 == 0.) {
        if (relres) *relres = 0.;
        return 0;
    }
    const double threshold = tol * tol * rhsNorm2;
    double residualNorm2 = rhsNorm2;
    if (residualNorm2 < threshold) {
        if (relres) *relres = std::sqrt(residualNorm2 / rhsNorm2);
        return 0;
    }
    p = r;
    double absNew = dotc(r, p).real();
    int i = 0;
    while (i < maxit) {
        apply(p.data(), tmp.data());
        cd alpha = absNew / dotc(p, tmp);
        for (size_t k = 0; k < dim; ++k) {
            x[k] += alpha * p[k];
            r[k] -= alpha * tmp[k];
        }
        residualNorm2 = 0.;
        for (size_t k = 0; k < dim; ++k) residualNorm2 += std::norm(r[k]);
        if (residualNorm2 < threshold) break;
        double absOld = absNew;
        absNew = dotc(r, r).real();
        double beta = absNew / absOld;
        for (size_t k = 0; k < dim; ++k) p[k] = r[k] + beta * p[k];
        ++i;
    }
    if (relres) *relres = std::sqrt(residualNorm2 / rhsNorm2);
    return i;
}

SRResult sr_step(const RBM& q, const Ham& H, int ns, const int8_t* sig, const cd* th, double shift, int mode,
                 int solver, double cgtol, int nthreads) {
    const int nt = nthreads_or_default(nthreads);
    const size_t P = q.dim();
    SRResult R;
    std::vector<cd> O(size_t(ns) * P);
    R.elocs.resize(ns);
    // GroundState/utils.hpp:12-51 (constructDelta) and :108-126 (constructObs -> Energy::eachSample)
#pragma omp parallel for schedule(static) num_threads(nt)
    for (int s = 0; s < ns; ++s) {
        q.logDeriv(sig + size_t(s) * q.n, th + size_t(s) * q.m, O.data() + size_t(s) * P);
        R.elocs[s] = ham_eloc(H, q, sig + size_t(s) * q.n, th + size_t(s) * q.m);
    }
    // Observables/Energy.hpp:53-58
    double e = 0., e2 = 0.;
    cd emean = 0.;
    for (int s = 0; s < ns; ++s) {
        e += R.elocs[s].real();
        e2 += R.elocs[s].real() * R.elocs[s].real();
        emean += R.elocs[s];
    }
    e /= ns;
    e2 /= ns;
    emean /= double(ns);
    R.energy = e;
    R.energy_var = e2 - e * e;
    // SRMat.hpp:97-102: column mean, centring, energyGrad = O~^H E / Ns
    R.oloc.assign(P, cd{});
    for (int s = 0; s < ns; ++s)
        for (size_t p = 0; p < P; ++p) R.oloc[p] += O[size_t(s) * P + p];
    for (size_t p = 0; p < P; ++p) R.oloc[p] /= double(ns);
#pragma omp parallel for schedule(static) num_threads(nt)
    for (int s = 0; s < ns; ++s)
        for (size_t p = 0; p < P; ++p) O[size_t(s) * P + p] -= R.oloc[p];
    R.grad.assign(P, cd{});
#pragma omp parallel for schedule(static) num_threads(nt)
    for (long long p = 0; p < (long long)P; ++p) {
        cd acc = 0.;
        for (int s = 0; s < ns; ++s) acc += std::conj(O[size_t(s) * P + p]) * R.elocs[s];
        R.grad[p] = acc / double(ns);
    }
    R.v.assign(P, cd{});
    if (mode == SR_S) {
        if (solver == SOLVE_LLT) {  // SRMat.hpp:142-149 corrMat + :231-237 solveExact
            std::vector<cd> S(P * P);
#pragma omp parallel for schedule(dynamic, 4) num_threads(nt)
            for (long long a = 0; a < (long long)P; ++a)
                for (size_t b = 0; b <= size_t(a); ++b) {
                    cd acc = 0.;
                    for (int s = 0; s < ns; ++s) acc += std::conj(O[size_t(s) * P + a]) * O[size_t(s) * P + b];
                    S[size_t(a) * P + b] = acc / double(ns);
                }
            for (size_t a = 0; a < P; ++a) S[a * P + a] += shift;
            R.status = cholesky_lower(int(P), S.data());
            if (R.status) return R;
            R.v = R.grad;
            cholesky_solve(int(P), S.data(), R.v.data());
        } else {  // SRMat.hpp:170-189 apply + :197-208 solveCG
            auto apply = [&](const cd* x, cd* y) {
                std::vector<cd> r(ns);
#pragma omp parallel for schedule(static) num_threads(nt)
                for (int s = 0; s < ns; ++s) {
                    cd acc = 0.;
                    for (size_t p = 0; p < P; ++p) acc += O[size_t(s) * P + p] * x[p];
                    r[s] = acc / double(ns);
                }
#pragma omp parallel for schedule(static) num_threads(nt)
                for (long long p = 0; p < (long long)P; ++p) {
                    cd acc = 0.;
                    for (int s = 0; s < ns; ++s) acc += std::conj(O[size_t(s) * P + p]) * r[s];
                    y[p] = acc + shift * x[p];
                }
            };
            R.cg_iters = conjugate_gradient(P, apply, R.grad.data(), R.v.data(), cgtol, int(2 * P), &R.cg_relres);
        }
    } else {  // sample-space dual (push-through identity); no reference counterpart
        std::vector<cd> T(size_t(ns) * ns);
#pragma omp parallel for schedule(dynamic, 4) num_threads(nt)
        for (int a = 0; a < ns; ++a)
            for (int b = 0; b <= a; ++b) {
                cd acc = 0.;
                const cd* ra = O.data() + size_t(a) * P;
                const cd* rb = O.data() + size_t(b) * P;
                for (size_t p = 0; p < P; ++p) acc += ra[p] * std::conj(rb[p]);
                T[size_t(a) * ns + b] = acc / double(ns);
            }
        for (int a = 0; a < ns; ++a) T[size_t(a) * ns + a] += shift;
        R.status = cholesky_lower(ns, T.data());
        if (R.status) return R;
        std::vector<cd> y(ns);
        for (int s = 0; s < ns; ++s) y[s] = (R.elocs[s] - emean) / double(ns);
        cholesky_solve(ns, T.data(), y.data());
#pragma omp parallel for schedule(static) num_threads(nt)
        for (long long p = 0; p < (long long)P; ++p) {
            cd acc = 0.;
            for (int s = 0; s < ns; ++s) acc += std::conj(O[size_t(s) * P + p]) * y[s];
            R.v[p] = acc;
        }
    }
    return R;
}

// ---------------------------------------------------------------------------
std::vector<uint64_t> basis_full(int n) {
    std::vector<uint64_t> b(size_t(1) << n);
    std::iota(b.begin(), b.end(), uint64_t(0));
    return b;
}

std::vector<uint64_t> basis_jz(int n, int nup) {
    // Basis/BasisJz.hpp:25-30: next integer with the same popcount (Gosper's hack)
    std::vector<uint64_t> b;
    if (nup == 0) {
        b.push_back(0);
        return b;
    }
    uint64_t v = (uint64_t(1) << nup) - 1;
    const uint64_t last = v << (n - nup);
    while (true) {
        b.push_back(v);
        if (v == last) break;
        uint64_t t = v | (v - 1);
        v = (t + 1) | (((~t & (t + 1)) - 1) >> (__builtin_ctzll(v) + 1));
    }
    return b;
}

namespace {
struct CSR {
    std::vector<size_t> ptr;
    std::vector<uint32_t> col;
    std::vector<double> val;
};
// ED/ConstructSparseMat.hpp:32-57: row idx gets the column map of basis[idx]
// restricted to the basis via lower_bound (duplicates summed).
CSR build_csr(const Ham& H, const std::vector<uint64_t>& basis, int nt) {
    const size_t dim = basis.size();
    std::vector<std::vector<std::pair<uint32_t, double>>> rows(dim);
#pragma omp parallel for schedule(dynamic, 256) num_threads(nt)
    for (long long idx = 0; idx < (long long)dim; ++idx) {
        auto mcol = ham_column(H, basis[idx]);
        auto it = basis.begin();
        std::map<uint32_t, double> acc;
        for (auto& kv : mcol) {
            it = std::lower_bound(it, basis.end(), kv.first);
            if (it == basis.end()) break;
            acc[uint32_t(it - basis.begin())] += kv.second;
        }
        rows[idx].assign(acc.begin(), acc.end());
    }
    CSR A;
    A.ptr.resize(dim + 1, 0);
    for (size_t i = 0; i < dim; ++i) A.ptr[i + 1] = A.ptr[i] + rows[i].size();
    A.col.resize(A.ptr[dim]);
    A.val.resize(A.ptr[dim]);
    for (size_t i = 0; i < dim; ++i)
        for (size_t k = 0; k < rows[i].size(); ++k) {
            A.col[A.ptr[i] + k] = rows[i][k].first;
            A.val[A.ptr[i] + k] = rows[i][k].second;
        }
    return A;
}
}  // namespace

ExactResult exact_sr(const RBM& q, const Ham& H, const std::vector<uint64_t>& basis, int nthreads, bool with_S) {
    const int nt = nthreads_or_default(nthreads);
    const size_t dim = basis.size(), P = q.dim();
    ExactResult X;
    std::vector<cd> psi(dim);
    std::vector<cd> O(dim * P);
#pragma omp parallel for schedule(static) num_threads(nt)
    for (long long s = 0; s < (long long)dim; ++s) {
        std::vector<int8_t> sg(q.n);
        std::vector<cd> th(q.m);
        for (int i = 0; i < q.n; ++i) sg[i] = ((basis[s] >> i) & 1u) ? int8_t(-1) : int8_t(1);
        q.theta(sg.data(), th.data());
        psi[s] = q.coeff(sg.data(), th.data());
        q.logDeriv(sg.data(), th.data(), O.data() + size_t(s) * P);
    }
    double nrm = 0.;
    for (auto& v : psi) nrm += std::norm(v);
    nrm = std::sqrt(nrm);
    for (auto& v : psi) v /= nrm;
    CSR A = build_csr(H, basis, nt);
    std::vector<cd> k(dim);
#pragma omp parallel for schedule(static) num_threads(nt)
    for (long long i = 0; i < (long long)dim; ++i) {
        cd acc = 0.;
        for (size_t e = A.ptr[i]; e < A.ptr[i + 1]; ++e) acc += A.val[e] * psi[A.col[e]];
        k[i] = acc;
    }
    cd t = 0.;
    double kk = 0.;
    for (size_t i = 0; i < dim; ++i) {
        t += std::conj(psi[i]) * k[i];
        kk += std::norm(k[i]);
    }
    X.energy = t.real();
    X.energy_var = kk - X.energy * X.energy;
    X.oloc.assign(P, cd{});
    X.grad.assign(P, cd{});
#pragma omp parallel for schedule(static) num_threads(nt)
    for (long long p = 0; p < (long long)P; ++p) {
        cd ol = 0., g = 0.;
        for (size_t s = 0; s < dim; ++s) {
            const cd o = O[s * P + p];
            ol += std::norm(psi[s]) * o;
            g += std::conj(psi[s] * o) * k[s];
        }
        X.oloc[p] = ol;
        X.grad[p] = g;
    }
    for (size_t p = 0; p < P; ++p) X.grad[p] -= t * std::conj(X.oloc[p]);
    if (!with_S) return X;
    X.S.assign(P * P, cd{});
#pragma omp parallel for schedule(dynamic, 4) num_threads(nt)
    for (long long a = 0; a < (long long)P; ++a)
        for (size_t b = 0; b < P; ++b) {
            cd acc = 0.;
            for (size_t s = 0; s < dim; ++s) acc += std::norm(psi[s]) * std::conj(O[s * P + a]) * O[s * P + b];
            X.S[size_t(a) * P + b] = acc - std::conj(X.oloc[a]) * X.oloc[b];
        }
    return X;
}

std::vector<uint32_t> exact_sample(const RBM& q, const std::vector<uint64_t>& basis, int nsamples, uint64_t seed,
                                   uint32_t epoch, int nthreads) {
    const int nt = nthreads_or_default(nthreads);
    const size_t dim = basis.size();
    std::vector<double> probs(dim);
#pragma omp parallel for schedule(static) num_threads(nt)
    for (long long s = 0; s < (long long)dim; ++s) {
        std::vector<int8_t> sg(q.n);
        std::vector<cd> th(q.m);
        for (int i = 0; i < q.n; ++i) sg[i] = ((basis[s] >> i) & 1u) ? int8_t(-1) : int8_t(1);
        q.theta(sg.data(), th.data());
        probs[s] = std::norm(q.coeff(sg.data(), th.data()));
    }
    std::vector<long double> accum;
    accum.reserve(dim);
    long double tot = 0.0L;
    for (size_t k = 0; k < dim; ++k) {
        tot += probs[k];
        accum.push_back(tot);
    }
    const long double total = accum.back();
    accum.back() += 1e-8L;
    std::vector<uint32_t> out(static_cast<size_t>(nsamples));
    for (int i = 0; i < nsamples; ++i) {
        uint32_t x[4];
        Philox4x32::draw(seed, uint32_t(i), epoch, 0u, TAG_EXACT, x);
        const long double r = (long double)draw_u53(x[2], x[3]) * total;
        out[size_t(i)] = uint32_t(std::lower_bound(accum.begin(), accum.end(), r) - accum.begin());
    }
    return out;
}

// Lanczos with full reorthogonalisation; smallest Ritz value by Sturm bisection.
static double tridiag_min_eig(const std::vector<double>& al, const std::vector<double>& be) {
    const int k = int(al.size());
    double lo = 1e300, hi = -1e300;
    for (int i = 0; i < k; ++i) {
        double r = (i > 0 ? std::fabs(be[i - 1]) : 0.) + (i + 1 < k ? std::fabs(be[i]) : 0.);
        lo = std::min(lo, al[i] - r);
        hi = std::max(hi, al[i] + r);
    }
    auto count_below = [&](double x) {
        int c = 0;
        double d = 1.;
        for (int i = 0; i < k; ++i) {
            double b2 = i > 0 ? be[i - 1] * be[i - 1] : 0.;
            d = al[i] - x - (i > 0 ? b2 / d : 0.);
            if (d == 0.) d = 1e-300;
            if (d < 0) ++c;
        }
        return c;
    };
    for (int it = 0; it < 200; ++it) {
        double mid = 0.5 * (lo + hi);
        if (count_below(mid) >= 1)
            hi = mid;
        else
            lo = mid;
        if (hi - lo < 1e-14 * std::max(1.0, std::fabs(mid))) break;
    }
    return 0.5 * (lo + hi);
}

double ed_ground_energy(const Ham& H, const std::vector<uint64_t>& basis, int maxit, int nthreads) {
    const int nt = nthreads_or_default(nthreads);
    CSR A = build_csr(H, basis, nt);
    const size_t dim = basis.size();
    if (dim == 1) return A.val.empty() ? 0. : A.val[0];
    maxit = std::min<int>(maxit, int(dim));
    std::vector<std::vector<double>> V;
    std::vector<double> v(dim), w(dim), al, be;
    double nrm = 0.;
    for (size_t i = 0; i < dim; ++i) {
        v[i] = normal_pair(0x4c414e43ULL, uint32_t(i), nullptr);
        nrm += v[i] * v[i];
    }
    nrm = std::sqrt(nrm);
    for (auto& x : v) x /= nrm;
    double prev = 0.;
    for (int it = 0; it < maxit; ++it) {
        V.push_back(v);
#pragma omp parallel for schedule(static) num_threads(nt)
        for (long long i = 0; i < (long long)dim; ++i) {
            double acc = 0.;
            for (size_t e = A.ptr[i]; e < A.ptr[i + 1]; ++e) acc += A.val[e] * v[A.col[e]];
            w[i] = acc;
        }
        double a = 0.;
        for (size_t i = 0; i < dim; ++i) a += w[i] * v[i];
        al.push_back(a);
        for (int pass = 0; pass < 2; ++pass)
            for (auto& u : V) {
                double c = 0.;
                for (size_t i = 0; i < dim; ++i) c += u[i] * w[i];
                for (size_t i = 0; i < dim; ++i) w[i] -= c * u[i];
            }
        double b = 0.;
        for (size_t i = 0; i < dim; ++i) b += w[i] * w[i];
        b = std::sqrt(b);
        double cur = tridiag_min_eig(al, be);
        if ((it > 10 && std::fabs(cur - prev) < 1e-13 * std::max(1.0, std::fabs(cur))) || b < 1e-12) return cur;
        prev = cur;
        be.push_back(b);
        for (size_t i = 0; i < dim; ++i) v[i] = w[i] / b;
    }
    return tridiag_min_eig(al, std::vector<double>(be.begin(), be.begin() + (al.size() - 1)));
}

// ---------------------------------------------------------------------------
namespace {
struct FFActs {
    std::vector<double> in, z1, a1, z2;
};
void ff_fwd(const FFNet& f, const int8_t* s, FFActs& A) {
    const int L = f.L, C = f.conv_out, K = f.conv_k, F = f.fc_out, I = L * C;
    A.in.assign(L, 0.);
    for (int r = 0; r < L; ++r) A.in[r] = double(s[r]);
    // layers/Conv1D.hpp:144-171 (inChannels = 1, stride 1, no bias)
    A.z1.assign(I, 0.);
    for (int oc = 0; oc < C; ++oc)
        for (int r = 0; r < L; ++r)
            for (int ki = 0; ki < K; ++ki)
                A.z1[r + oc * L] += f.p[ki + size_t(K) * oc] * A.in[(r + ki - K / 2 + L) % L];
    A.a1.resize(I);
    for (int i = 0; i < I; ++i) A.a1[i] = logCosh(A.z1[i]);  // activations.hpp:83-87
    // layers/FullyConnected.hpp:150-157: z = W^T x, W (I x F) column-major
    const double* Wfc = f.p + size_t(K) * C;
    A.z2.assign(F, 0.);
    for (int o = 0; o < F; ++o) {
        double acc = 0.;
        for (int i = 0; i < I; ++i) acc += Wfc[i + size_t(I) * o] * A.a1[i];
        A.z2[o] = acc;
    }
}
}  // namespace

double ff_forward(const FFNet& f, const int8_t* s) {
    FFActs A;
    ff_fwd(f, s, A);
    double r = 0.;
    for (double z : A.z2) r += logCosh(z);  // LnCosh then Sum (= fc_out * Mean, layers/Mean.hpp:92-103)
    return r;
}

void ff_backward(const FFNet& f, const int8_t* s, double* der) {
    // Machines/FeedForward.hpp:186-205 with dout = 1 at the output
    FFActs A;
    ff_fwd(f, s, A);
    const int L = f.L, C = f.conv_out, K = f.conv_k, F = f.fc_out, I = L * C;
    std::vector<double> d2(F), d1(I, 0.), dz1(I);
    for (int o = 0; o < F; ++o) d2[o] = 1.0 * std::tanh(A.z2[o]);  // Sum, then LnCosh Jacobian
    const double* Wfc = f.p + size_t(K) * C;
    double* der_fc = der + size_t(K) * C;
    for (int o = 0; o < F; ++o)  // FullyConnected.hpp:170-178
        for (int i = 0; i < I; ++i) der_fc[i + size_t(I) * o] = A.a1[i] * d2[o];
    for (int i = 0; i < I; ++i) {
        double acc = 0.;
        for (int o = 0; o < F; ++o) acc += Wfc[i + size_t(I) * o] * d2[o];
        d1[i] = acc;
    }
    for (int i = 0; i < I; ++i) dz1[i] = d1[i] * std::tanh(A.z1[i]);
    for (int k = 0; k < K * C; ++k) der[k] = 0.;  // Conv1D.hpp:197-212
    for (int oc = 0; oc < C; ++oc)
        for (int r = 0; r < L; ++r)
            for (int ki = 0; ki < K; ++ki)
                der[ki + size_t(K) * oc] += A.in[(r + ki - K / 2 + L) % L] * dz1[r + oc * L];
}


// ---------------------------------------------------------------------------
// AmplitudePhase machine and NGDExact.

void ap_layout(APNet& q) {
    q.Pa = size_t(q.n) * q.m + (q.bias ? size_t(q.n + q.m) : 0);
    int size = q.n;
    size_t off = q.Pa;
    for (Layer& L : q.layers) {
        L.in_size = size;
        L.off = off;
        if (L.type == L_CONV1D) {  // layers/Conv1D.hpp:57-65, :104-106
            if (L.a < 1 || L.b < 1 || L.k < 1 || L.stride < 1 || size % L.a) throw std::runtime_error("conv1d shape");
            const int in_len = size / L.a;
            if (L.k / 2 > in_len) throw std::runtime_error("conv1d kernel");
            L.out_size = (in_len / L.stride) * L.b;
            L.npar = size_t(L.a) * L.b * L.k + (L.bias ? size_t(L.b) : 0);
        } else if (L.type == L_FC) {  // layers/FullyConnected.hpp
            if (L.a != size || L.b < 1) throw std::runtime_error("fc shape");
            L.out_size = L.b;
            L.npar = size_t(L.a) * L.b + (L.bias ? size_t(L.b) : 0);
        } else {
            L.out_size = size;
            L.npar = 0;
        }
        off += L.npar;
        size = L.out_size;
    }
    if (size != 1) throw std::runtime_error("the phase network must end in one output");
    q.Pp = off - q.Pa;
}

// activations.hpp forward and ApplyJacobian, as written there
static double act_fwd(const Layer& L, double z) {
    switch (L.type) {
        case A_IDENTITY: return z;
        case A_LNCOSH: return logCosh(z);
        case A_TANH: return L.x * std::tanh(z / L.x);
        case A_WEAKTANH: return z - std::tanh(z) / 2.0;
        case A_SIGMOID: return std::exp(z) + 1.;  // activations.hpp:215-220 (the inverse() results are discarded)
        case A_RELU: return std::max(z, 0.0);
        case A_LEAKYRELU: return z > 0 ? z : L.x * z;
        case A_HARDTANH: return std::abs(z) > 1.0 ? std::copysign(1.0, z) : z;
        case A_SOFTSHRINK: return std::abs(z) < 1.0 ? 0.0 : (z - std::copysign(1.0, z));
        case A_LEAKYHARDTANH: {
            double v = std::abs(z) > 1.0 ? std::copysign(1.0, z) : z;
            v += std::abs(z) < 1.0 ? 0.0 : L.x * (z - std::copysign(1.0, z));
            return v;
        }
        case A_SOFTSIGN: return z / (std::abs(z) + 1.0);
        case A_COS: return L.x * std::cos(z * M_PI / L.x);
        default: throw std::runtime_error("unknown activation");
    }
}
static double act_jac(const Layer& L, double z, double a, double f) {
    switch (L.type) {
        case A_IDENTITY: return f;
        case A_LNCOSH: return f * std::tanh(z);
        case A_TANH: return f * (1. - a * a / (L.x * L.x));
        case A_WEAKTANH: {
            const double t = std::tanh(z);
            return f * (1.0 + t * t) / 2.0;
        }
        case A_SIGMOID: return (1. - a) * a;  // activations.hpp:226-229 (F unused)
        case A_RELU: return z > 0 ? f : 0.0;
        case A_LEAKYRELU: return z > 0 ? f : L.x * f;
        case A_HARDTANH: return std::abs(z) > 1.0 ? 0.0 : f;
        case A_SOFTSHRINK: return std::abs(z) < 1.0 ? 0.0 : f;
        case A_LEAKYHARDTANH: return std::abs(z) > 1.0 ? L.x * f : f;
        case A_SOFTSIGN: {
            const double d = 1.0 + std::abs(z);
            return (1.0 / (d * d)) * f;
        }
        case A_COS: return -M_PI * std::sin(M_PI * z / L.x) * f;
        default: throw std::runtime_error("unknown activation");
    }
}

std::vector<std::vector<double>> ap_phase_data(const APNet& q, const int8_t* s) {
    std::vector<std::vector<double>> data;
    data.emplace_back(s, s + q.n);
    for (const Layer& L : q.layers) {
        const std::vector<double>& in = data.back();
        std::vector<double> out(size_t(L.out_size), 0.0);
        const double* w = q.p + L.off;
        if (L.type == L_CONV1D) {  // Conv1D.hpp:144-171
            const int in_len = L.in_size / L.a, out_len = in_len / L.stride, K = L.k;
            for (int oc = 0; oc < L.b; ++oc)
                for (int r = 0; r < out_len; ++r)
                    for (int ic = 0; ic < L.a; ++ic)
                        for (int ki = 0; ki < K; ++ki)
                            out[size_t(r + oc * out_len)] +=
                                w[size_t(ki + ic * K) + size_t(oc) * L.a * K] *
                                in[size_t((r * L.stride + ki - K / 2 + in_len) % in_len + ic * in_len)];
            if (L.bias) {
                const double* b = w + size_t(L.a) * L.b * K;
                for (int oc = 0; oc < L.b; ++oc)
                    for (int r = 0; r < out_len; ++r) out[size_t(r + oc * out_len)] += b[oc];
            }
        } else if (L.type == L_FC) {  // FullyConnected.hpp forward: bias + W^T in
            for (int o = 0; o < L.b; ++o) {
                double acc = L.bias ? w[size_t(L.a) * L.b + o] : 0.0;
                double t = 0.;
                for (int i = 0; i < L.a; ++i) t += w[size_t(i) + size_t(o) * L.a] * in[size_t(i)];
                out[size_t(o)] = acc + t;
            }
        } else {
            for (int i = 0; i < L.in_size; ++i) out[size_t(i)] = act_fwd(L, in[size_t(i)]);
        }
        data.push_back(std::move(out));
    }
    return data;
}

// FeedForward::backward (FeedForward.hpp:186-205) with dout = 1
void ap_phase_backward(const APNet& q, const std::vector<std::vector<double>>& data, double* der) {
    std::vector<double> dout(1, 1.0);
    for (int idx = int(q.layers.size()) - 1; idx >= 0; --idx) {
        const Layer& L = q.layers[size_t(idx)];
        const std::vector<double>& prev = data[size_t(idx)];
        const std::vector<double>& cur = data[size_t(idx) + 1];
        std::vector<double> din(size_t(L.in_size), 0.0);
        const double* w = q.p + L.off;
        double* d = der + (L.off - q.Pa);
        if (L.type == L_CONV1D) {  // Conv1D.hpp:173-225
            const int in_len = L.in_size / L.a, out_len = in_len / L.stride, K = L.k;
            for (size_t e = 0; e < L.npar; ++e) d[e] = 0.0;
            for (int oc = 0; oc < L.b; ++oc)
                for (int r = 0; r < out_len; ++r)
                    for (int ic = 0; ic < L.a; ++ic)
                        for (int ki = 0; ki < K; ++ki) {
                            const size_t src = size_t((r * L.stride + ki - K / 2 + in_len) % in_len + ic * in_len);
                            const size_t wi = size_t(ki + ic * K) + size_t(oc) * L.a * K;
                            din[src] += w[wi] * dout[size_t(r + oc * out_len)];
                            d[wi] += prev[src] * dout[size_t(r + oc * out_len)];
                        }
            if (L.bias)
                for (int oc = 0; oc < L.b; ++oc)
                    for (int r = 0; r < out_len; ++r) d[size_t(L.a) * L.b * K + oc] += dout[size_t(r + oc * out_len)];
        } else if (L.type == L_FC) {  // FullyConnected.hpp backprop
            for (int o = 0; o < L.b; ++o)
                for (int i = 0; i < L.a; ++i) d[size_t(i) + size_t(o) * L.a] = prev[size_t(i)] * dout[size_t(o)];
            if (L.bias)
                for (int o = 0; o < L.b; ++o) d[size_t(L.a) * L.b + o] = dout[size_t(o)];
            for (int i = 0; i < L.a; ++i) {
                double t = 0.;
                for (int o = 0; o < L.b; ++o) t += w[size_t(i) + size_t(o) * L.a] * dout[size_t(o)];
                din[size_t(i)] = t;
            }
        } else {
            for (int i = 0; i < L.in_size; ++i)
                din[size_t(i)] = act_jac(L, prev[size_t(i)], cur[size_t(i)], dout[size_t(i)]);
        }
        dout = std::move(din);
    }
}

static void amp_theta(const APNet& q, const int8_t* s, std::vector<double>& th) {
    th.assign(size_t(q.m), 0.0);
    const size_t nm = size_t(q.n) * q.m;
    for (int j = 0; j < q.m; ++j) {
        double t = q.bias ? q.p[nm + q.n + j] : 0.0;
        for (int i = 0; i < q.n; ++i) t += q.p[size_t(j) + size_t(i) * q.m] * s[i];
        th[size_t(j)] = t;
    }
}

// Machines/RBM.hpp:367-378 for real T
double ap_log_amp(const APNet& q, const int8_t* s) {
    std::vector<double> th;
    amp_theta(q, s, th);
    const size_t nm = size_t(q.n) * q.m;
    double acc = 0.;
    if (q.bias)
        for (int i = 0; i < q.n; ++i) acc += q.p[nm + i] * s[i];
    for (int j = 0; j < q.m; ++j) acc += logCosh(th[size_t(j)]);
    return acc;
}

// AmplitudePhase::logDerivAmp = RBM::logDeriv / 2 (RBM.hpp:390-406)
void ap_log_deriv_amp(const APNet& q, const int8_t* s, double* out) {
    std::vector<double> th;
    amp_theta(q, s, th);
    const size_t nm = size_t(q.n) * q.m;
    for (int i = 0; i < q.n; ++i)
        for (int j = 0; j < q.m; ++j) out[size_t(i) * q.m + j] = s[i] * std::tanh(th[size_t(j)]) / 2.0;
    if (!q.bias) return;
    for (int i = 0; i < q.n; ++i) out[nm + i] = s[i] / 2.0;
    for (int j = 0; j < q.m; ++j) out[nm + q.n + j] = std::tanh(th[size_t(j)]) / 2.0;
}

// Real draws: entry e of the amplitude (order a, b, W by columns) and of the
// phase (layer by layer, FeedForward.hpp initializeRandom) uses the first normal
// of normal_pair(seed, e); the phase continues the counter after the amplitude.
void ap_init(const APNet& q, uint64_t seed, double sigma_amp, int mode, double* p) {
    uint32_t e = 0;
    const size_t nm = size_t(q.n) * q.m;
    if (q.bias) {
        for (int i = 0; i < q.n; ++i) p[nm + i] = sigma_amp * normal_pair(seed, e++, nullptr);
        for (int j = 0; j < q.m; ++j) p[nm + q.n + j] = sigma_amp * normal_pair(seed, e++, nullptr);
    }
    for (int i = 0; i < q.n; ++i)
        for (int j = 0; j < q.m; ++j) p[size_t(i) * q.m + j] = sigma_amp * normal_pair(seed, e++, nullptr);
    for (const Layer& L : q.layers) {
        if (L.npar == 0) continue;
        // fanIn / fanOut: Conv1D.hpp:227-234, FullyConnected.hpp
        const double fin = L.type == L_CONV1D ? double(L.a) * L.k : double(L.a);
        const double fout = L.type == L_CONV1D ? double(L.b) * L.k : double(L.b);
        const double sd = mode == 0 ? std::sqrt(1.0 / fin) : mode == 1 ? std::sqrt(2.0 / (fin + fout)) : std::sqrt(2.0 / fin);
        for (size_t k = 0; k < L.npar; ++k) p[L.off + k] = sd * normal_pair(seed, e++, nullptr);
    }
}

// GroundState/NGDExact.hpp:123-150 (constructExact), :177-189 (corrMat*)
NGDResult ngd_exact(const APNet& q, const Ham& H, const std::vector<uint64_t>& basis, bool with_corr, int nthreads) {
    const size_t dim = basis.size(), Pa = q.Pa, Pp = q.Pp;
    const int nt = nthreads_or_default(nthreads);
    std::vector<cd> psi(dim);
    std::vector<double> Da(dim * Pa), Dp(dim * Pp);
#pragma omp parallel for schedule(dynamic, 64) num_threads(nt)
    for (size_t k = 0; k < dim; ++k) {
        std::vector<int8_t> s(size_t(q.n));
        for (int i = 0; i < q.n; ++i) s[size_t(i)] = ((basis[k] >> i) & 1u) ? int8_t(-1) : int8_t(1);
        auto data = ap_phase_data(q, s.data());
        const double phi = data.back()[0];
        // AmplitudePhase::coeff: sqrt(A) exp(i pi phi)
        psi[k] = std::sqrt(std::exp(ap_log_amp(q, s.data()))) * std::exp(cd(0., M_PI * phi));
        ap_log_deriv_amp(q, s.data(), Da.data() + k * Pa);
        ap_phase_backward(q, data, Dp.data() + k * Pp);
        for (size_t c = 0; c < Pp; ++c) Dp[k * Pp + c] *= M_PI;  // logDerivPhase = pi * backward
    }
    double nrm = 0.;
    for (auto& z : psi) nrm += std::norm(z);
    nrm = std::sqrt(nrm);
    for (auto& z : psi) z /= nrm;
    // k = H_sub psi, H_sub(idx, j) = col(basis[idx])[basis[j]] (ED/ConstructSparseMat.hpp:31-56)
    std::vector<cd> kv(dim);
#pragma omp parallel for schedule(static) num_threads(nt)
    for (size_t idx = 0; idx < dim; ++idx) {
        auto col = ham_column(H, basis[idx]);
        cd acc = 0.;
        for (auto& e : col) {
            auto it = std::lower_bound(basis.begin(), basis.end(), e.first);
            if (it == basis.end() || *it != e.first) continue;
            acc += e.second * psi[size_t(it - basis.begin())];
        }
        kv[idx] = acc;
    }
    NGDResult R;
    cd e = 0.;
    for (size_t k = 0; k < dim; ++k) e += std::conj(psi[k]) * kv[k];
    R.energy = e.real();
    R.oloc_amp.assign(Pa, 0.);
    R.oloc_phase.assign(Pp, 0.);
    R.grad.assign(Pa + Pp, 0.);
    for (size_t k = 0; k < dim; ++k) {
        const double w = std::norm(psi[k]);
        const cd g = std::conj(psi[k]) * kv[k];
        for (size_t c = 0; c < Pa; ++c) {
            R.oloc_amp[c] += w * Da[k * Pa + c];
            R.grad[c] += 2.0 * Da[k * Pa + c] * g.real();
        }
        for (size_t c = 0; c < Pp; ++c) {
            R.oloc_phase[c] += w * Dp[k * Pp + c];
            R.grad[Pa + c] += 2.0 * Dp[k * Pp + c] * g.imag();
        }
    }
    for (size_t c = 0; c < Pa; ++c) R.grad[c] -= 2.0 * R.energy * R.oloc_amp[c];
    if (!with_corr) return R;
    auto corr = [&](const std::vector<double>& D, size_t P, const std::vector<double>& o, std::vector<double>& C) {
        C.assign(P * P, 0.);
#pragma omp parallel for schedule(dynamic, 4) num_threads(nt)
        for (size_t r = 0; r < P; ++r)
            for (size_t c = 0; c <= r; ++c) {
                double t = 0.;
                for (size_t k = 0; k < dim; ++k) t += D[k * P + r] * std::norm(psi[k]) * D[k * P + c];
                t -= o[r] * o[c];
                C[r * P + c] = t;
                C[c * P + r] = t;
            }
    };
    corr(Da, Pa, R.oloc_amp, R.corr_amp);
    corr(Dp, Pp, R.oloc_phase, R.corr_phase);
    return R;
}

}  // namespace orc
