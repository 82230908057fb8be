// C ABI of libyannq_b200 (include/yannq_b200.h): argument checks, host staging
// for the batch entry points, and the VMC iteration driver.
#include <cstring>
#include <memory>
#include <string>
#include <vector>

#include "chol.hpp"
#include "internal.hpp"

namespace yq {
std::atomic<unsigned long long> g_launches{0};
std::atomic<unsigned long long> g_device_allocs{0};
void record_error(const std::string& msg);
}

using namespace yq;

namespace {
thread_local std::string g_last_error;

template <class F>
int guard(F&& f) {
    try {
        f();
        return YQ_OK;
    } catch (const Error& e) {
        g_last_error = e.what();
        return e.code;
    } catch (const std::bad_alloc&) {
        g_last_error = "host allocation failed";
        return YQ_E_NOMEM;
    } catch (const std::exception& e) {
        g_last_error = e.what();
        return YQ_E_ARG;
    }
}

}  // namespace

// Lets entry points defined in other files report their failure to yq_last_error().
void yq::record_error(const std::string& msg) { g_last_error = msg; }

namespace {

void need(const void* p, const char* what) {
    if (!p) throw Error(YQ_E_ARG, std::string("null argument: ") + what);
}

// staging helpers
struct Staging {
    DevBuf buf;
    template <typename T>
    T* up(const T* host, size_t count, cudaStream_t st) {
        buf.ensure(count * sizeof(T) + 16);
        if (count) YQ_CUDA(cudaMemcpyAsync(buf.p, host, count * sizeof(T), cudaMemcpyHostToDevice, st));
        return buf.as<T>();
    }
    template <typename T>
    T* alloc(size_t count) {
        buf.ensure(count * sizeof(T) + 16);
        return buf.as<T>();
    }
};

template <typename T>
void down(T* host, const void* dev, size_t count, cudaStream_t st) {
    if (count) YQ_CUDA(cudaMemcpyAsync(host, dev, count * sizeof(T), cudaMemcpyDeviceToHost, st));
    YQ_CUDA(cudaStreamSynchronize(st));
}

__global__ void c128_to_c64_kernel(size_t n, const c128* __restrict__ a, c64* __restrict__ b) {
    for (size_t i = size_t(blockIdx.x) * blockDim.x + threadIdx.x; i < n; i += size_t(gridDim.x) * blockDim.x)
        b[i] = cast<float>(a[i]);
}
__global__ void c64_to_c128_kernel(size_t n, const c64* __restrict__ a, c128* __restrict__ b) {
    for (size_t i = size_t(blockIdx.x) * blockDim.x + threadIdx.x; i < n; i += size_t(gridDim.x) * blockDim.x)
        b[i] = cast<double>(a[i]);
}

// Upload a host theta (c128) as the RBM's compute type.
void* upload_theta(yq_rbm_s* q, const double* theta, size_t count, Staging& s64, Staging& sc) {
    cudaStream_t st = q->ctx->stream;
    c128* d64 = s64.up(reinterpret_cast<const c128*>(theta), count, st);
    if (q->dtype == YQ_C128) return d64;
    c64* d32 = sc.alloc<c64>(count);
    c128_to_c64_kernel<<<std::min<unsigned>(cdiv_u(count, 256), 4096u), 256, 0, st>>>(count, d64, d32);
    YQ_LAUNCH_CHECK();
    return d32;
}

void check_sigma(const int8_t* s, size_t count) {
    for (size_t i = 0; i < count; ++i)
        if (s[i] != 1 && s[i] != -1) throw Error(YQ_E_ARG, "sigma entries must be +1 or -1");
}

int status_to_code(int ds) {
    if (ds & DS_TIMEOUT) return YQ_E_TIMEOUT;
    if (ds & DS_NOT_PD) return YQ_E_NOT_PD;
    if (ds & DS_NONFINITE) return YQ_E_NONFINITE;
    return YQ_OK;
}
const char* status_msg(int code) {
    switch (code) {
        case YQ_E_TIMEOUT: return "a bounded device wait timed out";
        case YQ_E_NOT_PD: return "Cholesky met a non-positive pivot (matrix not positive definite)";
        case YQ_E_NONFINITE: return "non-finite value in E_loc, O, S/T or the update";
        default: return "ok";
    }
}
void raise_device_status(yq_ctx_s* ctx) {
    int code = status_to_code(ctx->read_status_and_clear());
    if (code != YQ_OK) throw Error(code, status_msg(code));
}
}  // namespace

// ---------------------------------------------------------------------------
void yq_ctx_s::stage_begin(int s) {
    if (timing) cudaEventRecord(ev_start[s], stream);
}
void yq_ctx_s::stage_end(int s) {
    if (!timing) return;
    cudaEventRecord(ev_stop[s], stream);
    ev_used[s] = true;
}
int yq_ctx_s::read_status_and_clear() {
    int h = 0;
    YQ_CUDA(cudaMemcpyAsync(&h, status.p, sizeof(int), cudaMemcpyDeviceToHost, stream));
    YQ_CUDA(cudaStreamSynchronize(stream));
    if (h) YQ_CUDA(cudaMemsetAsync(status.p, 0, sizeof(int), stream));
    return h;
}

extern "C" {

int yq_last_error(char* buf, size_t len) {
    if (!buf || len == 0) return YQ_E_ARG;
    std::strncpy(buf, g_last_error.c_str(), len - 1);
    buf[len - 1] = '\0';
    return YQ_OK;
}

const char* yq_version(void) { return "yannq_b200 0.1 sm_100a"; }

int yq_launch_count(uint64_t* out) {
    return guard([&] {
        need(out, "out");
        *out = g_launches.load(std::memory_order_relaxed);
    });
}

int yq_alloc_count(uint64_t* out) {
    return guard([&] {
        need(out, "out");
        *out = g_device_allocs.load(std::memory_order_relaxed);
    });
}

int yq_host_alloc(size_t bytes, void** out) {
    return guard([&] {
        need(out, "out");
        *out = nullptr;
        YQ_CUDA(cudaHostAlloc(out, bytes ? bytes : 1, cudaHostAllocDefault));
    });
}

int yq_host_free(void* p) {
    return guard([&] {
        if (p) YQ_CUDA(cudaFreeHost(p));
    });
}

int yq_ctx_create(int device, yq_ctx* out) {
    return guard([&] {
        need(out, "out");
        *out = nullptr;
        int ndev = 0;
        YQ_CUDA(cudaGetDeviceCount(&ndev));
        if (device < 0 || device >= ndev) throw Error(YQ_E_ARG, "device index out of range");
        YQ_CUDA(cudaSetDevice(device));
        auto* c = new yq_ctx_s();
        try {
            c->device = device;
            YQ_CUDA(cudaDeviceGetAttribute(&c->sm_count, cudaDevAttrMultiProcessorCount, device));
            int major = 0, minor = 0;
            YQ_CUDA(cudaDeviceGetAttribute(&major, cudaDevAttrComputeCapabilityMajor, device));
            YQ_CUDA(cudaDeviceGetAttribute(&minor, cudaDevAttrComputeCapabilityMinor, device));
            if (major != 10)
                throw Error(YQ_E_UNSUPPORTED, "libyannq_b200 is built for sm_100a; device is sm_" +
                                                  std::to_string(major) + std::to_string(minor));
            YQ_CUDA(cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking));
            for (int s = 0; s < ST_COUNT; ++s) {
                YQ_CUDA(cudaEventCreate(&c->ev_start[s]));
                YQ_CUDA(cudaEventCreate(&c->ev_stop[s]));
            }
            c->status.ensure(sizeof(int) * 4);
            YQ_CUDA(cudaMemset(c->status.p, 0, sizeof(int) * 4));
            c->scratch.ensure(64 * 1024);
        } catch (...) {
            delete c;
            throw;
        }
        *out = c;
    });
}

int yq_ctx_destroy(yq_ctx c) {
    return guard([&] {
        if (!c) return;
        cudaSetDevice(c->device);
        cudaStreamSynchronize(c->stream);
        for (int s = 0; s < ST_COUNT; ++s) {
            if (c->ev_start[s]) cudaEventDestroy(c->ev_start[s]);
            if (c->ev_stop[s]) cudaEventDestroy(c->ev_stop[s]);
        }
        if (c->stream) cudaStreamDestroy(c->stream);
        delete c;
    });
}

int yq_ctx_synchronize(yq_ctx c) {
    return guard([&] {
        need(c, "ctx");
        YQ_CUDA(cudaStreamSynchronize(c->stream));
    });
}

int yq_ctx_stage_ms(yq_ctx c, int stage, float* ms) {
    return guard([&] {
        need(c, "ctx");
        need(ms, "ms");
        if (stage < 0 || stage >= ST_COUNT) throw Error(YQ_E_ARG, "stage index out of range");
        if (!c->ev_used[stage]) {
            *ms = 0.f;
            return;
        }
        YQ_CUDA(cudaEventSynchronize(c->ev_stop[stage]));
        YQ_CUDA(cudaEventElapsedTime(ms, c->ev_start[stage], c->ev_stop[stage]));
    });
}

// ---- RBM --------------------------------------------------------------------
int yq_rbm_create(yq_ctx ctx, int n, int m, int use_bias, int dtype, yq_rbm* out) {
    return guard([&] {
        need(ctx, "ctx");
        need(out, "out");
        *out = nullptr;
        if (n < 1 || m < 1 || n > 65535 || m > 1024) throw Error(YQ_E_ARG, "rbm: need 1 <= n <= 65535, 1 <= m <= 1024");
        if (dtype != YQ_C64 && dtype != YQ_C128) throw Error(YQ_E_ARG, "rbm: dtype must be YQ_C64 or YQ_C128");
        YQ_CUDA(cudaSetDevice(ctx->device));
        auto* q = new yq_rbm_s();
        try {
            q->ctx = ctx;
            q->n = n;
            q->m = m;
            q->use_bias = use_bias != 0;
            q->dtype = dtype;
            q->P = size_t(n) * m + (q->use_bias ? size_t(n) + m : 0);
            const size_t nm = size_t(n) * m;
            // the master copy always carries a, b slots (zero without bias)
            q->p64.ensure((nm + n + m) * sizeof(c128));
            YQ_CUDA(cudaMemsetAsync(q->p64.p, 0, (nm + n + m) * sizeof(c128), ctx->stream));
            const size_t cs = q->csize();
            q->W.ensure(nm * cs);
            q->tau.ensure(nm * cs);
            q->tauT.ensure(nm * cs);
            q->a.ensure(size_t(n) * cs);
            q->b.ensure(size_t(m) * cs);
            q->Lk.ensure(size_t(n) * sizeof(c128));
        } catch (...) {
            delete q;
            throw;
        }
        *out = q;
    });
}

int yq_rbm_destroy(yq_rbm q) {
    return guard([&] {
        if (!q) return;
        cudaStreamSynchronize(q->ctx->stream);
        delete q;
    });
}

int yq_rbm_dim(yq_rbm q, size_t* dim) {
    return guard([&] {
        need(q, "rbm");
        need(dim, "dim");
        *dim = q->P;
    });
}

int yq_rbm_set_params(yq_rbm q, const double* params) {
    return guard([&] {
        need(q, "rbm");
        need(params, "params");
        YQ_CUDA(cudaMemcpyAsync(q->p64.p, params, q->P * sizeof(c128), cudaMemcpyHostToDevice, q->ctx->stream));
        q->version++;
    });
}

int yq_rbm_archive_size(yq_rbm q, int elem, size_t* size) {
    return guard([&] {
        need(q, "rbm");
        need(size, "size");
        *size = rbm_archive_size(q->n, q->m, q->use_bias, elem);
    });
}

int yq_rbm_save_archive(yq_rbm q, int elem, void* buf, size_t cap, size_t* size) {
    return guard([&] {
        need(q, "rbm");
        need(buf, "buf");
        std::vector<uint8_t> out;
        rbm_archive_write(q, elem, out);
        if (size) *size = out.size();
        if (cap < out.size()) throw Error(YQ_E_ARG, "archive: buffer smaller than yq_rbm_archive_size");
        std::memcpy(buf, out.data(), out.size());
    });
}

int yq_rbm_load_archive(yq_rbm q, int elem, const void* buf, size_t size) {
    return guard([&] {
        need(q, "rbm");
        need(buf, "buf");
        rbm_archive_read(q, elem, static_cast<const uint8_t*>(buf), size);
    });
}

int yq_rbm_archive_shape(const void* buf, size_t size, int* n, int* m, int* use_bias) {
    return guard([&] {
        need(buf, "buf");
        need(n, "n");
        need(m, "m");
        need(use_bias, "use_bias");
        rbm_archive_shape(static_cast<const uint8_t*>(buf), size, n, m, use_bias);
    });
}

int yq_rbm_save(yq_rbm q, int elem, const char* path) {
    return guard([&] {
        need(q, "rbm");
        need(path, "path");
        std::vector<uint8_t> out;
        rbm_archive_write(q, elem, out);
        write_file(path, out);
    });
}

int yq_rbm_load(yq_rbm q, int elem, const char* path) {
    return guard([&] {
        need(q, "rbm");
        need(path, "path");
        const std::vector<uint8_t> buf = read_file(path);
        rbm_archive_read(q, elem, buf.data(), buf.size());
    });
}

int yq_rbm_file_shape(const char* path, int* n, int* m, int* use_bias) {
    return guard([&] {
        need(path, "path");
        need(n, "n");
        need(m, "m");
        need(use_bias, "use_bias");
        const std::vector<uint8_t> buf = read_file(path);
        rbm_archive_shape(buf.data(), buf.size(), n, m, use_bias);
    });
}

int yq_rbm_get_params(yq_rbm q, double* params) {
    return guard([&] {
        need(q, "rbm");
        need(params, "params");
        down(reinterpret_cast<c128*>(params), q->p64.p, q->P, q->ctx->stream);
    });
}

int yq_rbm_update_params(yq_rbm q, const double* delta) {
    return guard([&] {
        need(q, "rbm");
        need(delta, "delta");
        std::vector<c128> cur(q->P);
        down(cur.data(), q->p64.p, q->P, q->ctx->stream);
        const c128* d = reinterpret_cast<const c128*>(delta);
        for (size_t i = 0; i < q->P; ++i) cur[i] = cur[i] + d[i];
        YQ_CUDA(cudaMemcpyAsync(q->p64.p, cur.data(), q->P * sizeof(c128), cudaMemcpyHostToDevice, q->ctx->stream));
        YQ_CUDA(cudaStreamSynchronize(q->ctx->stream));
        q->version++;
    });
}

int yq_rbm_init_random(yq_rbm q, uint64_t seed, double sd) {
    return guard([&] {
        need(q, "rbm");
        if (!(sd >= 0.0)) throw Error(YQ_E_ARG, "init_random: sd must be >= 0");
        std::vector<c128> p(q->P);
        rbm_init_params_host(q->n, q->m, q->use_bias, seed, sd, p.data());
        YQ_CUDA(cudaMemcpyAsync(q->p64.p, p.data(), q->P * sizeof(c128), cudaMemcpyHostToDevice, q->ctx->stream));
        YQ_CUDA(cudaStreamSynchronize(q->ctx->stream));
        q->version++;
    });
}

int yq_rbm_theta(yq_rbm q, int ns, const int8_t* sigma, double* theta) {
    return guard([&] {
        need(q, "rbm");
        need(sigma, "sigma");
        need(theta, "theta");
        if (ns < 0 || ns > 65535) throw Error(YQ_E_ARG, "theta: need 0 <= ns <= 65535 per call");
        check_sigma(sigma, size_t(ns) * q->n);
        Staging ss, so;
        cudaStream_t st = q->ctx->stream;
        int8_t* ds = ss.up(sigma, size_t(ns) * q->n, st);
        c128* dt = so.alloc<c128>(size_t(ns) * q->m);
        rbm_theta(q, ns, ds, dt, true);
        down(reinterpret_cast<c128*>(theta), dt, size_t(ns) * q->m, st);
    });
}

int yq_rbm_log_psi(yq_rbm q, int ns, const int8_t* sigma, double* out) {
    return guard([&] {
        need(q, "rbm");
        need(sigma, "sigma");
        need(out, "out");
        if (ns < 0) throw Error(YQ_E_ARG, "ns < 0");
        check_sigma(sigma, size_t(ns) * q->n);
        Staging ss, so;
        cudaStream_t st = q->ctx->stream;
        int8_t* ds = ss.up(sigma, size_t(ns) * q->n, st);
        c128* d = so.alloc<c128>(ns);
        rbm_log_psi(q, ns, ds, d);
        down(reinterpret_cast<c128*>(out), d, ns, st);
    });
}

int yq_rbm_log_ratio(yq_rbm q, int ns, const int8_t* sigma, const double* theta, int nflip, const int* flips,
                     double* out) {
    return guard([&] {
        need(q, "rbm");
        need(sigma, "sigma");
        need(theta, "theta");
        need(flips, "flips");
        need(out, "out");
        if (ns < 0) throw Error(YQ_E_ARG, "ns < 0");
        if (nflip != 1 && nflip != 2) throw Error(YQ_E_ARG, "log_ratio: nflip must be 1 or 2");
        check_sigma(sigma, size_t(ns) * q->n);
        for (size_t i = 0; i < size_t(ns) * nflip; ++i)
            if (flips[i] < 0 || flips[i] >= q->n) throw Error(YQ_E_ARG, "log_ratio: flip site out of range");
        if (nflip == 2)
            for (int s = 0; s < ns; ++s)
                if (flips[2 * s] == flips[2 * s + 1]) throw Error(YQ_E_ARG, "log_ratio: the two flip sites coincide");
        Staging ss, st64, sf, so;
        cudaStream_t st = q->ctx->stream;
        int8_t* ds = ss.up(sigma, size_t(ns) * q->n, st);
        c128* dth = st64.up(reinterpret_cast<const c128*>(theta), size_t(ns) * q->m, st);
        int* df = sf.up(flips, size_t(ns) * nflip, st);
        c128* d = so.alloc<c128>(ns);
        rbm_log_ratio(q, ns, ds, dth, nflip, df, d);
        down(reinterpret_cast<c128*>(out), d, ns, st);
    });
}

int yq_rbm_log_ratio_k(yq_rbm q, int ns, const int8_t* sigma, const double* theta, int k, const int* flips,
                       double* out) {
    return guard([&] {
        need(q, "rbm");
        need(sigma, "sigma");
        need(theta, "theta");
        need(flips, "flips");
        need(out, "out");
        if (ns < 0) throw Error(YQ_E_ARG, "ns < 0");
        if (k < 1 || k > q->n) throw Error(YQ_E_ARG, "log_ratio_k: k must lie in [1, n]");
        check_sigma(sigma, size_t(ns) * q->n);
        for (int s = 0; s < ns; ++s)
            for (int e = 0; e < k; ++e) {
                const int f = flips[size_t(s) * k + e];
                if (f < 0 || f >= q->n) throw Error(YQ_E_ARG, "log_ratio_k: flip site out of range");
                for (int d = 0; d < e; ++d)
                    if (flips[size_t(s) * k + d] == f) throw Error(YQ_E_ARG, "log_ratio_k: repeated flip site");
            }
        Staging ss, st64, sf, so;
        cudaStream_t st = q->ctx->stream;
        int8_t* ds = ss.up(sigma, size_t(ns) * q->n, st);
        c128* dth = st64.up(reinterpret_cast<const c128*>(theta), size_t(ns) * q->m, st);
        int* df = sf.up(flips, size_t(ns) * k, st);
        c128* d = so.alloc<c128>(ns);
        rbm_log_ratio_k(q, ns, ds, dth, k, df, d);
        down(reinterpret_cast<c128*>(out), d, ns, st);
    });
}

int yq_rbm_log_ratio_states(yq_rbm q, int ns, const int8_t* sigma, const double* theta, const int8_t* sigma_other,
                            const double* theta_other, double* out) {
    return guard([&] {
        need(q, "rbm");
        need(sigma, "sigma");
        need(theta, "theta");
        need(sigma_other, "sigma_other");
        need(theta_other, "theta_other");
        need(out, "out");
        if (ns < 0) throw Error(YQ_E_ARG, "ns < 0");
        check_sigma(sigma, size_t(ns) * q->n);
        check_sigma(sigma_other, size_t(ns) * q->n);
        Staging sa, ta, sb, tb, so;
        cudaStream_t st = q->ctx->stream;
        int8_t* dsa = sa.up(sigma, size_t(ns) * q->n, st);
        c128* dta = ta.up(reinterpret_cast<const c128*>(theta), size_t(ns) * q->m, st);
        int8_t* dsb = sb.up(sigma_other, size_t(ns) * q->n, st);
        c128* dtb = tb.up(reinterpret_cast<const c128*>(theta_other), size_t(ns) * q->m, st);
        c128* d = so.alloc<c128>(ns);
        rbm_log_ratio_states(q, ns, dsa, dta, dsb, dtb, d);
        down(reinterpret_cast<c128*>(out), d, ns, st);
    });
}

int yq_rbm_log_deriv(yq_rbm q, int ns, const int8_t* sigma, const double* theta, double* out) {
    return guard([&] {
        need(q, "rbm");
        need(sigma, "sigma");
        need(theta, "theta");
        need(out, "out");
        if (ns < 0 || ns > 65535) throw Error(YQ_E_ARG, "log_deriv: need 0 <= ns <= 65535 per call");
        check_sigma(sigma, size_t(ns) * q->n);
        Staging ss, st64, so;
        cudaStream_t st = q->ctx->stream;
        int8_t* ds = ss.up(sigma, size_t(ns) * q->n, st);
        c128* dth = st64.up(reinterpret_cast<const c128*>(theta), size_t(ns) * q->m, st);
        c128* d = so.alloc<c128>(size_t(ns) * q->P);
        rbm_log_deriv(q, ns, ds, dth, d);
        down(reinterpret_cast<c128*>(out), d, size_t(ns) * q->P, st);
    });
}

// ---- Hamiltonians -----------------------------------------------------------
int yq_ham_create(yq_ctx ctx, int kind, int n, int lx, int ly, double J, double h, int sign_rule, yq_ham* out) {
    return guard([&] {
        need(ctx, "ctx");
        need(out, "out");
        *out = nullptr;
        if (kind != YQ_HAM_TFI && kind != YQ_HAM_XXZ && kind != YQ_HAM_TFI2D && kind != YQ_HAM_XXX &&
            kind != YQ_HAM_J1J2 && kind != YQ_HAM_XYZNNN)
            throw Error(YQ_E_ARG, kind == YQ_HAM_KITAEV_HEX ? "ham: KitaevHex is made by yq_ham_create_kitaev_hex"
                                                            : "ham: unknown kind");
        if (n < 2) throw Error(YQ_E_ARG, "ham: need n >= 2");
        if ((kind == YQ_HAM_J1J2 || kind == YQ_HAM_XYZNNN) && n < 3)
            throw Error(YQ_E_ARG, "ham: next-nearest-neighbour models need n >= 3");
        if (kind == YQ_HAM_TFI2D && (lx < 2 || ly < 2 || lx * ly != n))
            throw Error(YQ_E_ARG, "ham: TFI2D needs lx, ly >= 2 and lx * ly == n");
        auto H = std::make_unique<yq_ham_s>();
        H->ctx = ctx;
        H->kind = kind;
        H->n = n;
        H->lx = kind == YQ_HAM_TFI2D ? lx : 0;
        H->ly = kind == YQ_HAM_TFI2D ? ly : 0;
        H->J = J;
        H->h = h;
        H->sign = sign_rule ? -1.0 : 1.0;
        H->conserves_sz = kind == YQ_HAM_XXZ;
        if (kind >= YQ_HAM_XXX) ham_build_terms(H.get(), 0.0, 0.0);
        ham_build_moves(H.get());
        *out = H.release();
    });
}

int yq_ham_create_kitaev_hex(yq_ctx ctx, int ncol, int nrow, double Jx, double Jy, double Jz, double h,
                             yq_ham* out) {
    return guard([&] {
        need(ctx, "ctx");
        need(out, "out");
        *out = nullptr;
        if (ncol < 2 || nrow < 2 || ncol % 2 || nrow % 2)
            throw Error(YQ_E_ARG, "ham: KitaevHex needs even ncol, nrow >= 2");
        if (ncol > 65535 || nrow > 65535 || ncol * nrow > 65535) throw Error(YQ_E_ARG, "ham: KitaevHex lattice too large");
        auto H = std::make_unique<yq_ham_s>();
        H->ctx = ctx;
        H->kind = YQ_HAM_KITAEV_HEX;
        H->n = ncol * nrow;
        H->lx = ncol;
        H->ly = nrow;
        H->J = Jx;
        H->h = h;
        ham_build_terms(H.get(), Jy, Jz);
        ham_build_moves(H.get());
        *out = H.release();
    });
}

int yq_ham_destroy(yq_ham H) {
    return guard([&] { delete H; });
}

int yq_ham_num_offdiag(yq_ham H, int* count) {
    return guard([&] {
        need(H, "ham");
        need(count, "count");
        *count = ham_num_offdiag(H);
    });
}

int yq_ham_enumerate(yq_ham H, int ns, const int8_t* sigma, int* site_a, int* site_b, double* coeff, double* diag) {
    return guard([&] {
        need(H, "ham");
        need(sigma, "sigma");
        need(site_a, "site_a");
        need(site_b, "site_b");
        need(coeff, "coeff");
        need(diag, "diag");
        if (ns < 0) throw Error(YQ_E_ARG, "ns < 0");
        check_sigma(sigma, size_t(ns) * H->n);
        cudaStream_t st = H->ctx->stream;
        const size_t K = size_t(ham_num_offdiag(H));
        Staging ss, sa, sb, sc, sd;
        int8_t* ds = ss.up(sigma, size_t(ns) * H->n, st);
        int* da = sa.alloc<int>(size_t(ns) * K);
        int* db = sb.alloc<int>(size_t(ns) * K);
        double* dc = sc.alloc<double>(size_t(ns) * K);
        double* dd = sd.alloc<double>(ns);
        ham_enumerate(H, ns, ds, da, db, dc, dd);
        down(site_a, da, size_t(ns) * K, st);
        down(site_b, db, size_t(ns) * K, st);
        down(coeff, dc, size_t(ns) * K, st);
        down(diag, dd, size_t(ns), st);
    });
}

int yq_eloc(yq_ham H, yq_rbm q, int ns, const int8_t* sigma, const double* theta, double* out) {
    return guard([&] {
        need(H, "ham");
        need(q, "rbm");
        need(sigma, "sigma");
        need(theta, "theta");
        need(out, "out");
        if (ns < 0) throw Error(YQ_E_ARG, "ns < 0");
        if (H->n != q->n) throw Error(YQ_E_ARG, "eloc: Hamiltonian and RBM sizes differ");
        check_sigma(sigma, size_t(ns) * q->n);
        cudaStream_t st = q->ctx->stream;
        Staging ss, s64, sc, so;
        int8_t* ds = ss.up(sigma, size_t(ns) * q->n, st);
        void* dth = upload_theta(q, theta, size_t(ns) * q->m, s64, sc);
        c128* d = so.alloc<c128>(ns);
        ham_eloc(H, q, ns, ds, dth, d);
        down(reinterpret_cast<c128*>(out), d, ns, st);
        raise_device_status(q->ctx);
    });
}

// ---- sampler ------------------------------------------------------------------
int yq_sampler_create(yq_rbm q, int n_chains, int move, int nup, int sweep_len, yq_sampler* out) {
    return guard([&] {
        need(q, "rbm");
        need(out, "out");
        *out = nullptr;
        if (n_chains < 1) throw Error(YQ_E_ARG, "sampler: n_chains must be >= 1");
        if (move != YQ_MOVE_LOCAL && move != YQ_MOVE_EXCHANGE_ANY && move != YQ_MOVE_EXCHANGE_NN &&
            move != YQ_MOVE_HAMILTONIAN)
            throw Error(YQ_E_ARG, "sampler: unknown move");
        if (nup > q->n) throw Error(YQ_E_ARG, "sampler: nup > n");
        if (sweep_len < 0) throw Error(YQ_E_ARG, "sampler: sweep_len < 0");
        auto* S = new yq_sampler_s();
        try {
            S->q = q;
            S->n_chains = n_chains;
            S->move = move;
            S->nup = nup;
            S->sweep_len = sweep_len;
            S->chains.ensure(size_t(n_chains) * q->n);
            S->acc.ensure(size_t(n_chains) * sizeof(unsigned long long));
        } catch (...) {
            delete S;
            throw;
        }
        *out = S;
    });
}

int yq_sampler_destroy(yq_sampler S) {
    return guard([&] {
        if (!S) return;
        cudaStreamSynchronize(S->q->ctx->stream);
        delete S;
    });
}

int yq_sampler_set_hamiltonian(yq_sampler S, yq_ham H) {
    return guard([&] {
        need(S, "sampler");
        need(H, "ham");
        if (S->move != YQ_MOVE_HAMILTONIAN) throw Error(YQ_E_ARG, "sampler: not a HamiltonianSweeper sampler");
        if (H->n != S->q->n) throw Error(YQ_E_ARG, "sampler: Hamiltonian and RBM sizes differ");
        if (H->ctx->device != S->q->ctx->device) throw Error(YQ_E_ARG, "sampler: Hamiltonian on another device");
        S->ham = H;
    });
}

int yq_sampler_set_resync(yq_sampler S, int every) {
    return guard([&] {
        need(S, "sampler");
        if (every < 0) throw Error(YQ_E_ARG, "resync interval must be >= 0");
        S->resync = every;
    });
}

int yq_sampler_set_chains(yq_sampler S, const int8_t* sigma) {
    return guard([&] {
        need(S, "sampler");
        need(sigma, "sigma");
        check_sigma(sigma, size_t(S->n_chains) * S->q->n);
        YQ_CUDA(cudaMemcpyAsync(S->chains.p, sigma, size_t(S->n_chains) * S->q->n, cudaMemcpyHostToDevice,
                                S->q->ctx->stream));
        YQ_CUDA(cudaStreamSynchronize(S->q->ctx->stream));
        S->have_chains = true;
    });
}

int yq_sampler_get_chains(yq_sampler S, int8_t* sigma) {
    return guard([&] {
        need(S, "sampler");
        need(sigma, "sigma");
        if (!S->have_chains) throw Error(YQ_E_STATE, "sampler has no chains yet");
        down(sigma, S->chains.p, size_t(S->n_chains) * S->q->n, S->q->ctx->stream);
    });
}

int yq_sample(yq_sampler S, int n_sweeps, int n_discard, uint64_t seed, uint32_t epoch, int reinit) {
    return guard([&] {
        need(S, "sampler");
        yq_ctx_s* ctx = S->q->ctx;
        ctx->stage_begin(ST_SAMPLE);
        sampler_run(S, n_sweeps, n_discard, seed, epoch, reinit);
        ctx->stage_end(ST_SAMPLE);
    });
}

int yq_sampler_num_samples(yq_sampler S, int* ns) {
    return guard([&] {
        need(S, "sampler");
        need(ns, "ns");
        *ns = S->ns;
    });
}

int yq_sampler_get_samples(yq_sampler S, int8_t* sigma, double* theta) {
    return guard([&] {
        need(S, "sampler");
        yq_rbm_s* q = S->q;
        cudaStream_t st = q->ctx->stream;
        if (sigma) down(sigma, S->sigma.p, size_t(S->ns) * q->n, st);
        if (theta) {
            const size_t cnt = size_t(S->ns) * q->m;
            if (q->dtype == YQ_C128) {
                down(reinterpret_cast<c128*>(theta), S->theta.p, cnt, st);
            } else {
                Staging tmp;
                c128* d = tmp.alloc<c128>(cnt);
                c64_to_c128_kernel<<<std::min<unsigned>(cdiv_u(cnt, 256), 4096u), 256, 0, st>>>(cnt, S->theta.as<c64>(),
                                                                                               d);
                YQ_LAUNCH_CHECK();
                down(reinterpret_cast<c128*>(theta), d, cnt, st);
            }
        }
    });
}

int yq_sampler_get_accepts(yq_sampler S, uint64_t* acc) {
    return guard([&] {
        need(S, "sampler");
        need(acc, "acc");
        down(reinterpret_cast<unsigned long long*>(acc), S->acc.p, size_t(S->n_chains), S->q->ctx->stream);
    });
}

int yq_sampler_set_tempering(yq_sampler S, int ntemps) {
    return guard([&] {
        need(S, "sampler");
        if (ntemps < 1 || ntemps > 64 || (ntemps > 1 && ntemps % 2 != 0))
            throw Error(YQ_E_ARG, "set_tempering: ntemps must be 1 or even and at most 64");
        if (S->n_chains % ntemps != 0) throw Error(YQ_E_ARG, "set_tempering: n_chains must be a multiple of ntemps");
        S->ntemps = ntemps;
        S->pt_ready = false;
        if (ntemps > 1) {
            S->pt_slot.ensure(size_t(S->n_chains) * sizeof(int));
            S->pt_beta.ensure(size_t(S->n_chains) * sizeof(double));
        }
    });
}

int yq_sampler_get_slots(yq_sampler S, int* slots) {
    return guard([&] {
        need(S, "sampler");
        need(slots, "slots");
        if (S->ntemps <= 1 || !S->pt_ready) {
            for (int c = 0; c < S->n_chains; ++c) slots[c] = S->ntemps > 1 ? c % S->ntemps : 0;
            return;
        }
        down(slots, S->pt_slot.p, size_t(S->n_chains), S->q->ctx->stream);
    });
}

int yq_sampler_chains_per_cta(yq_sampler S, int* out) {
    return guard([&] {
        need(S, "sampler");
        need(out, "out");
        *out = S->chains_per_cta;
    });
}

int yq_sampler_warps_per_chain(yq_sampler S, int* out) {
    return guard([&] {
        need(S, "sampler");
        need(out, "out");
        *out = S->warps_per_chain;
    });
}

int yq_sampler_sample_exact(yq_sampler S, int ns, uint64_t seed, uint32_t epoch, uint64_t* positions) {
    return guard([&] {
        need(S, "sampler");
        if (ns < 1) throw Error(YQ_E_ARG, "sample_exact: ns must be >= 1");
        DevBuf pos;
        if (positions) pos.ensure(size_t(ns) * sizeof(uint64_t));
        sampler_sample_exact(S, ns, seed, epoch, positions ? pos.as<uint64_t>() : nullptr);
        if (positions) down(positions, pos.p, size_t(ns), S->q->ctx->stream);
        raise_device_status(S->q->ctx);
    });
}

int yq_sampler_put_samples(yq_sampler S, int ns, const int8_t* sigma, const double* theta) {
    return guard([&] {
        need(S, "sampler");
        need(sigma, "sigma");
        need(theta, "theta");
        if (ns < 1) throw Error(YQ_E_ARG, "put_samples: ns must be >= 1");
        yq_rbm_s* q = S->q;
        check_sigma(sigma, size_t(ns) * q->n);
        cudaStream_t st = q->ctx->stream;
        S->sigma.ensure(size_t(ns) * q->n);
        S->theta.ensure(size_t(ns) * q->m * q->csize());
        YQ_CUDA(cudaMemcpyAsync(S->sigma.p, sigma, size_t(ns) * q->n, cudaMemcpyHostToDevice, st));
        const size_t cnt = size_t(ns) * q->m;
        if (q->dtype == YQ_C128) {
            YQ_CUDA(cudaMemcpyAsync(S->theta.p, theta, cnt * sizeof(c128), cudaMemcpyHostToDevice, st));
        } else {
            Staging tmp;
            c128* d = tmp.up(reinterpret_cast<const c128*>(theta), cnt, st);
            c128_to_c64_kernel<<<std::min<unsigned>(cdiv_u(cnt, 256), 4096u), 256, 0, st>>>(cnt, d, S->theta.as<c64>());
            YQ_LAUNCH_CHECK();
        }
        YQ_CUDA(cudaStreamSynchronize(st));
        S->ns = ns;
    });
}

int yq_debug_wait_timeout(yq_ctx ctx, int which, unsigned cap, int* published) {
    return guard([&] {
        need(ctx, "ctx");
        need(published, "published");
        if (which != 0 && which != 1) throw Error(YQ_E_ARG, "debug_wait_timeout: which must be 0 or 1");
        *published = chol_debug_unpublished_flag(which, cap, ctx->status.as<int>(), ctx->sm_count, ctx->stream);
        raise_device_status(ctx);
    });
}

// ---- SR ---------------------------------------------------------------------------
int yq_sr_create(yq_rbm q, yq_ham H, yq_sampler S, int mode, int precision, yq_sr* out) {
    return guard([&] {
        need(q, "rbm");
        need(H, "ham");
        need(S, "sampler");
        need(out, "out");
        *out = nullptr;
        if (S->q != q) throw Error(YQ_E_ARG, "sr: the sampler belongs to another RBM");
        if (H->n != q->n) throw Error(YQ_E_ARG, "sr: Hamiltonian and RBM sizes differ");
        if (mode != YQ_SR_AUTO && mode != YQ_SR_S && mode != YQ_SR_T) throw Error(YQ_E_ARG, "sr: unknown mode");
        if (precision != YQ_PREC_FP64 && precision != YQ_PREC_MIXED) throw Error(YQ_E_ARG, "sr: unknown precision");
        if (precision == YQ_PREC_MIXED && q->dtype != YQ_C64)
            throw Error(YQ_E_ARG, "sr: mixed precision needs a complex64 RBM");
        if (precision == YQ_PREC_FP64 && q->dtype != YQ_C128)
            throw Error(YQ_E_ARG, "sr: FP64 precision needs a complex128 RBM");
        auto* sr = new yq_sr_s();
        sr->q = q;
        sr->H = H;
        sr->S = S;
        sr->mode_req = mode;
        sr->precision = precision;
        *out = sr;
    });
}

int yq_sr_destroy(yq_sr sr) {
    return guard([&] {
        if (!sr) return;
        cudaStreamSynchronize(sr->q->ctx->stream);
        delete sr;
    });
}

int yq_sr_construct(yq_sr sr) {
    return guard([&] {
        need(sr, "sr");
        sr_construct(sr);
        raise_device_status(sr->q->ctx);
    });
}

int yq_sr_energy(yq_sr sr, double* energy, double* energy_var) {
    return guard([&] {
        need(sr, "sr");
        if (!sr->constructed) throw Error(YQ_E_STATE, "energy: call construct first");
        double h[4];
        down(h, sr->stats.p, 4, sr->q->ctx->stream);
        if (energy) *energy = h[0];
        if (energy_var) *energy_var = h[1];
    });
}

int yq_sr_get(yq_sr sr, int which, double* out) {
    return guard([&] {
        need(sr, "sr");
        need(out, "out");
        if (!sr->constructed) throw Error(YQ_E_STATE, "get: call construct first");
        cudaStream_t st = sr->q->ctx->stream;
        c128* o = reinterpret_cast<c128*>(out);
        switch (which) {
            case 0: down(o, sr->eloc.p, size_t(sr->ns), st); break;
            case 1: down(o, sr->oloc.p, sr->q->P, st); break;
            case 2: down(o, sr->grad.p, sr->q->P, st); break;
            case 3:
                if (!sr->solved) throw Error(YQ_E_STATE, "get: no solution yet");
                down(o, sr->v.p, sr->q->P, st);
                break;
            default: throw Error(YQ_E_ARG, "get: which must be 0..3");
        }
    });
}

int yq_sr_solve(yq_sr sr, double shift, int solver, double cg_tol, double* v, int* iterations, double* relres) {
    return guard([&] {
        need(sr, "sr");
        if (solver != YQ_SOLVE_LLT && solver != YQ_SOLVE_CG) throw Error(YQ_E_ARG, "solve: unknown solver");
        const int ir = sr->solve_steps >= 0 ? sr->solve_steps : sr->precision == YQ_PREC_MIXED ? 2 : 0;
        sr_solve(sr, shift, solver, cg_tol, ir, iterations, relres);
        raise_device_status(sr->q->ctx);
        if (v) down(reinterpret_cast<c128*>(v), sr->v.p, sr->q->P, sr->q->ctx->stream);
    });
}

int yq_sr_set_solve_steps(yq_sr sr, int steps) {
    return guard([&] {
        need(sr, "sr");
        if (steps < -1 || steps > 64) throw Error(YQ_E_ARG, "set_solve_steps: steps must be -1..64");
        sr->solve_steps = steps;
    });
}

int yq_exact(yq_rbm q, yq_ham H, int basis_kind, int nup, double* stats, double* oloc, double* grad, double* S) {
    return guard([&] {
        need(q, "rbm");
        need(H, "hamiltonian");
        need(stats, "stats");
        if (q->ctx != H->ctx) throw Error(YQ_E_ARG, "exact: RBM and Hamiltonian belong to different contexts");
        const size_t P = q->P;
        DevBuf d_ol, d_g, d_S;
        d_ol.ensure(P * sizeof(c128));
        d_g.ensure(P * sizeof(c128));
        if (S) d_S.ensure(P * P * sizeof(c128));
        exact_summation(q, H, basis_kind, nup, stats, d_ol.as<c128>(), d_g.as<c128>(), S ? d_S.as<c128>() : nullptr);
        cudaStream_t st = q->ctx->stream;
        if (oloc) down(reinterpret_cast<c128*>(oloc), d_ol.p, P, st);
        if (grad) down(reinterpret_cast<c128*>(grad), d_g.p, P, st);
        if (S) {
            c128* h = reinterpret_cast<c128*>(S);
            down(h, d_S.p, P * P, st);
            for (size_t a = 0; a < P; ++a)  // lower triangle computed; Hermitian upper part
                for (size_t b = a + 1; b < P; ++b) h[a * P + b] = conj(h[b * P + a]);
        }
        raise_device_status(q->ctx);
    });
}

int yq_exact_iteration(yq_rbm q, yq_ham H, int basis_kind, int nup, double shift, double lr, double* out) {
    return guard([&] {
        need(q, "rbm");
        need(H, "hamiltonian");
        need(out, "out");
        if (q->ctx != H->ctx) throw Error(YQ_E_ARG, "exact: RBM and Hamiltonian belong to different contexts");
        if (!(shift >= 0.0) || !(lr >= 0.0)) throw Error(YQ_E_ARG, "exact_iteration: shift and lr must be >= 0");
        exact_iteration(q, H, basis_kind, nup, shift, lr, out);
        raise_device_status(q->ctx);
    });
}

int yq_sr_matrix(yq_sr sr, int* dim, double* out) {
    return guard([&] {
        need(sr, "sr");
        need(dim, "dim");
        if (!sr->constructed) throw Error(YQ_E_STATE, "matrix: call construct first");
        *dim = sr->dim;
        if (!out) return;
        sr_form_matrix_public(sr, 0.0);
        sr->solved = false;
        cudaStream_t st = sr->q->ctx->stream;
        YQ_CUDA(cudaMemcpy2DAsync(out, size_t(sr->dim) * sizeof(c128), sr->G.p, size_t(sr->dim_pad) * sizeof(c128),
                                  size_t(sr->dim) * sizeof(c128), size_t(sr->dim), cudaMemcpyDeviceToHost, st));
        YQ_CUDA(cudaStreamSynchronize(st));
        raise_device_status(sr->q->ctx);
    });
}

int yq_sr_set_momentum(yq_sr sr, double beta1, double beta2) {
    return guard([&] {
        need(sr, "sr");
        if (!(beta1 >= 0.0 && beta1 < 1.0) || !(beta2 >= 0.0 && beta2 < 1.0))
            throw Error(YQ_E_ARG, "set_momentum: beta1 and beta2 must lie in [0, 1)");
        sr->beta1 = beta1;
        sr->beta2 = beta2;
        sr->t_grad = 0;
        sr->t_fisher = 0;
    });
}

int yq_sr_set_grad_clip(yq_sr sr, double clip) {
    return guard([&] {
        need(sr, "sr");
        if (!(clip >= 0.0)) throw Error(YQ_E_ARG, "set_grad_clip: clip must be >= 0");
        sr->grad_clip = clip;
    });
}

int yq_vmc_iteration(yq_sr sr, const yq_iter_params* p, yq_iter_result* r) {
    return guard([&] {
        need(sr, "sr");
        need(p, "params");
        need(r, "result");
        std::memset(r, 0, sizeof(*r));
        yq_ctx_s* ctx = sr->q->ctx;
        cudaStream_t st = ctx->stream;
        if (!(p->lr >= 0.0)) throw Error(YQ_E_ARG, "iteration: lr must be >= 0");
        ctx->stage_begin(ST_TOTAL);
        ctx->stage_begin(ST_SAMPLE);
        sampler_run(sr->S, p->n_sweeps, p->n_discard, p->seed, p->epoch, p->reinit);
        ctx->stage_end(ST_SAMPLE);
        sr_construct(sr);
        int iters = 0;
        double relres = 0., cg_err = 0.;
        sr_solve_runner(sr, p->shift, p->solver, p->cg_tol, p->ir_steps, &iters, &relres, &cg_err);
        sr_update_params(sr, p->lr);
        ctx->stage_end(ST_TOTAL);
        double h[8];
        YQ_CUDA(cudaMemcpyAsync(h, sr->stats.p, sizeof(h), cudaMemcpyDeviceToHost, st));
        std::vector<unsigned long long> acc(sr->S->n_chains);
        YQ_CUDA(cudaMemcpyAsync(acc.data(), sr->S->acc.p, acc.size() * sizeof(unsigned long long),
                                cudaMemcpyDeviceToHost, st));
        YQ_CUDA(cudaStreamSynchronize(st));
        double tot = 0.;
        for (auto a : acc) tot += double(a);
        r->energy = h[0];
        r->energy_var = h[1];
        r->update_norm = h[4];
        r->cg_err = cg_err;
        r->accept_rate = tot / (double(sr->S->n_chains) * double(sr->S->proposals));
        int code = status_to_code(ctx->read_status_and_clear());
        r->status = code;
        if (code != YQ_OK) throw Error(code, status_msg(code));
    });
}

int yq_batch_create(yq_ctx ctx, int nprob, const yq_sr* srs, yq_batch* out) {
    return guard([&] {
        need(ctx, "ctx");
        need(srs, "srs");
        need(out, "out");
        *out = nullptr;
        batch_create(ctx, nprob, srs, out);
    });
}

int yq_batch_destroy(yq_batch B) {
    return guard([&] {
        if (!B) return;
        YQ_CUDA(cudaStreamSynchronize(B->ctx->stream));
        batch_destroy(B);
    });
}

int yq_batch_iteration(yq_batch B, const yq_iter_params* p, yq_iter_result* results) {
    return guard([&] {
        need(B, "batch");
        need(p, "params");
        need(results, "results");
        std::memset(results, 0, B->srs.size() * sizeof(yq_iter_result));
        batch_iteration(B, *p, results);
        int first = YQ_OK;
        for (size_t k = 0; k < B->srs.size(); ++k) {
            results[k].status = status_to_code(results[k].status);
            if (first == YQ_OK) first = results[k].status;
        }
        if (first != YQ_OK) throw Error(first, status_msg(first));
    });
}

}  // extern "C"
