// Shared device/host utilities of libyannq_b200: complex arithmetic, Philox4x32-10,
// error plumbing and small RAII buffers.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

#include <atomic>
#include <cmath>
#include <cstdio>
#include <stdexcept>
#include <string>

#include "../../include/yannq_b200.h"

namespace yq {

// ---------------------------------------------------------------------------
// Errors.  Every C entry point converts a yq::Error into its status code and
// records the message for yq_last_error().
struct Error : std::runtime_error {
    int code;
    Error(int c, const std::string& m) : std::runtime_error(m), code(c) {}
};

#define YQ_CUDA(call)                                                                                      \
    do {                                                                                                   \
        cudaError_t e_ = (call);                                                                           \
        if (e_ != cudaSuccess)                                                                             \
            throw ::yq::Error(YQ_E_CUDA, std::string(#call) + ": " + cudaGetErrorString(e_) + " @" __FILE__ \
                                             ":" + std::to_string(__LINE__));                               \
    } while (0)

#define YQ_CHECK_ARG(cond, msg)                                  \
    do {                                                         \
        if (!(cond)) throw ::yq::Error(YQ_E_ARG, std::string(msg)); \
    } while (0)

// Counts the library's own kernel launches (reported by yq_launch_count) and its
// device allocations (every one goes through DevBuf::ensure; yq_alloc_count).
extern std::atomic<unsigned long long> g_launches;
extern std::atomic<unsigned long long> g_device_allocs;
#define YQ_LAUNCH_CHECK()                                               \
    do {                                                                \
        ::yq::g_launches.fetch_add(1, std::memory_order_relaxed);       \
        YQ_CUDA(cudaGetLastError());                                    \
    } while (0)

// ---------------------------------------------------------------------------
// Complex numbers (interleaved re, im; layout-compatible with std::complex).
template <typename R>
struct alignas(2 * sizeof(R)) cplx {
    R re, im;
};
using c64 = cplx<float>;
using c128 = cplx<double>;

template <typename R>
__host__ __device__ __forceinline__ cplx<R> mk(R a, R b) {
    cplx<R> z;
    z.re = a;
    z.im = b;
    return z;
}
template <typename R>
__host__ __device__ __forceinline__ cplx<R> operator+(cplx<R> a, cplx<R> b) {
    return mk(a.re + b.re, a.im + b.im);
}
template <typename R>
__host__ __device__ __forceinline__ cplx<R> operator-(cplx<R> a, cplx<R> b) {
    return mk(a.re - b.re, a.im - b.im);
}
template <typename R>
__host__ __device__ __forceinline__ cplx<R> operator*(cplx<R> a, cplx<R> b) {
    return mk(a.re * b.re - a.im * b.im, a.re * b.im + a.im * b.re);
}
template <typename R>
__host__ __device__ __forceinline__ cplx<R> operator*(R s, cplx<R> a) {
    return mk(s * a.re, s * a.im);
}
template <typename R>
__host__ __device__ __forceinline__ cplx<R> conj(cplx<R> a) {
    return mk(a.re, -a.im);
}
template <typename R>
__host__ __device__ __forceinline__ R norm2(cplx<R> a) {
    return a.re * a.re + a.im * a.im;
}
template <typename R>
__host__ __device__ __forceinline__ cplx<R> cdiv(cplx<R> a, cplx<R> b) {
    // Smith's algorithm (scaled to avoid overflow in |b|^2)
    if (fabs(b.re) >= fabs(b.im)) {
        R r = b.im / b.re, d = b.re + b.im * r;
        return mk((a.re + a.im * r) / d, (a.im - a.re * r) / d);
    } else {
        R r = b.re / b.im, d = b.re * r + b.im;
        return mk((a.re * r + a.im) / d, (a.im * r - a.re) / d);
    }
}
template <typename R, typename S>
__host__ __device__ __forceinline__ cplx<R> cast(cplx<S> a) {
    return mk(R(a.re), R(a.im));
}

// exp(z)
__device__ __forceinline__ c128 cexp(c128 z) {
    double s, c;
    sincos(z.im, &s, &c);
    double e = exp(z.re);
    return mk(e * c, e * s);
}
__device__ __forceinline__ c64 cexp(c64 z) {
    float s, c;
    sincosf(z.im, &s, &c);
    float e = expf(z.re);
    return mk(e * c, e * s);
}

// tanh(x + iy) by Kahan's formulation ("Branch cuts for complex elementary
// functions", 1987): t = tan y, b = 1 + t^2, s = sinh x, r = sqrt(1 + s^2),
// tanh = (b r s + i t) / (1 + b s^2); for large |x| the real part is +-1.
__device__ __forceinline__ c128 ctanh(c128 z) {
    const double x = z.re, y = z.im;
    if (fabs(x) > 22.0) {
        double s, c;
        sincos(y, &s, &c);
        double e = exp(-2.0 * fabs(x));
        return mk(copysign(1.0, x), 4.0 * s * c * e);
    }
    double t = tan(y);
    double b = 1.0 + t * t;
    double s = sinh(x);
    double r = sqrt(1.0 + s * s);
    double d = 1.0 + b * s * s;
    return mk(b * r * s / d, t / d);
}
__device__ __forceinline__ c64 ctanh(c64 z) {
    const float x = z.re, y = z.im;
    if (fabsf(x) > 9.0f) {
        float s, c;
        sincosf(y, &s, &c);
        float e = expf(-2.0f * fabsf(x));
        return mk(copysignf(1.0f, x), 4.0f * s * c * e);
    }
    float t = tanf(y);
    float b = 1.0f + t * t;
    float s = sinhf(x);
    float r = sqrtf(1.0f + s * s);
    float d = 1.0f + b * s * s;
    return mk(b * r * s / d, t / d);
}

// Stable log(cosh(z)) in the reference's form (Utilities/Utility.hpp:14-37):
// logCosh(Re) + log(cos(Im) + i tanh(Re) sin(Im)).
__device__ __forceinline__ double logcosh_real(double x) {
    double xp = fabs(x);
    return xp <= 12.0 ? log(cosh(xp)) : xp - 0.69314718055994530942;
}
__device__ __forceinline__ c128 clogcosh(c128 z) {
    double s, c;
    sincos(z.im, &s, &c);
    double wr = c, wi = tanh(z.re) * s;
    return mk(logcosh_real(z.re) + 0.5 * log(wr * wr + wi * wi), atan2(wi, wr));
}

// Running product with an exact power-of-two exponent, so that products of
// thousands of factors neither overflow nor underflow.
template <typename R>
struct ScaledProd {
    cplx<R> p;
    int e;
    __device__ __forceinline__ void init() {
        p = mk(R(1), R(0));
        e = 0;
    }
    __device__ __forceinline__ void renorm() {
        R a = fmax(fabs(p.re), fabs(p.im));
        if (a == R(0) || !isfinite(a)) return;
        int k;
        frexp(a, &k);
        p.re = ldexp(p.re, -k);
        p.im = ldexp(p.im, -k);
        e += k;
    }
};

// ---------------------------------------------------------------------------
// Philox4x32-10 (Salmon et al., SC'11); same stream convention as the oracle:
// key = seed, counter = (index, epoch, chain, tag).
enum : uint32_t {
    TAG_SWEEP = 0x53574550u,
    TAG_INIT = 0x494e4954u,
    TAG_SHUF = 0x53485546u,
    TAG_PARAM = 0x50415241u,
    TAG_EXACT = 0x45584143u,
    TAG_PT = 0x50544d58u,
};

struct U4 {
    uint32_t x, y, z, w;
};

__host__ __device__ __forceinline__ U4 philox4x32_10(uint32_t c0, uint32_t c1, uint32_t c2, uint32_t c3, uint32_t k0,
                                                     uint32_t k1) {
#pragma unroll
    for (int r = 0; r < 10; ++r) {
        if (r > 0) {
            k0 += 0x9E3779B9u;
            k1 += 0xBB67AE85u;
        }
#ifdef __CUDA_ARCH__
        uint32_t lo0 = 0xD2511F53u * c0, hi0 = __umulhi(0xD2511F53u, c0);
        uint32_t lo1 = 0xCD9E8D57u * c2, hi1 = __umulhi(0xCD9E8D57u, c2);
#else
        uint64_t p0 = uint64_t(0xD2511F53u) * c0, p1 = uint64_t(0xCD9E8D57u) * c2;
        uint32_t lo0 = uint32_t(p0), hi0 = uint32_t(p0 >> 32), lo1 = uint32_t(p1), hi1 = uint32_t(p1 >> 32);
#endif
        uint32_t n0 = hi1 ^ c1 ^ k0, n2 = hi0 ^ c3 ^ k1;
        c0 = n0;
        c1 = lo1;
        c2 = n2;
        c3 = lo0;
    }
    return U4{c0, c1, c2, c3};
}
__host__ __device__ __forceinline__ U4 draw(uint64_t seed, uint32_t index, uint32_t epoch, uint32_t chain,
                                            uint32_t tag) {
    return philox4x32_10(index, epoch, chain, tag, uint32_t(seed), uint32_t(seed >> 32));
}
__host__ __device__ __forceinline__ uint32_t draw_site(uint32_t x, uint32_t n) {
    return uint32_t((uint64_t(x) * n) >> 32);
}
__host__ __device__ __forceinline__ double draw_u53(uint32_t x2, uint32_t x3) {
    uint64_t v = (uint64_t(x2) << 21) | uint64_t(x3 >> 11);
    return double(v) * (1.0 / 9007199254740992.0);
}
__host__ __device__ __forceinline__ float draw_u24(uint32_t x2) { return float(x2 >> 8) * (1.0f / 16777216.0f); }
template <typename R>
__device__ __forceinline__ R draw_uniform(U4 x);
template <>
__device__ __forceinline__ double draw_uniform<double>(U4 x) {
    return draw_u53(x.z, x.w);
}
template <>
__device__ __forceinline__ float draw_uniform<float>(U4 x) {
    return draw_u24(x.z);
}

// ---------------------------------------------------------------------------
// Device buffer (RAII).
struct DevBuf {
    void* p = nullptr;
    size_t bytes = 0;
    DevBuf() = default;
    DevBuf(const DevBuf&) = delete;
    DevBuf& operator=(const DevBuf&) = delete;
    ~DevBuf() { release(); }
    void release() {
        if (p) cudaFree(p);
        p = nullptr;
        bytes = 0;
    }
    void ensure(size_t b) {
        if (b <= bytes && p) return;
        release();
        if (b == 0) return;
        g_device_allocs.fetch_add(1, std::memory_order_relaxed);
        cudaError_t e = cudaMalloc(&p, b);
        if (e != cudaSuccess) {
            p = nullptr;
            cudaGetLastError();
            throw Error(YQ_E_NOMEM, "cudaMalloc(" + std::to_string(b) + " bytes) failed: " + cudaGetErrorString(e));
        }
        bytes = b;
    }
    template <typename T>
    T* as() const {
        return reinterpret_cast<T*>(p);
    }
};

inline unsigned cdiv_u(size_t a, size_t b) { return unsigned((a + b - 1) / b); }

}  // namespace yq
