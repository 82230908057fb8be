// Micro-benchmarks of the device roofs used by the roofline reports that the
// copy/GEMM peaks measured outside this library do not cover: FP64 and FP32 FMA
// throughput (SIMT), FP64 tensor-core (DMMA m8n8k4) throughput, and complex
// logcosh evaluations per second (the transcendental roof of the reference-form
// psi-ratio, Utilities/Utility.hpp:27-37).
#include "internal.hpp"

namespace yq {

template <typename R, int CHAINS>
__global__ void fma_kernel(int iters, R seed, R* out) {
    R a[CHAINS];
#pragma unroll
    for (int c = 0; c < CHAINS; ++c) a[c] = seed + R(threadIdx.x + c);
    const R b = R(0.999999), d = R(1e-7);
    for (int i = 0; i < iters; ++i) {
#pragma unroll
        for (int c = 0; c < CHAINS; ++c) a[c] = fma(a[c], b, d);
    }
    R s = 0;
#pragma unroll
    for (int c = 0; c < CHAINS; ++c) s += a[c];
    if (s == R(-12345.678)) out[blockIdx.x] = s;  // keeps the loop alive
}

__global__ void dmma_kernel(int iters, double* out) {
    double c[8][2];
#pragma unroll
    for (int k = 0; k < 8; ++k) c[k][0] = c[k][1] = 0.0;
    double a = 1.0 + threadIdx.x * 1e-9, b = 0.5;
    for (int i = 0; i < iters; ++i) {
#pragma unroll
        for (int k = 0; k < 8; ++k)
            asm volatile("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0,%1}, {%2}, {%3}, {%0,%1};"
                         : "+d"(c[k][0]), "+d"(c[k][1])
                         : "d"(a), "d"(b));
    }
    double s = 0;
#pragma unroll
    for (int k = 0; k < 8; ++k) s += c[k][0] + c[k][1];
    if (s == -12345.678) out[blockIdx.x] = s;
}

__global__ void logcosh_kernel(int iters, double* out) {
    c128 z = mk(0.01 * threadIdx.x, 0.02 * blockIdx.x);
    c128 acc = mk(0., 0.);
    for (int i = 0; i < iters; ++i) {
        acc = acc + clogcosh(z);
        z.re += 1e-3;
        z.im -= 7e-4;
    }
    if (acc.re == -12345.678) out[blockIdx.x] = acc.re;
}

}  // namespace yq

using namespace yq;

extern "C" int yq_measure_peaks(yq_ctx ctx, double* out) {
    // out[0] FP64 SIMT TFLOP/s, out[1] FP32 SIMT TFLOP/s, out[2] FP64 DMMA TFLOP/s,
    // out[3] complex128 logcosh evaluations per second (x 1e9)
    if (!ctx || !out) return YQ_E_ARG;
    try {
        cudaStream_t st = ctx->stream;
        DevBuf sink;
        sink.ensure(1 << 20);
        cudaEvent_t e0, e1;
        YQ_CUDA(cudaEventCreate(&e0));
        YQ_CUDA(cudaEventCreate(&e1));
        const int blocks = ctx->sm_count * 8, threads = 256;
        auto timed = [&](auto launch) {
            launch();  // warm-up
            YQ_CUDA(cudaEventRecord(e0, st));
            launch();
            YQ_CUDA(cudaEventRecord(e1, st));
            YQ_CUDA(cudaEventSynchronize(e1));
            float ms = 0.f;
            YQ_CUDA(cudaEventElapsedTime(&ms, e0, e1));
            return double(ms) * 1e-3;
        };
        const int it = 4096;
        double t = timed([&] {
            fma_kernel<double, 8><<<blocks, threads, 0, st>>>(it, 1.0, sink.as<double>());
            YQ_LAUNCH_CHECK();
        });
        out[0] = 2.0 * double(blocks) * threads * 8 * it / t / 1e12;
        t = timed([&] {
            fma_kernel<float, 8><<<blocks, threads, 0, st>>>(it, 1.0f, sink.as<float>());
            YQ_LAUNCH_CHECK();
        });
        out[1] = 2.0 * double(blocks) * threads * 8 * it / t / 1e12;
        const int itd = 1024;
        t = timed([&] {
            dmma_kernel<<<blocks, threads, 0, st>>>(itd, sink.as<double>());
            YQ_LAUNCH_CHECK();
        });
        // one m8n8k4 per warp = 256 FMA
        out[2] = 2.0 * 256.0 * double(blocks) * (threads / 32) * 8 * itd / t / 1e12;
        const int itl = 256;
        t = timed([&] {
            logcosh_kernel<<<blocks, threads, 0, st>>>(itl, sink.as<double>());
            YQ_LAUNCH_CHECK();
        });
        out[3] = double(blocks) * threads * itl / t / 1e9;
        cudaEventDestroy(e0);
        cudaEventDestroy(e1);
        return YQ_OK;
    } catch (const Error& e) {
        return e.code;
    }
}
