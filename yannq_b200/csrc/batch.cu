// Batched VMC iterations over independent problems.
//
// A batch groups SR objects (each with its machine, Hamiltonian and sampler,
// normally each on its own context and stream) and advances all of them by one
// RunRBM iteration (Runners/RunRBM.hpp:166-214: sample, constructFromSamples,
// LLT solve, SGD update) per call.  The first call, and any call whose iteration
// parameters differ from the captured ones, runs the problems eagerly, each on
// its own stream, then captures the next iteration of every problem into one
// CUDA graph: a fork from the launching context's stream to every problem
// stream and a join back.  Later calls replay the graph, so the host enqueues
// one graph launch instead of every kernel of every problem, and problems
// overlap on the device.  Replays advance the sampler epoch through a device
// counter (the graph's first node), since kernel arguments are frozen at
// capture; problem k draws from seed + k.
#include <memory>
#include <vector>

#include "internal.hpp"

namespace yq {

namespace {

__global__ void epoch_step_kernel(uint32_t* e) { *e += 1u; }

__global__ void acc_sum_kernel(int n, const unsigned long long* __restrict__ acc, unsigned long long* __restrict__ out) {
    __shared__ unsigned long long red[8];
    unsigned long long t = 0;
    for (int i = threadIdx.x; i < n; i += blockDim.x) t += acc[i];
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) t += __shfl_xor_sync(0xffffffffu, t, o);
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = t;
    __syncthreads();
    if (threadIdx.x == 0) {
        unsigned long long s = 0;
        for (int w = 0; w < int(blockDim.x >> 5); ++w) s += red[w];
        *out = s;
    }
}

bool same_params(const yq_iter_params& a, const yq_iter_params& b) {
    return a.n_sweeps == b.n_sweeps && a.n_discard == b.n_discard && a.seed == b.seed && a.shift == b.shift &&
           a.lr == b.lr && a.solver == b.solver && a.ir_steps == b.ir_steps;
}

// sample + constructFromSamples + solve + update of problem k on its own stream
void advance(yq_sr_s* sr, const yq_iter_params& p, int k, uint32_t epoch, int reinit) {
    sampler_run(sr->S, p.n_sweeps, p.n_discard, p.seed + uint64_t(k), epoch, reinit);
    sr_construct(sr);
    int iters = 0;
    double relres = 0.;
    sr_solve(sr, p.shift, p.solver, p.cg_tol, p.ir_steps, &iters, &relres);
    sr_update_params(sr, p.lr);
}

// Per-problem statistics into the host arrays (copies queued on `st`).
void queue_results(yq_batch_s* B, cudaStream_t st) {
    const int np = int(B->srs.size());
    for (int k = 0; k < np; ++k) {
        yq_sr_s* sr = B->srs[size_t(k)];
        acc_sum_kernel<<<1, 256, 0, st>>>(sr->S->n_chains, sr->S->acc.as<unsigned long long>(),
                                          B->dev_acc_sum.as<unsigned long long>() + k);
        YQ_LAUNCH_CHECK();
        YQ_CUDA(cudaMemcpyAsync(B->host_stats.data() + 8 * size_t(k), sr->stats.p, 8 * sizeof(double),
                                cudaMemcpyDeviceToHost, st));
    }
    YQ_CUDA(cudaMemcpyAsync(B->host_acc.data(), B->dev_acc_sum.p, size_t(np) * sizeof(unsigned long long),
                            cudaMemcpyDeviceToHost, st));
}

}  // namespace

void batch_create(yq_ctx_s* ctx, int np, yq_sr_s* const* srs, yq_batch_s** out) {
    YQ_CHECK_ARG(np >= 1, "batch: at least one problem");
    auto B = std::make_unique<yq_batch_s>();
    B->ctx = ctx;
    for (int k = 0; k < np; ++k) {
        YQ_CHECK_ARG(srs[k] != nullptr, "batch: null SR handle");
        YQ_CHECK_ARG(srs[k]->q->ctx->device == ctx->device, "batch: every problem must be on the batch's device");
        for (int j = 0; j < k; ++j) YQ_CHECK_ARG(srs[j] != srs[k], "batch: an SR object appears twice");
        B->srs.push_back(srs[k]);
    }
    B->epoch.ensure(sizeof(uint32_t));
    YQ_CUDA(cudaMemsetAsync(B->epoch.p, 0, sizeof(uint32_t), ctx->stream));
    B->dev_acc_sum.ensure(size_t(np) * sizeof(unsigned long long));
    B->host_stats.assign(8 * size_t(np), 0.0);
    B->host_acc.assign(size_t(np), 0);
    YQ_CUDA(cudaEventCreateWithFlags(&B->fork, cudaEventDisableTiming));
    B->joins.assign(size_t(np), nullptr);
    for (int k = 0; k < np; ++k) YQ_CUDA(cudaEventCreateWithFlags(&B->joins[size_t(k)], cudaEventDisableTiming));
    YQ_CUDA(cudaStreamSynchronize(ctx->stream));
    *out = B.release();
}

void batch_destroy(yq_batch_s* B) { delete B; }

// Advances every problem once; returns per-problem statistics and device status.
void batch_iteration(yq_batch_s* B, const yq_iter_params& p, yq_iter_result* res) {
    YQ_CHECK_ARG(p.solver == YQ_SOLVE_LLT, "batch: the captured iteration needs the LLT solver");
    YQ_CHECK_ARG(p.lr >= 0.0, "batch: lr must be >= 0");
    const int np = int(B->srs.size());
    for (auto* sr : B->srs)
        if (sr->beta1 != 0.0 || sr->beta2 != 0.0)
            throw Error(YQ_E_UNSUPPORTED, "batch: momentum (yq_sr_set_momentum) is not captured in batch graphs");
    cudaStream_t master = B->ctx->stream;
    if (B->have_graph && same_params(B->captured, p)) {
        YQ_CUDA(cudaGraphLaunch(B->exec, master));
    } else {
        // eager iteration: every problem on its own stream
        YQ_CUDA(cudaEventRecord(B->fork, master));
        for (int k = 0; k < np; ++k) {
            yq_sr_s* sr = B->srs[size_t(k)];
            cudaStream_t st = sr->q->ctx->stream;
            YQ_CUDA(cudaStreamWaitEvent(st, B->fork, 0));
            sr->S->epoch_dev = nullptr;
            advance(sr, p, k, p.epoch, p.reinit);
            YQ_CUDA(cudaEventRecord(B->joins[size_t(k)], st));
            YQ_CUDA(cudaStreamWaitEvent(master, B->joins[size_t(k)], 0));
        }
        // capture the next iteration of every problem (chains kept, epoch + 1, + 2, ...)
        if (B->exec) YQ_CUDA(cudaGraphExecDestroy(B->exec));
        if (B->graph) YQ_CUDA(cudaGraphDestroy(B->graph));
        B->exec = nullptr;
        B->graph = nullptr;
        B->have_graph = false;
        YQ_CUDA(cudaMemsetAsync(B->epoch.p, 0, sizeof(uint32_t), master));
        YQ_CUDA(cudaStreamSynchronize(master));
        YQ_CUDA(cudaStreamBeginCapture(master, cudaStreamCaptureModeRelaxed));
        try {
            epoch_step_kernel<<<1, 1, 0, master>>>(B->epoch.as<uint32_t>());
            YQ_LAUNCH_CHECK();
            YQ_CUDA(cudaEventRecord(B->fork, master));
            for (int k = 0; k < np; ++k) {
                yq_sr_s* sr = B->srs[size_t(k)];
                cudaStream_t st = sr->q->ctx->stream;
                YQ_CUDA(cudaStreamWaitEvent(st, B->fork, 0));
                sr->q->ctx->timing = false;
                sr->S->epoch_dev = B->epoch.as<uint32_t>();
                advance(sr, p, k, p.epoch, 0);
                sr->S->epoch_dev = nullptr;
                sr->q->ctx->timing = true;
                YQ_CUDA(cudaEventRecord(B->joins[size_t(k)], st));
                YQ_CUDA(cudaStreamWaitEvent(master, B->joins[size_t(k)], 0));
            }
        } catch (...) {
            for (auto* sr : B->srs) {
                sr->S->epoch_dev = nullptr;
                sr->q->ctx->timing = true;
            }
            cudaGraph_t g = nullptr;
            cudaStreamEndCapture(master, &g);
            if (g) cudaGraphDestroy(g);
            throw;
        }
        YQ_CUDA(cudaStreamEndCapture(master, &B->graph));
        YQ_CUDA(cudaGraphInstantiate(&B->exec, B->graph, 0));
        B->captured = p;
        B->have_graph = true;
        // the captured iteration ran nothing yet: report the eager one below
    }
    queue_results(B, master);
    YQ_CUDA(cudaStreamSynchronize(master));
    for (int k = 0; k < np; ++k) {
        yq_sr_s* sr = B->srs[size_t(k)];
        const double* h = B->host_stats.data() + 8 * size_t(k);
        yq_iter_result& r = res[k];
        r.energy = h[0];
        r.energy_var = h[1];
        r.update_norm = h[4];
        r.cg_err = 0.;
        r.accept_rate = double(B->host_acc[size_t(k)]) / (double(sr->S->n_chains) * double(sr->S->proposals));
        r.status = sr->q->ctx->read_status_and_clear();  // raw device status bits; mapped by the caller
    }
}

}  // namespace yq
