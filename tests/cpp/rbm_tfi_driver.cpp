// A RunRBM-style driver written against the C++ adapters, following the call
// pattern of the reference example (Examples/RBMTFI.cpp:57-87): TFIsing(N, -1, -h),
// RunRBM(N, alpha), initializeRandom(0.01), SGD, SamplerMT(qs, 1, K, LocalSweeper),
// run(sampler, callback, ham, nSweeps, nDiscard).  Prints one line per epoch and a
// final "OK E/N" line; exits non-zero if the energy does not go down.
#include <cstdio>
#include <vector>

#include "yannq_gpu/yannq_gpu.hpp"

int main(int argc, char** argv) {
    using namespace yannq::gpu;
    const unsigned N = 10, alpha = 2;
    const double h = 1.0;
    const int epochs = argc > 1 ? std::atoi(argv[1]) : 40;
    Context ctx(0);
    TFIsing ham(ctx, int(N), -1.0, -h);
    RunRBM<std::complex<double>> runner(ctx, N, alpha, true);
    runner.initializeRandom(20261203, 0.01);
    runner.setLambda(1e-3, 1.0, 1e-3);
    runner.setIterParams(epochs, 0);
    runner.setOptimizer(SGD{0.05, 0.0});
    LocalSweeper sweeper{N};
    SamplerMT<RBM<std::complex<double>>, LocalSweeper> sampler(runner.getQs(), 1, 32, sweeper);
    std::vector<double> es;
    auto callback = [&](int ll, double e, double nv, double cgErr, float smp, float slv) {
        std::printf("%d\t%.10f\t%.4e\t%.1e\t%.3f\t%.3f\n", ll, e, nv, cgErr, smp, slv);
        es.push_back(e);
    };
    runner.run(sampler, callback, ham, 16, 16, 7);
    double first = es.front(), last = 0.0;
    for (size_t i = es.size() - 5; i < es.size(); ++i) last += es[i] / 5.0;
    std::printf("OK %.8f %.8f\n", first / N, last / N);
    return last < first ? 0 : 1;
}
