// The reference example's driver (Examples/RBMTFI.cpp:51-87) on the C++ adapters,
// with the call it makes: runner.run(sampler, callback, randomizer, std::move(ham),
// nSweeps, nDiscard) -- Runners/RunRBM.hpp:123 -- where randomizer is a host
// functor re -> randomSigma(N, re), a callback with auto-typed durations, parallel
// tempering (nTmp x K chains), and the RunRBM option setters.
// Prints one line per epoch, "RANDOMIZER <calls>" and a final "OK E_first/N E_last/N".
#include <cstdio>
#include <cstdlib>
#include <vector>

#include "yannq_gpu/yannq_gpu.hpp"

int main(int argc, char** argv) {
    using namespace yannq::gpu;
    using ValT = std::complex<double>;
    const uint32_t N = 10;
    const int alpha = 2, nTmp = 2, K = 16;
    const double h = 1.0;
    const int epochs = argc > 1 ? std::atoi(argv[1]) : 30;

    Context ctx(0);
    TFIsing ham(ctx, int(N), -1.0, -h);
    std::vector<double> es;
    auto callback = [&](int ll, double currE, double nv, double cgErr, auto smp_dur, auto slv_dur) {
        std::printf("%d\t%.10f\t%.4e\t%.1e\t%.3f\t%.3f\n", ll, currE, nv, cgErr, double(smp_dur), double(slv_dur));
        es.push_back(currE);
    };

    RunRBM<ValT> runner(ctx, N, alpha, true);
    runner.setSeed(20261203);
    runner.initializeRandom(0.01);
    runner.setIterParams(epochs, 0);
    runner.setOptimizer(SGD{0.05, 0.0});
    runner.setSolverParams(false, 1e-3);
    runner.setMomentum(0.0, 0.0);  // the reference's defaults; momentum runs are pinned against the oracle runner
    runner.setGradClip(0.0);

    long calls = 0;
    auto randomizer = [N, &calls](auto& re) {
        ++calls;
        return randomSigma(int(N), re);
    };
    LocalSweeper sweeper{N};
    auto sampler = SamplerMT<RBM<ValT>, LocalSweeper>(runner.getQs(), nTmp, K, sweeper);

    runner.run(sampler, callback, randomizer, std::move(ham), 16, 16);

    std::printf("RANDOMIZER %ld\n", calls);
    double first = es.front(), last = 0.0;
    for (size_t i = es.size() - 5; i < es.size(); ++i) last += es[i] / 5.0;
    std::printf("OK %.8f %.8f\n", first / N, last / N);
    return last < first ? 0 : 1;
}
