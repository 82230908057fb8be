// The reference's AmplitudePhase example (Examples/AmplitudePhase.cpp:39-79) on the
// C++ adapters: a Conv1D / LeakyHardTanh phase network ending in FullyConnected
// and SoftSign, J1J2(N, 1, j2, signRule), RunAmplitudePhaseExact with lambda
// 10 * 0.9^ll down to 1e-3 on the Jz basis at zero magnetisation.  N = 12 (the
// kernel of five taps needs N >= 5), 60 epochs; also checks NGDExact's getters.
// Prints one line per epoch and "OK first last" (energies per site); exits
// non-zero if the energy does not go down.
#include <cstdio>
#include <vector>

#include "yannq_gpu/yannq_gpu.hpp"

int main(int argc, char** argv) {
    using namespace yannq::gpu;
    const uint32_t N = 12;
    const int alpha = 1;
    const double j2 = 0.2;
    const int epochs = argc > 1 ? std::atoi(argv[1]) : 60;
    Context ctx(0);
    FeedForward ff;
    const int kernel_size = 5;
    ff.addLayer<Conv1D>(1, 6, kernel_size, 1, false);
    ff.addLayer<LeakyHardTanh>(0.01);
    ff.addLayer<Conv1D>(6, 4, kernel_size, 1, false);
    ff.addLayer<LeakyHardTanh>(0.01);
    ff.addLayer<Conv1D>(4, 2, kernel_size, 1, false);
    ff.addLayer<LeakyHardTanh>(0.01);
    ff.addLayer<FullyConnected>(2 * int(N), 1, false);
    ff.addLayer<SoftSign>();
    J1J2 ham(ctx, int(N), 1.0, j2, true);
    RunAmplitudePhaseExact runner(ctx, N, alpha, false, std::move(ff));
    runner.initializeRandom(20261205, 0.01);
    runner.setLambda(10.0, 0.9, 1e-3);
    runner.setIterParams(epochs, 0);
    runner.setOptimizer(SGD{0.05, 0.0});
    std::vector<double> es;
    runner.run([&](int ll, double e, double ng, double nv) {
        std::printf("%d\t%.10f\t%.4e\t%.4e\n", ll, e, ng, nv);
        es.push_back(e);
    }, BasisJz(N, N / 2), ham);
    NGDExact ngd(runner.getQs(), BasisJz(N, N / 2), ham);
    ngd.constructExact();
    const auto ca = ngd.corrMatAmp();
    const auto g = ngd.energyGrad();
    std::printf("GETTERS %zu %zu %.10f\n", ca.size(), g.size(), ngd.eloc() / N);
    std::printf("OK %.8f %.8f\n", es.front() / N, es.back() / N);
    return es.back() < es.front() ? 0 : 1;
}
