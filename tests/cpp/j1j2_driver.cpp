// The further Hamiltonian adapters (XXX, J1J2, XYZNNN, KitaevHex) in the
// reference's constructor forms, and a RunRBM-style run on the J1J2 chain
// (Hamiltonians/J1J2.hpp:14-56, N = 12, J1 = 1, J2 = 0.2, sign rule) with
// exchange moves at zero magnetisation, then a HamiltonianSweeper sampler on the
// trained machine; checkpoints every 20 epochs (w%04d.dat in the working
// directory) and a resumed runner.  Prints "TERMS <name> <n> <requests>" for
// every model, "HAMSWEEP <samples>", "RESUME <dim>" and a final "OK E/N first
// last" line; exits non-zero if the energy does not go down.
#include <cstdio>
#include <vector>

#include "yannq_gpu/yannq_gpu.hpp"

namespace {
void terms(const char* name, const yannq::gpu::Hamiltonian& h) {
    int k = 0;
    yannq::gpu::check(yq_ham_num_offdiag(h.handle(), &k));
    std::printf("TERMS %s %d %d\n", name, h.size(), k);
}
}  // namespace

int main(int argc, char** argv) {
    using namespace yannq::gpu;
    const unsigned N = 12, alpha = 1;
    const int epochs = argc > 1 ? std::atoi(argv[1]) : 40;
    Context ctx(0);
    {
        XXX xxx(ctx, 10);
        XYZNNN xyz(ctx, 10, 0.3, 0.7);
        KitaevHex kit(ctx, 4, 4, 1.0, 0.2);
        KitaevHex kita(ctx, 4, 4, 0.2, 0.4, 0.6);
        terms("XXX", xxx);
        terms("XYZNNN", xyz);
        terms("KitaevHex", kit);
        terms("KitaevHexAniso", kita);
    }
    J1J2 ham(ctx, int(N), 1.0, 0.2, true);
    terms("J1J2", ham);
    RunRBM<std::complex<double>> runner(ctx, N, alpha, true);
    runner.initializeRandom(20261204, 0.01);
    runner.setLambda(1e-3, 1.0, 1e-3);
    runner.setIterParams(epochs, 20);  // w0000.dat, w0020.dat, ... in the working directory
    runner.setOptimizer(SGD{0.05, 0.0});
    SwapSweeper sweeper{N};
    SamplerMT<RBM<std::complex<double>>, SwapSweeper> sampler(runner.getQs(), 1, 64, sweeper, int(N / 2));
    std::vector<double> es;
    auto callback = [&](int ll, double e, double nv, double cgErr, float smp, float slv) {
        std::printf("%d\t%.10f\t%.4e\t%.1e\t%.3f\t%.3f\n", ll, e, nv, cgErr, smp, slv);
        es.push_back(e);
    };
    runner.run(sampler, callback, ham, 16, 16, 7);
    // the same chain sampled with the HamiltonianSweeper (offDiagonals proposals)
    HamiltonianSweeper<J1J2> hsw(int(N), ham);
    SamplerMT<RBM<std::complex<double>>, HamiltonianSweeper<J1J2>> hsampler(runner.getQs(), 1, 16, hsw, int(N / 2));
    hsampler.initializeRandomEngine(5);
    std::printf("HAMSWEEP %zu\n", hsampler.sample(4, 8).size());
    // resume from a checkpoint (AbstractRunner::initializeFrom)
    RunRBM<std::complex<double>> resumed(ctx, N, alpha, true);
    resumed.initializeFrom("w0020.dat");
    std::printf("RESUME %u\n", resumed.getQs().getDim());
    double first = es.front(), last = 0.0;
    for (size_t i = es.size() - 5; i < es.size(); ++i) last += es[i] / 5.0;
    std::printf("OK %.8f %.8f\n", first / N, last / N);
    return last < first ? 0 : 1;
}
