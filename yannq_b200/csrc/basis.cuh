// Bases of spin configurations on the device (Basis/BasisFull.hpp:126-153,
// Basis/BasisJz.hpp:25-104): every configuration of n spins, or the configurations
// with nup spins down in increasing order of their index (bit i set <=> sigma_i =
// -1, Utilities/Utility.hpp:91-99), unranked and ranked by the combinatorial
// number system.
#pragma once
#include <vector>

#include "internal.hpp"

namespace yq {
namespace {

constexpr int MAX_N_FULL = 24;   // 2^24 configurations
constexpr int MAX_N_JZ = 62;
constexpr uint64_t MAX_DIM = uint64_t(1) << 24;

// Number of configurations of the basis and the binomial table C(c, i), c, i <= n.
struct Basis {
    int n = 0, kind = 0, nup = 0;
    uint64_t dim = 0;
    std::vector<uint64_t> binom;  // (n + 1) x (n + 1)
};

inline Basis make_basis(int n, int kind, int nup) {
    Basis b;
    b.n = n;
    b.kind = kind;
    b.nup = nup;
    if (kind == YQ_BASIS_FULL) {
        YQ_CHECK_ARG(n >= 1 && n <= MAX_N_FULL, "exact: the full basis needs 1 <= n <= 24");
        b.dim = uint64_t(1) << n;
    } else if (kind == YQ_BASIS_JZ) {
        YQ_CHECK_ARG(n >= 1 && n <= MAX_N_JZ && nup >= 0 && nup <= n, "exact: the Jz basis needs 0 <= nup <= n <= 62");
        b.binom.assign(size_t(n + 1) * (n + 1), 0);
        for (int c = 0; c <= n; ++c) {
            b.binom[size_t(c) * (n + 1)] = 1;
            for (int i = 1; i <= c; ++i)
                b.binom[size_t(c) * (n + 1) + i] =
                    b.binom[size_t(c - 1) * (n + 1) + i - 1] + (i <= c - 1 ? b.binom[size_t(c - 1) * (n + 1) + i] : 0);
        }
        b.dim = b.binom[size_t(n) * (n + 1) + nup];
    } else {
        throw Error(YQ_E_ARG, "exact: unknown basis kind");
    }
    YQ_CHECK_ARG(b.dim >= 1 && b.dim <= MAX_DIM, "exact: the basis must hold at most 2^24 configurations");
    return b;
}

// Configuration index of basis position k (bit i set <=> sigma_i = -1,
// Utilities/Utility.hpp:91-99) and its sigma row.
__global__ void basis_kernel(uint64_t dim, int n, int kind, int nup, const uint64_t* __restrict__ binom,
                             uint64_t* __restrict__ index, int8_t* __restrict__ sigma) {
    for (uint64_t k = uint64_t(blockIdx.x) * blockDim.x + threadIdx.x; k < dim; k += uint64_t(gridDim.x) * blockDim.x) {
        uint64_t v = 0;
        if (kind == YQ_BASIS_FULL) {
            v = k;
        } else {
            // increasing order of values with popcount nup = colex order of the set
            // bits: rank = sum_i C(c_i, i) over the set bits c_1 < ... < c_nup
            uint64_t r = k;
            int c = n - 1;
            for (int i = nup; i >= 1; --i) {
                while (binom[size_t(c) * (n + 1) + i] > r) --c;
                v |= uint64_t(1) << c;
                r -= binom[size_t(c) * (n + 1) + i];
                --c;
            }
        }
        if (index) index[k] = v;
        int8_t* row = sigma + k * n;
        for (int i = 0; i < n; ++i) row[i] = ((v >> i) & 1u) ? int8_t(-1) : int8_t(1);
    }
}

// Position of configuration v in the basis, or -1 when v is not in it.
__device__ __forceinline__ long long basis_rank(uint64_t v, int n, int kind, int nup, const uint64_t* __restrict__ binom) {
    if (kind == YQ_BASIS_FULL) return (n >= 64 || (v >> n) == 0) ? (long long)v : -1;
    if (__popcll(v) != nup) return -1;
    uint64_t r = 0;
    int i = 1;
    for (int c = 0; c < n; ++c)
        if ((v >> c) & 1u) r += binom[size_t(c) * (n + 1) + i++];
    return (long long)r;
}

}  // namespace
}  // namespace yq
