// Oracle-side Philox4x32-10 (test infrastructure: used only by the CPU oracle).
//
// Counter-based RNG of Salmon, Moraes, Dror, Shaw, "Parallel random numbers:
// as easy as 1, 2, 3", SC'11. Written here from the published round function:
//   (hi0, lo0) = mulhilo(0xD2511F53, c0); (hi1, lo1) = mulhilo(0xCD9E8D57, c2)
//   c' = (hi1 ^ c1 ^ k0, lo1, hi0 ^ c3 ^ k1, lo0)
//   k' = (k0 + 0x9E3779B9, k1 + 0xBB67AE85)
// ten rounds, key bumped between rounds.  The device library has its own copy
// (yannq_b200/csrc/philox.cuh); both are pinned to the Random123 known-answer
// vectors and to each other by the tests.
//
// Stream convention shared with the device sampler (the reference draws from
// std::default_random_engine seeded by std::random_device, so its streams are
// not reproducible; this convention replaces them):
//   key     = (seed & 0xffffffff, seed >> 32)
//   counter = (index, epoch, chain, tag)
//   site    = (uint64(x0) * n) >> 32            (multiply-shift, bias <= n/2^32)
//   u (f64) = ((uint64(x2) << 21) | (x3 >> 11)) * 2^-53   in [0, 1)
#pragma once
#include <cstdint>

namespace orc {

enum : uint32_t {
    TAG_SWEEP = 0x53574550u,  // proposals of a Metropolis sweep
    TAG_INIT = 0x494e4954u,   // random +-1 chain initialisation
    TAG_SHUF = 0x53485546u,   // fixed-magnetisation shuffle
    TAG_PARAM = 0x50415241u,  // normal draws for parameter initialisation
    TAG_EXACT = 0x45584143u,  // exact-sampler draws
    TAG_PT = 0x50544d58u,     // parallel-tempering swap draws
};

struct Philox4x32 {
    static inline void mulhilo(uint32_t a, uint32_t b, uint32_t& hi, uint32_t& lo) {
        uint64_t p = uint64_t(a) * uint64_t(b);
        hi = uint32_t(p >> 32);
        lo = uint32_t(p);
    }
    static inline void generate(const uint32_t ctr_in[4], const uint32_t key_in[2], uint32_t out[4]) {
        uint32_t c0 = ctr_in[0], c1 = ctr_in[1], c2 = ctr_in[2], c3 = ctr_in[3];
        uint32_t k0 = key_in[0], k1 = key_in[1];
        for (int r = 0; r < 10; ++r) {
            if (r > 0) {
                k0 += 0x9E3779B9u;
                k1 += 0xBB67AE85u;
            }
            uint32_t hi0, lo0, hi1, lo1;
            mulhilo(0xD2511F53u, c0, hi0, lo0);
            mulhilo(0xCD9E8D57u, c2, hi1, lo1);
            uint32_t n0 = hi1 ^ c1 ^ k0;
            uint32_t n2 = hi0 ^ c3 ^ k1;
            c0 = n0;
            c1 = lo1;
            c2 = n2;
            c3 = lo0;
        }
        out[0] = c0;
        out[1] = c1;
        out[2] = c2;
        out[3] = c3;
    }
    static inline void draw(uint64_t seed, uint32_t index, uint32_t epoch, uint32_t chain, uint32_t tag,
                            uint32_t out[4]) {
        uint32_t ctr[4] = {index, epoch, chain, tag};
        uint32_t key[2] = {uint32_t(seed), uint32_t(seed >> 32)};
        generate(ctr, key, out);
    }
};

inline uint32_t draw_site(uint32_t x, uint32_t n) { return uint32_t((uint64_t(x) * n) >> 32); }
inline double draw_u53(uint32_t x2, uint32_t x3) {
    uint64_t v = (uint64_t(x2) << 21) | uint64_t(x3 >> 11);
    return double(v) * (1.0 / 9007199254740992.0);
}
inline float draw_u24(uint32_t x2) { return float(x2 >> 8) * (1.0f / 16777216.0f); }

}  // namespace orc
