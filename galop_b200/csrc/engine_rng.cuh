// engine_rng.cuh -- the random streams of the reference's evolution engine,
// usable on the host and on the device, so that variation on the GPU draws
// exactly the numbers the engine draws on the CPU.
//
//   Pcg32       the engine's per-pair generator (src/LGPEngine.h:80-98):
//               O'Neill's pcg32 (XSH-RR output, 64-bit LCG state), seeded
//               with (seed, stream) as the engine seeds it.
//   uniform_u32 std::uniform_int_distribution over a 32-bit generator as
//               GCC's libstdc++ (13.x) computes it: the raw draw when the
//               range is the generator's full range, else Lemire's
//               nearly-divisionless method ("Fast Random Integer Generation
//               in an Interval", ACM TOMACS 2019) with 64-bit products.
//   unit_float  std::uniform_real_distribution<float>(0, 1) over a 32-bit
//               generator as libstdc++ computes it (generate_canonical<float,
//               24>: one draw, float(x) / 2^32, values that round up to 1
//               replaced by the largest float below 1).
//   Mt19937     the engine's master generator, std::mt19937 (Matsumoto &
//               Nishimura 1998, the parameters the C++ standard fixes); host
//               only.
#pragma once
#include <cstdint>

#ifdef __CUDACC__
#define GALOP_HD __host__ __device__ __forceinline__
#else
#define GALOP_HD inline
#endif

namespace galop {

struct Pcg32 {
    uint64_t state;
    uint64_t inc;
    GALOP_HD Pcg32(uint64_t seed, uint64_t stream) : state(0u), inc((stream << 1u) | 1u) {
        next();
        state += seed;
        next();
    }
    GALOP_HD uint32_t next() {
        const uint64_t old = state;
        state = old * 6364136223846793005ULL + inc;
        const uint32_t xs = (uint32_t)(((old >> 18u) ^ old) >> 27u);
        const uint32_t rot = (uint32_t)(old >> 59u);
        return (xs >> rot) | (xs << ((32u - rot) & 31u));
    }
};

// Uniform integer in [lo, hi] (hi - lo < 2^32), drawn from a generator G
// with a 32-bit full-range output G::next().
template <class G>
GALOP_HD uint32_t uniform_u32(G& g, uint32_t lo, uint32_t hi) {
    const uint32_t range = hi - lo;
    if (range == 0xFFFFFFFFu) return lo + g.next();
    const uint32_t n = range + 1u;
    uint64_t product = (uint64_t)g.next() * (uint64_t)n;
    uint32_t low = (uint32_t)product;
    if (low < n) {
        const uint32_t threshold = (0u - n) % n;
        while (low < threshold) {
            product = (uint64_t)g.next() * (uint64_t)n;
            low = (uint32_t)product;
        }
    }
    return lo + (uint32_t)(product >> 32);
}

template <class G>
GALOP_HD int uniform_int(G& g, int lo, int hi) {
    return (int)((uint32_t)lo + uniform_u32(g, 0u, (uint32_t)hi - (uint32_t)lo));
}

template <class G>
GALOP_HD float unit_float(G& g) {
    const float x = (float)g.next();               // rounded to nearest
    const float r = x / 4294967296.0f;             // exact: a power of two
    return r >= 1.0f ? 0x1.fffffep-1f : r;
}

// std::mt19937 (host only: the engine's master stream).
struct Mt19937 {
    uint32_t mt[624];
    int idx;
    explicit Mt19937(uint32_t seed) {
        mt[0] = seed;
        for (int i = 1; i < 624; ++i) mt[i] = 1812433253u * (mt[i - 1] ^ (mt[i - 1] >> 30)) + (uint32_t)i;
        idx = 624;
    }
    uint32_t next() {
        if (idx >= 624) {
            for (int i = 0; i < 624; ++i) {
                const uint32_t y = (mt[i] & 0x80000000u) | (mt[(i + 1) % 624] & 0x7FFFFFFFu);
                mt[i] = mt[(i + 397) % 624] ^ (y >> 1) ^ ((y & 1u) ? 0x9908B0DFu : 0u);
            }
            idx = 0;
        }
        uint32_t y = mt[idx++];
        y ^= y >> 11;
        y ^= (y << 7) & 0x9D2C5680u;
        y ^= (y << 15) & 0xEFC60000u;
        y ^= y >> 18;
        return y;
    }
};

}  // namespace galop
