// Checks galop_b200/csrc/engine_rng.cuh against the real thing: the
// reference's PCG32 (src/LGPEngine.h:80-98) and this compiler's libstdc++
// distributions and mt19937.  Built and run by tests/test_engine_rng.py.
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <random>

#include "LGPEngine.h"                                   // the reference's PCG32
#include "../../galop_b200/csrc/engine_rng.cuh"

int main() {
    long bad = 0, n = 0;
    const int ranges[] = {1, 2, 3, 5, 7, 64, 100, 999, 1000, 1001, 4096, 65537, 1000000, 99999989,
                          2147483647};
    for (uint64_t seed : {0ull, 1ull, 42ull, 0x9E3779B97F4A7C15ull, 0xFFFFFFFFFFFFFFFFull}) {
        for (uint64_t stream : {0ull, 1ull, 7ull, 123456789ull, 0x7FFFFFFFull}) {
            PCG32 ref(seed, stream);
            galop::Pcg32 mine(seed, stream);
            for (int i = 0; i < 2000; ++i, ++n) bad += ref() != mine.next();
            for (int hi : ranges) {
                std::uniform_int_distribution<int> d(0, hi - 1);
                for (int i = 0; i < 300; ++i, ++n) bad += d(ref) != galop::uniform_int(mine, 0, hi - 1);
                std::uniform_int_distribution<int> d1(1, hi);
                for (int i = 0; i < 100; ++i, ++n) bad += d1(ref) != galop::uniform_int(mine, 1, hi);
            }
            std::uniform_real_distribution<float> du(0.0f, 1.0f);
            for (int i = 0; i < 20000; ++i, ++n) {
                const float a = du(ref), b = galop::unit_float(mine);
                bad += std::memcmp(&a, &b, 4) != 0;
            }
            std::uniform_int_distribution<uint32_t> d32(0, UINT32_MAX);
            for (int i = 0; i < 2000; ++i, ++n) bad += d32(ref) != galop::uniform_u32(mine, 0u, 0xFFFFFFFFu);
        }
    }
    // mt19937 through the engine's full-range distribution (dist_32)
    for (uint32_t seed : {0u, 1u, 42u, 5489u, 4294967295u}) {
        std::mt19937 ref(seed);
        galop::Mt19937 mine(seed);
        std::uniform_int_distribution<uint32_t> d32(0, UINT32_MAX);
        for (int i = 0; i < 100000; ++i, ++n) bad += d32(ref) != mine.next();
    }
    std::printf("%ld %ld\n", n, bad);
    return bad != 0;
}
