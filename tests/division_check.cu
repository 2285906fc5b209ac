// division_check.cu -- checks the interpreter's fast division path against
// IEEE division on the GPU.  TEST INFRASTRUCTURE (built and run by
// tests/test_gpu_division.py); not part of the library.
//
// DivFast (dispatch_gen.cuh) is generated from the same lines as the DIV
// arms of the wide interpreter loop: q0 = a * y, r = a - b q0, q = q0 + r y
// with y = rcp.approx(b) refined by one Newton-Raphson step (Markstein's
// correction).  It claims its result (ok == 1) when 2^-63 <= |b| <= 2^63 and
// 2^-63 <= |a| <= 2^63 or a == 0, or when b == 0 (the protected 1.0).  The
// loop takes IEEE division (div.rn) for a warp in which any element is out
// of that range.
//
// Why these checks cover every in-range input: each step of the fast path
// is an IEEE operation whose result scales by a power of two with its
// inputs while nothing leaves the normal range, so fast(a, b) is
// fast(ma, mb) scaled by 2^(ea - eb) for significands ma, mb in [1, 2),
// provided rcp.approx itself scales, which mode `rcp` checks for every
// divisor in range.  Mode `pairs` checks all (or a stride of) the 2^46
// significand pairs; mode `random` random bit patterns over the whole float
// range plus a grid of special values, zero dividends included.
//
// Modes (one JSON line of counts on stdout):
//   rcp                 every b with 2^-63 <= |b| <= 2^63
//   pairs STEP          a significands 0, STEP, 2 STEP, ... x every b significand
//   random N SEED       N random pairs of bit patterns + the special grid
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <cstring>

#include "dispatch_gen.cuh"

using galop::DivFast;

__device__ __forceinline__ float rcp_approx(float b) {
    float y;
    asm("rcp.approx.ftz.f32 %0, %1;" : "=f"(y) : "f"(b));
    return y;
}

// the interpreter's semantics: protected, IEEE round to nearest
__device__ __forceinline__ float exact_div(float a, float b) { return b != 0.0f ? __fdiv_rn(a, b) : 1.0f; }

__device__ __forceinline__ bool same(float x, float y) {
    return __float_as_uint(x) == __float_as_uint(y) || (x != x && y != y);
}

struct Counts {
    unsigned long long checked, fast, mismatch, not_ok;
    unsigned int first_a, first_b, have_first, pad;
};

__device__ void note(Counts* c, float a, float b) {
    if (atomicCAS(&c->have_first, 0u, 1u) == 0u) {
        c->first_a = __float_as_uint(a);
        c->first_b = __float_as_uint(b);
    }
}

constexpr uint64_t kRcpCount = 127ull * 2ull * (1ull << 23);

// one thread per (exponent field 64..190, sign, significand) of b
__global__ void rcp_kernel(Counts* c) {
    const uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= kRcpCount) return;
    const uint32_t mant = (uint32_t)(i & 0x7fffffu);
    const uint32_t sign = (uint32_t)((i >> 23) & 1u) << 31;
    const uint32_t efield = 64u + (uint32_t)(i >> 24);
    const float b = __uint_as_float(sign | (efield << 23) | mant);
    const float bm = __uint_as_float(sign | (127u << 23) | mant);   // same significand in [1, 2)
    const uint32_t want = __float_as_uint(rcp_approx(bm)) - ((efield - 127u) << 23);
    if (__float_as_uint(rcp_approx(b)) != want) {
        atomicAdd(&c->mismatch, 1ull);
        note(c, 1.0f, b);
    }
}

// thread = b significand; loop over `count` a significands a0, a0 + step, ...
__global__ void pairs_kernel(uint32_t a0, uint32_t step, uint32_t count, Counts* c) {
    const uint32_t mb = blockIdx.x * blockDim.x + threadIdx.x;
    if (mb >= (1u << 23)) return;
    const float b = __uint_as_float(0x3f800000u | mb);
    unsigned long long bad = 0, nok = 0, n = 0;
    for (uint32_t j = 0; j < count; ++j) {
        const uint64_t ma = (uint64_t)a0 + (uint64_t)j * step;
        if (ma >= (1u << 23)) break;
        ++n;
        const float a = __uint_as_float(0x3f800000u | (uint32_t)ma);
        uint32_t ok = 0;
        const float q = DivFast::run(a, b, ok);
        if (!ok) {
            ++nok;
        } else if (!same(q, exact_div(a, b))) {
            ++bad;
            note(c, a, b);
        }
    }
    atomicAdd(&c->checked, n);
    if (bad) atomicAdd(&c->mismatch, bad);
    if (nok) atomicAdd(&c->not_ok, nok);
}

constexpr int kSpecialMax = 64;
__constant__ float kSpecial[kSpecialMax];

__device__ __forceinline__ uint32_t xorshift(uint32_t& s) {
    s ^= s << 13;
    s ^= s >> 17;
    s ^= s << 5;
    return s;
}

__global__ void random_kernel(uint32_t per_thread, uint32_t seed, uint32_t n_special, Counts* c) {
    const uint32_t t = blockIdx.x * blockDim.x + threadIdx.x;
    uint32_t s = seed ^ (t * 2654435761u) ^ 0x9e3779b9u;
    if (s == 0) s = 1;
    unsigned long long bad = 0, fast = 0;
    for (uint32_t j = 0; j < per_thread; ++j) {
        float a = __uint_as_float(xorshift(s));
        float b = __uint_as_float(xorshift(s));
        const uint32_t r = xorshift(s);
        // a quarter of the pairs take a special value on one side, a quarter
        // have both operands in the fast path's range
        if ((r & 3u) == 0u) {
            const float v = kSpecial[(r >> 2) % n_special];
            if (r & 0x100000u) a = v; else b = v;
        } else if ((r & 3u) == 1u) {
            a = __uint_as_float((__float_as_uint(a) & 0x807fffffu) | ((64u + (r >> 8) % 127u) << 23));
            b = __uint_as_float((__float_as_uint(b) & 0x807fffffu) | ((64u + (r >> 16) % 127u) << 23));
        }
        uint32_t ok = 0;
        const float q = DivFast::run(a, b, ok);
        if (ok) {
            ++fast;
            if (!same(q, exact_div(a, b))) {
                ++bad;
                note(c, a, b);
            }
        }
    }
    atomicAdd(&c->checked, (unsigned long long)per_thread);
    atomicAdd(&c->fast, fast);
    if (bad) atomicAdd(&c->mismatch, bad);
}

static void check(cudaError_t e, const char* what) {
    if (e != cudaSuccess) {
        std::printf("{\"error\": \"%s: %s\"}\n", what, cudaGetErrorString(e));
        std::exit(1);
    }
}

int main(int argc, char** argv) {
    if (argc < 2) return 2;
    Counts* d = nullptr;
    check(cudaMalloc(&d, sizeof(Counts)), "malloc");
    check(cudaMemset(d, 0, sizeof(Counts)), "memset");
    const char* mode = argv[1];
    unsigned long long checked_host = 0;
    if (!std::strcmp(mode, "rcp")) {
        rcp_kernel<<<(unsigned)((kRcpCount + 255) / 256), 256>>>(d);
        check(cudaGetLastError(), "launch");
        checked_host = kRcpCount;
    } else if (!std::strcmp(mode, "pairs") && argc >= 3) {
        const uint32_t step = (uint32_t)std::strtoul(argv[2], nullptr, 10);
        if (step == 0) return 2;
        const uint32_t per_launch = 256;
        for (uint64_t a0 = 0; a0 < (1ull << 23); a0 += (uint64_t)per_launch * step) {
            pairs_kernel<<<(1u << 23) / 256, 256>>>((uint32_t)a0, step, per_launch, d);
            check(cudaGetLastError(), "launch");
            check(cudaDeviceSynchronize(), "pairs");
        }
    } else if (!std::strcmp(mode, "random") && argc >= 4) {
        const uint64_t total = std::strtoull(argv[2], nullptr, 10);
        const uint32_t seed = (uint32_t)std::strtoul(argv[3], nullptr, 10);
        const float inf = __builtin_inff(), nan = __builtin_nanf("");
        const float sp[] = {0.0f, -0.0f, 1.0f, -1.0f, 2.0f, 0.5f, 3.0f, -3.0f, inf, -inf, nan, -nan,
                            1e-45f, -1e-45f, 1.17549435e-38f, 1.1754942e-38f, 3.4028235e38f, -3.4028235e38f,
                            0x1p-63f, -0x1p-63f, 0x1p63f, -0x1p63f, 0x1.fffffep-64f, 0x1.000002p63f,
                            0x1.fffffep62f, 0x1.000002p-63f, 1e-20f, 1e20f, 1e-19f, 1e19f, 7.0f, 0.1f,
                            -0.1f, 1e30f, 1e-30f, 0x1.fffffep0f, 0x1.000002p0f, 1.5f, -1.5f, 10.0f};
        const uint32_t n_special = (uint32_t)(sizeof sp / sizeof sp[0]);
        static_assert(sizeof sp / sizeof sp[0] <= kSpecialMax, "special grid");
        check(cudaMemcpyToSymbol(kSpecial, sp, sizeof sp), "special values");
        const uint32_t threads = 1u << 20;
        const uint64_t per_thread = (total + threads - 1) / threads;
        for (uint64_t done = 0; done < per_thread; done += 256) {
            const uint32_t chunk = (uint32_t)(per_thread - done < 256 ? per_thread - done : 256);
            random_kernel<<<threads / 256, 256>>>(chunk, seed + (uint32_t)done, n_special, d);
            check(cudaGetLastError(), "launch");
            check(cudaDeviceSynchronize(), "random");
        }
    } else {
        return 2;
    }
    check(cudaDeviceSynchronize(), "sync");
    Counts h{};
    check(cudaMemcpy(&h, d, sizeof h, cudaMemcpyDeviceToHost), "copy");
    if (checked_host) h.checked = checked_host;
    std::printf("{\"mode\": \"%s\", \"checked\": %llu, \"fast\": %llu, \"mismatch\": %llu, \"not_ok\": %llu, "
                "\"first_a\": %u, \"first_b\": %u}\n",
                mode, h.checked, h.fast, h.mismatch, h.not_ok, h.first_a, h.first_b);
    return 0;
}
