// fold.cuh -- constant folding and dead-code removal over the wide
// micro-ops of each program, after the intron pass.
//
// A register holds the same value in every fitness case until an
// instruction writes it from a case-dependent value: registers at or above
// the dataset's input count start at 0 (src/Interpreter.cpp:41-47), constant
// operands are constants.  An instruction all of whose operands are such
// known values computes the same number for every case, so it is evaluated
// once here -- with the very operations the interpreter would use (apply_op:
// __fadd_rn, IEEE division, sinf, ... on this device), hence the same bits --
// and becomes a broadcast micro-op (dest = that constant).  A second,
// backward liveness pass then drops instructions whose results no remaining
// instruction reads (broadcasts read nothing), and the survivors are packed
// to the front of the program's slot.  Per-case outputs and fitness are
// unchanged; only case-independent work is done once instead of per case.
#pragma once
#include <cstdint>
#include <cuda_runtime.h>
#include "isa.cuh"
#include "interp.cuh"

namespace galop {

constexpr uint32_t kWideDead = 0xFFFFFFFEu;   // dropped (never reaches the interpreter)

struct FoldParams {
    int profile;
    int num_registers;
    int output_reg;
    uint32_t stride_shift;       // log2 of the register stride S
    int num_inputs;              // single population; or per program through pops/prog_pop
    const PopDesc* pops;
    const int32_t* prog_pop;
};

static __global__ void fold_kernel(uint4* __restrict__ uops, const int64_t* __restrict__ eff_off, int64_t n,
                                   FoldParams fp, int32_t* __restrict__ interp_len,
                                   unsigned long long* __restrict__ total) {
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    int64_t kept = 0;
    if (i < n) {
        const int64_t p0 = eff_off[i];
        const int64_t L = eff_off[i + 1] - p0;
        uint4* __restrict__ u = uops + p0;
        const uint32_t sh = fp.stride_shift;
        const int k_in = fp.pops ? fp.pops[fp.prog_pop[i]].num_inputs : fp.num_inputs;
        float vals[kMaxRegisters];
        uint32_t known = 0;
        for (int r = 0; r < fp.num_registers; ++r) {
            vals[r] = 0.0f;
            if (r >= k_in) known |= 1u << r;
        }
        // forward: evaluate what is known
        for (int64_t j = 0; j < L; ++j) {
            const uint4 w = u[j];
            const uint32_t op = w.w & 7u;
            const bool is_const = (w.w & 8u) != 0;
            const bool unary = (w.w & kWideSpecial) != 0;
            const uint32_t s1 = w.x >> sh, s2 = w.y >> sh, d = w.z >> sh;
            const bool a_known = unary || ((known >> s1) & 1u);
            const bool b_known = is_const || ((known >> s2) & 1u);
            if (a_known && b_known) {
                const float a = unary ? 0.0f : vals[s1];
                const float b = is_const ? __uint_as_float(w.y) : vals[s2];
                const float v = fp.profile == kProfileBj ? apply_op<kProfileBj>(op, a, b)
                                                         : apply_op<kProfileRef>(op, a, b);
                vals[d] = v;
                known |= 1u << d;
                u[j] = make_uint4(0u, __float_as_uint(v), w.z, kWideBcast);
            } else {
                known &= ~(1u << d);
            }
        }
        // backward: drop what nothing reads
        uint32_t live = 1u << fp.output_reg;
        for (int64_t j = L - 1; j >= 0; --j) {
            const uint4 w = u[j];
            const uint32_t d = w.z >> sh;
            if (!((live >> d) & 1u)) {
                u[j].w = kWideDead;
                continue;
            }
            live &= ~(1u << d);
            if (w.w != kWideBcast) {
                if (!(w.w & kWideSpecial)) live |= 1u << (w.x >> sh);
                if (!(w.w & 8u)) live |= 1u << (w.y >> sh);
            }
        }
        for (int64_t j = 0; j < L; ++j) {
            const uint4 w = u[j];
            if (w.w != kWideDead) u[kept++] = w;
        }
        interp_len[i] = (int32_t)kept;
    }
    __shared__ unsigned long long sk;
    if (threadIdx.x == 0) sk = 0;
    __syncthreads();
    if (kept) atomicAdd(&sk, (unsigned long long)kept);
    __syncthreads();
    if (threadIdx.x == 0 && sk) atomicAdd(total, sk);
}

}  // namespace galop
