// interp_wide.cuh -- the wide-micro-op interpreter (dispatch 3).
//
// Same work decomposition as the shared-memory interpreter of interp.cuh
// (one warp per program or case chunk, K cases per lane, the lane's NR x K
// register file in shared memory), but every instruction is a 16-byte
// micro-op whose operand fields are already byte offsets into the register
// file (encode_wide in isa.cuh), and a constant operand carries its value.
// Runs of binary instructions execute inside one PTX loop (WideLoop); per
// instruction the warp does:
//   one broadcast 16-byte shared load of the micro-op (the 32-instruction
//     window is staged in shared memory; the next micro-op is prefetched
//     into a second register set, the loop body existing twice),
//   a sign test (unary ops and the window end leave the loop),
//   one jump table (16 arms: 8 ops x register/constant src2, each with
//     entry points that skip what the micro-op's flags make unnecessary)
//     whose arm stores the previous result if the flags ask for it, loads
//     src1 unless it is the previous result, loads src2 (register arms),
//     and computes into the result registers, which are also the src1
//     registers.
// The result registers a[K] and the address of the register they belong to
// live across the whole pass: the unary ops (SIN/COS, and EXP/LOG of the BJ
// profile), which run in C++ on the slow branch with the CUDA math library,
// read and write them too.  The last result is never stored: the output
// is taken from it when the last instruction wrote the output register.
// Each pass initialises only the registers the program reads before
// writing them (args.livein).  The folding pass sets the flags and the
// masks (isa.cuh, fold.cuh).
//
// Semantics are those of interp.cuh (src/Interpreter.cpp:36-59,
// src/ISA.h:219-231, src/Evaluator.cpp:11-45 and :88-91).
#pragma once
#include <cstdint>
#include <cuda_runtime.h>
#include "isa.cuh"
#include "interp.cuh"
#include "dispatch_gen.cuh"

namespace galop {

// The lane's view of one register: K floats as K/V vectors of V floats,
// vector q at byte offset q * 32 * V * 4 (lane l's V floats at l * V * 4).
template <int K>
struct WideRegs {
    static constexpr int V = K < 4 ? K : 4;
    static constexpr uint32_t kStride = 128u * K;          // bytes per register per warp
    static constexpr uint32_t kChunk = 128u * V;           // bytes between vectors

    static __device__ __forceinline__ void load(uint32_t addr, float (&v)[K]) {
#pragma unroll
        for (int q = 0; q < K / V; ++q) {
            const uint32_t p = addr + q * kChunk;
            if constexpr (V == 4) {
                asm volatile("ld.shared.v4.f32 {%0, %1, %2, %3}, [%4];"
                             : "=f"(v[4 * q]), "=f"(v[4 * q + 1]), "=f"(v[4 * q + 2]), "=f"(v[4 * q + 3])
                             : "r"(p) : "memory");
            } else if constexpr (V == 2) {
                asm volatile("ld.shared.v2.f32 {%0, %1}, [%2];" : "=f"(v[2 * q]), "=f"(v[2 * q + 1]) : "r"(p)
                             : "memory");
            } else {
                asm volatile("ld.shared.f32 %0, [%1];" : "=f"(v[q]) : "r"(p) : "memory");
            }
        }
    }

    static __device__ __forceinline__ void store(uint32_t addr, const float (&v)[K]) {
#pragma unroll
        for (int q = 0; q < K / V; ++q) {
            const uint32_t p = addr + q * kChunk;
            if constexpr (V == 4) {
                asm volatile("st.shared.v4.f32 [%0], {%1, %2, %3, %4};"
                             :: "r"(p), "f"(v[4 * q]), "f"(v[4 * q + 1]), "f"(v[4 * q + 2]), "f"(v[4 * q + 3])
                             : "memory");
            } else if constexpr (V == 2) {
                asm volatile("st.shared.v2.f32 [%0], {%1, %2};" :: "r"(p), "f"(v[2 * q]), "f"(v[2 * q + 1])
                             : "memory");
            } else {
                asm volatile("st.shared.f32 [%0], %1;" :: "r"(p), "f"(v[q]) : "memory");
            }
        }
    }
};

__device__ __forceinline__ uint4 lds_u4(uint32_t addr) {
    uint4 u;
    asm volatile("ld.shared.v4.u32 {%0, %1, %2, %3}, [%4];" : "=r"(u.x), "=r"(u.y), "=r"(u.z), "=r"(u.w)
                 : "r"(addr) : "memory");
    return u;
}

__device__ __forceinline__ void sts_u4(uint32_t addr, uint4 u) {
    asm volatile("st.shared.v4.u32 [%0], {%1, %2, %3, %4};" :: "r"(addr), "r"(u.x), "r"(u.y), "r"(u.z), "r"(u.w)
                 : "memory");
}

// Shared memory per warp: NR registers x stride, then a 33-entry micro-op
// stage (32 instructions + a permanent end marker).
constexpr uint32_t kWideStageBytes = 33u * 16u;

template <int NR, int K>
__host__ __device__ constexpr uint32_t wide_warp_bytes() {
    return (uint32_t)NR * 128u * K + kWideStageBytes;
}

inline size_t wide_smem_bytes(int nr, int k, int warps) {
    return (size_t)warps * ((size_t)nr * 128u * (size_t)k + kWideStageBytes);
}

// One work item of the persistent queue: which program, which cases, which
// dataset, where the result goes.
struct WideItem {
    int64_t prog, cbeg, cend, N, Np, out_index, partial_index;
    int num_inputs;
    const float* X;
    const float* y;
    float* fitness;
    double* sse;
    Objective obj;
};

__device__ __forceinline__ WideItem resolve_item(const InterpArgs& args, unsigned long long item) {
    WideItem w;
    w.partial_index = -1;
    if (args.pops != nullptr) {
        const unsigned long long it = args.items[item];
        w.prog = (int64_t)(it >> 20);
        const int chunk = (int)(it & 0xFFFFFull);
        const PopDesc* d = args.pops + args.prog_pop[w.prog];
        w.X = d->X;
        w.y = d->y;
        w.N = d->N;
        w.Np = d->Np;
        w.num_inputs = d->num_inputs;
        w.cbeg = (int64_t)chunk * d->chunk_cases;
        w.cend = w.cbeg + d->chunk_cases;
        w.fitness = d->fitness;
        w.sse = d->sse;
        w.obj = d->obj;
        w.out_index = w.prog - d->prog_base;
        if (d->n_chunks > 1) w.partial_index = (int64_t)item;
    } else {
        const int64_t slot = (int64_t)item / args.n_chunks;
        const int chunk = (int)((int64_t)item % args.n_chunks);
        w.prog = args.order ? (int64_t)args.order[slot] : slot;
        w.X = args.X;
        w.y = args.y;
        w.N = args.N;
        w.Np = args.Np;
        w.num_inputs = args.num_inputs;
        w.cbeg = (int64_t)chunk * args.chunk_cases;
        w.cend = w.cbeg + args.chunk_cases;
        w.fitness = args.fitness;
        w.sse = args.sse;
        w.obj = args.obj;
        w.out_index = w.prog;
        if (args.n_chunks > 1) w.partial_index = w.prog * args.n_chunks + chunk;
    }
    if (w.cend > w.N) w.cend = w.N;
    return w;
}

// Trace mode: all NR registers of the lane's cases after instruction `row`
// (row 0 = initial state), at trace[(row * NR + r) * 32K + case].
template <int NR, int K>
__device__ __forceinline__ void wide_trace(float* __restrict__ trace, int64_t row, uint32_t base, int lane) {
    using WR = WideRegs<K>;
    constexpr int V = WR::V;
#pragma unroll
    for (int r = 0; r < NR; ++r) {
        float v[K];
        WR::load(base + r * WR::kStride, v);
#pragma unroll
        for (int q = 0; q < K / V; ++q)
#pragma unroll
            for (int e = 0; e < V; ++e)
                trace[(row * NR + r) * (32 * K) + (q * 32 + lane) * V + e] = v[q * V + e];
    }
}

// The unary ops of the profile on K cases: SIN/COS (REF), SIN/COS/EXP/LOG
// (BJ), with the CUDA math library as everywhere else.
template <int K, int PROFILE>
__device__ __forceinline__ void unary_op(uint32_t op, const float (&b)[K], float (&t)[K]) {
    if constexpr (PROFILE == kProfileRef) {
        if (op == kSin) {
#pragma unroll
            for (int k = 0; k < K; ++k) t[k] = sinf(b[k]);
        } else {
#pragma unroll
            for (int k = 0; k < K; ++k) t[k] = cosf(b[k]);
        }
    } else {
        slow_op<K, PROFILE>(op, b, b, t);
    }
}

template <int NR, int K, int PROFILE, int REDUCE, int MODE>
__global__ void __launch_bounds__(256, 3)
interp_wide_kernel(InterpArgs args) {
    extern __shared__ float4 galop_smem4[];
    using WR = WideRegs<K>;
    constexpr int V = WR::V;
    constexpr uint32_t S = WR::kStride;
    constexpr int kPass = 32 * K;
    const int lane = threadIdx.x & 31;
    const uint32_t warp_base = (uint32_t)__cvta_generic_to_shared(galop_smem4) +
                               (threadIdx.x >> 5) * wide_warp_bytes<NR, K>();
    const uint32_t base = warp_base + (uint32_t)lane * V * 4u;   // this lane's register 0
    const uint32_t stage = warp_base + NR * S;
    const uint4 kEnd4 = make_uint4(0u, 0u, 0u, kWideEnd);
    if (lane == 0) sts_u4(stage + 32u * 16u, kEnd4);
    __syncwarp();

    const int64_t n_work = args.n_skipped ? args.n_programs - (int64_t)*args.n_skipped : args.n_programs;
    const int64_t total_items = args.pops != nullptr ? (args.n_items_dev ? *args.n_items_dev : args.n_items)
                                                     : n_work * (int64_t)args.n_chunks;
    const uint4* __restrict__ uops4 = reinterpret_cast<const uint4*>(args.uops);

    for (;;) {
        unsigned long long item = 0;
        if (lane == 0) item = atomicAdd(args.counter, 1ull);
        item = __shfl_sync(0xffffffffu, item, 0);
        if ((int64_t)item >= total_items) break;
        const WideItem w = resolve_item(args, item);
        // folded programs are packed against the end of their slot (fold.cuh)
        const int64_t L = args.interp_len ? (int64_t)args.interp_len[w.prog]
                                          : args.eff_off[w.prog + 1] - args.eff_off[w.prog];
        const int64_t p0 = args.eff_off[w.prog + 1] - L;
        const uint4* __restrict__ pw = uops4 + p0;
        const uint32_t livein = (MODE == kModeTrace || args.livein == nullptr) ? (1u << NR) - 1u
                                                                              : args.livein[w.prog];

        float ks = 0.0f, kc = 0.0f;
        double big = 0.0;
        double acc = 0.0;

        for (int64_t cb = w.cbeg; cb < w.cend; cb += kPass) {
            // Case of element q*V+e of this lane: cb + (q*32 + lane)*V + e.
            const int64_t c0 = cb + (int64_t)lane * V;
            // Only the registers the program reads before writing them are
            // initialised (all of them for a register trace).
            for (uint32_t m = livein; m != 0u; m &= m - 1u) {
                const int f = __ffs(m) - 1;
                float v[K];
                if (f < w.num_inputs) {
#pragma unroll
                    for (int q = 0; q < K / V; ++q) {
                        float t[V];
                        load_cases<V>(w.X + (int64_t)f * w.Np + c0 + q * 32 * V, t);
#pragma unroll
                        for (int e = 0; e < V; ++e) v[q * V + e] = t[e];
                    }
                } else {
#pragma unroll
                    for (int k = 0; k < K; ++k) v[k] = 0.0f;
                }
                WR::store(base + f * S, v);
            }
            if constexpr (MODE == kModeTrace) wide_trace<NR, K>(args.trace, 0, base, lane);

            float a[K];       // result of the last instruction executed
            uint32_t pt = 0;  // its register's address
#pragma unroll
            for (int k = 0; k < K; ++k) a[k] = 0.0f;
            for (int64_t wb = 0; wb < L; wb += 32) {
                const int64_t n = (L - wb < 32) ? L - wb : 32;
                const uint4 mine = (lane < n) ? __ldg(pw + wb + lane) : kEnd4;
                sts_u4(stage + (uint32_t)lane * 16u, mine);
                __syncwarp();
                uint32_t sp = stage;
                if constexpr (MODE == kModeTrace) {
                    // One instruction at a time, the register file dumped after
                    // each; every result is stored, the flags do not apply.
                    for (;;) {
                        uint4 u = lds_u4(sp);
                        while ((int32_t)u.w >= 0) {
                            WideOps<K, PROFILE>::run(u.w & 15u, base + u.x, base + u.y, base + u.z, u.y);
                            wide_trace<NR, K>(args.trace, wb + (sp - stage) / 16u + 1, base, lane);
                            sp += 16u;
                            u = lds_u4(sp);
                        }
                        if (u.w == kWideEnd) break;
                        float b[K];
                        if (u.w & 8u) {
                            const float c = __uint_as_float(u.y);
#pragma unroll
                            for (int k = 0; k < K; ++k) b[k] = c;
                        } else {
                            WR::load(base + u.y, b);
                        }
                        slow_op<K, PROFILE>(u.w & 7u, b, b, a);
                        WR::store(base + u.z, a);
                        wide_trace<NR, K>(args.trace, wb + (sp - stage) / 16u + 1, base, lane);
                        sp += 16u;
                    }
                } else {
                    uint4 cur = lds_u4(sp);
                    for (;;) {
                        // Every binary instruction up to the next unary op or the
                        // end marker; u is the micro-op that stopped the loop.
                        uint4 u;
                        WideLoop<K, PROFILE>::run(sp, a, pt, base, cur, u);
                        if (u.w == kWideEnd) break;
                        const uint4 next = lds_u4(sp + 16u);   // the end marker at most
                        // Unary op on src2 (register, constant or the previous result).
                        if (u.w & kWideStorePrev) WR::store(pt, a);
                        float b[K];
                        if (u.w & 8u) {
                            const float c = __uint_as_float(u.y);
#pragma unroll
                            for (int k = 0; k < K; ++k) b[k] = c;
                        } else if (u.w & kWideFwd2) {
#pragma unroll
                            for (int k = 0; k < K; ++k) b[k] = a[k];
                        } else {
                            WR::load(base + u.y, b);
                        }
                        unary_op<K, PROFILE>(u.w & 7u, b, a);
                        pt = base + u.z;
                        sp += 16u;
                        cur = next;
                    }
                }
                __syncwarp();
            }
            // The output register: the last result when the last instruction
            // wrote it (never stored), else the register file.
            float o[K];
            const uint32_t out_addr = base + (uint32_t)args.output_reg * S;
            if (MODE != kModeTrace && L > 0 && pt == out_addr) {
#pragma unroll
                for (int k = 0; k < K; ++k) o[k] = a[k];
            } else {
                WR::load(out_addr, o);
            }
            if constexpr (MODE == kModeOutputs) {
#pragma unroll
                for (int q = 0; q < K / V; ++q)
#pragma unroll
                    for (int e = 0; e < V; ++e) {
                        const int64_t c = cb + (int64_t)(q * 32 + lane) * V + e;
                        if (c < w.cend) args.outputs[w.prog * w.N + c] = o[q * V + e];
                    }
            } else if constexpr (MODE == kModeFitness) {
                float t[K];
#pragma unroll
                for (int q = 0; q < K / V; ++q) {
                    float tv[V];
                    load_cases<V>(w.y + c0 + q * 32 * V, tv);
#pragma unroll
                    for (int e = 0; e < V; ++e) t[q * V + e] = tv[e];
                }
                if constexpr (REDUCE == kReduceKahan32) {
#pragma unroll
                    for (int k = 0; k < K; ++k) {
                        const int64_t c = cb + (int64_t)((k / V) * 32 + lane) * V + (k % V);
                        const float e = __fsub_rn(o[k], t[k]);
                        const bool valid = c < w.cend;
                        const bool huge = !(fabsf(e) <= kKahanMaxError);
                        const float qv = (valid && !huge) ? __fmul_rn(e, e) : 0.0f;
                        if (valid && huge) big = __dadd_rn(big, __dmul_rn((double)e, (double)e));
                        const float yk = __fsub_rn(qv, kc);
                        const float tt = __fadd_rn(ks, yk);
                        kc = __fsub_rn(__fsub_rn(tt, ks), yk);
                        ks = tt;
                    }
                } else if constexpr (REDUCE == kReduceFp64) {
#pragma unroll
                    for (int k = 0; k < K; ++k) {
                        const int64_t c = cb + (int64_t)((k / V) * 32 + lane) * V + (k % V);
                        const double e = (double)o[k] - (double)t[k];
                        if (c < w.cend) acc = __dadd_rn(acc, __dmul_rn(e, e));
                    }
                } else {
                    // Strict case order: vector q, lane j, element e.
                    double qd[K];
#pragma unroll
                    for (int k = 0; k < K; ++k) {
                        const double e = (double)o[k] - (double)t[k];
                        qd[k] = __dmul_rn(e, e);
                    }
#pragma unroll
                    for (int q = 0; q < K / V; ++q) {
                        for (int j = 0; j < 32; ++j) {
#pragma unroll
                            for (int e = 0; e < V; ++e) {
                                const double v = __shfl_sync(0xffffffffu, qd[q * V + e], j);
                                if (cb + (int64_t)(q * 32 + j) * V + e < w.cend) acc = __dadd_rn(acc, v);
                            }
                        }
                    }
                }
            }
            if constexpr (MODE == kModeTrace) break;
        }

        if constexpr (MODE == kModeFitness) {
            double sse;
            if constexpr (REDUCE == kReduceKahan32) sse = warp_sum_f64((double)ks - (double)kc + big);
            else if constexpr (REDUCE == kReduceFp64) sse = warp_sum_f64(acc);
            else sse = acc;
            if (lane == 0) {
                if (w.partial_index < 0) {
                    w.fitness[w.out_index] = fitness_of(sse, w.N, w.obj);
                    if (w.sse) w.sse[w.out_index] = sse;
                } else {
                    args.partial[w.partial_index] = sse;
                }
            }
        }
        if constexpr (MODE == kModeTrace) break;
    }
}

}  // namespace galop
