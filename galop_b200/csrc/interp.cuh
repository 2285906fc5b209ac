// interp.cuh -- shared definitions of the warp-per-individual interpreters
// and the compact interpreter (dispatch 2).
//
// One warp evaluates one program (or one case chunk of it); lane l of the warp
// owns K fitness cases of every 32*K-case pass.  The LGP register file of
// those cases lives in shared memory, so a register index is an address
// offset: no local-memory register array (the reference's
// program_partial_sse keeps reg[] in local memory, src/EvaluatorCuda.cu:127,
// :151-153) and no select chains over NR registers.
//
// Fitness cases: feature-major (SoA) arrays padded to a multiple of 1024
// cases; a lane reads its cases of a feature with 8/16-byte vector loads,
// so a warp reads 32*K contiguous floats per feature.
//
// Semantics per case follow src/Interpreter.cpp:36-59: r0..k-1 = inputs, the
// rest 0, execute every instruction in order, output r[OUTPUT_REG].  Fitness
// follows src/Evaluator.cpp:11-45 and :88-91 (see galop_reduce in the header
// for the three accumulation modes).
//
// The default interpreter (dispatch 3) is interp_wide.cuh; this file keeps
// the compact one (dispatch 2: 32-bit micro-ops, one instruction at a time),
// which the no-allocation entry point uses and the parity tests hold to the
// same bar.
#pragma once
#include <cstdint>
#include <cuda_runtime.h>
#include "isa.cuh"
#include "dispatch_gen.cuh"
#include "fitness.cuh"

namespace galop {

enum Reduce : int { kReduceKahan32 = 0, kReduceFp64 = 1, kReduceOrdered = 2 };
enum Mode : int { kModeFitness = 0, kModeOutputs = 1, kModeTrace = 2 };

// One population of a batched evaluation (galop_batch_*): its resident
// dataset, case chunking and outputs.  Programs of all populations are
// numbered globally; prog_base is this population's first.
struct PopDesc {
    const float* X;                // [num_inputs][Np]
    const float* y;                // [Np]
    int64_t N;
    int64_t Np;
    float* fitness;                // [n_programs of the population]
    double* sse;                   // or null
    int64_t prog_base;
    int64_t chunk_cases;           // cases per work item (multiple of 1024)
    int32_t n_chunks;              // work items per program
    int32_t num_inputs;
    Objective obj;                 // fitness from SSE for this population's dataset
};

struct InterpArgs {
    const uint32_t* uops;          // micro-ops, CSR by eff_off
    const int64_t* eff_off;        // [n_programs + 1]
    const int32_t* interp_len;     // interpreted length per program after folding (the last interp_len
                                   // micro-ops of the program's slot), or null
    const uint32_t* livein;        // per program: registers read before written (wide kernel), or null: all
    const unsigned long long* n_skipped;  // copies left out of the order (dedup), or null
    const int32_t* order;          // slot -> program (longest first), or null
    int64_t n_programs;
    int32_t n_chunks;              // work items per program
    int64_t chunk_cases;           // cases per item (multiple of 32*K)
    const float* X;                // [num_inputs][Np] feature-major
    const float* y;                // [Np]
    int64_t N;                     // real case count
    int64_t Np;                    // padded case count (multiple of 1024)
    int32_t num_inputs;
    int32_t output_reg;
    ConstPool consts;
    Objective obj;                 // fitness from SSE (single-population mode)
    unsigned long long* counter;   // work-queue head (zeroed before launch)
    float* fitness;                // [n_programs] (n_chunks == 1)
    double* sse;                   // [n_programs] or null (n_chunks == 1)
    double* partial;               // [n_programs * n_chunks] (n_chunks > 1)
    float* outputs;                // kModeOutputs: [n_programs * N]
    float* trace;                  // kModeTrace: [(L+1) * NR][n_traced]
    // Batched mode (pops != null, fitness mode, shared-memory kernel only):
    // work item i is items[i] = global program << 20 | chunk, longest work
    // first; partial sums of chunked programs go to partial[i].
    const PopDesc* pops;
    const int32_t* prog_pop;       // global program -> population
    const unsigned long long* items;
    int64_t n_items;
    const int64_t* n_items_dev;    // the item count computed on the device (dedup), or null
    // Plain schedule (single population): warp w of the grid evaluates
    // program w over all its cases (n_chunks 1, no order, no queue), and a
    // dedup copy (interp_len < 0) is skipped.
    int32_t plain;
    // Register-file classes (wide kernel): the order lists the programs
    // whose values fit in 8 slots first.  Single population: *class_split is
    // their count, class_part 0 covers those slots of the order, 1 the rest.
    // Batched: their work items come first in `items`, *class_split is the
    // first item of the others, class_part 0 covers the items before it, 1
    // the rest.  class_split null: one launch covers everything.
    const unsigned long long* class_split;
    int32_t class_part;
};

template <int K>
__device__ __forceinline__ void load_cases(const float* __restrict__ p, float (&v)[K]) {
    if constexpr (K % 4 == 0) {
#pragma unroll
        for (int k = 0; k < K; k += 4) {
            const float4 q = __ldg(reinterpret_cast<const float4*>(p + k));
            v[k] = q.x; v[k + 1] = q.y; v[k + 2] = q.z; v[k + 3] = q.w;
        }
    } else if constexpr (K == 2) {
        const float2 q = __ldg(reinterpret_cast<const float2*>(p));
        v[0] = q.x; v[1] = q.y;
    } else {
#pragma unroll
        for (int k = 0; k < K; ++k) v[k] = __ldg(p + k);
    }
}

// Most cases one work item of the persistent interpreter covers (a
// multiple of every pass width 32*K): longer case ranges are split into
// chunks whose partial sums are added in chunk order.
constexpr int64_t kMaxItemCases = 16384;

// KAHAN32 keeps squared errors in FP32 only while |error| <= 2^52: a square
// is then <= 2^104 and a lane's compensated sum of up to 2^20 of them stays
// finite.  Larger (or non-finite) errors are squared and summed in FP64, so
// the FP32 path never overflows where the CPU's double sum would not.
constexpr float kKahanMaxError = 4503599627370496.0f;   // 2^52

__device__ __forceinline__ double warp_sum_f64(double v) {
#pragma unroll
    for (int off = 16; off > 0; off >>= 1) v += __shfl_down_sync(0xffffffffu, v, off);
    return v;
}

// ---- dispatch 2: the LGP register file in shared memory, 32-bit micro-ops -----
//
// Each lane keeps its K cases' NR registers in its own shared-memory slots:
// register j of the warp is a block of 32*K floats, lane l owns the K
// consecutive floats at l*V of every V-wide chunk (V = min(K, 4)), so a
// register read or write is one conflict-free 64/128-bit LDS/STS per chunk
// and the register index is just an address offset -- no branches, no
// select chains.  The opcode is the only dispatch: one jump table
// (CheapOps, 8 entries) for the single-instruction ops, a C++ switch for
// DIV and the unary ops.  No lane reads another lane's slots, so no
// barrier is needed.
template <int K>
struct SmemRegs {
    static constexpr int V = K < 4 ? K : 4;     // floats per vector access
    static constexpr int kStride = 32 * K;       // floats per register per warp
    static __device__ __forceinline__ void load(const float* p, float (&v)[K]) {
#pragma unroll
        for (int q = 0; q < K / V; ++q) {
            if constexpr (V == 4) {
                const float4 x = *reinterpret_cast<const float4*>(p + q * 32 * V);
                v[q * 4] = x.x; v[q * 4 + 1] = x.y; v[q * 4 + 2] = x.z; v[q * 4 + 3] = x.w;
            } else if constexpr (V == 2) {
                const float2 x = *reinterpret_cast<const float2*>(p + q * 32 * V);
                v[q * 2] = x.x; v[q * 2 + 1] = x.y;
            } else {
                v[q] = p[q * 32];
            }
        }
    }
    static __device__ __forceinline__ void store(float* p, const float (&v)[K]) {
#pragma unroll
        for (int q = 0; q < K / V; ++q) {
            if constexpr (V == 4) {
                *reinterpret_cast<float4*>(p + q * 32 * V) = make_float4(v[q * 4], v[q * 4 + 1], v[q * 4 + 2],
                                                                         v[q * 4 + 3]);
            } else if constexpr (V == 2) {
                *reinterpret_cast<float2*>(p + q * 32 * V) = make_float2(v[q * 2], v[q * 2 + 1]);
            } else {
                p[q * 32] = v[q];
            }
        }
    }
};

template <int K, int PROFILE>
__device__ __forceinline__ void slow_op(uint32_t op, const float (&a)[K], const float (&b)[K], float (&t)[K]) {
    switch (op) {
        case kDiv:
#pragma unroll
            for (int k = 0; k < K; ++k) t[k] = (b[k] != 0.0f) ? __fdiv_rn(a[k], b[k]) : 1.0f;
            break;
        case kSin:
            galop_trig_k<K>(b, t, 0u);
            break;
        case kCos:
            galop_trig_k<K>(b, t, 1u);
            break;
        case kOp6:
#pragma unroll
            for (int k = 0; k < K; ++k) t[k] = apply_op<PROFILE>(kOp6, a[k], b[k]);
            break;
        default:
#pragma unroll
            for (int k = 0; k < K; ++k) t[k] = apply_op<PROFILE>(kOp7, a[k], b[k]);
            break;
    }
}

// 64 registers per thread (4 blocks of 256 threads per SM) hold every
// instantiation without spills; residency is then bounded by shared memory.
template <int NR, int K, int PROFILE, int REDUCE, int MODE>
__global__ void __launch_bounds__(256, 4)
interp_smem_kernel(InterpArgs args) {
    // Shared memory: [constant pool: NR registers x 32 lanes x K][warp 0
    // registers][warp 1 registers]...  The pool is written once per block
    // with every value in every lane slot, so "src2 = constant i" is just a
    // load of pool register i: operand fetch has no branch.
    extern __shared__ float4 galop_smem4[];
    using SR = SmemRegs<K>;
    constexpr int V = SR::V;
    constexpr int RS = SR::kStride;
    const int lane = threadIdx.x & 31;
    float* pool = reinterpret_cast<float*>(galop_smem4) + lane * V;
    float* regs = reinterpret_cast<float*>(galop_smem4) + NR * RS + (threadIdx.x >> 5) * NR * RS + lane * V;
    for (int i = threadIdx.x; i < NR * RS; i += blockDim.x)
        reinterpret_cast<float*>(galop_smem4)[i] = args.consts.c[i / RS];
    __syncthreads();
    const bool batched = args.pops != nullptr;
    const bool plain = args.plain != 0;
    const int64_t total_items = batched ? args.n_items : args.n_programs * (int64_t)args.n_chunks;
    constexpr int kPass = 32 * K;

    for (int round = 0;; ++round) {
        unsigned long long item = 0;
        if (plain) {
            if (round > 0) break;
            item = (unsigned long long)blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5);
        } else {
            if (lane == 0) item = atomicAdd(args.counter, 1ull);
            item = __shfl_sync(0xffffffffu, item, 0);
        }
        if ((int64_t)item >= total_items) break;

        // Resolve the work item: program, case range, dataset, output slot.
        int64_t prog, cbeg, cend, N, Np, out_index, partial_index = -1;
        int chunk, num_inputs;
        const float* __restrict__ Xd;
        const float* __restrict__ yd;
        float* out_fitness;
        double* out_sse;
        Objective obj;
        if (batched) {
            const unsigned long long it = args.items[item];
            prog = (int64_t)(it >> 20);
            chunk = (int)(it & 0xFFFFFull);
            const PopDesc* d = args.pops + args.prog_pop[prog];
            Xd = d->X;
            yd = d->y;
            N = d->N;
            Np = d->Np;
            num_inputs = d->num_inputs;
            cbeg = (int64_t)chunk * d->chunk_cases;
            cend = cbeg + d->chunk_cases;
            out_fitness = d->fitness;
            out_sse = d->sse;
            obj = d->obj;
            out_index = prog - d->prog_base;
            if (d->n_chunks > 1) partial_index = (int64_t)item;
        } else {
            const int64_t slot = (int64_t)item / args.n_chunks;
            chunk = (int)((int64_t)item % args.n_chunks);
            prog = args.order ? (int64_t)args.order[slot] : slot;
            Xd = args.X;
            yd = args.y;
            N = args.N;
            Np = args.Np;
            num_inputs = args.num_inputs;
            cbeg = (int64_t)chunk * args.chunk_cases;
            cend = cbeg + args.chunk_cases;
            out_fitness = args.fitness;
            out_sse = args.sse;
            obj = args.obj;
            out_index = prog;
            if (args.n_chunks > 1) partial_index = prog * args.n_chunks + chunk;
        }
        if (cend > N) cend = N;
        const int64_t p0 = args.eff_off[prog];
        const int64_t L = args.eff_off[prog + 1] - p0;
        const uint32_t* __restrict__ pw = args.uops + p0;

        float ks = 0.0f, kc = 0.0f;
        double big = 0.0;
        double acc = 0.0;

        for (int64_t base = cbeg; base < cend; base += kPass) {
            // Case c of this lane: base + (q*32 + lane)*V + e for chunk q,
            // element e -- the same layout as the registers, so the inputs
            // are copied with the same vector width.
            const int64_t c0 = base + (int64_t)lane * V;
#pragma unroll
            for (int f = 0; f < NR; ++f) {
                float v[K];
                if (f < num_inputs) {
#pragma unroll
                    for (int q = 0; q < K / V; ++q) {
                        float w[V];
                        load_cases<V>(Xd + (int64_t)f * Np + c0 + q * 32 * V, w);
#pragma unroll
                        for (int e = 0; e < V; ++e) v[q * V + e] = w[e];
                    }
                } else {
#pragma unroll
                    for (int k = 0; k < K; ++k) v[k] = 0.0f;
                }
                SR::store(regs + f * RS, v);
                if constexpr (MODE == kModeTrace) {
#pragma unroll
                    for (int q = 0; q < K / V; ++q)
#pragma unroll
                        for (int e = 0; e < V; ++e)
                            args.trace[(int64_t)f * kPass + (q * 32 + lane) * V + e] = v[q * V + e];
                }
            }

            for (int64_t wb = 0; wb < L; wb += 32) {
                const uint32_t win = (wb + lane < L) ? __ldg(pw + wb + lane) : 0u;
                const int n = (L - wb < 32) ? (int)(L - wb) : 32;
                for (int j = 0; j < n; ++j) {
                    const uint32_t u = __shfl_sync(0xffffffffu, win, j);
                    const uint32_t op = uop_op(u);
                    float a[K], b[K], t[K];
                    // src1 is loaded for unary ops too (ignored): no branch.
                    SR::load(regs + uop_src1(u) * RS, a);
                    SR::load((uop_is_const(u) ? pool : regs) + uop_src2(u) * RS, b);
                    if ((u & 0x40u) == 0 && op != kDiv) CheapOps<K, PROFILE>::cheap(op, a, b, t);
                    else slow_op<K, PROFILE>(op, a, b, t);
                    SR::store(regs + uop_dest(u) * RS, t);
                    if constexpr (MODE == kModeTrace) {
                        const int64_t row = (wb + j + 1) * NR;
#pragma unroll
                        for (int r2 = 0; r2 < NR; ++r2) {
                            float v[K];
                            SR::load(regs + r2 * RS, v);
#pragma unroll
                            for (int q = 0; q < K / V; ++q)
#pragma unroll
                                for (int e = 0; e < V; ++e)
                                    args.trace[(row + r2) * kPass + (q * 32 + lane) * V + e] = v[q * V + e];
                        }
                    }
                }
            }

            float o[K];
            SR::load(regs + args.output_reg * RS, o);
            // case index of element k: base + (q*32 + lane)*V + e, k = q*V + e
            if constexpr (MODE == kModeOutputs) {
#pragma unroll
                for (int q = 0; q < K / V; ++q)
#pragma unroll
                    for (int e = 0; e < V; ++e) {
                        const int64_t c = base + (int64_t)(q * 32 + lane) * V + e;
                        if (c < cend) args.outputs[prog * N + c] = o[q * V + e];
                    }
            } else if constexpr (MODE == kModeFitness) {
                float t[K];
#pragma unroll
                for (int q = 0; q < K / V; ++q) {
                    float w[V];
                    load_cases<V>(yd + c0 + q * 32 * V, w);
#pragma unroll
                    for (int e = 0; e < V; ++e) t[q * V + e] = w[e];
                }
                if constexpr (REDUCE == kReduceKahan32) {
#pragma unroll
                    for (int k = 0; k < K; ++k) {
                        const int64_t c = base + (int64_t)((k / V) * 32 + lane) * V + (k % V);
                        const float e = __fsub_rn(o[k], t[k]);
                        const bool valid = c < cend;
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
                        const int64_t c = base + (int64_t)((k / V) * 32 + lane) * V + (k % V);
                        const double e = (double)o[k] - (double)t[k];
                        if (c < cend) acc = __dadd_rn(acc, __dmul_rn(e, e));
                    }
                } else {
                    // Strict case order: chunk q, lane j, element e.
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
                                if (base + (int64_t)(q * 32 + j) * V + e < cend) acc = __dadd_rn(acc, v);
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
                if (partial_index < 0) {
                    out_fitness[out_index] = fitness_of(sse, N, obj);
                    if (out_sse) out_sse[out_index] = sse;
                } else {
                    args.partial[partial_index] = sse;
                }
            }
        }
        if constexpr (MODE == kModeTrace) break;
    }
}

}  // namespace galop
