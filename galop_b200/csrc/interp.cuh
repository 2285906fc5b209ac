// interp.cuh -- the warp-per-individual LGP interpreter for sm_100a.
//
// One warp evaluates one program (or one case chunk of it); lane l of the warp
// owns K consecutive fitness cases of every 32*K-case pass and keeps their
// NR-entry register files in real registers (float r[NR][K]).  Register
// indices in an instruction are warp-uniform, so "read register s1" is a
// switch whose every arm moves K values with static indices: no local-memory
// register array (the reference's program_partial_sse keeps reg[] in local
// memory, src/EvaluatorCuda.cu:127, :151-153).
//
// Instruction stream: 32 micro-ops at a time are read with one coalesced load
// (lane j holds word j) and broadcast with a shuffle.
//
// Fitness cases: feature-major (SoA) arrays padded to a multiple of 1024
// cases; a lane reads its K consecutive cases of a feature with one 8/16-byte
// vector load, so a warp reads 32*K contiguous floats per feature.
//
// Semantics per case follow src/Interpreter.cpp:36-59: r0..k-1 = inputs, the
// rest 0, execute every instruction in order, output r[OUTPUT_REG].  Fitness
// follows src/Evaluator.cpp:11-45 and :88-91 (see galop_reduce in the header
// for the three accumulation modes).
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
};

#define GALOP_CASES16(X) X(0) X(1) X(2) X(3) X(4) X(5) X(6) X(7) \
                         X(8) X(9) X(10) X(11) X(12) X(13) X(14) X(15)

template <int NR, int K>
__device__ __forceinline__ void read_reg(const float (&r)[NR][K], uint32_t idx, float (&out)[K]) {
    switch (idx) {
#define GALOP_RD(j)                                                        \
        case j:                                                            \
            if constexpr (j < NR) {                                        \
                _Pragma("unroll") for (int k = 0; k < K; ++k) out[k] = r[j][k]; \
            }                                                              \
            break;
        GALOP_CASES16(GALOP_RD)
#undef GALOP_RD
        default: break;
    }
}

template <int NR, int K>
__device__ __forceinline__ void write_reg(float (&r)[NR][K], uint32_t idx, const float (&v)[K]) {
    switch (idx) {
#define GALOP_WR(j)                                                        \
        case j:                                                            \
            if constexpr (j < NR) {                                        \
                _Pragma("unroll") for (int k = 0; k < K; ++k) r[j][k] = v[k]; \
            }                                                              \
            break;
        GALOP_CASES16(GALOP_WR)
#undef GALOP_WR
        default: break;
    }
}

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

// One instruction over the lane's K cases.
template <int NR, int K, int PROFILE>
__device__ __forceinline__ void step(float (&r)[NR][K], uint32_t u, const ConstPool& cp) {
    const uint32_t op = uop_op(u);
    float a[K], b[K], t[K];
    read_reg<NR, K>(r, uop_src1(u), a);
    if (uop_is_const(u)) {
        const float c = cp.c[uop_src2(u)];
#pragma unroll
        for (int k = 0; k < K; ++k) b[k] = c;
    } else {
        read_reg<NR, K>(r, uop_src2(u), b);
    }
    switch (op) {
        case kAdd:
#pragma unroll
            for (int k = 0; k < K; ++k) t[k] = __fadd_rn(a[k], b[k]);
            break;
        case kSub:
#pragma unroll
            for (int k = 0; k < K; ++k) t[k] = __fsub_rn(a[k], b[k]);
            break;
        case kMul:
#pragma unroll
            for (int k = 0; k < K; ++k) t[k] = __fmul_rn(a[k], b[k]);
            break;
        case kDiv:
#pragma unroll
            for (int k = 0; k < K; ++k) t[k] = (b[k] != 0.0f) ? __fdiv_rn(a[k], b[k]) : 1.0f;
            break;
        case kSin:
#pragma unroll
            for (int k = 0; k < K; ++k) t[k] = sinf(b[k]);
            break;
        case kCos:
#pragma unroll
            for (int k = 0; k < K; ++k) t[k] = cosf(b[k]);
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
    write_reg<NR, K>(r, uop_dest(u), t);
}

// ---- dispatch strategy 1: jump tables (default) --------------------------------
//
// The C++ switches above are compiled into predicated select chains: every
// register read or write costs NR*K instructions.  Strategy 1 uses the PTX
// brx.idx helpers of dispatch_gen.cuh instead: one indirect branch per
// access, then K moves.  Single-instruction binary ops (ADD, SUB, MUL, and
// LT, GT in the REF profile) are fused with their destination: one branch on
// op*NR+dest lands on K arithmetic instructions that write r[dest] directly,
// with a constant src2 kept as one scalar.  DIV and the unary ops gather,
// compute in C++ and scatter: their own cost dwarfs the moves.
template <int NR, int K, int PROFILE>
__device__ __forceinline__ void step_brx(float (&r)[NR][K], uint32_t u, const ConstPool& cp) {
    using B = Brx<NR, K, PROFILE>;
    const uint32_t op = uop_op(u);
    const uint32_t dest = uop_dest(u);
    const bool konst = uop_is_const(u);
    const uint32_t s2 = uop_src2(u);
    if (u & 0x40u) {                       // unary: reads src2 only
        float b[K], t[K];
        if (konst) {
            const float c = cp.c[s2];
#pragma unroll
            for (int k = 0; k < K; ++k) b[k] = c;
        } else {
            B::gather(r, s2, b);
        }
        switch (op) {
            case kSin:
#pragma unroll
                for (int k = 0; k < K; ++k) t[k] = sinf(b[k]);
                break;
            case kCos:
#pragma unroll
                for (int k = 0; k < K; ++k) t[k] = cosf(b[k]);
                break;
            case kOp6:
#pragma unroll
                for (int k = 0; k < K; ++k) t[k] = apply_op<PROFILE>(kOp6, 0.0f, b[k]);
                break;
            default:
#pragma unroll
                for (int k = 0; k < K; ++k) t[k] = apply_op<PROFILE>(kOp7, 0.0f, b[k]);
                break;
        }
        B::scatter(r, dest, t);
        return;
    }
    float a[K];
    B::gather(r, uop_src1(u), a);
    if (op == kDiv) {
        float t[K];
        if (konst) {
            const float c = cp.c[s2];
#pragma unroll
            for (int k = 0; k < K; ++k) t[k] = (c != 0.0f) ? __fdiv_rn(a[k], c) : 1.0f;
        } else {
            float b[K];
            B::gather(r, s2, b);
#pragma unroll
            for (int k = 0; k < K; ++k) t[k] = (b[k] != 0.0f) ? __fdiv_rn(a[k], b[k]) : 1.0f;
        }
        B::scatter(r, dest, t);
        return;
    }
    const uint32_t od = op * NR + dest;
    if (konst) {
        B::od_sca(r, od, a, cp.c[s2]);
    } else {
        float b[K];
        B::gather(r, s2, b);
        B::od_vec(r, od, a, b);
    }
}

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

// src/Evaluator.cpp:44 then :88-91.

template <int NR, int K, int PROFILE, int REDUCE, int MODE, int DISPATCH>
__global__ void __launch_bounds__(256, 1)
interp_kernel(InterpArgs args) {
    const int lane = threadIdx.x & 31;
    const int64_t total_items = args.n_programs * (int64_t)args.n_chunks;
    constexpr int kPass = 32 * K;

    for (;;) {
        unsigned long long item = 0;
        if (lane == 0) item = atomicAdd(args.counter, 1ull);
        item = __shfl_sync(0xffffffffu, item, 0);
        if ((int64_t)item >= total_items) break;

        const int64_t slot = (int64_t)item / args.n_chunks;
        const int chunk = (int)((int64_t)item % args.n_chunks);
        const int64_t prog = args.order ? (int64_t)args.order[slot] : slot;
        const int64_t p0 = args.eff_off[prog];
        const int64_t L = args.eff_off[prog + 1] - p0;
        const uint32_t* __restrict__ pw = args.uops + p0;

        const int64_t cbeg = (int64_t)chunk * args.chunk_cases;
        int64_t cend = cbeg + args.chunk_cases;
        if (cend > args.N) cend = args.N;

        float ks = 0.0f, kc = 0.0f;   // Kahan sum / compensation (KAHAN32)
        double big = 0.0;             // KAHAN32: squares of errors beyond kKahanMaxError
        double acc = 0.0;             // FP64 / ORDERED accumulator

        for (int64_t base = cbeg; base < cend; base += kPass) {
            const int64_t c0 = base + (int64_t)lane * K;
            float r[NR][K];
#pragma unroll
            for (int f = 0; f < NR; ++f) {
                if (f < args.num_inputs) {
                    load_cases<K>(args.X + (int64_t)f * args.Np + c0, r[f]);
                } else {
#pragma unroll
                    for (int k = 0; k < K; ++k) r[f][k] = 0.0f;
                }
            }
            if constexpr (MODE == kModeTrace) {
#pragma unroll
                for (int j = 0; j < NR; ++j)
#pragma unroll
                    for (int k = 0; k < K; ++k)
                        args.trace[(int64_t)j * kPass + lane * K + k] = r[j][k];
            }

            for (int64_t wb = 0; wb < L; wb += 32) {
                const uint32_t win = (wb + lane < L) ? __ldg(pw + wb + lane) : 0u;
                const int n = (L - wb < 32) ? (int)(L - wb) : 32;
                for (int j = 0; j < n; ++j) {
                    const uint32_t u = __shfl_sync(0xffffffffu, win, j);
                    if constexpr (DISPATCH == 1) step_brx<NR, K, PROFILE>(r, u, args.consts);
                    else step<NR, K, PROFILE>(r, u, args.consts);
                    if constexpr (MODE == kModeTrace) {
                        const int64_t row = (wb + j + 1) * NR;
#pragma unroll
                        for (int q = 0; q < NR; ++q)
#pragma unroll
                            for (int k = 0; k < K; ++k)
                                args.trace[(row + q) * kPass + lane * K + k] = r[q][k];
                    }
                }
            }

            float o[K];
            if constexpr (DISPATCH >= 1) Brx<NR, K, PROFILE>::gather(r, (uint32_t)args.output_reg, o);
            else read_reg<NR, K>(r, (uint32_t)args.output_reg, o);

            if constexpr (MODE == kModeOutputs) {
#pragma unroll
                for (int k = 0; k < K; ++k)
                    if (c0 + k < cend) args.outputs[prog * args.N + c0 + k] = o[k];
            } else if constexpr (MODE == kModeFitness) {
                float t[K];
                load_cases<K>(args.y + c0, t);
                if constexpr (REDUCE == kReduceKahan32) {
#pragma unroll
                    for (int k = 0; k < K; ++k) {
                        const float e = __fsub_rn(o[k], t[k]);
                        const bool valid = c0 + k < cend;
                        const bool huge = !(fabsf(e) <= kKahanMaxError);
                        const float q = (valid && !huge) ? __fmul_rn(e, e) : 0.0f;
                        if (valid && huge) big = __dadd_rn(big, __dmul_rn((double)e, (double)e));
                        const float yk = __fsub_rn(q, kc);
                        const float tt = __fadd_rn(ks, yk);
                        kc = __fsub_rn(__fsub_rn(tt, ks), yk);
                        ks = tt;
                    }
                } else if constexpr (REDUCE == kReduceFp64) {
#pragma unroll
                    for (int k = 0; k < K; ++k) {
                        const double e = (double)o[k] - (double)t[k];
                        if (c0 + k < cend) acc = __dadd_rn(acc, __dmul_rn(e, e));
                    }
                } else {
                    // Strict case order: base+0, base+1, ... (lane-major, K per lane).
                    double q[K];
#pragma unroll
                    for (int k = 0; k < K; ++k) {
                        const double e = (double)o[k] - (double)t[k];
                        q[k] = __dmul_rn(e, e);
                    }
                    for (int j = 0; j < 32; ++j) {
#pragma unroll
                        for (int k = 0; k < K; ++k) {
                            const double v = __shfl_sync(0xffffffffu, q[k], j);
                            if (base + (int64_t)j * K + k < cend) acc = __dadd_rn(acc, v);
                        }
                    }
                }
            }
            if constexpr (MODE == kModeTrace) break;  // one pass
        }

        if constexpr (MODE == kModeFitness) {
            double sse;
            if constexpr (REDUCE == kReduceKahan32) {
                sse = warp_sum_f64((double)ks - (double)kc + big);
            } else if constexpr (REDUCE == kReduceFp64) {
                sse = warp_sum_f64(acc);
            } else {
                sse = acc;  // identical in every lane
            }
            if (lane == 0) {
                if (args.n_chunks == 1) {
                    args.fitness[prog] = fitness_of(sse, args.N, args.obj);
                    if (args.sse) args.sse[prog] = sse;
                } else {
                    args.partial[prog * args.n_chunks + chunk] = sse;
                }
            }
        }
        if constexpr (MODE == kModeTrace) break;
    }
}


// ---- dispatch strategy 2 (default): the LGP register file in shared memory -----
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
#pragma unroll
            for (int k = 0; k < K; ++k) t[k] = sinf(b[k]);
            break;
        case kCos:
#pragma unroll
            for (int k = 0; k < K; ++k) t[k] = cosf(b[k]);
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
    const int64_t total_items = batched ? args.n_items : args.n_programs * (int64_t)args.n_chunks;
    constexpr int kPass = 32 * K;

    for (;;) {
        unsigned long long item = 0;
        if (lane == 0) item = atomicAdd(args.counter, 1ull);
        item = __shfl_sync(0xffffffffu, item, 0);
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
