// interp_wide.cuh -- the wide-micro-op interpreter (dispatch 3).
//
// Same work decomposition as the shared-memory interpreter of interp.cuh
// (one warp per program or case chunk, K cases per lane, the lane's
// register file in shared memory), but every instruction is a 16-byte
// micro-op whose operand fields are already byte offsets into the register
// file (encode_wide in isa.cuh), and a constant operand carries its value.
// The register file has NSLOT slots per lane, not the ISA's NR registers:
// the folding pass renames each program's values into as few slots as it
// keeps live at once (fold.cuh), and the runtime runs the programs that fit
// in 8 slots on the 8-slot instance, which needs half the shared memory per
// warp.  Runs of binary instructions and of SIN/COS of a register execute
// inside one PTX loop (WideLoop); per instruction the warp does:
//   one broadcast 16-byte shared load of the micro-op (32-instruction
//     windows are staged in shared memory with cp.async, the next window
//     copied while the current one runs; the next micro-op is prefetched
//     into a second register set, the loop body existing twice),
//   a sign test (other unary ops and the window end leave the loop),
//   one jump table (arms for the 8 ops x register/constant src2, each with
//     entry points that skip what the micro-op's flags make unnecessary)
//     whose arm stores the previous result if the flags ask for it, loads
//     src1 unless it is the previous result, loads src2 (register arms),
//     and computes into the result registers, which are also the src1
//     registers (DIV with its own fast division, IEEE division only for a
//     warp with an operand out of that path's range; SIN/COS with
//     trig.cuh's Cody-Waite path, their operand taken as src1;
//     gen_dispatch.py).
// The result registers a[K] and the address of the register they belong to
// live across the whole pass: the unary ops the loop leaves to C++ (EXP/LOG
// of the BJ profile from the CUDA math library, a constant's SIN/COS when
// folding is off, and SIN/COS for a warp with an argument that needs
// trig.cuh's Payne-Hanek path) read and write them too.  The last result
// is never stored: the output is taken from it when the last instruction
// wrote the output register.
// Each pass initialises only the values the program reads before writing
// them (args.livein: registers, slots used, output slot).  The folding pass
// sets the flags and these words (isa.cuh, fold.cuh).
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

// Shared memory per warp: NSLOT register slots x stride, then two 33-entry
// micro-op stages (32 instructions + a permanent end marker each).
constexpr uint32_t kWideStageBytes = 33u * 16u;

template <int NSLOT, int K>
__host__ __device__ constexpr uint32_t wide_warp_bytes() {
    return (uint32_t)NSLOT * 128u * K + 2u * kWideStageBytes;
}

inline size_t wide_smem_bytes(int nslot, int k, int warps) {
    return (size_t)warps * ((size_t)nslot * 128u * (size_t)k + 2u * kWideStageBytes);
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

__device__ __forceinline__ WideItem resolve_item(const InterpArgs& args, unsigned long long item,
                                                int64_t slot_lo) {
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
        const int64_t slot = slot_lo + (int64_t)item / args.n_chunks;
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
// (BJ); sine and cosine from trig.cuh, EXP/LOG from the CUDA math library.
template <int K, int PROFILE>
__device__ __forceinline__ void unary_op(uint32_t op, const float (&b)[K], float (&t)[K]) {
    if constexpr (PROFILE == kProfileRef) {
        if (op == kSin) galop_trig_k<K>(b, t, 0u);
        else galop_trig_k<K>(b, t, 1u);
    } else {
        slow_op<K, PROFILE>(op, b, b, t);
    }
}

// Launch bounds: at most 256 threads per block and at least kMinBlocks
// blocks of 256 threads per SM, which caps the registers per thread.  The
// 8-slot instance needs 5,152 bytes of shared memory per warp at K = 4, so
// 40 warps fit on an SM; 5 blocks of 8 warps cap it at 48 registers per
// thread, which those 40 warps need (65,536 / (40 x 32) = 51).  At K = 8 it
// needs 9,248 bytes per warp (24 warps), and the 16-slot instance fits at
// most 24 warps by shared memory at any K, which 3 blocks' cap of 85
// registers per thread allows.
template <int NSLOT, int K>
struct WideBounds {
    static constexpr int kMaxThreads = 256;
    static constexpr int kMinBlocks = (NSLOT <= 8 && K <= 4) ? 5 : 3;
};

// Asynchronous copy of one 16-byte micro-op into shared memory (cached in
// L2 only), and the waits.
__device__ __forceinline__ void cp_async16(uint32_t dst, const void* src) {
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" :: "r"(dst), "l"(src) : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
__device__ __forceinline__ void cp_async_wait_all() { asm volatile("cp.async.wait_all;" ::: "memory"); }

// Stage window w of a program (micro-ops [32w, min(32w + 32, L))) into the
// stage at st: lane l copies micro-op 32w + l asynchronously; in a partial
// window the first slot past the program gets the end marker (a full
// window ends at the stage's permanent marker, slot 32).
__device__ __forceinline__ void stage_window(uint32_t st, const uint4* __restrict__ pw, int64_t L, int64_t w,
                                             int lane) {
    const int64_t j = w * 32 + lane;
    if (j < L) cp_async16(st + (uint32_t)lane * 16u, pw + j);
    else if (j == L) sts_u4(st + (uint32_t)lane * 16u, make_uint4(0u, 0u, 0u, kWideEnd));
    cp_async_commit();
}

// NSLOT: register-file slots per warp.  The folding pass renames each
// program's values into slots (rename_slots in fold.cuh); a program whose
// values need at most NSLOT slots runs here.  Trace mode interprets the raw
// program in the ISA's own register layout (NSLOT = NR).
//
// Micro-op staging: each warp has two 33-entry stages.  A program of at
// most two 32-instruction windows is staged once per work item and stays in
// shared memory for all its passes over the cases; a longer one is streamed
// window by window, the next window (the first one again at the end of a
// pass) copied with cp.async into the other stage while the current one
// runs.
template <int NSLOT, int K, int PROFILE, int REDUCE, int MODE>
__global__ void __launch_bounds__(WideBounds<NSLOT, K>::kMaxThreads, WideBounds<NSLOT, K>::kMinBlocks)
interp_wide_kernel(InterpArgs args) {
    extern __shared__ float4 galop_smem4[];
    using WR = WideRegs<K>;
    constexpr int V = WR::V;
    constexpr uint32_t S = WR::kStride;
    constexpr int kPass = 32 * K;
    const int lane = threadIdx.x & 31;
    const uint32_t warp_base = (uint32_t)__cvta_generic_to_shared(galop_smem4) +
                               (threadIdx.x >> 5) * wide_warp_bytes<NSLOT, K>();
    const uint32_t base = warp_base + (uint32_t)lane * V * 4u;   // this lane's slot 0
    const uint32_t stage0 = warp_base + NSLOT * S;
    const uint32_t stage1 = stage0 + kWideStageBytes;
    const uint4 kEnd4 = make_uint4(0u, 0u, 0u, kWideEnd);
    if (lane == 0) {
        sts_u4(stage0 + 32u * 16u, kEnd4);
        sts_u4(stage1 + 32u * 16u, kEnd4);
    }
    __syncwarp();

    const bool plain = args.plain != 0;
    const int64_t n_work = args.n_skipped ? args.n_programs - (int64_t)*args.n_skipped : args.n_programs;
    // the slots of the order this launch covers (one register-file class)
    int64_t slot_lo = 0, slot_hi = n_work;
    if (args.class_split != nullptr && args.pops == nullptr) {
        const int64_t n0 = (int64_t)*args.class_split;
        if (args.class_part == 0) slot_hi = n0 < n_work ? n0 : n_work;
        else slot_lo = n0 < n_work ? n0 : n_work;
    }
    int64_t total_items = args.pops != nullptr ? (args.n_items_dev ? *args.n_items_dev : args.n_items)
                        : plain ? args.n_programs : (slot_hi - slot_lo) * (int64_t)args.n_chunks;
    // batched items: the first class's items come first in the item list,
    // the split is the first item of the second class
    int64_t item_lo = 0;
    if (args.pops != nullptr && args.class_split != nullptr) {
        const int64_t b = (int64_t)*args.class_split < total_items ? (int64_t)*args.class_split : total_items;
        if (args.class_part == 0) total_items = b;
        else item_lo = b;
    }
    const uint4* __restrict__ uops4 = reinterpret_cast<const uint4*>(args.uops);

    for (int round = 0;; ++round) {
        unsigned long long item = 0;
        if (plain) {
            if (round > 0) break;
            item = (unsigned long long)blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5);
        } else {
            if (lane == 0) item = (unsigned long long)item_lo + atomicAdd(args.counter, 1ull);
            item = __shfl_sync(0xffffffffu, item, 0);
        }
        if ((int64_t)item >= total_items) break;
        const WideItem w = resolve_item(args, item, slot_lo);
        if (plain && args.interp_len != nullptr && args.interp_len[w.prog] < 0) continue;   // a dedup copy
        // folded programs are packed against the end of their slot (fold.cuh)
        const int64_t L = args.interp_len ? (int64_t)args.interp_len[w.prog]
                                          : args.eff_off[w.prog + 1] - args.eff_off[w.prog];
        const int64_t p0 = args.eff_off[w.prog + 1] - L;
        const uint4* __restrict__ pw = uops4 + p0;
        // live-in registers (loaded into slots 0..m-1 in register order) and
        // the output value's slot; a trace uses the ISA's layout
        const bool arch = MODE == kModeTrace || args.livein == nullptr;
        const uint32_t lv = arch ? (1u << NSLOT) - 1u : args.livein[w.prog];
        const uint32_t live_regs = arch ? lv : livein_regs(lv);
        const uint32_t out_addr = base + (arch ? (uint32_t)args.output_reg : livein_out_slot(lv)) * S;
        const int64_t nwin = (L + 31) / 32;
        const bool resident = nwin <= 2;
        if (resident) {
            for (int64_t wi = 0; wi < nwin; ++wi) stage_window(wi == 0 ? stage0 : stage1, pw, L, wi, lane);
        } else {
            stage_window(stage0, pw, L, 0, lane);
        }
        int64_t gw = 0;   // windows of this item streamed so far (stage = gw & 1)

        float ks = 0.0f, kc = 0.0f;
        double big = 0.0;
        double acc = 0.0;

        for (int64_t cb = w.cbeg; cb < w.cend; cb += kPass) {
            // Case of element q*V+e of this lane: cb + (q*32 + lane)*V + e.
            const int64_t c0 = cb + (int64_t)lane * V;
            // Only the values the program reads before writing them are
            // initialised (all registers for a register trace).
            uint32_t slot_addr = base;
            for (uint32_t m = live_regs; m != 0u; m &= m - 1u) {
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
                WR::store(slot_addr, v);
                slot_addr += S;
            }
            if constexpr (MODE == kModeTrace) wide_trace<NSLOT, K>(args.trace, 0, base, lane);

            float a[K];       // result of the last instruction executed
            uint32_t pt = 0;  // its slot's address
#pragma unroll
            for (int k = 0; k < K; ++k) a[k] = 0.0f;
            for (int64_t wi = 0; wi < nwin; ++wi) {
                cp_async_wait_all();
                __syncwarp();   // the window has landed, and every lane is done with the other stage
                uint32_t stage;
                if (resident) {
                    stage = wi == 0 ? stage0 : stage1;
                } else {
                    stage = (gw & 1) ? stage1 : stage0;
                    const bool last = wi + 1 == nwin;
                    if (!last || cb + kPass < w.cend)
                        stage_window((gw & 1) ? stage0 : stage1, pw, L, last ? 0 : wi + 1, lane);
                    ++gw;
                }
                const int64_t wb = wi * 32;
                uint32_t sp = stage;
                if constexpr (MODE == kModeTrace) {
                    // One instruction at a time, the register file dumped after
                    // each; every result is stored, the flags do not apply.
                    for (;;) {
                        uint4 u = lds_u4(sp);
                        while ((int32_t)u.w >= 0) {
                            WideOps<K, PROFILE>::run(u.w & 15u, base + u.x, base + u.y, base + u.z, u.y);
                            wide_trace<NSLOT, K>(args.trace, wb + (sp - stage) / 16u + 1, base, lane);
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
                        wide_trace<NSLOT, K>(args.trace, wb + (sp - stage) / 16u + 1, base, lane);
                        sp += 16u;
                    }
                } else {
                    uint4 cur = lds_u4(sp);
                    for (;;) {
                        // Every binary instruction and SIN/COS up to the next other
                        // unary op, a SIN/COS with an argument for trig.cuh's slow
                        // path, or the end marker; u is the micro-op that stopped
                        // the loop.
                        uint4 u;
                        WideLoop<K, PROFILE>::run(sp, a, pt, base, cur, u);
                        if (u.w == kWideEnd) break;
                        const uint4 next = lds_u4(sp + 16u);   // the end marker at most
                        float b[K];
                        if (!(u.w & kWideSpecial)) {
                            // a SIN/COS the loop left for trig.cuh's slow path:
                            // the previous result is stored, a holds the operand
#pragma unroll
                            for (int k = 0; k < K; ++k) b[k] = a[k];
                        } else {
                            // unary op on src2 (register, constant or the previous result)
                            if (u.w & kWideStorePrev) WR::store(pt, a);
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
                        }
                        unary_op<K, PROFILE>(u.w & 7u, b, a);
                        pt = base + u.z;
                        sp += 16u;
                        cur = next;
                    }
                }
            }
            // The output: the last result when the last instruction wrote the
            // output's slot (never stored), else the register file.
            float o[K];
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
                    float ev[K];
                    bool small = true;
#pragma unroll
                    for (int k = 0; k < K; ++k) {
                        ev[k] = __fsub_rn(o[k], t[k]);
                        small = small && fabsf(ev[k]) <= kKahanMaxError;
                    }
                    if (cb + kPass <= w.cend && small) {
                        // every case of the pass counts and no square can
                        // overflow: the lane's K squares summed pairwise
                        // (each passes through at most four roundings at
                        // K = 8), then one compensated step into the lane's sum
                        float s[K / 2 > 0 ? K / 2 : 1];
                        if constexpr (K == 1) {
                            s[0] = __fmul_rn(ev[0], ev[0]);
                        } else {
#pragma unroll
                            for (int h = 0; h < K / 2; ++h)
                                s[h] = __fmaf_rn(ev[2 * h + 1], ev[2 * h + 1], __fmul_rn(ev[2 * h], ev[2 * h]));
#pragma unroll
                            for (int h = K / 4; h >= 1; h /= 2)
#pragma unroll
                                for (int j = 0; j < h; ++j) s[j] = __fadd_rn(s[j], s[j + h]);
                        }
                        const float yk = __fsub_rn(s[0], kc);
                        const float tt = __fadd_rn(ks, yk);
                        kc = __fsub_rn(__fsub_rn(tt, ks), yk);
                        ks = tt;
                    } else {
#pragma unroll
                        for (int k = 0; k < K; ++k) {
                            const int64_t c = cb + (int64_t)((k / V) * 32 + lane) * V + (k % V);
                            const float e = ev[k];
                            const bool valid = c < w.cend;
                            const bool huge = !(fabsf(e) <= kKahanMaxError);
                            const float qv = (valid && !huge) ? __fmul_rn(e, e) : 0.0f;
                            if (valid && huge) big = __dadd_rn(big, __dmul_rn((double)e, (double)e));
                            const float yk = __fsub_rn(qv, kc);
                            const float tt = __fadd_rn(ks, yk);
                            kc = __fsub_rn(__fsub_rn(tt, ks), yk);
                            ks = tt;
                        }
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
        cp_async_wait_all();   // nothing of this item may still be landing in a stage
        __syncwarp();

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
