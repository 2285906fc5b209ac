// fold.cuh -- constant folding and dead-code removal over the wide
// micro-ops of each program, after the intron pass.
//
// A register holds the same value in every fitness case until an
// instruction writes it from a case-dependent value: registers at or above
// the dataset's input count start at 0 (src/Interpreter.cpp:41-47), constant
// operands are constants.  An instruction all of whose operands are such
// known values computes the same number for every case, so it is evaluated
// once here -- with the very operations the interpreter would use (apply_op:
// __fadd_rn, IEEE division, galop_sinf, ... on this device), hence the same bits --
// and becomes a broadcast micro-op (dest = that constant).  A second,
// backward liveness pass then drops instructions whose results no remaining
// instruction reads (broadcasts read nothing) and packs the survivors
// against the end of the program's slot: the interpreted micro-ops of
// program i are u[eff_off[i + 1] - interp_len[i], eff_off[i + 1]).
// Per-case outputs and fitness are unchanged; only case-independent work is
// done once instead of per case.
//
// Two rewrites make the survivors cheaper without changing any result:
//   - a known value read by an instruction that is not folded becomes that
//     instruction's constant operand: as src2 always (the constant arms
//     compute OP(a, c) with c the register's exact value), as src1 when the
//     op is ADD or MUL (IEEE sum and product are commutative) or LT/GT of
//     the REF profile (a < b is b > a, both false on NaN), by swapping the
//     operands; the broadcast that wrote the register then usually dies;
//   - on the final order (in the same backward pass), each operand that is
//     the previous instruction's destination is marked as forwarded
//     (kWideFwd1 / kWideFwd2), and a result is marked to reach the register
//     file (kWideStorePrev on the next instruction) only when something
//     other than the next instruction's forwarded operand reads it.
// With folding off (intron pass off) the kernel only marks forwarding:
// every stream the interpreter loop runs carries the flags.
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
    int fold;                    // 0: forwarding flags only (no folding, no dead-code removal)
    int rename;                  // 1: values renamed into register-file slots (rename_slots);
                                 // 0: the ISA's register layout (register traces)
};

// Operand swap that keeps the result bits: ADD, MUL, and LT <-> GT of REF.
__host__ __device__ __forceinline__ bool swaps(int profile, uint32_t op) {
    return op == kAdd || op == kMul || (profile == kProfileRef && (op == kOp6 || op == kOp7));
}

// Registers a micro-op reads (broadcasts none, unary ops only src2, a
// constant src2 none).
__host__ __device__ __forceinline__ uint32_t uop_reads(const uint4& w, uint32_t sh) {
    if ((w.w & ~kWideFlags) == kWideBcast) return 0u;
    uint32_t r = 0u;
    if (!(w.w & kWideSpecial)) r |= 1u << (w.x >> sh);
    if (!(w.w & 8u)) r |= 1u << (w.y >> sh);
    return r;
}

// fwd1 / fwd2 on micro-op w whose predecessor wrote the register at byte
// offset prev, swapping the operands of a binary op first when only src2
// is that register and the swap keeps the result bits.
__host__ __device__ __forceinline__ void set_fwd(uint4& w, uint32_t prev, int profile) {
    if (w.w == kWideBcast) return;
    const bool reg2 = !(w.w & 8u);
    if (w.w & kWideSpecial) {
        if (reg2 && w.y == prev) w.w |= kWideFwd2;
        return;
    }
    const uint32_t op = w.w & 7u;
    if (w.x != prev && reg2 && w.y == prev && swaps(profile, op)) {
        const uint32_t sop = op == kOp6 ? (uint32_t)kOp7 : op == kOp7 ? (uint32_t)kOp6 : op;
        const uint32_t x = w.x;
        w.x = w.y;
        w.y = x;
        w.w = (w.w & ~7u) | sop;
    }
    if (w.x == prev) w.w |= kWideFwd1;
}

// Whether the result of the instruction before nx (register d) must reach
// the register file: unless nx takes it forwarded, loads no copy of it, and
// nothing after nx reads it (live_after_next: registers live after nx).
__host__ __device__ __forceinline__ bool needs_store(const uint4& nx, uint32_t d, uint32_t live_after_next, uint32_t sh) {
    const uint32_t nd = nx.z >> sh;
    const bool fwd = (nx.w & (kWideFwd1 | kWideFwd2)) != 0;
    // a binary op loads src2 (never forwarded); src1 equal to d is forwarded
    const bool loads_d = !(nx.w & kWideSpecial) && !(nx.w & 8u) && (nx.y >> sh) == d &&
                         (nx.w & ~kWideFlags) != kWideBcast;
    const bool read_later = d != nd && ((live_after_next >> d) & 1u);
    return !(fwd && !loads_d && !read_later);
}

// Forwarding flags over a program u[0, n) in its final order (see the
// micro-op format in isa.cuh).  The interpreter loop keeps the last result
// in registers; an instruction takes it as src1 (binary ops, fwd1) or src2
// (unary ops, fwd2) when that operand is the previous destination, and a
// binary op whose src2 is the previous destination swaps its operands first
// where that keeps the result bits (swaps).  The previous result is written
// to the register file (store_prev on this instruction) unless this
// instruction is its only reader: it takes the value forwarded, loads no
// copy of it, and the value is not read after it (overwritten by it, or
// dead below it; the output register counts as read after the last
// instruction).  The first instruction carries no flag: every pass over the
// cases starts there with nothing pending.  The last result is never
// stored: the interpreter takes the output from it when the last
// instruction wrote the output register.
// Returns the registers the program reads before writing them (the
// output register counts as read after the last instruction): the only
// ones the interpreter must initialise before each pass over the cases.
__host__ __device__ __forceinline__ uint32_t mark_forwarding(uint4* __restrict__ u, int64_t n, uint32_t sh, int output_reg,
                                                    int profile) {
    for (int64_t j = 1; j < n; ++j) set_fwd(u[j], u[j - 1].z, profile);
    uint32_t live = 1u << output_reg;      // live after instruction j
    uint32_t live_after_next = 0u;
    for (int64_t j = n - 1; j >= 0; --j) {
        const uint4 w = u[j];
        const uint32_t d = w.z >> sh;
        if (j < n - 1 && needs_store(u[j + 1], d, live_after_next, sh)) u[j + 1].w |= kWideStorePrev;
        live_after_next = live;
        live = (live & ~(1u << d)) | uop_reads(w, sh);
    }
    return live;
}

// Folds one program in place (constants, dead code, packing, forwarding
// flags), returns its interpreted length and sets its live-in registers.
__host__ __device__ __forceinline__ int64_t fold_program(uint4* __restrict__ u, int64_t L, const FoldParams& fp,
                                                 int k_in, uint32_t& livein) {
    const uint32_t sh = fp.stride_shift;
    int64_t kept = 0;
    float vals[kMaxRegisters];
    uint32_t known = 0;
    for (int r = 0; r < fp.num_registers; ++r) {
        vals[r] = 0.0f;
        if (r >= k_in) known |= 1u << r;
    }
    // forward: evaluate what is known (micro-ops read four at a time, so
    // that several loads are in flight; each step writes only u[j])
    auto forward = [&](const uint4 w, const int64_t j) {
        const uint32_t op = w.w & 7u;
        const bool is_const = (w.w & 8u) != 0;
        const bool unary = (w.w & kWideSpecial) != 0;
        const uint32_t s1 = w.x >> sh, s2 = w.y >> sh, d = w.z >> sh;
        const bool a_known = unary || ((known >> s1) & 1u);
        const bool b_known = is_const || ((known >> s2) & 1u);
        const float a = a_known && !unary ? vals[s1] : 0.0f;
        const float b = is_const ? galop_float(w.y) : (b_known ? vals[s2] : 0.0f);
        // Results known whatever the other operand: protected division by a
        // zero (src/ISA.h:224: 1.0 for every dividend, NaN included), and
        // LT/GT of the REF profile with a NaN operand (0.0: ordered
        // comparisons with NaN are false).
        const bool div0 = !unary && op == kDiv && b_known && b == 0.0f;
        const bool cmp_nan = fp.profile == kProfileRef && (op == kOp6 || op == kOp7) &&
                             ((a_known && a != a) || (b_known && b != b));
        if ((a_known && b_known) || div0 || cmp_nan) {
            const float v = div0 ? 1.0f
                          : cmp_nan ? 0.0f
                          : fp.profile == kProfileBj ? apply_op<kProfileBj>(op, a, b)
                                                     : apply_op<kProfileRef>(op, a, b);
            vals[d] = v;
            known |= 1u << d;
            u[j] = make_uint4(0u, galop_bits(v), w.z, kWideBcast);
        } else {
            if (!unary && b_known && !is_const) {
                u[j] = make_uint4(w.x, galop_bits(b), w.z, w.w | 8u);
            } else if (!unary && a_known && swaps(fp.profile, op)) {
                const uint32_t sop = op == kOp6 ? (uint32_t)kOp7 : op == kOp7 ? (uint32_t)kOp6 : op;
                u[j] = make_uint4(w.y, galop_bits(a), w.z, (w.w & ~7u) | sop | 8u);
            }
            known &= ~(1u << d);
        }
    };
    for (int64_t j0 = 0; j0 < L; j0 += 4) {
        uint4 g[4];
#pragma unroll
        for (int q = 0; q < 4; ++q) g[q] = j0 + q < L ? u[j0 + q] : make_uint4(0u, 0u, 0u, 0u);
#pragma unroll
        for (int q = 0; q < 4; ++q)
            if (j0 + q < L) forward(g[q], j0 + q);
    }
    // backward: drop what nothing reads, pack the survivors against the end
    // of the slot, and set each survivor's forwarding flags once its
    // predecessor (the next survivor met) is known
    uint32_t live = 1u << fp.output_reg;   // live after instruction j
    int64_t pos = L;                       // survivors occupy u[pos, L)
    bool pending = false;
    uint4 nx = make_uint4(0u, 0u, 0u, 0u); // the survivor after j, not yet written
    uint32_t live_after_nx = 0u;
    auto backward = [&](const uint4 w) {
        const uint32_t d = w.z >> sh;
        if (!((live >> d) & 1u)) return;
        if (pending) {
            set_fwd(nx, w.z, fp.profile);
            if (needs_store(nx, d, live_after_nx, sh)) nx.w |= kWideStorePrev;
            u[--pos] = nx;              // past the micro-op in hand: never one still to be read
        }
        nx = w;
        pending = true;
        live_after_nx = live;
        live = (live & ~(1u << d)) | uop_reads(w, sh);
    };
    for (int64_t j0 = L - 1; j0 >= 0; j0 -= 4) {
        uint4 g[4];                     // u[j0 - 3 .. j0], read before any of them is processed
#pragma unroll
        for (int q = 0; q < 4; ++q) g[q] = j0 - q >= 0 ? u[j0 - q] : make_uint4(0u, 0u, 0u, 0u);
#pragma unroll
        for (int q = 0; q < 4; ++q)
            if (j0 - q >= 0) backward(g[q]);
    }
    if (pending) u[--pos] = nx;         // the first survivor: no flags
    livein = live;
    kept = L - pos;
    return kept;
}

// ---- register renaming ------------------------------------------------------
//
// The interpreter's register file is per warp in shared memory, so the
// registers a program needs -- not the ISA's NR -- set how many warps fit on
// an SM.  rename_slots assigns every value of the program's final micro-op
// order u[0, n) a slot of the file: each register the program reads before
// writing it gets one of slots 0..m-1 (in register order: the interpreter
// loads the i-th set bit of the live-in mask into slot i), each result gets
// the lowest free slot, and a slot is free again after the last instruction
// that reads its value, or when its register is overwritten.  On
// straight-line code this linear scan uses as many slots as there are
// values live at once.  An instruction's operands whose values end there
// are freed before its result is placed, so the result may take an
// operand's slot: the interpreter loads every operand of an instruction
// before that instruction's result is stored (results are stored, if at
// all, at the start of the next instruction, before it loads anything).
// The forwarding flags, set on registers before renaming, stay valid: they
// name the previous instruction's value, whatever slot it gets.  Renamed
// SIN/COS micro-ops with a register operand take the loop's unary form
// (isa.cuh).
constexpr uint32_t kDies1 = 1u << 8;    // src1's value is not read after this instruction
constexpr uint32_t kDies2 = 1u << 9;    // the same for a register src2

__host__ __device__ __forceinline__ uint32_t rename_slots(uint4* __restrict__ u, int64_t n, uint32_t sh, int output_reg,
                                                 uint32_t livein) {
    // backward: mark the reads whose values end at their instruction
    uint32_t live = 1u << output_reg;   // registers live after instruction j
    for (int64_t j = n - 1; j >= 0; --j) {
        uint4 w = u[j];
        const uint32_t d = w.z >> sh;
        const bool bcast = (w.w & ~kWideFlags) == kWideBcast;
        const uint32_t reads = uop_reads(w, sh);
        if (!bcast && !(w.w & kWideSpecial)) {
            const uint32_t r = w.x >> sh;
            if (r == d || !((live >> r) & 1u)) w.w |= kDies1;
        }
        if (!bcast && !(w.w & 8u)) {
            const uint32_t r = w.y >> sh;
            if (r == d || !((live >> r) & 1u)) w.w |= kDies2;
        }
        u[j] = w;
        live = (live & ~(1u << d)) | reads;
    }
    // forward: linear-scan slot assignment
    int8_t slot_of[kMaxRegisters];
    for (int r = 0; r < kMaxRegisters; ++r) slot_of[r] = -1;
    uint32_t used = 0u, top = 0u;
    for (uint32_t m = livein & 0xFFFFu; m != 0u; m &= m - 1u) {
        const int r = galop_ffs(m) - 1;
        slot_of[r] = (int8_t)top;
        used |= 1u << top;
        ++top;
    }
    for (int64_t j = 0; j < n; ++j) {
        uint4 w = u[j];
        const uint32_t d = w.z >> sh;
        const bool bcast = (w.w & ~(kWideFlags | kDies1 | kDies2)) == kWideBcast;
        const bool reads1 = !bcast && !(w.w & kWideSpecial);
        const bool reads2 = !bcast && !(w.w & 8u);
        const uint32_t r1 = w.x >> sh, r2 = w.y >> sh;
        if (reads1) w.x = (uint32_t)slot_of[r1] << sh;
        if (reads2) w.y = (uint32_t)slot_of[r2] << sh;
        if (reads1 && (w.w & kDies1) && slot_of[r1] >= 0) {
            used &= ~(1u << slot_of[r1]);
            slot_of[r1] = -1;
        }
        if (reads2 && (w.w & kDies2) && slot_of[r2] >= 0) {
            used &= ~(1u << slot_of[r2]);
            slot_of[r2] = -1;
        }
        if (slot_of[d] >= 0) {           // the register's old value, never read again
            used &= ~(1u << slot_of[d]);
            slot_of[d] = -1;
        }
        const uint32_t p = (uint32_t)(galop_ffs(~used) - 1);
        used |= 1u << p;
        slot_of[d] = (int8_t)p;
        if (p + 1u > top) top = p + 1u;
        w.z = p << sh;
        w.w &= ~(kDies1 | kDies2);
        // SIN/COS of a register run inside the interpreter loop, which takes
        // a unary operand the way it takes a binary op's src1: the operand's
        // slot into x, fwd2 into fwd1, the unary bit cleared
        const uint32_t op = w.w & 7u;
        if ((w.w & kWideSpecial) && reads2 && (op == kSin || op == kCos)) {
            w.x = w.y;
            w.w = op | ((w.w & kWideFwd2) ? kWideFwd1 : 0u) | (w.w & kWideStorePrev);
        }
        u[j] = w;
    }
    const uint32_t out = slot_of[output_reg] >= 0 ? (uint32_t)slot_of[output_reg] : 0u;
    if (top < 1u) top = 1u;
    return pack_livein(livein, top, out);
}

// One program of fold_kernel: folds u[0, L) in place (forwarding flags only
// when fp.fold is 0), sets its live-in word and returns its interpreted
// length.  Host builds run the same code (tests).
__host__ __device__ __forceinline__ int64_t fold_one(uint4* __restrict__ u, int64_t L, const FoldParams& fp,
                                                     int k_in, uint32_t& livein) {
    const uint32_t sh = fp.stride_shift;
    uint32_t in = 0u;
    int64_t kept;
    if (!fp.fold) {
        in = mark_forwarding(u, L, sh, fp.output_reg, fp.profile);
        kept = L;
    } else {
        kept = fold_program(u, L, fp, k_in, in);
    }
    livein = fp.rename ? rename_slots(u + (L - kept), kept, sh, fp.output_reg, in)
                       : pack_livein(in, (uint32_t)fp.num_registers, (uint32_t)fp.output_reg);
    return kept;
}

static __global__ void fold_kernel(uint4* __restrict__ uops, const int64_t* __restrict__ eff_off, int64_t n,
                                   FoldParams fp, int32_t* __restrict__ interp_len,
                                   uint32_t* __restrict__ livein, unsigned long long* __restrict__ total) {
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    int64_t kept = 0;
    if (i < n) {
        const int64_t p0 = eff_off[i];
        const int64_t L = eff_off[i + 1] - p0;
        const int k_in = fp.pops ? fp.pops[fp.prog_pop[i]].num_inputs : fp.num_inputs;
        uint32_t lv;
        kept = fold_one(uops + p0, L, fp, k_in, lv);
        livein[i] = lv;
        interp_len[i] = (int32_t)kept;
        if (!fp.fold) kept = 0;
    }
    __shared__ unsigned long long sk;
    if (threadIdx.x == 0) sk = 0;
    __syncthreads();
    if (kept) atomicAdd(&sk, (unsigned long long)kept);
    __syncthreads();
    if (threadIdx.x == 0 && sk) atomicAdd(total, sk);
}

}  // namespace galop
