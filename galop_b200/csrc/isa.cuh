// isa.cuh -- device-side view of Galop's instruction encoding and op
// semantics.
//
// Raw word (src/ISA.h:20-41):  [31:24 SRC2 mode|idx][23:16 SRC1][15:8 DEST][7:0 OP]
// Only the low 3 bits of OP (src/LGPConfig.h:189-191) and the low log2(NR)
// bits of each register field are meaningful; bit 31 selects the constant
// pool for src2 (src/ISA.h:84, :201-206).
//
// The pre-pass rewrites every interpreted instruction into a "micro-op" with
// the same byte layout but every field already masked, the INPUT_PROTECT dest
// fold (src/ISA.h:181-187) applied, and bit 6 of the OP byte set for unary
// ops, so the interpreter decodes with plain byte extracts.
#pragma once
#include <cstdint>
#include <cstring>
#include <cmath>
#include <cuda_runtime.h>

#include "trig.cuh"

namespace galop {

constexpr int kMaxRegisters = 16;

enum Profile : int { kProfileRef = 0, kProfileBj = 1 };
enum Op : uint32_t { kAdd = 0, kSub, kMul, kDiv, kSin, kCos, kOp6, kOp7 };

// Runtime ISA parameters shared by the pre-pass kernels.
struct IsaParams {
    int profile;
    int num_registers;   // power of two <= kMaxRegisters
    int input_protect;
    int output_reg;      // 0, or num_registers/2 under input protection
};

// Constant pool passed by value as a kernel parameter (it lands in the
// constant bank, so a warp-uniform index is a single broadcast load).
struct ConstPool {
    float c[kMaxRegisters];
};

struct Decoded {
    uint32_t op, dest, src1, src2, is_const, unary;
};

__host__ __device__ __forceinline__ bool op_is_unary(int profile, uint32_t op) {
    return op == kSin || op == kCos || (profile == kProfileBj && (op == kOp6 || op == kOp7));
}

// src/ISA.h:176-206 with runtime NR / INPUT_PROTECT.
__host__ __device__ __forceinline__ Decoded decode_raw(const IsaParams& p, uint32_t w) {
    const uint32_t rmask = (uint32_t)p.num_registers - 1u;
    Decoded d;
    d.op = w & 7u;
    d.dest = p.input_protect ? (uint32_t)p.output_reg + ((w >> 8) & (rmask >> 1))
                             : ((w >> 8) & rmask);
    d.src1 = (w >> 16) & rmask;
    d.src2 = (w >> 24) & rmask;
    d.is_const = (w >> 31) & 1u;
    d.unary = op_is_unary(p.profile, d.op) ? 1u : 0u;
    return d;
}

// Micro-op: byte0 = op | unary<<6, byte1 = dest, byte2 = src1,
// byte3 = src2 | const<<7.
__host__ __device__ __forceinline__ uint32_t encode_uop(const Decoded& d) {
    return (d.op | (d.unary << 6)) | (d.dest << 8) | (d.src1 << 16) | ((d.src2 | (d.is_const << 7)) << 24);
}

// Wide micro-op (16 bytes, interp_wide_kernel): the operand fields are
// already byte offsets into the warp's shared-memory register file and a
// constant operand carries its value, so the interpreter decodes nothing.
//   x = src1 * stride            (0 for unary ops)
//   y = src2 * stride, or the constant's bits when src2 is a constant
//   z = dest * stride
//   w = op | const << 3 | fwd1 << 4 | store_prev << 5 | fwd2 << 6
//       | unary << 31   (kWideEnd ends a window)
// stride = bytes per register per warp (32 lanes x K cases x 4 bytes).
// The flag bits describe the program's final instruction order (fold.cuh
// sets them) for the interpreter loop, which keeps the last result in
// registers and writes it to the register file only when the next
// instruction says so:
//   fwd1        src1 (binary op) is the previous instruction's destination:
//               the operand is the previous result, not loaded;
//   fwd2        the same for src2 of a unary op;
//   store_prev  the previous result must reach the register file (something
//               other than this instruction's forwarded operand reads it);
//               it is stored before this instruction reads any operand.
// Renamed streams (register-file slots, fold.cuh) carry SIN and COS of a
// register in the interpreter loop's unary form: x = the operand's slot,
// y unused, w = op | fwd1 << 4 | store_prev << 5 (fwd1: the operand is the
// previous result), unary bit clear.
constexpr uint32_t kWideSpecial = 0x80000000u;
constexpr uint32_t kWideEnd = 0xFFFFFFFFu;
constexpr uint32_t kWideFwd1 = 16u;
constexpr uint32_t kWideStorePrev = 32u;
constexpr uint32_t kWideFwd2 = 64u;
constexpr uint32_t kWideFlags = kWideFwd1 | kWideStorePrev | kWideFwd2;
// Broadcast micro-op (table slot 12): dest = the constant in y, for an
// instruction whose operands are all known before any case is read.
constexpr uint32_t kWideBcast = 12u;

__device__ __forceinline__ uint4 encode_wide(const Decoded& d, uint32_t stride, const ConstPool& cp) {
    uint4 u;
    u.x = d.unary ? 0u : d.src1 * stride;
    u.y = d.is_const ? __float_as_uint(cp.c[d.src2]) : d.src2 * stride;
    u.z = d.dest * stride;
    u.w = d.op | (d.is_const << 3) | (d.unary ? kWideSpecial : 0u);
    return u;
}

// Per-program word the folding pass writes for the interpreter (one uint32
// per program): registers read before written (bits 0-15; the i-th set bit
// is loaded into register-file slot i), slots the program's values use
// (bits 16-20), slot that holds the output value at the end (bits 24-27).
__host__ __device__ __forceinline__ uint32_t pack_livein(uint32_t regs, uint32_t slots, uint32_t out_slot) {
    return (regs & 0xFFFFu) | (slots << 16) | (out_slot << 24);
}
__host__ __device__ __forceinline__ uint32_t livein_regs(uint32_t w) { return w & 0xFFFFu; }
__host__ __device__ __forceinline__ uint32_t livein_slots(uint32_t w) { return (w >> 16) & 31u; }
__host__ __device__ __forceinline__ uint32_t livein_out_slot(uint32_t w) { return (w >> 24) & 15u; }

// Which micro-op form the pre-pass writes.
struct UopFormat {
    int wide;              // 0: 32-bit micro-ops, 1: 16-byte wide micro-ops
    uint32_t stride;       // wide: bytes per register per warp
    ConstPool consts;      // wide: constant values folded into the micro-ops
};

__device__ __forceinline__ uint32_t uop_op(uint32_t u) { return u & 7u; }
__device__ __forceinline__ uint32_t uop_dest(uint32_t u) { return (u >> 8) & 0xffu; }
__device__ __forceinline__ uint32_t uop_src1(uint32_t u) { return (u >> 16) & 0xffu; }
__device__ __forceinline__ uint32_t uop_src2(uint32_t u) { return (u >> 24) & 0x7fu; }
__device__ __forceinline__ bool uop_is_const(uint32_t u) { return (u >> 31) != 0u; }

// Bit casts and find-first-set for code that also runs on the host (the
// folding pass, which tests build for the CPU).
__host__ __device__ __forceinline__ uint32_t galop_bits(float f) {
#if defined(__CUDA_ARCH__)
    return __float_as_uint(f);
#else
    uint32_t u;
    std::memcpy(&u, &f, sizeof u);
    return u;
#endif
}
__host__ __device__ __forceinline__ float galop_float(uint32_t u) {
#if defined(__CUDA_ARCH__)
    return __uint_as_float(u);
#else
    float f;
    std::memcpy(&f, &u, sizeof f);
    return f;
#endif
}
__host__ __device__ __forceinline__ int galop_ffs(uint32_t x) {
#if defined(__CUDA_ARCH__)
    return __ffs(x);
#else
    return __builtin_ffs((int)x);
#endif
}

// Op semantics, src/ISA.h:219-231 (REF) and the BJ profile's EXP/LOG.
// Explicit round-to-nearest intrinsics: no FMA contraction, IEEE division,
// matching the CPU build (ISO C++, no contraction, SSE2 arithmetic).  SIN
// and COS are trig.cuh's (within 1.56 ulp of the exact value, as the C
// library's are within 1 ulp); EXP and LOG are CUDA's.  A host build
// (tests) computes the IEEE ops with the host's single-precision
// arithmetic, the same bits, and EXP/LOG with the C library.
template <int PROFILE>
__host__ __device__ __forceinline__ float apply_op(uint32_t op, float a, float b) {
    switch (op) {
#if defined(__CUDA_ARCH__)
        case kAdd: return __fadd_rn(a, b);
        case kSub: return __fsub_rn(a, b);
        case kMul: return __fmul_rn(a, b);
        case kDiv: return (b != 0.0f) ? __fdiv_rn(a, b) : 1.0f;
#else
        case kAdd: return a + b;
        case kSub: return a - b;
        case kMul: return a * b;
        case kDiv: return (b != 0.0f) ? a / b : 1.0f;
#endif
        case kSin: return galop_sinf(b);
        case kCos: return galop_cosf(b);
        case kOp6:
            if constexpr (PROFILE == kProfileBj) return expf(b);
            else return (a < b) ? 1.0f : 0.0f;
        default:
            if constexpr (PROFILE == kProfileBj) return (b != 0.0f) ? logf(fabsf(b)) : 0.0f;
            else return (a > b) ? 1.0f : 0.0f;
    }
}

}  // namespace galop
