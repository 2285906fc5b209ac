"""Generate dispatch_gen.cuh: PTX jump tables of the interpreters.

The LGP register file of a warp lives in shared memory and an instruction's
operands are addresses, so the only run-time dispatch is on the opcode.
These helpers emit PTX ``brx.idx`` over a ``.branchtargets`` table: one
indirect branch, then the K arithmetic instructions of the selected op.

Emitted for K in {1, 2, 4, 8} and both ISA profiles:
  cheap    t[k] = OP(a[k], b[k]) on the opcode alone (dispatch 2: operands
           already loaded from the shared-memory register file)
  wide     one whole binary instruction of the 16-byte micro-op kernel
           (dispatch 3, one instruction at a time: register traces):
           load a (and b) from the shared-memory register file, compute,
           store t -- the table index is op | constant-src2 << 3, and
           protected DIV is one of the arms
  wide loop  the same ops as one PTX loop over consecutive binary
           instructions and SIN/COS of a register (returns at any other
           unary op or the window end), with the last result kept in
           registers: forwarded src1 operands are not loaded and results
           only reach the register file when the next instruction's
           store_prev flag asks for it.  Its DIV arms divide with a fast
           path of their own (div_group: rcp.approx, one Newton-Raphson
           step, Markstein's correction) and take the exact div.rn path
           only for a warp with an operand out of its range; its SIN/COS
           arms run trig.cuh's Cody-Waite path (trig_blocks) and leave the
           loop to the caller for a warp with an argument beyond it.  ADD,
           SUB and MUL, the division's Newton-Raphson and Markstein steps
           and the trig polynomials take two elements per instruction
           (sm_100a's f32x2 forms, rounded per half like the f32 ones)
  both wide forms also have the broadcast arm (table index 12): t[k] = the
  micro-op's constant, for instructions folded by the pre-pass
where OP is one of the single-instruction ops: ADD, SUB, MUL (add/sub/mul
with explicit .rn rounding, which ptxas never contracts into FMA) and, for
the REF profile, LT, GT (set.lt/set.gt .f32.f32: 1.0 if the ordered
comparison holds, else 0.0 -- false for NaN operands, like the C++ `a < b ?
1.0f : 0.0f`).  Table entries of other opcodes fall through to the end
label (never taken: the interpreter routes those ops elsewhere).

The build (galop_b200/build.py) calls render() and rewrites dispatch_gen.cuh
whenever its text differs, so the header cannot drift from this generator.
Run by hand: python galop_b200/csrc/gen_dispatch.py
"""
from __future__ import annotations

import re
import struct
from pathlib import Path

KS = (1, 2, 4, 8)
CHEAP = {0: "add.rn.f32", 1: "sub.rn.f32", 2: "mul.rn.f32", 6: "set.lt.f32.f32", 7: "set.gt.f32.f32"}
PROFILES = {0: (0, 1, 2, 6, 7), 1: (0, 1, 2)}   # REF, BJ
# Table slot 8 + BCAST_OP (a SIN "with constant operand", which the pre-pass
# never emits as such) is the broadcast arm: t = the micro-op's constant, for
# instructions the pre-pass has evaluated once because every operand is known.
BCAST_OP = 4


def asm_block(lines: list[str], outs: list[str], ins: list[str]) -> str:
    body = "\\n\\t".join(lines)
    return (f'    asm("{{\\n\\t{body}\\n\\t}}"\n'
            f'        : {", ".join(outs) if outs else ""}\n'
            f'        : {", ".join(ins)});\n')


def cheap_table(k: int, profile: int) -> str:
    """t[q] = OP(a[q], b[q]) for the single-instruction ops, one table on
    the opcode (8 entries, other opcodes jump to the end)."""
    ops = PROFILES[profile]
    # outputs t %0..k-1 ; inputs op %k, a %(k+1+q), b %(2k+1+q)
    L = ["T%=: .branchtargets " + ", ".join(f"C{op}_%=" if op in ops else "E%=" for op in range(8)) + ";",
         f"brx.idx %{k}, T%=;"]
    for op in ops:
        body = " ".join(f"{CHEAP[op]} %{q}, %{k + 1 + q}, %{2 * k + 1 + q};" for q in range(k))
        L.append(f"C{op}_%=: {body} bra.uni E%=;")
    L.append("E%=:")
    outs = [f'"=f"(t[{q}])' for q in range(k)]
    ins = ['"r"(op)'] + [f'"f"(a[{q}])' for q in range(k)] + [f'"f"(b[{q}])' for q in range(k)]
    return (f"    static __device__ __forceinline__ void cheap(uint32_t op, const float (&a)[{k}], "
            f"const float (&b)[{k}], float (&t)[{k}]) {{\n" + asm_block(L, outs, ins) + "    }\n")


# Scratch registers of the wide arms (declared once per asm block).
WIDE_TEMPS = ".reg .pred dp, dn, dz; .reg .f32 da, db, dq; .reg .b32 ds, dbb;"


def wide_body(k: int, op: int, const: bool, a=None, b=None, t=None) -> list[str]:
    """t[q] = OP(a[q], b[q]) (b = the scalar c for a constant src2).

    a, b, t map q to register names (default a{q}, b{q}, t{q}); t[q] is
    written once, after the last read of a[q] and b[q], so an operand may be
    the result register itself (a forwarded operand).

    DIV is b != 0 ? a / b : 1.0 (src/ISA.h:224) with IEEE round-to-nearest
    (div.rn.f32), evaluated as:
      dp = b != 0 or NaN (setp.neu: NaN counts as nonzero, like C's b != 0)
      dz = a == +-0 and b is not NaN: the quotient is a zero whose sign is
           sign(a) xor sign(b) (IEEE 754: 0/x = +-0 for every nonzero,
           non-NaN x, infinities included), formed with one xor/and;
      otherwise div.rn on (a, b), with a zero dividend or divisor replaced by
      1.0 so the division only ever sees the operands whose quotient is used.
    Zero dividends are common in LGP code (LT/GT results, x - x)."""
    a = a or (lambda q: f"a{q}")
    t = t or (lambda q: f"t{q}")
    if const:
        b = lambda q: "c"
    else:
        b = b or (lambda q: f"b{q}")
    out = []
    for q in range(k):
        aq, bq, tq = a(q), b(q), t(q)
        if op != 3:
            out.append(f"{CHEAP[op]} {tq}, {aq}, {bq};")
            continue
        out += [f"setp.neu.f32 dp, {bq}, 0f00000000;",
                f"setp.num.f32 dn, {bq}, {bq};",
                f"setp.eq.and.f32 dz, {aq}, 0f00000000, dn;",
                f"selp.f32 da, 0f3F800000, {aq}, dz;",
                f"selp.f32 db, {bq}, 0f3F800000, dp;",
                "div.rn.f32 dq, da, db;",
                f"mov.b32 ds, {aq};",
                f"mov.b32 dbb, {bq};",
                "xor.b32 ds, ds, dbb;",
                "and.b32 ds, ds, 0x80000000;",
                f"selp.f32 {tq}, dq, 0f3F800000, dp;",
                "and.pred dz, dz, dp;",
                f"@dz mov.b32 {tq}, ds;"]
    return out


# Fast path of protected DIV in the wide loop (div_group).
DIV_TEMPS = (".reg .f32 fy, fe, fnb, fr, fab, fq; .reg .b32 fs, fw; "
             ".reg .pred fz, fa, fb0, fall, funi, fbok;")
DIV_LO, DIV_HI = "0f20000000", "0f5F000000"      # 2^-63, 2^63
# Paired (f32x2) temporaries of the wide loop's arithmetic: sm_100a's
# add/sub/mul/fma.rn.f32x2 round each half exactly as the f32 instruction
# does, so two elements take one instruction with the same bits.
PAIR_TEMPS = (".reg .b64 xa, xb, xc, xy, xnb, xe, xq, xr, xone; "
              ".reg .f32 fy0, fy1, fnb0, fnb1, fq0, fq1, fg0, fg1;")
X2 = {0: "add.rn.f32x2", 1: "sub.rn.f32x2", 2: "mul.rn.f32x2"}


def pair_body(k: int, op: int, const: bool, a, b) -> list[str]:
    """a[q] = OP(a[q], b[q]) for ADD/SUB/MUL, two elements per f32x2
    instruction (b = the scalar c for a constant src2)."""
    out = ["mov.b64 xc, {c, c};"] if const else []
    for j in range(k // 2):
        a0, a1 = a(2 * j), a(2 * j + 1)
        out.append(f"mov.b64 xa, {{{a0}, {a1}}};")
        if not const:
            out.append(f"mov.b64 xb, {{{b(2 * j)}, {b(2 * j + 1)}}};")
        out += [f"{X2[op]} xa, xa, {'xc' if const else 'xb'};", f"mov.b64 {{{a0}, {a1}}}, xa;"]
    return out


def div_divisor_lines(b: str) -> list[str]:
    """The divisor's half of the fast path (once per instruction for a
    constant divisor, per element otherwise): fy ~ 1/b refined by one
    Newton-Raphson step, fnb = -b, fbok = 2^-63 <= |b| <= 2^63, fb0 = (b == 0)."""
    return [f"rcp.approx.ftz.f32 fy, {b};",
            f"neg.f32 fnb, {b};",
            "fma.rn.f32 fe, fnb, fy, 0f3F800000;",
            "fma.rn.f32 fy, fy, fe, fy;",
            f"abs.f32 fab, {b};",
            f"setp.ge.f32 fbok, fab, {DIV_LO};",
            f"setp.le.and.f32 fbok, fab, {DIV_HI}, fbok;",
            f"setp.eq.f32 fb0, {b}, 0f00000000;"]


def div_fast_lines(a: str, out: str) -> list[str]:
    """The dividend's half: q0 = a * fy, r = a - b q0 (exact), q = q0 + r fy
    (the correction step of P. Markstein, "Computation of elementary
    functions on the IBM RISC System/6000 processor", IBM J. Res. Dev.
    34(1), 1990, which rounds correctly from a faithful q0 and an accurate
    reciprocal), the sign of q0 kept on a zero quotient; out = q, or 1.0 for
    a zero divisor.  fall &= this element is in the fast path's range:
    2^-63 <= |a| <= 2^63 or a == 0, and the divisor's fbok, or b == 0."""
    return [f"mul.rn.f32 fq, {a}, fy;",
            "mov.b32 fs, fq;",
            "and.b32 fs, fs, 0x80000000;",
            f"fma.rn.f32 fr, fnb, fq, {a};",
            "fma.rn.f32 fq, fr, fy, fq;",
            "mov.b32 fw, fq;",
            "or.b32 fw, fw, fs;",
            "mov.b32 fq, fw;",
            f"selp.f32 {out}, 0f3F800000, fq, fb0;",
            f"setp.eq.f32 fz, {a}, 0f00000000;",
            f"abs.f32 fab, {a};",
            f"setp.ge.or.f32 fa, fab, {DIV_LO}, fz;",
            f"setp.le.and.f32 fa, fab, {DIV_HI}, fa;",
            "and.pred fa, fa, fbok;",
            "or.pred fa, fa, fb0;",
            "and.pred fall, fall, fa;"]


# Scratch registers of the SIN/COS block (trig_blocks): per element, per
# element pair, and the register pairs that hold the constants.
TRIG_TEMPS = (".reg .f32 tax, tjr, tj, tr, tz, tp, trz, ts, tc, ty; .reg .b32 tq, tb, tt, tw, th, tcos, tmask; "
              ".reg .pred tpq, tslow, tany; "
              ".reg .f32 tax0, tax1, tjr0, tjr1, ts0, ts1, tc0, tc1; "
              ".reg .b64 k2pi, kround, knp1, knp2, knp3, ks3, ks2, ks1, kc4, kc3, kc2, kc1, kone, "
              "xax, xjr, xj, xtr, xz, xp, xrz, xs, xtc;")


def trig_pair_constants(c: dict) -> dict:
    """The Cody-Waite path's constants by the register-pair names of the
    paired (f32x2) form, which takes no immediate operands."""
    return {"k2pi": c["GT_TWO_OVER_PI"], "kround": c["GT_ROUND"], "knp1": neg_imm(c["GT_P1"]),
            "knp2": neg_imm(c["GT_P2"]), "knp3": neg_imm(c["GT_P3"]), "ks3": c["GT_S3"], "ks2": c["GT_S2"],
            "ks1": c["GT_S1"], "kc4": c["GT_C4"], "kc3": c["GT_C3"], "kc2": c["GT_C2"], "kc1": c["GT_C1"],
            "kone": "0f3F800000"}


def trig_constants() -> dict:
    """The single-precision constants of trig.cuh's Cody-Waite path as PTX
    immediates (0fXXXXXXXX), read from the header itself so the loop's copy
    of the fast path cannot drift from it."""
    text = (Path(__file__).resolve().parent / "trig.cuh").read_text()
    out = {}
    for name, lit in re.findall(r"#define (GT_[A-Z0-9_]+|GALOP_TRIG_FAST_LIMIT) (-?0x[0-9a-fA-Fp.+-]+f|[0-9.]+f)\n", text):
        v = float.fromhex(lit[:-1]) if "0x" in lit else float(lit[:-1])
        out[name] = "0f%08X" % struct.unpack("<I", struct.pack("<f", v))[0]
    need = {"GALOP_TRIG_FAST_LIMIT", "GT_TWO_OVER_PI", "GT_ROUND", "GT_P1", "GT_P2", "GT_P3",
            "GT_S1", "GT_S2", "GT_S3", "GT_C1", "GT_C2", "GT_C3", "GT_C4"}
    if not need <= out.keys():
        raise RuntimeError(f"trig.cuh: constants not found: {sorted(need - out.keys())}")
    return out


def neg_imm(imm: str) -> str:
    """The PTX immediate of -x for the float immediate x."""
    return "0f%08X" % (int(imm[2:], 16) ^ 0x80000000)


TRIG_OPS = (4, 5)      # SIN, COS: unary in both profiles


def trig_blocks(k: int, a) -> list[str]:
    """The wide loop's SIN and COS of the lane's K elements of the result
    registers a(q), in place: trig.cuh's Cody-Waite path (galop_trig_fast)
    restated operation for operation, so the bits are the same.  One block
    (R) serves both ops and both copies of the loop body: the arms jump here
    after putting the operand into a(q) and the destination address into the
    result-address register, with th = 1 when they are copy A's and
    tcos = 1 for COS (the quadrant moves by one, and the argument's sign
    does not enter the result's: tmask = 0).

    For K >= 2 the float steps run on element pairs (f32x2: each half
    rounded as the f32 instruction rounds it, so the bits do not change),
    with the constants in register pairs set at the block's start; the
    quadrant, selection and sign stay per element.

    Each element goes into fo<q>.  When an element of any lane is out of
    the fast path's range (|x| >= 2^17, infinities, NaN; vote.any, so the
    branch is uniform) the warp jumps to block Z, which steps the micro-op
    pointer back to the trig micro-op and leaves the loop through its
    copy's exit, with a(q) still the operand: the caller evaluates the op
    with galop_trig_k, which takes the Payne-Hanek path where needed.
    Otherwise the results move into a(q) and the loop goes on with the next
    micro-op, already loaded into the other copy's registers."""
    c = trig_constants()
    lim = c["GALOP_TRIG_FAST_LIMIT"]

    def tail(q: int, jr: str, sv: str, cv: str, ax: str) -> list[str]:
        # quadrant, sine or cosine polynomial, sign; the range test
        x = a(q)
        return [f"mov.b32 tq, {jr};",
                "add.u32 tq, tq, tcos;",
                "and.b32 tb, tq, 1;",
                "setp.ne.u32 tpq, tb, 0;",
                f"selp.f32 ty, {cv}, {sv}, tpq;",
                "shl.b32 tt, tq, 30;",
                f"mov.b32 tw, {x};",
                "and.b32 tw, tw, tmask;",
                "xor.b32 tt, tt, tw;",
                "and.b32 tt, tt, 0x80000000;",
                "mov.b32 tw, ty;",
                "xor.b32 tw, tw, tt;",
                f"mov.b32 fo{q}, tw;",
                f"setp.geu.f32 tslow, {ax}, {lim};" if q == 0 else
                f"setp.geu.or.f32 tslow, {ax}, {lim}, tslow;"]

    R = ["R_%=:", "sub.u32 tmask, tcos, 1;"]
    if k >= 2:
        # two elements per f32x2 instruction; the constants as register pairs
        R += [f"mov.b64 {n}, 0x{v[2:] * 2};" for n, v in trig_pair_constants(c).items()]
        for j in range(k // 2):
            R += [f"abs.f32 tax0, {a(2 * j)};", f"abs.f32 tax1, {a(2 * j + 1)};", "mov.b64 xax, {tax0, tax1};",
                  "fma.rn.f32x2 xjr, xax, k2pi, kround;",
                  "sub.rn.f32x2 xj, xjr, kround;",
                  "fma.rn.f32x2 xtr, xj, knp1, xax;",
                  "fma.rn.f32x2 xtr, xj, knp2, xtr;",
                  "fma.rn.f32x2 xtr, xj, knp3, xtr;",
                  "mul.rn.f32x2 xz, xtr, xtr;",
                  "fma.rn.f32x2 xp, xz, ks3, ks2;",
                  "fma.rn.f32x2 xp, xp, xz, ks1;",
                  "mul.rn.f32x2 xrz, xtr, xz;",
                  "fma.rn.f32x2 xs, xrz, xp, xtr;",
                  "fma.rn.f32x2 xtc, xz, kc4, kc3;",
                  "fma.rn.f32x2 xtc, xtc, xz, kc2;",
                  "fma.rn.f32x2 xtc, xtc, xz, kc1;",
                  "fma.rn.f32x2 xtc, xtc, xz, kone;",
                  "mov.b64 {tjr0, tjr1}, xjr;", "mov.b64 {ts0, ts1}, xs;", "mov.b64 {tc0, tc1}, xtc;"]
            for e in (0, 1):
                R += tail(2 * j + e, f"tjr{e}", f"ts{e}", f"tc{e}", f"tax{e}")
    else:
        for q in range(k):
            R += [f"abs.f32 tax, {a(q)};",
                  f"fma.rn.f32 tjr, tax, {c['GT_TWO_OVER_PI']}, {c['GT_ROUND']};",
                  f"sub.rn.f32 tj, tjr, {c['GT_ROUND']};",
                  f"fma.rn.f32 tr, tj, {neg_imm(c['GT_P1'])}, tax;",
                  f"fma.rn.f32 tr, tj, {neg_imm(c['GT_P2'])}, tr;",
                  f"fma.rn.f32 tr, tj, {neg_imm(c['GT_P3'])}, tr;",
                  "mul.rn.f32 tz, tr, tr;",
                  f"fma.rn.f32 tp, tz, {c['GT_S3']}, {c['GT_S2']};",
                  f"fma.rn.f32 tp, tp, tz, {c['GT_S1']};",
                  "mul.rn.f32 trz, tr, tz;",
                  "fma.rn.f32 ts, trz, tp, tr;",
                  f"fma.rn.f32 tc, tz, {c['GT_C4']}, {c['GT_C3']};",
                  f"fma.rn.f32 tc, tc, tz, {c['GT_C2']};",
                  f"fma.rn.f32 tc, tc, tz, {c['GT_C1']};",
                  "fma.rn.f32 tc, tc, tz, 0f3F800000;"]
            R += tail(q, "tjr", "ts", "tc", "tax")
    R += ["vote.sync.any.pred tany, tslow, 0xffffffff;", "@tany bra.uni Z_%=;"]
    R += [f"mov.f32 {a(q)}, fo{q};" for q in range(k)]
    R += ["setp.ne.u32 tpq, th, 0;", "@tpq bra.uni LB%=;", "bra.uni LA%=;"]
    Z = ["Z_%=: sub.u32 %0, %0, 16;", "setp.ne.u32 tpq, th, 0;", "@tpq bra.uni DA%=;", "bra.uni DB%=;"]
    return [" ".join(R), " ".join(Z)]


def div_group(k: int, const: bool, a, b, nm: str) -> tuple[list[str], list[str]]:
    """Protected DIV of the wide loop on the lane's K elements, in place
    (a[q] = a[q] / b[q], or 1.0 for b[q] == 0): (hot lines, exact lines).

    Hot: every element through the fast path into fo<q>; when every element
    of every lane is in the fast path's range (vote.all, so the branch is
    uniform), the results move into a[q] and the arm goes on at W<nm>.
    Otherwise the exact lines (block V<nm>, placed away from the hot code)
    evaluate all K elements with wide_body's div.rn path, which reads a[q]
    and b[q] unchanged, and jump back to W<nm>.  Fast and exact agree bit
    for bit wherever the fast path is in range (tests/test_gpu_division.py).
    For K >= 2 the Newton-Raphson and Markstein steps run on element pairs
    (div_pair_lines), the same operations two at a time.
    (Leaving the loop for a division in C++ instead, to keep the V blocks
    out of the loop's code, was slower.)"""
    bq = (lambda q: "c") if const else b
    hot = []
    if k >= 2:
        hot += ["mov.b64 xone, 0x3F8000003F800000;"]
        if const:
            hot += div_divisor_lines("c")
            hot += ["mov.b64 xy, {fy, fy};", "mov.b64 xnb, {fnb, fnb};"]
        for j in range(k // 2):
            hot += div_pair_lines(a(2 * j), a(2 * j + 1), bq(2 * j), bq(2 * j + 1), f"fo{2 * j}",
                                  f"fo{2 * j + 1}", const, first=(j == 0))
    else:
        if const:
            hot += div_divisor_lines("c")
        for q in range(k):
            if not const:
                hot += div_divisor_lines(bq(q))
            lines = div_fast_lines(a(q), f"fo{q}")
            if q == 0:
                lines[-1] = "mov.pred fall, fa;"
            hot += lines
    hot += ["vote.sync.all.pred funi, fall, 0xffffffff;", f"@!funi bra.uni V{nm};"]
    hot += [f"mov.f32 {a(q)}, fo{q};" for q in range(k)]
    hot.append(f"W{nm}:")
    exact = wide_body(k, 3, const, a=a, b=b, t=a)
    return hot, exact


def div_pair_lines(a0: str, a1: str, b0: str, b1: str, o0: str, o1: str, const: bool,
                   first: bool) -> list[str]:
    """div_divisor_lines and div_fast_lines for two elements, the float
    steps as f32x2 pairs: the reciprocal refinement (register divisors; a
    constant divisor's xy/xnb are set once), then q0 = a y, r = a - b q0,
    q = q0 + r y.  The per-element rest (sign of a zero quotient, the zero
    divisor's 1.0, the range tests) is div_fast_lines' own.  fall starts
    with the first pair."""
    L = []
    if not const:
        L += [f"rcp.approx.ftz.f32 fy0, {b0};", f"rcp.approx.ftz.f32 fy1, {b1};",
              f"neg.f32 fnb0, {b0};", f"neg.f32 fnb1, {b1};",
              "mov.b64 xy, {fy0, fy1};", "mov.b64 xnb, {fnb0, fnb1};",
              "fma.rn.f32x2 xe, xnb, xy, xone;",
              "fma.rn.f32x2 xy, xy, xe, xy;"]
    L += [f"mov.b64 xa, {{{a0}, {a1}}};",
          "mul.rn.f32x2 xq, xa, xy;",
          "fma.rn.f32x2 xr, xnb, xq, xa;",
          "fma.rn.f32x2 xr, xr, xy, xq;",
          "mov.b64 {fq0, fq1}, xq;",
          "mov.b64 {fg0, fg1}, xr;"]
    for e, (ae, be, oe, fqe, fge) in enumerate(((a0, b0, o0, "fq0", "fg0"), (a1, b1, o1, "fq1", "fg1"))):
        if not const:
            L += [f"abs.f32 fab, {be};",
                  f"setp.ge.f32 fbok, fab, {DIV_LO};",
                  f"setp.le.and.f32 fbok, fab, {DIV_HI}, fbok;",
                  f"setp.eq.f32 fb0, {be}, 0f00000000;"]
        L += [f"mov.b32 fs, {fqe};",
              "and.b32 fs, fs, 0x80000000;",
              f"mov.b32 fw, {fge};",
              "or.b32 fw, fw, fs;",
              "mov.b32 fq, fw;",
              f"selp.f32 {oe}, 0f3F800000, fq, fb0;",
              f"setp.eq.f32 fz, {ae}, 0f00000000;",
              f"abs.f32 fab, {ae};",
              f"setp.ge.or.f32 fa, fab, {DIV_LO}, fz;",
              f"setp.le.and.f32 fa, fab, {DIV_HI}, fa;",
              "and.pred fa, fa, fbok;",
              "or.pred fa, fa, fb0;",
              "mov.pred fall, fa;" if first and e == 0 else "and.pred fall, fall, fa;"]
    return L


def _vec(regs: list[str]) -> str:
    return regs[0] if len(regs) == 1 else "{" + ", ".join(regs) + "}"


def wide_ops(k: int, profile: int) -> str:
    """One binary instruction of the 16-byte micro-op kernel, start to end.

    Inputs: %0 table index (op | const << 3), %1/%2/%3 shared-memory byte
    addresses of the lane's src1 / src2 / dest register (V floats per vector,
    vectors 32*V floats apart), %4 the constant's bits (const arms).  src1 is
    loaded before the branch so its latency overlaps the dispatch; src2 only
    in the register arms (its address is meaningless for a constant).  DIV is
    b != 0 ? a / b (div.rn.f32) : 1.0, as src/ISA.h:224; setp.neu treats a
    NaN divisor as nonzero, like C's b != 0.0f."""
    v = min(k, 4)
    nq = k // v
    ops = tuple(sorted(PROFILES[profile] + (3,)))
    vs = "" if v == 1 else f".v{v}"

    def ld(dst: str, addr: str) -> list[str]:
        return [f"ld.shared{vs}.f32 {_vec([f'{dst}{q * v + e}' for e in range(v)])}, [{addr}+{q * 128 * v}];"
                for q in range(nq)]

    def st(addr: str) -> list[str]:
        return [f"st.shared{vs}.f32 [{addr}+{q * 128 * v}], {_vec([f't{q * v + e}' for e in range(v)])};"
                for q in range(nq)]

    def body(op: int, const: bool) -> list[str]:
        return wide_body(k, op, const)

    regs = ", ".join(f"{n}<{k}>" for n in "abt")
    L = [f".reg .f32 {regs}, c;", WIDE_TEMPS, "mov.b32 c, %4;"]
    L += ld("a", "%1")
    targets = [f"R{op}_%=" if op in ops else "E%=" for op in range(8)] + \
              [f"C{op}_%=" if op in ops else ("B%=" if op == BCAST_OP else "E%=") for op in range(8)]
    L += ["T%=: .branchtargets " + ", ".join(targets) + ";", "brx.idx.uni %0, T%=;"]
    for op in ops:
        L.append(f"R{op}_%=: " + " ".join(ld("b", "%2") + body(op, False) + st("%3")) + " bra.uni E%=;")
        L.append(f"C{op}_%=: " + " ".join(body(op, True) + st("%3")) + " bra.uni E%=;")
    L.append("B%=: " + " ".join([f"mov.f32 t{q}, c;" for q in range(k)] + st("%3")) + " bra.uni E%=;")
    L.append("E%=:")
    text = "\\n\\t".join(L)
    return ("    static __device__ __forceinline__ void run(uint32_t idx, uint32_t pa, uint32_t pb, uint32_t pt, "
            "uint32_t cbits) {\n"
            f'    asm volatile("{{\\n\\t{text}\\n\\t}}"\n'
            '        :\n        : "r"(idx), "r"(pa), "r"(pb), "r"(pt), "r"(cbits)\n        : "memory");\n    }\n')


def wide_loop(k: int, profile: int) -> str:
    """The fast path of the 16-byte micro-op kernel as one PTX loop: execute
    binary instructions (and SIN/COS of a register) from the staged micro-op
    at byte address %0 on, until a micro-op whose word w is negative (an
    other unary op or the window's end marker) or a SIN/COS whose argument
    needs the caller's Payne-Hanek path; return with %0 pointing at it.
    Such a SIN/COS leaves with its pending store done and a = its operand.

    Operands: %0 the micro-op address (in/out); %1..%K the lane's K values of
    the last result (in/out); %K+1 the register-file address that result
    belongs to (in/out); %K+2 the lane's register-file base.  The caller's
    unary ops and the next call continue from the same result registers.

    The result registers double as the src1 registers: an arm computes
    a = OP(a, b).  Each (op, constant src2) arm has three entry points, in
    this order: S stores the pending result to its register, L loads src1,
    F loads src2 (register arms) then computes, remembers the destination
    address and jumps on; a fourth, G, stores and jumps to F.  The jump
    table has 64 entries, indexed by w's low 6 bits (op | const << 3 |
    fwd1 << 4 | store_prev << 5):
      store_prev, not fwd1 -> S     neither -> L
      fwd1, not store_prev -> F     both    -> G
    The broadcast arm (index 12, | 32) has S and L only: a = the constant.
    SIN and COS with a register operand (indices 4 and 5, | 16 | 32) are
    arms too: the folding pass rewrites such a micro-op with its operand as
    src1 and fwd2 as fwd1 (fold.cuh), so S/L/F/G load or forward it like a
    src1 into a, and F jumps to the one block both ops and both copies
    share (trig_blocks), which computes a = SIN(a) or COS(a) and goes on -- or
    leaves the loop at that micro-op, a holding the operand, when an
    argument needs trig.cuh's slow path.

    Two copies of the loop body alternate between two micro-op register sets
    (u, v): each body prefetches the next micro-op into the other set, so no
    micro-op is ever copied between registers."""
    v = min(k, 4)
    nq = k // v
    ops = tuple(sorted(PROFILES[profile] + (3,)))
    vs = "" if v == 1 else f".v{v}"
    A = lambda q: f"%{1 + q}"
    PT = f"%{k + 1}"
    LV = [f"%{k + 2 + i}" for i in range(4)]      # out: the micro-op that leaves
    base = f"%{k + 6}"
    CUR = [f"%{k + 7 + i}" for i in range(4)]     # in: the micro-op at %0

    def ld(names, addr: str) -> list[str]:
        return [f"ld.shared{vs}.f32 {_vec([names(q * v + e) for e in range(v)])}, [{addr}+{q * 128 * v}];"
                for q in range(nq)]

    def st(addr: str) -> list[str]:
        return [f"st.shared{vs}.f32 [{addr}+{q * 128 * v}], {_vec([A(q * v + e) for e in range(v)])};"
                for q in range(nq)]

    bregs = lambda q: f"b{q}"
    L = [f".reg .f32 b<{k}>, fo<{k}>, c;", WIDE_TEMPS, DIV_TEMPS, PAIR_TEMPS, TRIG_TEMPS, ".reg .pred q;",
         ".reg .u32 ux, uy, uz, uw, vx, vy, vz, vw, pa, pb;",
         f"mov.b32 ux, {CUR[0]}; mov.b32 uy, {CUR[1]}; mov.b32 uz, {CUR[2]}; mov.b32 uw, {CUR[3]};"]
    entry = {(1, 0): "S", (0, 0): "L", (0, 1): "F", (1, 1): "G"}
    cold = []           # the DIV arms' exact paths, kept out of the hot code
    for cur, nxt, here, there in (("u", "v", "A", "B"), ("v", "u", "B", "A")):
        x, y, z, w = (f"{cur}{f}" for f in "xyzw")
        L += [f"L{here}%=: setp.lt.s32 q, {w}, 0;", f"@q bra.uni D{here}%=;",
              f"ld.shared.v4.u32 {{{nxt}x, {nxt}y, {nxt}z, {nxt}w}}, [%0+16];",
              "add.u32 %0, %0, 16;", f"mov.b32 c, {y};"]
        nxt_jump = [f"add.u32 {PT}, {base}, {z};", f"bra.uni L{there}%=;"]
        targets = []
        for idx in range(64):
            op, cst, f1, sp = idx & 7, (idx >> 3) & 1, (idx >> 4) & 1, (idx >> 5) & 1
            if op == BCAST_OP and cst and not f1:
                targets.append(f"{'S' if sp else 'L'}{here}B_%=")
            elif op in TRIG_OPS and not cst:
                targets.append(f"{entry[(sp, f1)]}{here}{op}0_%=")
            elif op in ops:
                targets.append(f"{entry[(sp, f1)]}{here}{op}{cst}_%=")
            else:
                targets.append(f"X{here}%=")
        L += [f"T{here}%=: .branchtargets " + ", ".join(targets) + ";", f"brx.idx.uni {w}, T{here}%=;"]
        for op in ops:
            for cst in (0, 1):
                nm = f"{here}{op}{cst}_%="
                L.append(f"S{nm}: " + " ".join(st(PT)))
                L.append(f"L{nm}: " + " ".join([f"add.u32 pa, {base}, {x};"] + ld(A, "pa")))
                body = [] if cst else [f"add.u32 pb, {base}, {y};"] + ld(bregs, "pb")
                if op == 3:
                    hot, exact = div_group(k, bool(cst), A, bregs, nm)
                    body += hot
                    cold.append(f"V{nm}: " + " ".join(exact + [f"bra.uni W{nm};"]))
                elif op in X2 and k >= 2:
                    body += pair_body(k, op, bool(cst), A, bregs)
                else:
                    body += wide_body(k, op, bool(cst), a=A, b=bregs, t=A)
                L.append(f"F{nm}: " + " ".join(body + nxt_jump))
                L.append(f"G{nm}: " + " ".join(st(PT) + [f"bra.uni F{nm};"]))
        for op in TRIG_OPS:
            # unary: the operand comes in as src1 (x, fwd1); the math is shared
            nm = f"{here}{op}0_%="
            L.append(f"S{nm}: " + " ".join(st(PT)))
            L.append(f"L{nm}: " + " ".join([f"add.u32 pa, {base}, {x};"] + ld(A, "pa")))
            L.append(f"F{nm}: add.u32 {PT}, {base}, {z}; mov.u32 th, {1 if here == 'A' else 0}; "
                     f"mov.u32 tcos, {op - 4}; bra.uni R_%=;")
            L.append(f"G{nm}: " + " ".join(st(PT) + [f"bra.uni F{nm};"]))
        L.append(f"S{here}B_%=: " + " ".join(st(PT)))
        L.append(f"L{here}B_%=: " + " ".join([f"mov.f32 {A(q)}, c;" for q in range(k)] + nxt_jump))
    # The DIV arms' exact paths (each block ends in a jump back into its arm)
    # and the shared SIN/COS block and its exit (each ends in jumps to a loop
    # head or an exit).  They sit between the loop bodies (whose lines all
    # end in unconditional jumps) and the exit blocks, because DB falls
    # through into D%= and nothing may fall into them.
    L += cold
    L += trig_blocks(k, A)
    # Table entries no micro-op uses (the pre-pass never writes them) leave
    # too, after the dispatch has already stepped to the next micro-op: X
    # steps back so that the caller gets this micro-op and %0 at it.
    for here in ("A", "B"):
        L.append(f"X{here}%=: sub.u32 %0, %0, 16; bra.uni D{here}%=;")
    for here, cur in (("A", "u"), ("B", "v")):
        L.append(f"D{here}%=: " + " ".join(f"mov.b32 {LV[i]}, {cur}{f};" for i, f in enumerate("xyzw"))
                 + (" bra.uni D%=;" if here == "A" else ""))
    L.append("D%=:")
    text = "\\n\\t".join(L)
    outs = ", ".join(['"+r"(sp)'] + [f'"+f"(a[{q}])' for q in range(k)] + ['"+r"(pt)']
                     + [f'"=r"(lv.{f})' for f in "xyzw"])
    ins = ", ".join(['"r"(base)'] + [f'"r"(cur.{f})' for f in "xyzw"])
    return (f"    static __device__ __forceinline__ void run(uint32_t& sp, float (&a)[{k}], uint32_t& pt, "
            f"uint32_t base, uint4 cur, uint4& lv) {{\n"
            f'    asm volatile("{{\\n\\t{text}\\n\\t}}"\n'
            f'        : {outs}\n        : {ins}\n        : "memory");\n    }}\n')


def div_fast_function() -> str:
    """The wide loop's fast DIV path for one element as a standalone device
    function, from the same generator lines.  The library does not call it;
    tests/division_check.cu checks the fast path with it."""
    L = [DIV_TEMPS] + div_divisor_lines("%3") + div_fast_lines("%2", "%0")
    L[-1] = "mov.pred fall, fa;"
    L += ["selp.u32 %1, 1, 0, fall;"]
    text = "\\n\\t".join(L)
    return ("struct DivFast {\n"
            "    // q = a / b (1.0 for b == 0) when ok == 1, else q is not defined\n"
            "    static __device__ __forceinline__ float run(float a, float b, uint32_t& ok) {\n"
            "        float q;\n"
            f'        asm volatile("{{\\n\\t{text}\\n\\t}}"\n'
            '            : "=f"(q), "=r"(ok) : "f"(a), "f"(b));\n'
            "        return q;\n    }\n};\n")


HEADER_PATH = Path(__file__).resolve().parent / "dispatch_gen.cuh"


def render() -> str:
    out = ["// dispatch_gen.cuh -- GENERATED by gen_dispatch.py; do not edit by hand.",
           "// PTX jump tables (brx.idx) of the LGP interpreters; see gen_dispatch.py",
           "// for what each helper does.",
           "#pragma once", "#include <cstdint>", "", "namespace galop {", ""]
    out.append("template <int K, int PROFILE>\nstruct CheapOps;\n")
    for k in KS:
        for prof in PROFILES:
            out.append(f"template <>\nstruct CheapOps<{k}, {prof}> {{")
            out.append(cheap_table(k, prof))
            out.append("};\n")
    out.append("template <int K, int PROFILE>\nstruct WideOps;\n")
    for k in KS:
        for prof in PROFILES:
            out.append(f"template <>\nstruct WideOps<{k}, {prof}> {{")
            out.append(wide_ops(k, prof))
            out.append("};\n")
    out.append("template <int K, int PROFILE>\nstruct WideLoop;\n")
    for k in KS:
        for prof in PROFILES:
            out.append(f"template <>\nstruct WideLoop<{k}, {prof}> {{")
            out.append(wide_loop(k, prof))
            out.append("};\n")
    out.append(div_fast_function())
    out.append("}  // namespace galop\n")
    return "\n".join(out)


def write_if_changed(path: Path = HEADER_PATH) -> bool:
    """Rewrite the header when its text differs from render(); True if it did."""
    text = render()
    if path.exists() and path.read_text() == text:
        return False
    path.write_text(text)
    return True


def main() -> None:
    changed = write_if_changed()
    print(HEADER_PATH, "(rewritten)" if changed else "(up to date)")


if __name__ == "__main__":
    main()
