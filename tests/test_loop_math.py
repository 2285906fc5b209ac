"""The interpreter loop's generated math, executed on the CPU
(galop_b200/csrc/gen_dispatch.py).

A small evaluator of the PTX subset used by the loop's shared SIN/COS block
(trig_blocks) and the DIV arms' fast path (div_group) runs the generated
statements over arrays of lanes, with IEEE single-precision rounding (FMA
exactly, by integer arithmetic).  For every K, in both forms (per element
for K = 1, f32x2 pairs otherwise):
  - the SIN/COS block equals trig.cuh's host build (the oracle's
    TRIG_DEVICE mode) bit for bit on arguments below 2^17, and its
    slow-path vote fires exactly when an argument of some lane is 2^17 or
    more, infinite or NaN;
  - the DIV fast path equals IEEE division (1.0 for a zero divisor) on
    operands in its range, register and constant divisors, and its vote
    fails for an operand out of range.  rcp.approx is taken here as the
    correctly rounded reciprocal (flushed like .ftz); the instruction itself
    is checked on the B200 by tests/test_gpu_division.py;
  - the whole loop (jump tables, both copies, the S/L/F/G entry points,
    the exact-division blocks, the trig exits, the window end), run with a
    shared memory of words under a restatement of the kernel's pass for one
    warp, gives the oracle's per-case outputs on random and chained
    programs; a loop that does not end fails on a step limit.
"""
from __future__ import annotations

import functools
import re
import sys

import numpy as np
import pytest

from conftest import ROOT, bits

sys.path.insert(0, str(ROOT / "galop_b200" / "csrc"))
import gen_dispatch as G  # noqa: E402

M32 = 0xFFFFFFFF


# --- IEEE single precision ---------------------------------------------------------------

def _f(u: np.ndarray) -> np.ndarray:
    return np.asarray(u, dtype=np.uint32).view(np.float32)


def _u(x: np.ndarray) -> np.ndarray:
    return np.asarray(x, dtype=np.float32).view(np.uint32)


def _decode(b: int):
    s, e, m = b >> 31, (b >> 23) & 0xFF, b & 0x7FFFFF
    return (s, m, -149) if e == 0 else (s, m | 0x800000, e - 150)


def _round(num: int, e2: int) -> int:
    """num * 2^e2 rounded to the nearest float32 (ties to even), as bits."""
    s = 1 if num < 0 else 0
    n = abs(num)
    exp = max(e2 + n.bit_length() - 24, -149)
    shift = exp - e2
    if shift > 0:
        q, r = divmod(n, 1 << shift)
        half = 1 << (shift - 1)
        if r > half or (r == half and q & 1):
            q += 1
    else:
        q = n << -shift
    if q >= 1 << 24:
        q >>= 1
        exp += 1
    if q < 1 << 23:
        return (s << 31) | q
    e_field = exp + 150
    if e_field >= 255:
        return (s << 31) | 0x7F800000
    return (s << 31) | (e_field << 23) | (q - (1 << 23))


def _fma1(a: int, b: int, c: int) -> int:
    fa, fb, fc = (float(np.uint32(v).view(np.float32)) for v in (a, b, c))
    if not all(np.isfinite(v) for v in (fa, fb, fc)):
        with np.errstate(all="ignore"):
            return int(np.float32(fa * fb + fc).view(np.uint32))
    sa, ma, ea = _decode(a)
    sb, mb, eb = _decode(b)
    sc, mc, ec = _decode(c)
    sp, mp, ep = sa ^ sb, ma * mb, ea + eb
    if mp == 0 and mc == 0:
        return (sp & sc) << 31
    e = min(ep, ec)
    num = (-1 if sp else 1) * (mp << (ep - e)) + (-1 if sc else 1) * (mc << (ec - e))
    if num == 0:
        return 0
    return _round(num, e)


def fma(a, b, c) -> np.ndarray:
    return np.array([_fma1(int(x), int(y), int(z)) for x, y, z in zip(a, b, c)], dtype=np.uint32)


def _ftz(u: np.ndarray) -> np.ndarray:
    u = np.asarray(u, dtype=np.uint32)
    sub = ((u >> 23) & 0xFF) == 0
    return np.where(sub, u & 0x80000000, u).astype(np.uint32)


# --- the PTX subset -----------------------------------------------------------------------

class Ptx:
    """Registers hold arrays over lanes: uint32 for .f32/.b32/.u32 values,
    (lo, hi) pairs for .b64, bool for predicates.  Execution stops at the
    first branch that leaves straight-line code; `stopped` names it."""

    def __init__(self, n: int, regs: dict):
        self.n = n
        self.r = dict(regs)
        self.stopped = None

    def val(self, t: str):
        t = t.strip()
        if t.startswith("0f"):
            return np.full(self.n, int(t[2:], 16), dtype=np.uint32)
        if t.startswith("0x"):
            v = int(t, 16)
            if v > M32:
                return (np.full(self.n, v & M32, np.uint32), np.full(self.n, v >> 32, np.uint32))
            return np.full(self.n, v, dtype=np.uint32)
        if re.fullmatch(r"\d+", t):
            return np.full(self.n, int(t), dtype=np.uint32)
        return self.r[t]

    def run(self, statements: list[str]) -> None:
        for st in statements:
            if self.stopped:
                return
            self.step(st)

    def step(self, st: str) -> None:
        st = re.sub(r"^[A-Za-z_][\w%=]*:\s*", "", st.strip())
        if not st or st.startswith(".reg"):
            return
        m = re.match(r"(@!?\w+\s+)?(\S+)\s*(.*)$", st)
        guard, op, rest = m.group(1), m.group(2), m.group(3)
        if op.startswith("bra"):
            take = True
            if guard:
                p = self.r[guard.strip()[1:].lstrip("!")]
                assert p.all() or not p.any(), "a branch that is not uniform"
                take = bool(p[0]) != guard.strip().startswith("@!")
            if take:
                self.stopped = rest.strip()
            return
        args = [a.strip() for a in re.findall(r"\s*(\{[^}]*\}|[^,{]+)", rest)]
        getattr(self, "op_" + op.replace(".", "_"))(*args)

    # moves and bits
    def op_mov_b32(self, d, a): self.r[d] = self.val(a).copy()
    op_mov_f32 = op_mov_b32
    op_mov_u32 = op_mov_b32
    op_mov_pred = op_mov_b32

    def op_mov_b64(self, d, a):
        if d.startswith("{"):
            lo, hi = (x.strip() for x in d[1:-1].split(","))
            self.r[lo], self.r[hi] = self.val(a)
        elif a.startswith("{"):
            lo, hi = (x.strip() for x in a[1:-1].split(","))
            self.r[d] = (self.val(lo).copy(), self.val(hi).copy())
        else:
            self.r[d] = self.val(a)

    def op_abs_f32(self, d, a): self.r[d] = self.val(a) & np.uint32(0x7FFFFFFF)
    def op_neg_f32(self, d, a): self.r[d] = self.val(a) ^ np.uint32(0x80000000)
    def op_add_u32(self, d, a, b): self.r[d] = (self.val(a) + self.val(b)).astype(np.uint32)
    def op_sub_u32(self, d, a, b): self.r[d] = (self.val(a) - self.val(b)).astype(np.uint32)
    def op_and_b32(self, d, a, b): self.r[d] = self.val(a) & self.val(b)
    def op_or_b32(self, d, a, b): self.r[d] = self.val(a) | self.val(b)
    def op_xor_b32(self, d, a, b): self.r[d] = self.val(a) ^ self.val(b)
    def op_shl_b32(self, d, a, b): self.r[d] = (self.val(a) << self.val(b)).astype(np.uint32)

    # single precision, round to nearest even
    def _arith(self, fn, d, *xs):
        with np.errstate(all="ignore"):
            self.r[d] = _u(fn(*[_f(self.val(x)) for x in xs]))

    def op_add_rn_f32(self, d, a, b): self._arith(lambda x, y: x + y, d, a, b)
    def op_sub_rn_f32(self, d, a, b): self._arith(lambda x, y: x - y, d, a, b)
    def op_mul_rn_f32(self, d, a, b): self._arith(lambda x, y: x * y, d, a, b)
    def op_fma_rn_f32(self, d, a, b, c): self.r[d] = fma(self.val(a), self.val(b), self.val(c))

    def op_rcp_approx_ftz_f32(self, d, a):
        with np.errstate(all="ignore"):
            self.r[d] = _ftz(_u(np.float32(1.0) / _f(_ftz(self.val(a)))))

    def _pair(self, one, d, *xs):
        vals = [self.val(x) for x in xs]
        halves = []
        for h in (0, 1):
            names = []
            for i, v in enumerate(vals):
                self.r[f"_x{i}"] = v[h]
                names.append(f"_x{i}")
            one(f"_y{h}", *names)
            halves.append(self.r[f"_y{h}"])
        self.r[d] = tuple(halves)

    def op_add_rn_f32x2(self, d, a, b): self._pair(self.op_add_rn_f32, d, a, b)
    def op_sub_rn_f32x2(self, d, a, b): self._pair(self.op_sub_rn_f32, d, a, b)
    def op_mul_rn_f32x2(self, d, a, b): self._pair(self.op_mul_rn_f32, d, a, b)
    def op_fma_rn_f32x2(self, d, a, b, c): self._pair(self.op_fma_rn_f32, d, a, b, c)

    # predicates
    def _cmp(self, cmp: str, typ: str, a, b):
        if typ == "f32":
            x, y = _f(self.val(a)), _f(self.val(b))
            nan = np.isnan(x) | np.isnan(y)
            with np.errstate(all="ignore"):
                base = {"eq": x == y, "ne": x != y, "lt": x < y, "le": x <= y, "gt": x > y, "ge": x >= y}
            if cmp == "num":
                return ~nan
            if cmp.endswith("u"):
                return base[cmp[:-1]] | nan
            return base[cmp] & ~nan
        x, y = self.val(a), self.val(b)
        if typ == "s32":
            x, y = x.view(np.int32), y.view(np.int32)
        return {"eq": x == y, "ne": x != y, "lt": x < y, "le": x <= y, "gt": x > y, "ge": x >= y}[cmp]

    def __getattr__(self, name):
        m = re.fullmatch(r"op_setp_(\w+?)(?:_(and|or))?_(f32|u32|s32)", name)
        if m:
            cmp, bop, typ = m.groups()

            def setp(d, a, b, c=None):
                p = self._cmp(cmp, typ, a, b)
                if bop == "and":
                    p = p & self.r[c]
                elif bop == "or":
                    p = p | self.r[c]
                self.r[d] = p
            return setp
        raise AttributeError(name)

    def op_selp_f32(self, d, a, b, p): self.r[d] = np.where(self.r[p], self.val(a), self.val(b)).astype(np.uint32)
    op_selp_u32 = op_selp_f32
    def op_and_pred(self, d, a, b): self.r[d] = self.r[a] & self.r[b]
    def op_or_pred(self, d, a, b): self.r[d] = self.r[a] | self.r[b]
    def op_vote_sync_any_pred(self, d, p, mask): self.r[d] = np.full(self.n, bool(self.r[p].any()))
    def op_vote_sync_all_pred(self, d, p, mask): self.r[d] = np.full(self.n, bool(self.r[p].all()))


def statements(lines: list[str]) -> list[str]:
    return [s for ln in lines for s in ln.split(";") if s.strip()]


A = lambda q: f"%{1 + q}"      # the loop's result registers


# --- SIN / COS ----------------------------------------------------------------------------

def trig_arguments(rng, n: int) -> np.ndarray:
    parts = [rng.uniform(-4, 4, n // 4), rng.uniform(-2e3, 2e3, n // 4),
             np.ldexp(rng.uniform(0.5, 1.0, n // 4), rng.integers(-30, 17, n // 4)) * rng.choice([-1, 1], n // 4)]
    k = rng.integers(-80_000, 80_000, n // 8).astype(np.float64)
    parts.append((k * (np.pi / 2)).astype(np.float32).view(np.int32) + rng.integers(-2, 3, k.size).astype(np.int32))
    parts[-1] = parts[-1].view(np.float32)
    x = np.concatenate([p.astype(np.float32) for p in parts])
    x = np.concatenate([x, np.float32([0.0, -0.0, 1e-45, -1e-45, 1e-38, 131071.99, -131071.99])])
    x = x[np.abs(x) < 131072.0]
    return x[rng.permutation(x.size)][:n]


@pytest.mark.parametrize("k", G.KS)
@pytest.mark.parametrize("op", G.TRIG_OPS)
def test_trig_block_equals_trig_cuh(oracle_lib, k, op):
    rng = np.random.default_rng(100 * k + op)
    n = 256
    x = [trig_arguments(rng, n) for _ in range(k)]
    n = min(len(v) for v in x)
    x = [v[:n] for v in x]
    R, Z = G.trig_blocks(k, A)
    regs = {A(q): _u(x[q]) for q in range(k)}
    regs["tcos"] = np.full(n, op - 4, np.uint32)
    regs["th"] = np.ones(n, np.uint32)
    e = Ptx(n, regs)
    e.run(statements([R]))
    assert e.stopped in ("LB%=", "LA%="), e.stopped          # no slow-path exit
    dev = oracle_lib.Oracle(oracle_lib.PROFILE_REF, 8, trig=oracle_lib.TRIG_DEVICE)
    for q in range(k):
        want = dev.apply_op_n(op, x[q], x[q])
        assert np.array_equal(e.r[A(q)], bits(want)), (k, op, q)
    assert Z.startswith("Z_%=:")


@pytest.mark.parametrize("k", G.KS)
def test_trig_block_leaves_for_the_slow_path(k):
    rng = np.random.default_rng(7 + k)
    n = 32
    for big in (131072.0, -3e38, np.inf, np.nan):
        x = [rng.uniform(-3, 3, n).astype(np.float32) for _ in range(k)]
        x[k - 1][n // 2] = big
        regs = {A(q): _u(x[q]) for q in range(k)}
        regs["tcos"] = np.zeros(n, np.uint32)
        regs["th"] = np.zeros(n, np.uint32)
        e = Ptx(n, regs)
        e.run(statements([G.trig_blocks(k, A)[0]]))
        assert e.stopped == "Z_%=", (k, big)
        for q in range(k):                   # the operands are left in place
            assert np.array_equal(e.r[A(q)], _u(x[q]))


# --- DIV ----------------------------------------------------------------------------------

def in_range(rng, n: int) -> np.ndarray:
    v = np.ldexp(rng.uniform(1.0, 2.0, n), rng.integers(-62, 62, n)) * rng.choice([-1, 1], n)
    return v.astype(np.float32)


def ieee_div(a: np.ndarray, b: np.ndarray) -> np.ndarray:
    with np.errstate(all="ignore"):
        return np.where(b != 0, a / b, np.float32(1.0)).astype(np.float32)


@pytest.mark.parametrize("k", G.KS)
@pytest.mark.parametrize("const", [False, True])
def test_div_fast_path_equals_ieee_division(k, const):
    rng = np.random.default_rng(30 + k + 10 * const)
    n = 256
    a = [in_range(rng, n) for _ in range(k)]
    for q in range(k):
        a[q][rng.choice(n, 8, replace=False)] = rng.choice(np.float32([0.0, -0.0]), 8)
    if const:
        c = np.float32(in_range(rng, 1)[0])
        b = [np.full(n, c, np.float32) for _ in range(k)]
    else:
        b = [in_range(rng, n) for _ in range(k)]
        for q in range(k):
            b[q][rng.choice(n, 4, replace=False)] = np.float32(0.0)
    hot, _ = G.div_group(k, const, A, lambda q: f"b{q}", "A30_%=")
    regs = {A(q): _u(a[q]) for q in range(k)}
    regs.update({f"b{q}": _u(b[q]) for q in range(k)})
    regs["c"] = _u(b[0])
    e = Ptx(n, regs)
    e.run(statements(hot))
    assert e.stopped is None                 # every lane in range: no exact path
    for q in range(k):
        assert np.array_equal(e.r[A(q)], bits(ieee_div(a[q], b[q]))), (k, const, q)


@pytest.mark.parametrize("k", G.KS)
def test_div_vote_fails_out_of_range(k):
    rng = np.random.default_rng(50 + k)
    n = 32
    for bad_a, bad_b in ((np.float32(1e-30), None), (np.float32(3e20), None), (None, np.float32(1e30)),
                         (None, np.float32(np.inf)), (np.float32(np.nan), None)):
        a = [in_range(rng, n) for _ in range(k)]
        b = [in_range(rng, n) for _ in range(k)]
        if bad_a is not None:
            a[k - 1][3] = bad_a
        if bad_b is not None:
            b[k - 1][3] = bad_b
        hot, _ = G.div_group(k, False, A, lambda q: f"b{q}", "A30_%=")
        regs = {A(q): _u(a[q]) for q in range(k)}
        regs.update({f"b{q}": _u(b[q]) for q in range(k)})
        e = Ptx(n, regs)
        e.run(statements(hot))
        assert e.stopped == "VA30_%=", (k, bad_a, bad_b)


# --- the whole loop -----------------------------------------------------------------------

@functools.lru_cache(maxsize=None)
def loop_statements(k: int, profile: int):
    """The WideLoop asm block of (k, profile), parsed by parse_asm."""
    return parse_asm(G.wide_loop(k, profile))


def parse_asm(text: str):
    """The one asm block of a generated function: executable statements as
    (guard, op, operands), the statement index of every label, and the jump
    tables."""
    body = re.split(r'asm(?: volatile)?\("\{\\n\\t', text, maxsplit=1)[1].split('\\n\\t}"', 1)[0]
    prog, labels, tables = [], {}, {}
    for ln in body.split("\\n\\t"):
        for st in ln.split(";"):
            st = st.strip()
            while True:
                m = re.match(r"^([A-Za-z_][\w%=]*):\s*(.*)$", st)
                if not m:
                    break
                lab, st = m.group(1), m.group(2).strip()
                if st.startswith(".branchtargets"):
                    tables[lab] = [t.strip() for t in st[len(".branchtargets"):].split(",")]
                    st = ""
                    break
                labels[lab] = len(prog)
            if st and not st.startswith(".reg"):
                m = re.match(r"(@!?\w+\s+)?(\S+)\s*(.*)$", st)
                args = [a.strip() for a in re.findall(r"\s*(\{[^}]*\}|\[[^\]]*\]|[^,{\[]+)", m.group(3))]
                prog.append(((m.group(1) or "").strip(), m.group(2), tuple(args)))
    return prog, labels, tables


class Loop(Ptx):
    """Ptx with control flow and a shared memory of 32-bit words."""

    def __init__(self, k: int, profile: int, n: int, regs: dict, mem: np.ndarray, parsed=None):
        super().__init__(n, regs)
        self.prog, self.labels, self.tables = parsed or loop_statements(k, profile)
        self.mem = mem
        self.hits = set()                  # jump-table entries taken

    def execute(self, limit: int = 100_000) -> None:
        pc, steps = 0, 0
        while pc < len(self.prog):
            steps += 1
            assert steps < limit, "the loop does not end"
            guard, op, args = self.prog[pc]
            pc += 1
            p = None
            if guard:
                p = self.r[guard[1:].lstrip("!")]
                if guard.startswith("@!"):
                    p = ~p
            if op.startswith("bra"):
                if p is not None:
                    assert p.all() or not p.any(), "a branch that is not uniform"
                if p is None or p[0]:
                    pc = self.labels[args[0]]
                continue
            if op in ("brx.idx.uni", "brx.idx"):
                idx = self.val(args[0])
                assert (idx == idx[0]).all(), "a jump that is not uniform"
                target = self.tables[args[1]][int(idx[0])]
                self.hits.add(target)
                pc = self.labels[target]
                continue
            if p is None:
                getattr(self, "op_" + op.replace(".", "_"))(*args)
            else:                           # a guarded instruction: per-lane result
                old = self.r.get(args[0])
                getattr(self, "op_" + op.replace(".", "_"))(*args)
                self.r[args[0]] = np.where(p, self.r[args[0]], old).astype(np.uint32)

    def _addr(self, a: str) -> np.ndarray:
        reg, _, off = a.strip()[1:-1].partition("+")
        return (self.val(reg).astype(np.int64) + int(off or 0)) // 4

    def _regs(self, t: str) -> list[str]:
        t = t.strip()
        return [x.strip() for x in t[1:-1].split(",")] if t.startswith("{") else [t]

    def _ld(self, d, a):
        w = self._addr(a)
        for i, name in enumerate(self._regs(d)):
            self.r[name] = self.mem[w + i].copy()

    def _st(self, a, s):
        w = self._addr(a)
        for i, name in enumerate(self._regs(s)):
            self.mem[w + i] = self.val(name)

    op_ld_shared_v4_u32 = op_ld_shared_v4_f32 = op_ld_shared_v2_f32 = op_ld_shared_f32 = _ld
    op_st_shared_v4_f32 = op_st_shared_v2_f32 = op_st_shared_f32 = _st

    def op_set_lt_f32_f32(self, d, a, b):
        with np.errstate(all="ignore"):
            self.r[d] = np.where(_f(self.val(a)) < _f(self.val(b)), np.uint32(0x3F800000), np.uint32(0))

    def op_set_gt_f32_f32(self, d, a, b):
        with np.errstate(all="ignore"):
            self.r[d] = np.where(_f(self.val(a)) > _f(self.val(b)), np.uint32(0x3F800000), np.uint32(0))

    def op_div_rn_f32(self, d, a, b): self._arith(lambda x, y: x / y, d, a, b)


END = 0xFFFFFFFF


def micro_ops(words: np.ndarray, S: int, consts: np.ndarray, profile: int = 0) -> np.ndarray:
    """The 16-byte micro-ops of a raw program without folding or
    renaming (register r at slot r): encode_wide, the forwarding flags as
    the folding pass sets them (fwd1/fwd2 where the operand is the previous
    destination; store_prev unless the next instruction is the previous
    result's only reader, through its forwarded operand -- fold.cuh's
    needs_store, with the output register read after the last
    instruction), and SIN/COS of a register in the loop's unary form."""
    ins = []
    for w in (int(x) for x in words):
        op, dest, s1, s2, c = w & 7, (w >> 8) & 15, (w >> 16) & 15, (w >> 24) & 15, w >> 31
        ins.append((op, dest, s1, s2, c, op in (4, 5) or (profile == 1 and op in (6, 7))))
    n = len(ins)
    live_after = [set() for _ in range(n)]
    live = {0}
    for j in range(n - 1, -1, -1):
        live_after[j] = set(live)
        op, dest, s1, s2, c, unary = ins[j]
        live = (live - {dest}) | ({s1} if not unary else set()) | ({s2} if not c else set())
    u = []
    for j, (op, dest, s1, s2, c, unary) in enumerate(ins):
        flags = 0
        if j > 0:
            d = ins[j - 1][1]
            fwd = (not unary and s1 == d) or (unary and not c and s2 == d)
            if fwd:
                flags |= 64 if unary else 16
            loads_d = not unary and not c and s2 == d
            read_later = d != dest and d in live_after[j]
            if not (fwd and not loads_d and not read_later):
                flags |= 32
        y = int(consts[s2].view(np.uint32)) if c else s2 * S
        if op in (4, 5) and not c:
            u.append([y, 0, dest * S, op | (16 if flags & 64 else 0) | (flags & 32)])
        else:
            u.append([0 if unary else s1 * S, y, dest * S, op | (c << 3) | flags | (0x80000000 if unary else 0)])
    return np.array(u, dtype=np.uint32).reshape(-1, 4)


def emulate(k: int, u: np.ndarray, X: np.ndarray, init: dict, out_slot: int, unary, profile: int = 0):
    """interp_wide_kernel's pass over 32*K cases for one warp, with the
    generated loop emulated: a 16-slot register file whose slot s starts as
    input column init[s] (-1: zero), the micro-ops u staged in 32-entry
    windows, the caller's handling of the micro-ops that leave the loop, and
    the output taken from the result registers when the last instruction
    wrote the output slot.  Returns the per-case outputs and the jump-table
    entries taken."""
    nslot, V, S = 16, min(k, 4), 128 * k
    stage = nslot * S
    mem = np.zeros((stage + 34 * 16) // 4, dtype=np.uint32)
    lanes = np.arange(32)
    base = (lanes * V * 4).astype(np.uint32)

    def slot_words(r):   # word index of element e of every lane in slot r
        return [(base.astype(np.int64) + r * S + (e // V) * 128 * V + (e % V) * 4) // 4 for e in range(k)]

    case = [(e // V) * 32 * V + lanes * V + (e % V) for e in range(k)]
    for r, col in init.items():
        for e, w in enumerate(slot_words(r)):
            mem[w] = _u(X[case[e], col]) if col >= 0 else 0
    hits = set()
    A = [np.zeros(32, np.uint32) for _ in range(k)]
    pt = np.zeros(32, np.uint32)
    for w0 in range(0, len(u), 32):
        win = u[w0:w0 + 32]
        mem[stage // 4: stage // 4 + 4 * len(win)] = win.ravel()
        mem[stage // 4 + 4 * len(win): stage // 4 + 4 * len(win) + 4] = [0, 0, 0, END]
        sp = stage
        while True:
            cur = mem[sp // 4: sp // 4 + 4]
            regs = {"%0": np.full(32, sp, np.uint32), f"%{k + 1}": pt, f"%{k + 6}": base}
            regs.update({f"%{1 + q}": A[q] for q in range(k)})
            regs.update({f"%{k + 7 + i}": np.full(32, cur[i], np.uint32) for i in range(4)})
            e = Loop(k, profile, 32, regs, mem)
            e.execute()
            hits |= e.hits
            sp = int(e.r["%0"][0])
            A = [e.r[f"%{1 + q}"] for q in range(k)]
            pt = e.r[f"%{k + 1}"]
            lv = [int(e.r[f"%{k + 2 + i}"][0]) for i in range(4)]
            if lv[3] == END:
                break
            op = lv[3] & 7
            if not lv[3] & 0x80000000:     # a SIN/COS left for the slow path
                b = A
            else:
                if lv[3] & 32:
                    for q, wq in enumerate(slot_words(0)):
                        mem[(pt.astype(np.int64) - base) // 4 + wq] = A[q]
                if lv[3] & 8:
                    b = [np.full(32, lv[1], np.uint32) for _ in range(k)]
                elif lv[3] & 64:
                    b = A
                else:
                    b = [mem[w + lv[1] // 4] for w in slot_words(0)]
            A = [_u(unary(op, _f(b[q]))) for q in range(k)]
            pt = (base + lv[2]).astype(np.uint32)
            sp += 16
    out_addr = base + out_slot * S
    if len(u) and (pt == out_addr).all():
        o = A
    else:
        o = [mem[w] for w in slot_words(out_slot)]
    res = np.empty(32 * k, np.float32)
    for e in range(k):
        res[case[e]] = _f(o[e])
    return res, hits


def run_program(k: int, words: np.ndarray, X: np.ndarray, unary, profile: int = 0):
    """A raw program without folding or renaming (register r in slot r)
    through emulate()."""
    from galop_b200 import REF_CONSTANTS_16
    u = micro_ops(words, 128 * k, REF_CONSTANTS_16, profile)
    init = {r: (r if r < X.shape[1] else -1) for r in range(16)}
    return emulate(k, u, X, init, 0, unary, profile)


def chained(rng, L: int) -> np.ndarray:
    """L instructions over registers 0-5, each reading the previous result
    with probability 0.6 (forwarded src1, or a unary op's operand) and
    otherwise an earlier register, the last one writing the output
    register: nearly every instruction reaches the output, stored results
    are read again further down."""
    from galop_b200 import workloads as W
    prev, ins = 0, []
    for _ in range(L):
        s1 = prev if rng.random() < 0.6 else int(rng.integers(0, 6))
        s2 = prev if rng.random() < 0.3 else int(rng.integers(0, 6))
        ins.append([int(rng.integers(0, 8)), int(rng.integers(0, 6)), s1, s2, int(rng.random() < 0.2)])
        prev = ins[-1][1]
    ins[-1][1] = 0
    return W.encode(*np.array(ins, dtype=np.int64).T)


@pytest.mark.parametrize("k", G.KS)
@pytest.mark.parametrize("profile", [0, 1])
def test_whole_loop_against_the_oracle(oracle_lib, k, profile):
    """Random REF programs (every op, register and constant operands) and
    chained ones (forwarded operands, deferred stores read back), of 1 to 80
    instructions across 32-instruction windows, through the emulated loop
    and its caller equal the oracle with trig.cuh's host build, per case,
    bit for bit, until every jump-table entry of both loop copies that
    these micro-ops can select has run.  A few cases hold arguments for the
    slow trig path and operands for the exact division.  The BJ profile's
    EXP/LOG leave the loop for the caller, which evaluates them here with
    the oracle's own functions."""
    from galop_b200 import workloads as W
    rng = np.random.default_rng(90 + k + 7 * profile)
    dev = oracle_lib.Oracle(profile, 16, trig=oracle_lib.TRIG_DEVICE)
    unary = lambda op, x: dev.apply_op_n(op, x, x)
    n = 32 * k
    X = rng.uniform(-3, 3, (n, 4)).astype(np.float32)
    X[rng.choice(n, 3, replace=False), 1] = np.float32([2e5, 1e-30, 0.0])
    progs = [W.random_words(rng, L, 16) for L in (1, 2, 7, 31, 32, 33, 80)]
    # every entry of both copies' tables that these micro-ops can select:
    # no broadcast arms (nothing is folded here), and copy B's L entries
    # (neither flag) never run -- such a micro-op is the first of a pass or
    # the first after the loop was left, and those run in copy A
    _, _, tables = loop_statements(k, profile)
    reachable = {t for tab in tables.values() for t in tab
                 if not t.startswith(("X", "LB")) and "B_" not in t}
    hit = set()
    i = 0
    while True:
        words = progs[i] if i < len(progs) else chained(rng, int(rng.integers(3, 80)))
        i += 1
        want = dev.case_outputs(words, X)
        got, h = run_program(k, words, X, unary, profile)
        hit |= h
        same = (bits(got) == bits(want)) | (np.isnan(got) & np.isnan(want))
        assert same.all(), (k, len(words), int((~same).sum()))
        if i >= len(progs) and hit >= reachable:
            break
        assert i < 400, sorted(reachable - hit)[:8]


@pytest.mark.parametrize("k", G.KS)
@pytest.mark.parametrize("profile", [0, 1])
def test_cheap_tables(k, profile):
    """The 32-bit micro-op interpreter's jump tables (CheapOps, dispatch 2 and
    the no-allocation entry point): each single-instruction op of the
    profile gives IEEE single-precision ADD/SUB/MUL and the 1.0/0.0 LT/GT
    (false on NaN), per element."""
    parsed = parse_asm(G.cheap_table(k, profile))
    rng = np.random.default_rng(k + 10 * profile)
    n = 64
    a = [rng.standard_normal(n).astype(np.float32) * 10 for _ in range(k)]
    b = [rng.standard_normal(n).astype(np.float32) * 10 for _ in range(k)]
    for q in range(k):
        a[q][:4] = np.float32([np.nan, 0.0, -0.0, np.inf])
        b[q][2:6] = np.float32([0.0, np.nan, 1e-45, -np.inf])
    want = {0: lambda x, y: x + y, 1: lambda x, y: x - y, 2: lambda x, y: x * y,
            6: lambda x, y: np.where(x < y, np.float32(1), np.float32(0)),
            7: lambda x, y: np.where(x > y, np.float32(1), np.float32(0))}
    for op in G.PROFILES[profile]:
        regs = {f"%{k}": np.full(n, op, np.uint32)}
        regs.update({f"%{k + 1 + q}": _u(a[q]) for q in range(k)})
        regs.update({f"%{2 * k + 1 + q}": _u(b[q]) for q in range(k)})
        e = Loop(k, profile, n, regs, np.zeros(4, np.uint32), parsed=parsed)
        e.execute()
        for q in range(k):
            with np.errstate(all="ignore"):
                w = want[op](a[q], b[q]).astype(np.float32)
            got = _f(e.r[f"%{q}"])
            assert ((bits(got) == bits(w)) | (np.isnan(got) & np.isnan(w))).all(), (k, profile, op, q)


@pytest.mark.parametrize("k", G.KS)
@pytest.mark.parametrize("profile", [0, 1])
def test_one_instruction_tables(k, profile):
    """The trace interpreter's one-instruction tables (WideOps): every arm of
    the profile, register and constant src2, and the broadcast arm, read the
    operands from the shared-memory register file and store the IEEE result
    (DIV: b != 0 ? a / b : 1.0) in the destination's slot."""
    parsed = parse_asm(G.wide_ops(k, profile))
    rng = np.random.default_rng(200 + k + 10 * profile)
    V, S = min(k, 4), 128 * k
    lanes = np.arange(32)
    base = (lanes * V * 4).astype(np.uint32)

    def words(slot):
        return [(base.astype(np.int64) + slot * S + (e // V) * 128 * V + (e % V) * 4) // 4 for e in range(k)]

    def div(x, y):
        with np.errstate(all="ignore"):
            return np.where(y != 0, x / y, np.float32(1.0)).astype(np.float32)

    want = {0: lambda x, y: x + y, 1: lambda x, y: x - y, 2: lambda x, y: x * y, 3: div,
            6: lambda x, y: np.where(x < y, np.float32(1), np.float32(0)),
            7: lambda x, y: np.where(x > y, np.float32(1), np.float32(0))}
    c = np.float32(-2.5)
    for op in sorted(G.PROFILES[profile] + (3,)):
        for const in (0, 1):
            mem = np.zeros(4 * S // 4, np.uint32)
            a = [rng.standard_normal(32).astype(np.float32) * 4 for _ in range(k)]
            b = [rng.standard_normal(32).astype(np.float32) * 4 for _ in range(k)]
            for q in range(k):
                a[q][:3] = np.float32([0.0, -0.0, np.nan])
                b[q][1:5] = np.float32([0.0, np.nan, -0.0, np.inf])
                mem[words(1)[q]] = _u(a[q])
                mem[words(2)[q]] = _u(b[q])
            regs = {"%0": np.full(32, op | (const << 3), np.uint32), "%1": base + 1 * S, "%2": base + 2 * S,
                    "%3": base + 3 * S, "%4": np.full(32, int(np.float32(c).view(np.uint32)), np.uint32)}
            e = Loop(k, profile, 32, regs, mem, parsed=parsed)
            e.execute()
            for q in range(k):
                with np.errstate(all="ignore"):
                    w = want[op](a[q], np.full(32, c, np.float32) if const else b[q]).astype(np.float32)
                got = _f(mem[words(3)[q]])
                assert ((bits(got) == bits(w)) | (np.isnan(got) & np.isnan(w))).all(), (k, profile, op, const, q)
    mem = np.zeros(4 * S // 4, np.uint32)
    regs = {"%0": np.full(32, G.BCAST_OP | 8, np.uint32), "%1": base + S, "%2": base + 2 * S, "%3": base + 3 * S,
            "%4": np.full(32, int(np.float32(c).view(np.uint32)), np.uint32)}
    Loop(k, profile, 32, regs, mem, parsed=parsed).execute()
    for q in range(k):
        assert (_f(mem[words(3)[q]]) == c).all()
