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
    is checked on the B200 by tests/test_gpu_division.py.
"""
from __future__ import annotations

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
