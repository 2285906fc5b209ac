"""Seeded synthetic workloads: random LGP populations and regression datasets.

Programs use the reference's encoding (src/ISA.h:20-41); random words are
masked field by field exactly as ``ISA::encode_from_random`` does
(src/ISA.h:106-138).  ``structured_population`` controls the effective
(non-intron) fraction by construction: it draws an effective/intron mask per
instruction and then, walking backwards with the liveness rule of
src/Introns.h:28-46, picks each destination inside (effective) or outside
(intron) the live set.

The regression target of a dataset is the output of a seeded random program
whose every instruction is effective.  ``program_outputs`` below computes it
with numpy while the dataset is built; it is workload synthesis only -- the
evaluator never calls it and it is not an evaluation path.

The configurations reproduce the shapes and value distributions of the
workloads the reference is compared on (population sizes, length
distributions, feature counts and ranges, case counts, noise); all data are
synthetic and seeded.
"""
from __future__ import annotations

from dataclasses import dataclass, field
from typing import Optional

import numpy as np

from . import PROFILE_BJ, PROFILE_REF, REF_CONSTANTS_8, REF_CONSTANTS_16

OP_ADD, OP_SUB, OP_MUL, OP_DIV, OP_SIN, OP_COS, OP_6, OP_7 = range(8)


@dataclass
class IsaSpec:
    profile: int = PROFILE_REF
    num_registers: int = 8
    input_protect: bool = False
    constants: np.ndarray = field(default=None)

    def __post_init__(self):
        if self.constants is None:
            self.constants = REF_CONSTANTS_16 if self.num_registers == 16 else REF_CONSTANTS_8
        self.constants = np.asarray(self.constants, dtype=np.float32)

    @property
    def output_reg(self) -> int:
        return self.num_registers // 2 if self.input_protect else 0

    def unary(self, op: np.ndarray) -> np.ndarray:
        u = (op == OP_SIN) | (op == OP_COS)
        if self.profile == PROFILE_BJ:
            u |= (op == OP_6) | (op == OP_7)
        return u


def encode(op, dest, src1, src2, is_const) -> np.ndarray:
    """Field values -> instruction words (src/ISA.h:150-166 layout)."""
    op = np.asarray(op, dtype=np.uint32)
    w = (op & 7) | (np.asarray(dest, np.uint32) << 8) | (np.asarray(src1, np.uint32) << 16)
    w |= (np.asarray(src2, np.uint32) & 0x7F) << 24
    w |= np.asarray(is_const, np.uint32) << 31
    return w.astype(np.uint32)


def mask_random_words(raw: np.ndarray, num_registers: int) -> np.ndarray:
    """ISA::encode_from_random (src/ISA.h:106-138) on an array of uint32."""
    raw = np.asarray(raw, dtype=np.uint32)
    m = np.uint32(num_registers - 1)
    keep = (np.uint32(7) | (m << np.uint32(8)) | (m << np.uint32(16)) | (m << np.uint32(24))
            | (np.uint32(0x80) << np.uint32(24)))
    return raw & keep


def random_words(rng: np.random.Generator, n: int, num_registers: int) -> np.ndarray:
    if n < (1 << 24):
        return mask_random_words(rng.integers(0, 2**32, size=n, dtype=np.uint64).astype(np.uint32), num_registers)
    # large populations: 32-bit draws in chunks, masked in place (bounded memory)
    out = np.empty(n, dtype=np.uint32)
    step = 1 << 26
    for i in range(0, n, step):
        m = min(step, n - i)
        out[i:i + m] = mask_random_words(rng.integers(0, 2**32, size=m, dtype=np.uint32), num_registers)
    return out


def csr_offsets(lengths: np.ndarray) -> np.ndarray:
    off = np.zeros(len(lengths) + 1, dtype=np.int64)
    np.cumsum(np.asarray(lengths, dtype=np.int64), out=off[1:])
    return off


def uniform_lengths(rng, n, lo, hi) -> np.ndarray:
    return rng.integers(lo, hi + 1, size=n, dtype=np.int64)


def log_uniform_lengths(rng, n, lo, hi) -> np.ndarray:
    v = np.exp(rng.uniform(np.log(lo), np.log(hi + 1), size=n))
    return np.clip(np.floor(v).astype(np.int64), lo, hi)


def random_population(rng, lengths, num_registers: int):
    """Uniform random words (any word is a valid instruction)."""
    off = csr_offsets(lengths)
    return random_words(rng, int(off[-1]), num_registers), off


_SELECT_CACHE: dict = {}


def _select_tables(bits_: int):
    """popcount[m] and select[m, k] = index of the k-th set bit of m, for
    all masks m < 2**bits_."""
    if bits_ not in _SELECT_CACHE:
        m = np.arange(1 << bits_, dtype=np.uint32)
        bitmat = ((m[:, None] >> np.arange(bits_, dtype=np.uint32)) & 1).astype(bool)
        pop = bitmat.sum(1).astype(np.int64)
        sel = np.zeros((1 << bits_, bits_), dtype=np.uint8)
        cum = np.cumsum(bitmat, axis=1)
        for k in range(bits_):
            sel[:, k] = np.argmax(cum > k, axis=1)
        _SELECT_CACHE[bits_] = (pop, sel)
    return _SELECT_CACHE[bits_]


def structured_population(rng, lengths, isa: IsaSpec, eff_frac: float, reg_limit: Optional[int] = None,
                          const_limit: Optional[int] = None, ops=None):
    """Random programs whose effective fraction is ``eff_frac`` by
    construction.  Walking each program backwards with the liveness rule of
    src/Introns.h:28-46, an instruction drawn effective takes its destination
    from the live set, an intron from outside it; opcodes, sources and the
    constant flag are uniform (an effective unary op that would leave nothing
    live reads a register instead of a constant).  The last instruction is
    always effective.  ``ops`` restricts the opcodes drawn (default: all 8).
    Vectorised over programs: programs are sorted by length, so at backward
    step t the programs still running are a prefix."""
    assert not isa.input_protect, "structured programs assume the default dest decode"
    lengths = np.asarray(lengths, dtype=np.int64)
    nr = isa.num_registers
    rl = reg_limit or nr
    cl = const_limit or nr
    pop, sel = _select_tables(rl)
    full = np.uint32((1 << rl) - 1)
    off = csr_offsets(lengths)
    words = np.empty(int(off[-1]), dtype=np.uint32)
    order = np.argsort(-lengths, kind="stable")
    Ls = lengths[order]
    base = off[order] + Ls - 1            # position of the last instruction
    live = np.full(order.shape[0], np.uint32(1 << isa.output_reg), dtype=np.uint32)
    neg = -Ls
    Lmax = int(Ls[0]) if Ls.size else 0
    op_set = np.arange(8, dtype=np.uint32) if ops is None else np.asarray(ops, dtype=np.uint32)
    for t in range(Lmax):
        a = int(np.searchsorted(neg, -t, side="left"))     # programs with L > t
        if a == 0:
            break
        lv = live[:a]
        op = op_set[rng.integers(0, op_set.size, size=a)]
        s1 = rng.integers(0, rl, size=a, dtype=np.uint32)
        kc = rng.random(a) < 0.5
        s2r = rng.integers(0, rl, size=a, dtype=np.uint32)
        s2c = rng.integers(0, cl, size=a, dtype=np.uint32)
        want = (rng.random(a) < eff_frac) | (t == 0)
        n_live = pop[lv]
        want &= n_live > 0
        want |= n_live == rl
        pool = np.where(want, lv, ~lv & full)
        k = (rng.random(a) * pop[pool]).astype(np.int64)
        dest = sel[pool, k].astype(np.uint32)
        unary = (op == OP_SIN) | (op == OP_COS)
        if isa.profile == PROFILE_BJ:
            unary |= (op == OP_6) | (op == OP_7)
        kc &= ~(want & unary & (n_live == 1))
        s2 = np.where(kc, s2c, s2r)
        one = np.uint32(1)
        upd = np.where(want, lv & ~(one << dest), lv)
        upd |= np.where(want & ~unary, one << s1, np.uint32(0))
        upd |= np.where(want & ~kc, one << s2, np.uint32(0))
        live[:a] = upd
        words[base[:a] - t] = encode(op, dest, s1, s2, kc)
    return words, off


def effective_program(rng, n_eff: int, isa: IsaSpec, num_inputs: int, reg_limit: Optional[int] = None,
                      const_limit: Optional[int] = None, ops=None) -> np.ndarray:
    """A program of n_eff instructions, all effective, that reads at least
    one input register."""
    nr = isa.num_registers
    rl = reg_limit or nr
    cl = const_limit or nr
    ops = np.arange(8) if ops is None else np.asarray(ops)
    for _ in range(1000):
        live = np.zeros(nr, dtype=bool)
        live[isa.output_reg] = True
        prog = []
        for _i in range(n_eff):
            cands = np.nonzero(live[:rl])[0]
            dest = int(rng.choice(cands))
            op = int(rng.choice(ops))
            kc = bool(rng.random() < 0.3)
            s1 = int(rng.integers(0, rl))
            s2 = int(rng.integers(0, cl if kc else rl))
            live[dest] = False
            if not isa.unary(np.array([op]))[0]:
                live[s1] = True
            if not kc:
                live[s2] = True
            if not live[:rl].any():
                live[isa.output_reg] = True
            prog.append(int(encode(op, dest, s1, s2, kc)))
        prog = np.array(prog[::-1], dtype=np.uint32)
        if live[:num_inputs].any():
            return prog
    return prog


def program_outputs(prog: np.ndarray, X: np.ndarray, isa: IsaSpec) -> np.ndarray:
    """Output r[OUTPUT_REG] of one program on every case (numpy, float32);
    used only to synthesise regression targets."""
    n, k = X.shape
    nr = isa.num_registers
    r = np.zeros((nr, n), dtype=np.float32)
    r[:k] = X.T
    with np.errstate(all="ignore"):
        for w in np.asarray(prog, dtype=np.uint32):
            w = int(w)
            op = w & 7
            d = (w >> 8) & (nr - 1)
            if isa.input_protect:
                d = isa.output_reg + ((w >> 8) & ((nr - 1) >> 1))
            a = r[(w >> 16) & (nr - 1)]
            i2 = (w >> 24) & (nr - 1)
            b = np.full(n, isa.constants[i2], dtype=np.float32) if (w >> 31) else r[i2]
            if op == OP_ADD:
                v = a + b
            elif op == OP_SUB:
                v = a - b
            elif op == OP_MUL:
                v = a * b
            elif op == OP_DIV:
                v = np.where(b != 0, a / np.where(b != 0, b, 1), np.float32(1))
            elif op == OP_SIN:
                v = np.sin(b)
            elif op == OP_COS:
                v = np.cos(b)
            elif op == OP_6:
                v = np.exp(b) if isa.profile == PROFILE_BJ else (a < b).astype(np.float32)
            else:
                v = (np.where(b != 0, np.log(np.abs(np.where(b != 0, b, 1))), np.float32(0))
                     if isa.profile == PROFILE_BJ else (a > b).astype(np.float32))
            r[d] = v.astype(np.float32)
    return r[isa.output_reg].copy()


def regression_target(rng, X: np.ndarray, isa: IsaSpec, n_eff: int, noise_sigma: float = 0.0,
                      scale: float = 1.0, reg_limit=None, const_limit=None, ops=None):
    """y = scale * f(x) + N(0, sigma^2) with f a random all-effective program;
    redrawn until f is finite and non-constant on the sample."""
    k = X.shape[1]
    for _ in range(200):
        prog = effective_program(rng, n_eff, isa, k, reg_limit, const_limit, ops)
        y = program_outputs(prog, X, isa)
        if np.all(np.isfinite(y)) and float(np.std(y)) > 1e-3 and float(np.max(np.abs(y))) < 1e6:
            break
    y = y.astype(np.float64)
    if scale != 1.0:
        y = (y - float(np.mean(y))) / max(float(np.std(y)), 1e-12) * scale
    if noise_sigma:
        y = y + rng.normal(0.0, noise_sigma, size=y.shape)
    return y.astype(np.float32), prog


@dataclass
class Workload:
    name: str
    isa: IsaSpec
    words: np.ndarray
    offsets: np.ndarray
    X: np.ndarray          # (N, k) case-major
    y: np.ndarray          # (N,)
    target_program: np.ndarray
    description: str = ""

    @property
    def n_programs(self) -> int:
        return self.offsets.shape[0] - 1

    @property
    def n_cases(self) -> int:
        return self.y.shape[0]

    def subsample(self, idx: np.ndarray) -> "Workload":
        idx = np.asarray(idx, dtype=np.int64)
        lens = self.offsets[idx + 1] - self.offsets[idx]
        off = csr_offsets(lens)
        words = np.concatenate([self.words[self.offsets[i]:self.offsets[i + 1]] for i in idx]) \
            if idx.size else np.empty(0, np.uint32)
        return Workload(self.name + f"[{idx.size}]", self.isa, words.astype(np.uint32), off, self.X, self.y,
                        self.target_program, self.description)


def single_generation(seed: int = 2, n_programs: int = 1 << 20, n_cases: int = 4096, len_lo: int = 16,
                      len_hi: int = 256, eff_frac: float = 0.6, num_inputs: int = 5, x_lo: float = -3.0,
                      x_hi: float = 3.0, target_eff: int = 16, noise: float = 0.01, ops=None) -> Workload:
    """One generation: 2^20 random programs, lengths U[16,256] with ~40%
    introns by construction, 5 features U[-3,3], 4096 cases, target = a
    random 16-effective-instruction program + N(0, 0.01^2).  REF ISA with 16
    registers (5 inputs + 11 scratch) and the reference's 16-entry pool.
    ``ops`` restricts the opcodes of the population (not of the target)."""
    rng = np.random.default_rng(seed)
    isa = IsaSpec(PROFILE_REF, 16)
    X = rng.uniform(x_lo, x_hi, size=(n_cases, num_inputs)).astype(np.float32)
    y, tp = regression_target(rng, X, isa, target_eff, noise)
    lens = uniform_lengths(rng, n_programs, len_lo, len_hi)
    words, off = structured_population(rng, lens, isa, eff_frac, ops=ops)
    return Workload("single_generation", isa, words, off, X, y, tp,
                    f"{n_programs} programs, L~U[{len_lo},{len_hi}], {eff_frac:.0%} effective, "
                    f"{num_inputs} features U[{x_lo},{x_hi}], {n_cases} cases")


def hbm_streaming(seed: int = 3, n_programs: int = 1 << 22, n_cases: int = 1 << 20, len_lo: int = 32,
                  len_hi: int = 1024, num_inputs: int = 8, target_eff: int = 24,
                  prefix_programs: Optional[int] = None) -> Workload:
    """2^22 programs, lengths log-uniform [32,1024] (uniform random words, so
    the intron fraction is whatever random code has, ~90%), 8 features
    U[-1,1], 2^20 cases, target = random 24-effective-instruction program.
    Words are drawn as 32-bit values in order, so ``prefix_programs`` = m
    materialises exactly the first m programs of the full population."""
    rng = np.random.default_rng(seed)
    isa = IsaSpec(PROFILE_REF, 16)
    X = rng.uniform(-1.0, 1.0, size=(n_cases, num_inputs)).astype(np.float32)
    y, tp = regression_target(rng, X, isa, target_eff)
    lens = log_uniform_lengths(rng, n_programs, len_lo, len_hi)
    m = n_programs if prefix_programs is None else min(prefix_programs, n_programs)
    off = csr_offsets(lens[:m])
    n_words = int(off[-1])
    words = np.empty(n_words, dtype=np.uint32)
    step = 1 << 26
    for i in range(0, n_words, step):
        k = min(step, n_words - i)
        words[i:i + k] = mask_random_words(rng.integers(0, 2**32, size=k, dtype=np.uint32), isa.num_registers)
    return Workload("hbm_streaming", isa, words, off, X, y, tp,
                    f"{n_programs} programs, L log-uniform [{len_lo},{len_hi}], {num_inputs} features, "
                    f"{n_cases} cases" + (f" (first {m} materialised)" if m < n_programs else ""))


def plain_cpu(seed: int = 0, n_programs: int = 1000, n_cases: int = 64) -> Workload:
    """The small CPU case: 1 feature x~U[-1,1], 64 cases, BJ op set
    {+,-,*,/p,sin,cos,exp,log_p}; registers r0 = input and r1..r8 calculation
    registers (field values < 9 of a 16-register file); 4 constants U[-5,5];
    lengths U[8,64]; target = a random 8-effective-instruction program."""
    rng = np.random.default_rng(seed)
    consts = np.zeros(16, dtype=np.float32)
    consts[:4] = rng.uniform(-5.0, 5.0, size=4).astype(np.float32)
    isa = IsaSpec(PROFILE_BJ, 16, False, consts)
    X = rng.uniform(-1.0, 1.0, size=(n_cases, 1)).astype(np.float32)
    y, tp = regression_target(rng, X, isa, 8, 0.0, reg_limit=9, const_limit=4)
    lens = uniform_lengths(rng, n_programs, 8, 64)
    words, off = structured_population(rng, lens, isa, 0.5, reg_limit=9, const_limit=4)
    return Workload("plain_cpu", isa, words, off, X, y, tp, "1000 programs, L~U[8,64], 64 cases, BJ ops")


def many_populations(seed: int = 4, n_pops: int = 64, size_lo: int = 1000, size_hi: int = 1 << 20,
                     len_lo: int = 8, len_hi: int = 2048, n_cases: int = 1 << 22, num_inputs: int = 4,
                     x_sigma: float = 10.0, target_scale: float = 1e4, noise: float = 1.0, target_eff: int = 16):
    """Batched populations on one shared dataset: population sizes and program
    lengths log-uniform, 4 features N(0, x_sigma^2) (sigma 10 reads "N(0,100)"
    as a variance), targets a random program rescaled to ~1e4 plus N(0, 1)
    noise.  Returns (isa, X, y, [(words, offsets)] per population)."""
    rng = np.random.default_rng(seed)
    isa = IsaSpec(PROFILE_REF, 16)
    X = (rng.standard_normal((n_cases, num_inputs)) * x_sigma).astype(np.float32)
    y, _ = regression_target(rng, X, isa, target_eff, noise, scale=target_scale)
    pops = []
    for _ in range(n_pops):
        n = int(log_uniform_lengths(rng, 1, size_lo, size_hi)[0])
        lens = log_uniform_lengths(rng, n, len_lo, len_hi)
        pops.append(random_population(rng, lens, isa.num_registers))
    return isa, X, y, pops


def serving_run_specs(seed: int = 5, n_runs: int = 256, cases_lo: int = 256, cases_hi: int = 1 << 20,
                      pop_lo: int = 1000, pop_hi: int = 1 << 18, len_lo: int = 8, len_hi: int = 512):
    """Shapes of independent GP runs for the serving loop (cases log-uniform,
    1-8 features, population log-uniform, lengths U[len_lo, len_hi]) and a
    seed for each; serving_run_data materialises one."""
    rng = np.random.default_rng(seed)
    specs = []
    for i in range(n_runs):
        specs.append({"n_cases": int(log_uniform_lengths(rng, 1, cases_lo, cases_hi)[0]),
                      "num_inputs": int(rng.integers(1, 9)),
                      "programs": int(log_uniform_lengths(rng, 1, pop_lo, pop_hi)[0]),
                      "len_lo": len_lo, "len_hi": len_hi, "seed": seed * 100003 + i})
    return specs


def serving_run_data(spec: dict):
    """(X, y, (words, offsets)) of one serving run: X U[-1,1], y a random
    12-effective-instruction program, uniform random words (REF ISA, 16
    registers)."""
    rng = np.random.default_rng(spec["seed"])
    isa = IsaSpec(PROFILE_REF, 16)
    X = rng.uniform(-1.0, 1.0, (spec["n_cases"], spec["num_inputs"])).astype(np.float32)
    y, _ = regression_target(rng, X, isa, 12)
    lens = uniform_lengths(rng, spec["programs"], spec["len_lo"], spec["len_hi"])
    return X, y, random_population(rng, lens, isa.num_registers)


def vary_words(rng, words: np.ndarray, frac: float, num_registers: int) -> None:
    """Redraw a fraction of the words in place (a next generation's
    variation, for serving workloads)."""
    k = int(words.size * frac)
    if k:
        idx = rng.integers(0, words.size, size=k)
        words[idx] = random_words(rng, k, num_registers)


def serving_runs(seed: int = 5, n_runs: int = 256, cases_lo: int = 256, cases_hi: int = 1 << 20,
                 pop_lo: int = 1000, pop_hi: int = 1 << 18, len_lo: int = 8, len_hi: int = 512,
                 generations: int = 1):
    """Independent GP runs for the serving loop: each has its own seeded
    dataset (cases log-uniform, 1-8 features U[-1,1], target a random
    program) and `generations` populations (size log-uniform, lengths
    U[len_lo, len_hi], uniform random words)."""
    rng = np.random.default_rng(seed)
    isa = IsaSpec(PROFILE_REF, 16)
    runs = []
    for _ in range(n_runs):
        N = int(log_uniform_lengths(rng, 1, cases_lo, cases_hi)[0])
        k = int(rng.integers(1, 9))
        X = rng.uniform(-1.0, 1.0, (N, k)).astype(np.float32)
        y, _ = regression_target(rng, X, isa, 12)
        gens = []
        for _g in range(generations):
            n = int(log_uniform_lengths(rng, 1, pop_lo, pop_hi)[0])
            gens.append(random_population(rng, uniform_lengths(rng, n, len_lo, len_hi), isa.num_registers))
        runs.append((X, y, gens))
    return isa, runs
