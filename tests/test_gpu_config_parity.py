"""Parity on the shapes of the workloads the throughput is measured on.

The reference semantics are src/Interpreter.cpp:36-59 (per-case outputs),
src/ISA.h:219-231 (ops) and src/Evaluator.cpp:11-45, :88-91 (fitness); the
oracle is their C restatement (oracle/oracle.c, pinned to the reference's
own vectors and golden histories by tests/test_oracle.py).  Bars:

* programs whose effective code uses only ADD, SUB, MUL, protected DIV, LT
  and GT: every per-case output bit-identical (NaN compares as NaN) and the
  ORDERED fitness bit-identical; KAHAN32 fitness within 1e-6 relative;
* programs with SIN/COS: each transcendental op is within 2 ulp (checked one
  instruction at a time by replaying GPU register traces, here on programs
  up to 2,048 instructions long); a program's output can move further,
  because an ulp of difference propagates through the rest of the program,
  so the per-case ulp distance is reported as a histogram, the fitness must
  be bit-identical wherever all of a program's outputs are, and the
  fitness is held to the reference's own GPU gate (tests/cuda_diff.cu:82:
  |d fitness| < 1e-4, at most 1% of programs over);
* the same programs against the oracle with the device's own sine and
  cosine (trig.cuh built for the host, Oracle(trig=TRIG_DEVICE)): every
  per-case output and every ORDERED fitness bit-identical, so the only
  difference from the reference is in the SIN/COS results themselves;
* the production path (intron pass, constant folding, operand forwarding,
  register renaming, 16-byte micro-ops) gives the same bits as the plain
  one-instruction-at-a-time interpreter on the raw programs (dispatch 2,
  intron pass off), so its rewrites change nothing on long programs with
  transcendental ops either;
* at the batching configuration's magnitudes (inputs N(0, 10^2), targets
  ~1e4 + N(0,1), 2^22 cases) the compensated-FP32 fitness is within 1e-6
  relative of the FP64 oracle.

Set GALOP_PARITY_REPORT to a file path to write the ulp histograms as JSON.
"""
from __future__ import annotations

import json
import os

import numpy as np
import pytest

import galop_b200 as g
from galop_b200 import workloads as W
from conftest import bits

pytestmark = pytest.mark.gpu

IEEE_REF_OPS = [0, 1, 2, 3, 6, 7]
ULP_EDGES = [0, 1, 2, 3, 17, 1025, 1 << 20, 1 << 40]
ULP_NAMES = ["0", "1", "2", "3-16", "17-1024", "1025-2^20", ">2^20", "nan/not-nan"]
_REPORT: dict = {}


def _ordered(x):
    i = np.ascontiguousarray(x, dtype=np.float32).view(np.int32).astype(np.int64)
    return np.where(i < 0, -(i & 0x7FFFFFFF), i)


def ulp_dist(a, b):
    a = np.asarray(a, np.float32)
    b = np.asarray(b, np.float32)
    d = np.abs(_ordered(a) - _ordered(b))
    both_nan = np.isnan(a) & np.isnan(b)
    one_nan = np.isnan(a) ^ np.isnan(b)
    return np.where(both_nan, 0, np.where(one_nan, 1 << 40, d))


def histogram(d) -> dict:
    counts, _ = np.histogram(np.minimum(d, (1 << 40)), bins=ULP_EDGES + [(1 << 40) + 1])
    return {name: int(c) for name, c in zip(ULP_NAMES, counts)}


def compare_rows(got, want, rows=64):
    """Per-case ulp distances of two (programs, cases) arrays, a few rows at
    a time: (histogram, per-program 'all outputs exact', max distance)."""
    hist = {name: 0 for name in ULP_NAMES}
    exact = np.empty(got.shape[0], bool)
    dmax = 0
    for r in range(0, got.shape[0], rows):
        d = ulp_dist(got[r:r + rows], want[r:r + rows])
        for name, c in histogram(d.ravel()).items():
            hist[name] += c
        exact[r:r + rows] = (d == 0).all(axis=1)
        dmax = max(dmax, int(d.max()))
    return hist, exact, dmax


def report(key: str, value) -> None:
    _REPORT[key] = value
    path = os.environ.get("GALOP_PARITY_REPORT")
    if path:
        with open(path, "w") as f:
            json.dump(_REPORT, f, indent=1, sort_keys=True)


def same_or_nan(a, b):
    a = np.asarray(a, np.float32)
    b = np.asarray(b, np.float32)
    return (bits(a) == bits(b)) | (np.isnan(a) & np.isnan(b))


def ieee_only(words):
    """SIN -> ADD and COS -> DIV: the same programs with IEEE-exact ops only."""
    w = np.asarray(words, np.uint32).copy()
    op = w & 7
    w = np.where(op == 4, w & ~np.uint32(7), w)
    w = np.where(op == 5, (w & ~np.uint32(7)) | np.uint32(3), w)
    return w.astype(np.uint32)


def effective_ops_ieee(o, words, off):
    out = np.empty(len(off) - 1, bool)
    for i in range(len(off) - 1):
        p = words[off[i]:off[i + 1]]
        out[i] = set((p[o.effective_mask(p)] & 7).tolist()) <= set(IEEE_REF_OPS)
    return out


def reference_gate(fit, want, n):
    over = np.abs(fit.astype(np.float64) - want.astype(np.float64)) > 1e-4
    return int(over.sum()) <= max(1, n // 100)


def gpu_outputs(words, off, ds, nr=16, dispatch=3, prepass=True):
    with g.Evaluator(num_registers=nr, dispatch=dispatch, intron_prepass=prepass) as ev:
        return ev.case_outputs(words, off, ds)


def gpu_fitness(words, off, ds, reduce, nr=16):
    with g.Evaluator(num_registers=nr, reduce=reduce) as ev:
        return ev.evaluate_csr(words, off, ds, with_sse=True)


# --- the single-generation configuration: 4,096 programs x 4,096 cases ---------------

def test_config2_ieee_only_programs_bit_exact(native, oracle_lib):
    """Config-2-shaped programs (L ~ U[16,256], ~40% introns, 5 features
    U[-3,3], 4,096 cases) drawn over the IEEE-exact ops: all 16.8 M outputs
    and every ORDERED fitness bit-identical to the oracle."""
    wl = W.single_generation(seed=2, n_programs=4096, ops=IEEE_REF_OPS)
    o = oracle_lib.Oracle(oracle_lib.PROFILE_REF, 16)
    ds = g.Dataset(wl.X, wl.y)
    outs = gpu_outputs(wl.words, wl.offsets, ds)
    fo, so = gpu_fitness(wl.words, wl.offsets, ds, g.REDUCE_ORDERED)
    fk, _ = gpu_fitness(wl.words, wl.offsets, ds, g.REDUCE_KAHAN32)
    want = o.case_outputs_csr(wl.words, wl.offsets, wl.X)
    wfit, wsse = o.evaluate_csr_opt(wl.words, wl.offsets, wl.X, wl.y)
    ok = same_or_nan(outs, want)
    report("config2_ieee_only", {"programs": 4096, "cases": 4096, "outputs_differing": int((~ok).sum())})
    assert ok.all(), int((~ok).sum())
    assert np.array_equal(bits(fo), bits(wfit))
    assert np.array_equal(so.view(np.uint64), wsse.view(np.uint64))
    fin = wfit > 0
    rel = np.abs(fk[fin].astype(np.float64) - wfit[fin]) / wfit[fin]
    assert rel.max() <= 1e-6
    assert np.array_equal(fk[~fin] > 0, wfit[~fin] > 0)


def test_config2_sample_ulp_histogram_and_fitness(native, oracle_lib):
    """The unmodified config-2 sample (4,096 programs, most with SIN/COS in
    their effective code): per-case ulp histogram against the oracle;
    outputs of IEEE-only programs exact; fitness bit-identical wherever a
    program's outputs are; the production path equals the plain
    interpreter on the raw programs bit for bit; the reference's gate."""
    wl = W.single_generation(seed=2, n_programs=4096)
    o = oracle_lib.Oracle(oracle_lib.PROFILE_REF, 16)
    ds = g.Dataset(wl.X, wl.y)
    outs = gpu_outputs(wl.words, wl.offsets, ds)
    plain = gpu_outputs(wl.words, wl.offsets, ds, dispatch=2, prepass=False)
    fo, _ = gpu_fitness(wl.words, wl.offsets, ds, g.REDUCE_ORDERED)
    want = o.case_outputs_csr(wl.words, wl.offsets, wl.X)
    wfit, _ = o.evaluate_csr_opt(wl.words, wl.offsets, wl.X, wl.y)
    od = oracle_lib.Oracle(oracle_lib.PROFILE_REF, 16, trig=oracle_lib.TRIG_DEVICE)
    dev_ok = same_or_nan(outs, od.case_outputs_csr(wl.words, wl.offsets, wl.X))
    dfit, dsse = od.evaluate_csr_opt(wl.words, wl.offsets, wl.X, wl.y)
    ieee = effective_ops_ieee(o, wl.words, wl.offsets)
    hist, exact_prog, _ = compare_rows(outs, want)
    report("config2_sample", {"programs": 4096, "cases": 4096, "ieee_only_programs": int(ieee.sum()),
                              "outputs_differing_from_device_trig_oracle": int((~dev_ok).sum()),
                              "programs_all_outputs_exact": int(exact_prog.sum()),
                              "ulp_histogram_per_case": hist,
                              "fitness_bit_exact_programs": int((bits(fo) == bits(wfit)).sum()),
                              "fitness_over_1e-4": int((np.abs(fo.astype(np.float64) - wfit) > 1e-4).sum())})
    assert np.array_equal(bits(outs), bits(plain))
    assert dev_ok.all(), int((~dev_ok).sum())
    assert np.array_equal(bits(fo), bits(dfit))
    assert exact_prog[ieee].all()
    assert np.array_equal(bits(fo)[exact_prog], bits(wfit)[exact_prog])
    assert reference_gate(fo, wfit, 4096)


# --- long programs: configs 3 and 4 lengths, 65,536 cases ------------------------------

@pytest.mark.parametrize("kind", ["ieee", "mixed"])
@pytest.mark.parametrize("lo,hi,k,sigma", [(32, 1024, 8, None), (8, 2048, 4, 10.0)])
def test_long_programs_against_oracle(native, oracle_lib, lo, hi, k, sigma, kind):
    """1,024 random programs with lengths log-uniform [32,1024] (8 features
    U[-1,1]) or [8,2048] (4 features N(0,10^2)) over 65,536 cases."""
    rng = np.random.default_rng(lo + hi)
    N = 65_536
    lens = W.log_uniform_lengths(rng, 1024, lo, hi)
    words, off = W.random_population(rng, lens, 16)
    if kind == "ieee":
        words = ieee_only(words)
    X = (rng.standard_normal((N, k)) * sigma if sigma else rng.uniform(-1, 1, (N, k))).astype(np.float32)
    y = rng.uniform(-1, 1, N).astype(np.float32)
    ds = g.Dataset(X, y)
    o = oracle_lib.Oracle(oracle_lib.PROFILE_REF, 16)
    outs = gpu_outputs(words, off, ds)
    fo, _ = gpu_fitness(words, off, ds, g.REDUCE_ORDERED)
    want = o.case_outputs_csr(words, off, X, effective_only=True)
    wfit, _ = o.evaluate_csr_opt(words, off, X, y, effective_only=True)
    hist, exact_prog, dmax = compare_rows(outs, want)
    report(f"long_L{lo}-{hi}_{kind}", {"programs": 1024, "cases": N, "max_length": int(lens.max()),
                                        "mean_length": float(lens.mean()),
                                        "programs_all_outputs_exact": int(exact_prog.sum()),
                                        "ulp_histogram_per_case": hist})
    assert lens.max() > 0.6 * hi
    if kind == "ieee":
        assert dmax == 0
        assert np.array_equal(bits(fo), bits(wfit))
    else:
        plain = gpu_outputs(words, off, ds, dispatch=2, prepass=False)
        assert np.array_equal(bits(outs), bits(plain))
        od = oracle_lib.Oracle(oracle_lib.PROFILE_REF, 16, trig=oracle_lib.TRIG_DEVICE)
        assert same_or_nan(outs, od.case_outputs_csr(words, off, X, effective_only=True)).all()
        assert np.array_equal(bits(fo), bits(od.evaluate_csr_opt(words, off, X, y, effective_only=True)[0]))
        assert np.array_equal(bits(fo)[exact_prog], bits(wfit)[exact_prog])
        assert reference_gate(fo, wfit, 1024)


@pytest.mark.parametrize("profile", [g.PROFILE_REF, g.PROFILE_BJ])
def test_trace_replay_long_programs(native, oracle_lib, profile):
    """Programs of 700 to 2,048 instructions: every GPU instruction, fed the
    GPU's own register file, reproduces the CPU's apply_op (bit-exact for
    IEEE ops and, against the device-trig oracle, for SIN/COS; <= 2 ulp
    for SIN/COS against the C library and for EXP/LOG); the production
    path's outputs equal the trace's final output register bit for bit."""
    rng = np.random.default_rng(70 + profile)
    o = oracle_lib.Oracle(profile, 16)
    od = oracle_lib.Oracle(profile, 16, trig=oracle_lib.TRIG_DEVICE)
    X = rng.uniform(-3, 3, size=(128, 5)).astype(np.float32)
    ds = g.Dataset(X, np.zeros(128, np.float32))
    ieee = {0, 1, 2, 3, 6, 7} if profile == g.PROFILE_REF else {0, 1, 2, 3}
    with g.Evaluator(profile=profile, num_registers=16, cases_per_lane=4) as ev:
        ev.set_dataset(ds)
        for L in (700, 1500, 2048):
            prog = W.random_words(rng, L, 16)
            st = ev.trace(prog)                          # (L+1, 16, n)
            n = st.shape[2]
            for pc, w in enumerate(prog):
                op, dd, s1, s2, kc, _ = o.decode(int(w))
                a = st[pc, s1]
                b = np.full(n, o.constants[s2], np.float32) if kc else st[pc, s2]
                want = o.apply_op_n(op, a, b)
                got = st[pc + 1, dd]
                if op in ieee:
                    assert same_or_nan(got, want).all(), (L, pc, op)
                else:
                    assert ulp_dist(got, want).max() <= 2, (L, pc, op)
                    if op in (4, 5):
                        assert same_or_nan(got, od.apply_op_n(op, a, b)).all(), (L, pc, op)
            final = ev.case_outputs(prog, np.array([0, L], np.int64))[0][:n]
            assert np.array_equal(bits(final), bits(st[L, o.output_reg]))


# --- the batching configuration's magnitudes: 2^22 cases ------------------------------

@pytest.mark.parametrize("kind", ["ieee", "mixed"])
def test_config4_magnitudes_kahan32_within_1e6(native, oracle_lib, kind):
    """2^22 cases of 4 features N(0, 10^2), targets a random program scaled
    to ~1e4 plus N(0,1), 192 programs of lengths log-uniform [8,2048]: the
    KAHAN32 fitness (compensated FP32 per lane, FP64 across lanes) is
    within 1e-6 relative of the FP64 case-order oracle, and the ORDERED SSE
    equals the oracle's bit for bit (for programs with SIN/COS, the oracle
    with the device's sine and cosine)."""
    rng = np.random.default_rng(404)
    N = 1 << 22
    X = (rng.standard_normal((N, 4)) * 10.0).astype(np.float32)
    isa = W.IsaSpec(g.PROFILE_REF, 16)
    y_full, _ = W.regression_target(rng, X, isa, 16, 1.0, scale=1e4)
    assert np.isfinite(y_full).all()
    lens = W.log_uniform_lengths(rng, 192, 8, 2048)
    words, off = W.random_population(rng, lens, 16)
    if kind == "ieee":
        words = ieee_only(words)
    ds = g.Dataset(X, y_full)
    fk, sk = gpu_fitness(words, off, ds, g.REDUCE_KAHAN32)
    fo, so = gpu_fitness(words, off, ds, g.REDUCE_ORDERED)
    o = oracle_lib.Oracle(oracle_lib.PROFILE_REF, 16)
    wfit, wsse = o.evaluate_csr_opt(words, off, X, y_full, effective_only=True)
    # IEEE-only: against the oracle itself; mixed: against the oracle with
    # the device's sine and cosine, whose outputs are the GPU's bit for bit,
    # which isolates the accumulation error from the transcendental ops'
    # last-ulp differences
    if kind == "ieee":
        ref, ref_sse = wfit, wsse
    else:
        od = oracle_lib.Oracle(oracle_lib.PROFILE_REF, 16, trig=oracle_lib.TRIG_DEVICE)
        ref, ref_sse = od.evaluate_csr_opt(words, off, X, y_full, effective_only=True)
    fin = np.isfinite(ref_sse) & (ref > 0)
    rel = np.abs(fk[fin].astype(np.float64) - ref[fin]) / ref[fin]
    rel_sse = np.abs(sk[fin] - ref_sse[fin]) / ref_sse[fin]
    report(f"config4_magnitudes_{kind}", {"programs": 192, "cases": N, "finite": int(fin.sum()),
                                          "max_rel_err_fitness": float(rel.max()) if rel.size else 0.0,
                                          "max_rel_err_sse": float(rel_sse.max()) if rel_sse.size else 0.0})
    assert fin.sum() >= 50
    assert rel.max() <= 1e-6
    assert np.array_equal(fk[~fin] > 0, ref[~fin] > 0)
    assert np.array_equal(so.view(np.uint64), ref_sse.view(np.uint64))
    if kind == "mixed":
        assert reference_gate(fo, wfit, 192)
