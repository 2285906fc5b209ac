"""The oracle (C restatement, oracle/oracle.c) against the reference's own
results: golden vectors recorded from the reference's code, the known-answer
tests of tests/test_bed.cpp, and the 1000-generation golden histories."""
from __future__ import annotations

import gzip
import os
import subprocess

import numpy as np
import pytest

from conftest import GOLDEN, ROOT, bits, load_vectors, same_bits

VARIANTS = {"nr8": (8, False), "nr16": (16, False), "ip16": (16, True)}


def make_oracle(orc, variant):
    nr, ip = VARIANTS[variant]
    return orc.Oracle(orc.PROFILE_REF, nr, ip)


@pytest.mark.parametrize("variant", list(VARIANTS))
def test_decode_matches_reference_fields(oracle_lib, variant):
    """Field extraction incl. the INPUT_PROTECT dest fold (src/ISA.h:176-206)."""
    v = load_vectors(variant)
    o = make_oracle(oracle_lib, variant)
    assert o.output_reg == int(v["output_reg"])
    rng = np.random.default_rng(1)
    for w in rng.integers(0, 2**32, size=2000, dtype=np.uint64).astype(np.uint32):
        op, d, s1, s2, kc, _ = o.decode(int(w))
        nr = o.num_registers
        assert op == (w & 7)
        assert s1 == (w >> 16) & (nr - 1) and s2 == (w >> 24) & (nr - 1) and kc == (w >> 31)
        if o.input_protect:
            assert d == nr // 2 + ((w >> 8) & ((nr - 1) >> 1))
        else:
            assert d == (w >> 8) & (nr - 1)


def test_apply_op_bit_exact_vs_reference(oracle_lib):
    """ISA::apply_op (src/ISA.h:219-231) on special and random operands,
    including NaN, infinities, signed zeros and denormals."""
    with np.load(GOLDEN / "ops_ref.npz") as z:
        a, b, out = z["a"], z["b"], z["out"]
    o = oracle_lib.Oracle(oracle_lib.PROFILE_REF, 8)
    for op in range(8):
        mine = np.array([o.apply_op(op, float(x), float(y)) for x, y in zip(a, b)], dtype=np.float32)
        assert same_bits(mine, out[op]), f"op {op}"


@pytest.mark.parametrize("variant", list(VARIANTS))
def test_case_outputs_and_fitness_bit_exact(oracle_lib, variant):
    """Per-case outputs (Interpreter::run_stateless) and fitness
    (CpuEvaluator) of 370 programs x 4 datasets, bit for bit."""
    v = load_vectors(variant)
    o = make_oracle(oracle_lib, variant)
    words, off = v["words"], v["offsets"]
    for d in ("d1", "d2", "d3", "d4"):
        X, y = v[f"{d}_X"], v[f"{d}_y"]
        outs = np.stack([o.case_outputs(words[off[i]:off[i + 1]], X) for i in range(len(off) - 1)])
        assert same_bits(outs, v[f"{d}_outputs"]), d
        fit, sse = o.evaluate_csr(words, off, X, y, threads=1, with_sse=True)
        assert same_bits(fit, v[f"{d}_fitness"]), d
        mse = (sse / X.shape[0]).astype(np.float32)
        assert same_bits(mse, v[f"{d}_mse"]), d
        # the threaded population forms, full and effective-code-only, give
        # the same bits (the config-sized GPU parity tests use them)
        for eff in (False, True):
            assert same_bits(o.case_outputs_csr(words, off, X, threads=4, effective_only=eff),
                             v[f"{d}_outputs"]), (d, eff)
            fit2, sse2 = o.evaluate_csr_opt(words, off, X, y, threads=4, effective_only=eff)
            assert same_bits(fit2, v[f"{d}_fitness"]), (d, eff)
            assert np.array_equal(sse2.view(np.uint64), sse.view(np.uint64)), (d, eff)
        ew, eo = o.extract_effective_csr(words, off)
        for i in range(0, len(off) - 1, 7):
            p = words[off[i]:off[i + 1]]
            assert np.array_equal(ew[eo[i]:eo[i + 1]], p[o.effective_mask(p)])


@pytest.mark.parametrize("variant", list(VARIANTS))
def test_effective_mask_matches_reference(oracle_lib, variant):
    """Introns::effective_mask (src/Introns.h:28-46)."""
    v = load_vectors(variant)
    o = make_oracle(oracle_lib, variant)
    words, off = v["words"], v["offsets"]
    mine = np.concatenate([o.effective_mask(words[off[i]:off[i + 1]]) for i in range(len(off) - 1)])
    assert np.array_equal(mine.astype(np.uint8), v["masks"])


def test_intron_removal_preserves_outputs_bitwise(oracle_lib):
    """Executing only the effective instructions gives bit-identical outputs
    (the claim of src/Introns.h:8-12 and tests/test_bed.cpp:1355-1381)."""
    v = load_vectors("nr8")
    o = make_oracle(oracle_lib, "nr8")
    words, off = v["words"], v["offsets"]
    X = v["d3_X"]
    for i in range(len(off) - 1):
        p = words[off[i]:off[i + 1]]
        m = o.effective_mask(p)
        assert same_bits(o.case_outputs(p, X), o.case_outputs(p[m], X))


# --- known-answer tests restated from tests/test_bed.cpp:91-381 ------------------

def enc(op, d, s1, s2, kc):
    from galop_b200.workloads import encode
    return int(encode(op, d, s1, s2, kc))


ADD, SUB, MUL, DIV, SIN, COS, LT, GT = range(8)
C = np.arange(32, dtype=np.float32)


def run(o, prog, xs):
    return o.case_outputs(np.array(prog, np.uint32), np.asarray(xs, np.float32).reshape(-1, 1))


def test_kat_interpreter(oracle_lib):
    o = oracle_lib.Oracle(oracle_lib.PROFILE_REF, 8)
    assert np.array_equal(run(o, [enc(ADD, 0, 0, 0, 0)], C), 2 * C)                      # doubling :91-112
    assert np.array_equal(run(o, [enc(ADD, 0, 0, 1, 0)], C + 1), C + 1)                  # zero init :114-136
    assert np.array_equal(run(o, [enc(ADD, 0, 0, 1, 1)], C), C + 1)                      # constant :138-160
    assert np.array_equal(run(o, [enc(SUB, 0, 0, 1, 1)], C), C - 1)                      # sub :162-180
    assert np.array_equal(run(o, [enc(MUL, 0, 0, 5, 1)], C), C * 2)                      # mul :182-198
    out = run(o, [enc(DIV, 0, 0, 1, 0)], C + 1)                                         # protected :200-222
    assert np.all(out == 1.0) and np.all(np.isfinite(out))
    assert np.array_equal(run(o, [enc(DIV, 0, 0, 5, 1)], C * 2), C)                      # div :224-241
    assert np.array_equal(run(o, [enc(LT, 0, 0, 5, 1)], C), (C < 2).astype(np.float32))  # lt :243-261
    assert np.array_equal(run(o, [enc(GT, 0, 0, 5, 1)], C), (C > 2).astype(np.float32))  # gt :263-281
    assert np.all(np.abs(run(o, [enc(SIN, 0, 0, 0, 0)], C) - np.sin(C)) < 1e-5)         # sin :283-302
    assert np.array_equal(run(o, [enc(ADD, 1, 0, 1, 1), enc(MUL, 0, 1, 5, 1)], C), 2 * C + 2)  # :304-327
    assert np.array_equal(run(o, [enc(MUL, 0, 0, 0, 0)], C), C * C)                      # :329-346
    assert same_bits(run(o, [enc(ADD, 0, 0, 0, 0)], C), run(o, [enc(ADD, 0, 0, 0, 0)], C))  # :348-362
    assert np.array_equal(run(o, [], C + 1), C + 1)                                      # zero length :364-381


def test_kat_introns(oracle_lib):
    o = oracle_lib.Oracle(oracle_lib.PROFILE_REF, 8)
    m = o.effective_mask(np.array([enc(ADD, 1, 0, 1, 1), enc(MUL, 0, 0, 5, 1)], np.uint32))   # :1304-1320
    assert m.tolist() == [False, True]
    m = o.effective_mask(np.array([enc(ADD, 2, 0, 0, 0), enc(ADD, 3, 0, 0, 0), enc(SIN, 0, 3, 2, 0)],
                                  np.uint32))                                                   # :1322-1339
    assert m.tolist() == [True, False, True]
    m = o.effective_mask(np.array([enc(MUL, 1, 0, 0, 0), enc(ADD, 0, 0, 1, 0)], np.uint32))    # :1341-1353
    assert m.tolist() == [True, True]
    prog = np.array([enc(MUL, 1, 0, 0, 0), enc(ADD, 4, 3, 6, 1), enc(ADD, 1, 1, 0, 0), enc(SUB, 5, 5, 2, 1),
                     enc(ADD, 0, 1, 1, 1)], np.uint32)                                          # :1355-1381
    m = o.effective_mask(prog)
    assert m.sum() == 3
    x = (0.13 * np.arange(32, dtype=np.float32) - 1.7).astype(np.float32)
    assert same_bits(run(o, prog, x), run(o, prog[m], x))


def test_bj_profile_semantics(oracle_lib):
    """BJ profile: EXP and protected LOG replace LT and GT; both unary on src2."""
    o = oracle_lib.Oracle(oracle_lib.PROFILE_BJ, 8)
    x = np.array([0.0, -0.0, 1.0, -2.5, 3.0, 1e-3, 100.0, -1e30], np.float32)
    with np.errstate(over="ignore"):
        want = np.exp(x.astype(np.float64)).astype(np.float32)
    np.testing.assert_allclose(run(o, [enc(6, 0, 3, 0, 0)], x), want, rtol=1e-6)
    lg = run(o, [enc(7, 0, 3, 0, 0)], x)
    assert lg[0] == 0.0 and lg[1] == 0.0
    np.testing.assert_allclose(lg[2:], np.log(np.abs(x[2:].astype(np.float64))), rtol=1e-6)
    m = o.effective_mask(np.array([enc(ADD, 3, 0, 0, 0), enc(6, 0, 3, 1, 0)], np.uint32))
    assert m.tolist() == [False, True]   # EXP reads src2 (r1) only, not src1 (r3)


# --- golden histories through the reference engine ---------------------------

def _golden_cells():
    return [(t, s) for t in ("nguyen1", "nguyen2", "nguyen3") for s in (0, 1, 2)]


def run_golden(exe, tmp_path, cells, env=None):
    procs = []
    for t, s in cells:
        procs.append(subprocess.Popen(
            [str(exe), str(GOLDEN / "datasets" / f"{t}_train.csv"), str(GOLDEN / "datasets" / f"{t}_test.csv"),
             t, str(s), str(tmp_path / "results.csv"), str(tmp_path / f"prog_{t}_s{s}.txt"),
             str(tmp_path / f"hist_{t}_s{s}.csv")], env=env, stdout=subprocess.DEVNULL,
            stderr=subprocess.PIPE))
    for p in procs:
        _, err = p.communicate()
        assert p.returncode == 0, err.decode()


def golden_bytes(name):
    with gzip.open(GOLDEN / "histories" / (name + ".gz")) as f:
        return f.read()


@pytest.mark.skipif(not (ROOT / "oracle" / "_ref" / "lgp_run_oracle").exists(),
                    reason="oracle/_ref not built (needs the reference sources)")
def test_golden_histories_through_engine_with_oracle_backend(tmp_path):
    """The reference's LGPEngine with the C restatement as its EvalBackend
    reproduces all 9 golden cells (1000 generations) byte for byte."""
    env = dict(os.environ, OMP_NUM_THREADS="1")
    run_golden(ROOT / "oracle" / "_ref" / "lgp_run_oracle", tmp_path, _golden_cells(), env)
    for t, s in _golden_cells():
        for name in (f"hist_{t}_s{s}.csv", f"prog_{t}_s{s}.txt"):
            assert (tmp_path / name).read_bytes() == golden_bytes(name), name
