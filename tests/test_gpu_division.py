"""The interpreter's division (src/ISA.h:224: b != 0 ? a / b : 1.0, IEEE
round to nearest) on the device.

The wide loop divides with its own fast path (rcp.approx refined by one
Newton-Raphson step, Markstein's correction q + (a - b q) y) and falls back
to IEEE division (div.rn) for a warp with an operand outside 2^-63..2^63.
tests/division_check.cu compares the fast path with div.rn (its header says
why these checks cover every in-range input): every divisor's rcp.approx
scaling, a stride of the 2^46 significand pairs (all of them with
GALOP_DIV_EXHAUSTIVE=1, about a minute), and random bit patterns over the
whole float range with special values.  Then the interpreter's outputs are
compared with numpy's IEEE division on operands that mix both paths, with
register and constant divisors.
"""
from __future__ import annotations

import json
import os
import shutil
import subprocess

import numpy as np
import pytest

import galop_b200 as g
from galop_b200 import workloads as W
from conftest import ROOT, bits

pytestmark = pytest.mark.gpu

EXHAUSTIVE = os.environ.get("GALOP_DIV_EXHAUSTIVE") == "1"


@pytest.fixture(scope="module")
def checker(tmp_path_factory):
    nvcc = shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc"
    exe = tmp_path_factory.mktemp("div") / "division_check"
    subprocess.run([nvcc, "-gencode", "arch=compute_100a,code=sm_100a", "-O3", "-std=c++17", "--fmad=false",
                    "-I", str(ROOT / "galop_b200" / "csrc"), str(ROOT / "tests" / "division_check.cu"),
                    "-o", str(exe)], check=True)
    return exe


def run(exe, *args) -> dict:
    out = subprocess.run([str(exe), *map(str, args)], capture_output=True, text=True, timeout=900)
    assert out.returncode == 0, out.stdout + out.stderr
    return json.loads(out.stdout.strip().splitlines()[-1])


def test_rcp_approx_scales_with_the_divisor(checker):
    r = run(checker, "rcp")
    assert r["checked"] == 127 * 2 * (1 << 23)
    assert r["mismatch"] == 0, r


def test_fast_path_on_significand_pairs(checker):
    step = 1 if EXHAUSTIVE else 4099
    r = run(checker, "pairs", step)
    n_a = -(-(1 << 23) // step)
    assert r["checked"] == n_a * (1 << 23)
    assert r["not_ok"] == 0 and r["mismatch"] == 0, r


def test_fast_path_on_random_and_special_operands(checker):
    r = run(checker, "random", 1 << 30, 7)
    assert r["checked"] >= 1 << 30
    assert r["fast"] > r["checked"] // 4            # at least the in-range quarter
    assert r["mismatch"] == 0, r


def _operands(n: int):
    rng = np.random.default_rng(11)
    a = rng.standard_normal(n).astype(np.float32) * 10
    b = rng.standard_normal(n).astype(np.float32) * 10
    # about one warp in eight gets out-of-range or special operands
    hit = (np.arange(n) // 256) % 8 == 3
    pick = rng.integers(0, 6, n)
    special = np.array([0.0, np.inf, np.nan, 1e-30, 3e38, 1e-42], np.float32)
    a = np.where(hit & (pick < 3), special[rng.integers(0, 6, n)], a).astype(np.float32)
    b = np.where(hit & (pick >= 3), special[rng.integers(0, 6, n)], b).astype(np.float32)
    a[::97] = 0.0                                   # zero dividends everywhere
    a[1::89] = -0.0
    b[::101] = 0.0                                  # protected divisions
    return a, b


def _want(a, b):
    with np.errstate(all="ignore"):
        return np.where(b != 0, a / b, np.float32(1.0)).astype(np.float32)


def _same(got, want):
    return (bits(got) == bits(want)) | (np.isnan(got) & np.isnan(want))


def test_interpreter_division_bit_exact(native):
    n = 1 << 20
    a, b = _operands(n)
    ds = g.Dataset(np.stack([a, b], 1), np.zeros(n, np.float32))
    cases = [(np.array([W.encode(3, 0, 0, 1, 0)], np.uint32), _want(a, b)),                 # r0 = r0 / r1
             (np.array([W.encode(3, 2, 0, 1, 0), W.encode(3, 0, 2, 1, 0)], np.uint32),      # twice
              _want(_want(a, b), b))]
    with g.Evaluator(num_registers=8) as ev:
        for prog, want in cases:
            got = ev.case_outputs(prog, np.array([0, prog.size], np.int64), ds)[0]
            ok = _same(got, want)
            assert ok.all(), (int((~ok).sum()), a[~ok][:4], b[~ok][:4])


def test_interpreter_division_by_constants_bit_exact(native):
    """Constant divisors (the divisor's half of the fast path runs once per
    instruction): every entry of the reference pool."""
    n = 1 << 18
    a, _ = _operands(n)
    ds = g.Dataset(a.reshape(-1, 1), np.zeros(n, np.float32))
    with g.Evaluator(num_registers=8) as ev:
        for j, c in enumerate(np.asarray(g.REF_CONSTANTS_8, np.float32)):
            prog = np.array([W.encode(3, 0, 0, j, 1)], np.uint32)
            got = ev.case_outputs(prog, np.array([0, 1], np.int64), ds)[0]
            ok = _same(got, _want(a, np.full(n, c, np.float32)))
            assert ok.all(), (j, float(c), int((~ok).sum()))
