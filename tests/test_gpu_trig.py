"""SIN and COS on the device equal the host build of the same functions
(galop_b200/csrc/trig.cuh compiled into the oracle) bit for bit, in both
interpreters.  Arguments mix both reduction paths inside every warp:
random bit patterns over all floats, values near multiples of pi/2, the
2^17 boundary between the paths, denormals and specials.  Compared with
the C library's sinf/cosf (the reference's), every result is within 2 ulp.
"""
from __future__ import annotations

import numpy as np
import pytest

import galop_b200 as g
from galop_b200 import workloads as W
from conftest import bits

pytestmark = pytest.mark.gpu


def _ordered(x):
    i = np.ascontiguousarray(x, dtype=np.float32).view(np.int32).astype(np.int64)
    return np.where(i < 0, -(i & 0x7FFFFFFF), i)


def arguments(n: int = 1 << 20) -> np.ndarray:
    rng = np.random.default_rng(17)
    parts = [
        rng.integers(0, 1 << 32, n // 4, dtype=np.uint64).astype(np.uint32).view(np.float32),
        rng.uniform(-200.0, 200.0, n // 4).astype(np.float32),
        rng.uniform(-3e5, 3e5, n // 8).astype(np.float32),
    ]
    k = rng.integers(-200_000, 200_000, n // 8).astype(np.float64)
    near = (k * (np.pi / 2)).astype(np.float32).view(np.int32) + rng.integers(-3, 4, k.size).astype(np.int32)
    parts.append(near.view(np.float32))
    edge = np.float32(131072.0).view(np.int32) + np.arange(-4096, 4096, dtype=np.int32)
    parts += [edge.view(np.float32), -edge.view(np.float32)]
    parts.append(np.array([0.0, -0.0, np.inf, -np.inf, np.nan, 1e-45, -1e-45, 1e-38, 3.4e38, -3.4e38],
                          np.float32))
    x = np.concatenate(parts).astype(np.float32)
    fill = n - x.size
    x = np.concatenate([x, rng.standard_normal(fill).astype(np.float32) * 10]) if fill > 0 else x[:n]
    return x[rng.permutation(x.size)]


@pytest.mark.parametrize("dispatch", [2, 3])
def test_sin_cos_device_equals_host_build(native, oracle_lib, dispatch):
    x = arguments()
    ds = g.Dataset(x.reshape(-1, 1), np.zeros(x.size, np.float32))
    dev = oracle_lib.Oracle(oracle_lib.PROFILE_REF, 8, trig=oracle_lib.TRIG_DEVICE)
    lib = oracle_lib.Oracle(oracle_lib.PROFILE_REF, 8)
    for op in (4, 5):
        prog = np.array([W.encode(op, 0, 0, 0, 0)], np.uint32)
        with g.Evaluator(num_registers=8, dispatch=dispatch) as ev:
            got = ev.case_outputs(prog, np.array([0, 1], np.int64), ds)[0]
        want = dev.apply_op_n(op, x, x)
        same = (bits(got) == bits(want)) | (np.isnan(got) & np.isnan(want))
        assert same.all(), (op, int((~same).sum()), x[~same][:8])
        ref = lib.apply_op_n(op, x, x)
        fin = np.isfinite(ref)
        assert np.array_equal(np.isnan(got), np.isnan(ref))
        assert np.abs(_ordered(got[fin]) - _ordered(ref[fin])).max() <= 2


def _trig_chain(rng, nr: int, L: int) -> np.ndarray:
    """L instructions, mostly SIN/COS, each reading the previous result with
    probability 0.6 (forwarded operands, deferred stores) and otherwise an
    earlier register; a few constant operands (folded with the intron pass
    on, left to the C++ path with it off)."""
    ops = rng.choice([W.OP_SIN, W.OP_COS, W.OP_ADD, W.OP_SUB, W.OP_MUL, W.OP_DIV], L,
                     p=[0.35, 0.35, 0.08, 0.06, 0.1, 0.06])
    ins, prev = [], 0
    for op in ops:
        dest = int(rng.integers(0, nr))
        s1 = prev if rng.random() < 0.6 else int(rng.integers(0, nr))
        s2 = prev if rng.random() < 0.6 else int(rng.integers(0, nr))
        c = int(rng.random() < 0.05)
        ins.append((int(op), dest, s1, s2, c))
        prev = dest
    return W.encode(*np.array(ins, dtype=np.int64).T)


@pytest.mark.parametrize("profile", [g.PROFILE_REF, g.PROFILE_BJ])
def test_trig_chains_in_the_interpreter_loop(native, oracle_lib, profile):
    """Chains of SIN/COS with forwarded operands and deferred stores, run by
    the micro-op loop's own trig arms (dispatch 3), equal the 32-bit
    micro-op kernel (dispatch 2, trig.cuh called from C++) and the oracle
    with trig.cuh's host build, bit for bit.  Warps of 256 cases alternate
    between all arguments on the Cody-Waite path and a few cases that need
    Payne-Hanek (2^20, 3e38, infinities, NaN), so the loop both completes
    its trig arms and leaves them to the caller, after loaded and after
    forwarded operands, in both copies of the loop body and across
    32-instruction windows."""
    nr = 8
    rng = np.random.default_rng(71 + profile)
    progs = [_trig_chain(rng, nr, int(L)) for L in rng.integers(1, 100, 300)]
    words = np.concatenate(progs).astype(np.uint32)
    off = W.csr_offsets(np.array([len(p) for p in progs]))
    n = 4096
    X = rng.uniform(-60, 60, (n, 1)).astype(np.float32)
    big = np.array([1048576.0, -3e38, np.inf, -np.inf, np.nan, 2e5, -131072.0], np.float32)
    for blk in range(1, n // 256, 2):
        at = blk * 256 + rng.choice(256, 3, replace=False)
        X[at, 0] = rng.choice(big, 3)
    y = rng.uniform(-1, 1, n).astype(np.float32)
    ds = g.Dataset(X, y)
    res = {}
    for disp, pre in ((3, True), (3, False), (2, False)):
        with g.Evaluator(num_registers=nr, profile=profile, intron_prepass=pre, reduce=g.REDUCE_ORDERED,
                         dispatch=disp) as ev:
            res[disp, pre] = (ev.case_outputs(words, off, ds), ev.evaluate_csr(words, off, ds))
    od = oracle_lib.Oracle(profile, nr, trig=oracle_lib.TRIG_DEVICE)
    want = od.case_outputs_csr(words, off, X)
    for key, (outs, fit) in res.items():
        same = (bits(outs) == bits(want)) | (np.isnan(outs) & np.isnan(want))
        assert same.all(), (key, int((~same).sum()))
        assert np.array_equal(bits(fit), bits(res[2, False][1])), key
