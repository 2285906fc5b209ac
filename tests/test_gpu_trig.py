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
