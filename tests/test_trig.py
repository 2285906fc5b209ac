"""The device's sine and cosine (galop_b200/csrc/trig.cuh), host build.

The reference's SIN/COS are the C library's sinf/cosf (src/ISA.h:219-231);
the bar for the GPU is 2 ulp.  trig.cuh is compiled into the oracle for
the host, where it gives the same bits as on the device (every step is an
IEEE-rounded operation; tests/test_gpu_trig.py checks the device against
this build).  Here its accuracy is measured against the correctly rounded
values (sinl/cosl rounded to float) on a stride through the bit patterns of
all floats, and against glibc.  Set GALOP_TRIG_EXHAUSTIVE=1 to check every
float (a minute or two on 8 cores).
"""
from __future__ import annotations

import ctypes
import ctypes.util
import os

import numpy as np
import pytest

FAST_LIMIT = 131072.0          # 2^17: the Cody-Waite path below, Payne-Hanek at and above
F32_MAX = float(np.finfo(np.float32).max)
EXHAUSTIVE = os.environ.get("GALOP_TRIG_EXHAUSTIVE") == "1"


@pytest.mark.parametrize("cosine", [False, True])
def test_fast_path_within_1_56_ulp(oracle_lib, cosine):
    """|x| < 2^17 (every float below, or every 7th bit pattern): the
    Cody-Waite path stays within 1.56 ulp of the exact value (the bar is
    2); between 0.5 and 2^17, where the reduction rounds, it rounds
    correctly at least 83% of the time (CUDA's sinf/cosf: 80%)."""
    stride = 1 if EXHAUSTIVE else 7
    below = np.nextafter(np.float32(FAST_LIMIT), np.float32(0))
    a = oracle_lib.Oracle.trig_accuracy(cosine, 0.0, float(below), stride)
    assert a["max_ulp"] <= 1.56, a
    assert a["asymmetric"] == 0, a
    assert a["correctly_rounded"] >= 0.97, a        # most floats are below 0.5
    mid = oracle_lib.Oracle.trig_accuracy(cosine, 0.5, float(below), stride)
    assert mid["correctly_rounded"] >= 0.83, mid
    small = oracle_lib.Oracle.trig_accuracy(cosine, 0.0, 0.78, stride)
    assert small["max_ulp"] <= 0.91, small           # no reduction below pi/4
    assert small["correctly_rounded"] >= 0.99, small


@pytest.mark.parametrize("cosine", [False, True])
def test_slow_path_correctly_rounded(oracle_lib, cosine):
    """2^17 <= |x| <= FLT_MAX: Payne-Hanek reduction with 62 fraction bits
    and double-precision polynomials round correctly."""
    stride = 1 if EXHAUSTIVE else 4099
    a = oracle_lib.Oracle.trig_accuracy(cosine, FAST_LIMIT, F32_MAX, stride)
    assert a["max_ulp"] <= 0.5 + 1e-6, a
    assert a["correctly_rounded"] >= 0.9999, a
    assert a["asymmetric"] == 0, a


def test_specials(oracle_lib):
    o = oracle_lib.Oracle(oracle_lib.PROFILE_REF, 8, trig=oracle_lib.TRIG_DEVICE)
    x = np.array([0.0, -0.0, np.inf, -np.inf, np.nan, 1e-45, -1e-45, 1e-30, FAST_LIMIT, -FAST_LIMIT,
                  np.nextafter(np.float32(FAST_LIMIT), np.float32(0)), F32_MAX, -F32_MAX], np.float32)
    s = o.apply_op_n(4, x, x)
    c = o.apply_op_n(5, x, x)
    bits = lambda v: np.asarray(v, np.float32).view(np.uint32)   # noqa: E731
    assert bits(s[:2]).tolist() == [0x00000000, 0x80000000]        # sin(+-0) = +-0
    assert (c[:2] == 1.0).all()
    assert np.isnan(s[2:5]).all() and np.isnan(c[2:5]).all()
    assert np.array_equal(s[5:8], x[5:8])                           # sin x = x for tiny x
    want_s = np.sin(x[8:].astype(np.float64))
    want_c = np.cos(x[8:].astype(np.float64))
    np.testing.assert_allclose(s[8:], want_s, rtol=3e-7, atol=0)
    np.testing.assert_allclose(c[8:], want_c, rtol=3e-7, atol=0)


def test_libm_mode_is_the_reference(oracle_lib):
    """The oracle's default mode keeps the C library's sinf/cosf (the
    reference's); the device mode differs from it in some last bits."""
    rng = np.random.default_rng(5)
    x = rng.uniform(-100, 100, 4096).astype(np.float32)
    lib = oracle_lib.Oracle(oracle_lib.PROFILE_REF, 8)
    dev = oracle_lib.Oracle(oracle_lib.PROFILE_REF, 8, trig=oracle_lib.TRIG_DEVICE)
    libm = ctypes.CDLL(ctypes.util.find_library("m"))
    libm.sinf.restype = ctypes.c_float
    libm.sinf.argtypes = [ctypes.c_float]
    assert np.array_equal(lib.apply_op_n(4, x, x), np.array([libm.sinf(float(v)) for v in x], np.float32))
    d = dev.apply_op_n(4, x, x)
    l = lib.apply_op_n(4, x, x)
    assert 0.5 < (d == l).mean() < 1.0
    for op in (0, 1, 2, 3, 6, 7):
        assert np.array_equal(dev.apply_op_n(op, x, x[::-1].copy()), lib.apply_op_n(op, x, x[::-1].copy()))
