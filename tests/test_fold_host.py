"""The folding pass (galop_b200/csrc/fold.cuh: constant folding, dead-code
removal, register renaming, forwarding and store flags, the loop's form of
SIN/COS), built for the host from the same source, followed by the emulated
interpreter loop of tests/test_loop_math.py: per-case outputs equal the
oracle's (trig.cuh's host build for SIN/COS) bit for bit.

The pass's input is what the intron pre-pass writes: the effective
instructions of each program (the oracle's effective mask,
src/Introns.h:28-57) as 16-byte micro-ops (encode_wide, isa.cuh).  The
emulated pass loads the live-in registers into slots 0..m-1 in register
order and takes the output from the output slot the pass reports.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np
import pytest

from conftest import ROOT, bits
from test_loop_math import chained, emulate

NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")


@pytest.fixture(scope="session")
def fold_lib(tmp_path_factory):
    if not os.path.exists(NVCC):
        pytest.skip("nvcc not found")
    out = tmp_path_factory.mktemp("fold") / "libfold_host.so"
    cmd = [NVCC, "-gencode", "arch=compute_100a,code=sm_100a", "-O2", "-std=c++17", "--fmad=false", "-ftz=false",
           "-prec-div=true", "-Xcompiler", "-fPIC,-ffp-contract=off", "-shared",
           "-I", str(ROOT / "galop_b200" / "csrc"), "-I", str(ROOT / "include"),
           str(ROOT / "tests" / "fold_host.cu"), "-o", str(out)]
    res = subprocess.run(cmd, capture_output=True, text=True)
    assert res.returncode == 0, res.stderr[-2000:]
    lib = C.CDLL(str(out))
    lib.fold_host.restype = C.c_int64
    lib.fold_host.argtypes = [C.POINTER(C.c_uint32), C.c_int64, C.c_int, C.c_int, C.c_int, C.c_uint32, C.c_int,
                              C.c_int, C.c_int, C.POINTER(C.c_uint32)]
    return lib


def effective_uops(o, words: np.ndarray, S: int, consts: np.ndarray, profile: int) -> np.ndarray:
    """The intron pre-pass's output for one program: its effective
    instructions in order as wide micro-ops (no flags)."""
    keep = o.effective_mask(words).astype(bool)
    u = []
    for w in (int(x) for x, m in zip(words, keep) if m):
        op, dest, s1, s2, c = w & 7, (w >> 8) & 15, (w >> 16) & 15, (w >> 24) & 15, w >> 31
        unary = op in (4, 5) or (profile == 1 and op in (6, 7))
        u.append([0 if unary else s1 * S, int(consts[s2].view(np.uint32)) if c else s2 * S, dest * S,
                  op | (c << 3) | (0x80000000 if unary else 0)])
    return np.array(u, dtype=np.uint32).reshape(-1, 4)


def fold(lib, u: np.ndarray, k: int, k_in: int, profile: int):
    """(interpreted micro-ops, live-in word) of one program."""
    buf = np.ascontiguousarray(u.copy())
    lv = C.c_uint32()
    kept = lib.fold_host(buf.ctypes.data_as(C.POINTER(C.c_uint32)), len(u), profile, 16, 0,
                         7 + (k.bit_length() - 1), k_in, 1, 1, C.byref(lv))
    assert 0 <= kept <= len(u)
    return buf[len(u) - kept:], lv.value


@pytest.mark.parametrize("k", [1, 8])
@pytest.mark.parametrize("profile", [0, 1])
def test_folded_programs_through_the_loop(oracle_lib, fold_lib, k, profile):
    """REF and BJ (whose EXP/LOG fold here with the host's C library, the
    oracle's own functions, and leave the loop for the caller)."""
    from galop_b200 import REF_CONSTANTS_16
    from galop_b200 import workloads as W
    rng = np.random.default_rng(400 + k + 50 * profile)
    dev = oracle_lib.Oracle(profile, 16, trig=oracle_lib.TRIG_DEVICE)
    unary = lambda op, x: dev.apply_op_n(op, x, x)
    n, k_in = 32 * k, 3
    X = rng.uniform(-3, 3, (n, k_in)).astype(np.float32)
    X[rng.choice(n, 3, replace=False), 1] = np.float32([2e5, 1e-30, 0.0])
    progs = [W.random_words(rng, int(L), 16) for L in rng.integers(1, 120, 40)]
    progs += [chained(rng, int(L)) for L in rng.integers(2, 80, 40)]
    folded = bcast = 0
    for words in progs:
        u = effective_uops(dev, words, 128 * k, REF_CONSTANTS_16, profile)
        if len(u) == 0:
            continue
        ui, lv = fold(fold_lib, u, k, k_in, profile)
        folded += len(u) - len(ui)
        bcast += int(((ui[:, 3] & ~np.uint32(0x70)) == 12).sum())
        regs = [r for r in range(16) if (lv >> r) & 1]
        init = {i: (r if r < k_in else -1) for i, r in enumerate(regs)}
        got, _ = emulate(k, ui, X, init, (lv >> 24) & 15, unary, profile)
        want = dev.case_outputs(words, X)
        same = (bits(got) == bits(want)) | (np.isnan(got) & np.isnan(want))
        assert same.all(), (k, len(words), int((~same).sum()))
    assert folded > 0 and bcast > 0          # the pass did fold, and broadcasts ran
