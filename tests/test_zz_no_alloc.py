"""galop_evaluate_csr_noalloc: evaluation for callers that cannot allocate.

Hosts that own all device memory through their own pool allocator, or that
run loops which must not stall on cudaMalloc/cudaFree (both can synchronise
the device), need an entry point that allocates nothing.  This one keeps its
working buffers in a fixed __device__ array.  The test calls it through the C
ABI twice in a row -- the second call reuses the first call's scratch -- over
more cases than one work item covers (so programs are split into case
chunks), and checks both against the regular entry point at the tolerance the
other KAHAN32 tests use (1e-6 relative).  The second call must leave the
device's free memory unchanged.  Offsets that disagree with the stated total
give NaN fitness, with nothing read beyond the stated sizes.  The file is
named to be collected last so that a run stopping at the first failure has
run everything else already; it passes alone in a fresh process too.  The
buffers it hands the entry point (inputs and outputs) are the test's own."""
from __future__ import annotations

import ctypes as C

import numpy as np
import pytest

import galop_b200 as g
from galop_b200 import workloads as W

pytestmark = pytest.mark.gpu


def _cudart():
    return C.CDLL("libcudart.so")


def _free_bytes() -> int:
    free, total = C.c_size_t(), C.c_size_t()
    assert _cudart().cudaMemGetInfo(C.byref(free), C.byref(total)) == 0
    return free.value


def test_noalloc_matches_regular_entry_point_on_two_calls(native):
    wl = W.single_generation(seed=11, n_programs=3000, n_cases=40_000)
    n, N, k = wl.n_programs, wl.n_cases, wl.X.shape[1]
    Np = (N + 1023) // 1024 * 1024
    X_fm = np.zeros((k, Np), np.float32)
    X_fm[:, :N] = wl.X.T
    y_p = np.zeros(Np, np.float32)
    y_p[:N] = wl.y
    lib = native
    total = int(wl.offsets[-1])
    with g.Evaluator(num_registers=16) as ev:
        want = ev.evaluate_csr(wl.words, wl.offsets, g.Dataset(wl.X, wl.y))
        bufs = {name: ev.device_alloc(arr.nbytes) for name, arr in
                (("w", wl.words), ("o", wl.offsets), ("x", X_fm), ("y", y_p))}
        d_fit = ev.device_alloc(4 * n)
        ev.h2d(bufs["w"], wl.words)
        ev.h2d(bufs["o"], wl.offsets)
        ev.h2d(bufs["x"], X_fm)
        ev.h2d(bufs["y"], y_p)
        opt = g._Options()
        lib.galop_options_init(C.byref(opt))
        opt.num_registers = 16
        got, free_delta = [], None
        for call in range(2):
            ev.h2d(d_fit, np.full(n, -1.0, np.float32))
            _cudart().cudaDeviceSynchronize()
            free_before = _free_bytes()
            rc = lib.galop_evaluate_csr_noalloc(C.byref(opt), bufs["w"], bufs["o"], n, total,
                                                bufs["x"], bufs["y"], N, Np, k, d_fit, None, None)
            assert rc == g.OK
            assert _cudart().cudaDeviceSynchronize() == 0
            if call == 1:
                free_delta = free_before - _free_bytes()
            fit = np.empty(n, np.float32)
            ev.d2h(fit, d_fit)
            got.append(fit)
        # offsets that disagree with the stated total: nothing is read beyond
        # the stated sizes and every fitness is NaN
        rc = lib.galop_evaluate_csr_noalloc(C.byref(opt), bufs["w"], bufs["o"], n, total - 1,
                                            bufs["x"], bufs["y"], N, Np, k, d_fit, None, None)
        assert rc == g.OK
        assert _cudart().cudaDeviceSynchronize() == 0
        poisoned = np.empty(n, np.float32)
        ev.d2h(poisoned, d_fit)
        # beyond the stated maximum: refused, nothing queued
        rc = lib.galop_evaluate_csr_noalloc(C.byref(opt), bufs["w"], bufs["o"], 65537, total,
                                            bufs["x"], bufs["y"], N, Np, k, d_fit, None, None)
        assert rc == g.E_CAPACITY
        for p in list(bufs.values()) + [d_fit]:
            ev.device_free(p)
    assert free_delta == 0
    assert np.isnan(poisoned).all()
    for fit in got:
        rel = np.abs(fit.astype(np.float64) - want) / np.maximum(np.abs(want.astype(np.float64)), 1e-30)
        assert rel.max() <= 1e-6
    assert np.array_equal(got[0].view(np.uint32), got[1].view(np.uint32))
