"""galop_evaluate_csr_device: asynchronous on the caller's stream, offsets
checked on the device.

The reference's evaluate_population synchronises every call
(src/EvaluatorCuda.cu:452).  The device-resident entry point must instead
return as soon as its work is queued, so a caller can overlap it with its
own work; the caller states total_words (the size of its words buffer) and
the device checks the offsets against it before reading any word.
"""
from __future__ import annotations

import ctypes as C

import numpy as np
import pytest

import galop_b200 as g
from galop_b200 import workloads as W
from conftest import bits

pytestmark = pytest.mark.gpu

CUDA_ERROR_NOT_READY = 600


def _cudart():
    return C.CDLL("libcudart.so")


def test_device_call_returns_before_its_work_is_done(native):
    wl = W.single_generation(seed=31, n_programs=60_000, n_cases=65_536)
    n = wl.n_programs
    rt = _cudart()
    stream = C.c_void_p()
    assert rt.cudaStreamCreate(C.byref(stream)) == 0
    try:
        with g.Evaluator(num_registers=16) as ev:
            ev.set_dataset(g.Dataset(wl.X, wl.y))
            want = ev.evaluate_csr(wl.words, wl.offsets)
            dw, do, df = (ev.device_alloc(wl.words.nbytes), ev.device_alloc(wl.offsets.nbytes),
                          ev.device_alloc(4 * n))
            try:
                ev.h2d(dw, wl.words)
                ev.h2d(do, wl.offsets)
                total = int(wl.offsets[-1])
                # first call sizes the working buffers (it may block while they grow)
                ev.evaluate_csr_device(dw, do, n, total, df, stream=stream.value)
                assert rt.cudaStreamSynchronize(stream) == 0
                ev.evaluate_csr_device(dw, do, n, total, df, stream=stream.value)
                pending = rt.cudaStreamQuery(stream)
                assert rt.cudaStreamSynchronize(stream) == 0
                st = ev.stats
                got = np.empty(n, np.float32)
                ev.d2h(got, df)
            finally:
                for p in (dw, do, df):
                    ev.device_free(p)
    finally:
        rt.cudaStreamDestroy(stream)
    # the call came back while the stream still had its work queued
    assert pending == CUDA_ERROR_NOT_READY
    assert st.interp_ms > 1.0
    assert np.array_equal(bits(got), bits(want))


@pytest.mark.parametrize("defect", ["total", "decreasing", "first"])
def test_device_offsets_are_checked_on_the_device(native, defect):
    wl = W.single_generation(seed=32, n_programs=5000, n_cases=3000)
    n = wl.n_programs
    off = wl.offsets.copy()
    total = int(off[-1])
    if defect == "total":
        total -= 1                      # offsets[n] disagrees with the stated size
    elif defect == "decreasing":
        off[7] = off[6] - 1
    else:
        off[0] = 1
    with g.Evaluator(num_registers=16) as ev:
        ev.set_dataset(g.Dataset(wl.X, wl.y))
        want = ev.evaluate_csr(wl.words, wl.offsets)
        dw, do, df = ev.device_alloc(wl.words.nbytes), ev.device_alloc(off.nbytes), ev.device_alloc(4 * n)
        try:
            ev.h2d(dw, wl.words)
            ev.h2d(do, off)
            ev.evaluate_csr_device(dw, do, n, total, df)
            with pytest.raises(g.GalopError) as e:
                ev.stats
            assert e.value.status == g.E_INVALID
            got = np.empty(n, np.float32)
            ev.d2h(got, df)
            assert np.isnan(got).all()
            # the context stays usable: the consistent call gives the right fitness
            ev.h2d(do, wl.offsets)
            ev.evaluate_csr_device(dw, do, n, int(wl.offsets[-1]), df)
            ev.stats
            ev.d2h(got, df)
        finally:
            for p in (dw, do, df):
                ev.device_free(p)
    assert np.array_equal(bits(got), bits(want))
