"""The plain schedule (the reference's launch shape: one warp per program
over all its cases, src/EvaluatorCuda.cu:433-441) gives the persistent
schedule's results: bit for bit in ORDERED mode (both sum each program's
cases in case order), within 1e-6 relative in KAHAN32 mode (the case
chunking differs), with dedup copies receiving their representative's
fitness either way."""
from __future__ import annotations

import numpy as np
import pytest

import galop_b200 as g
from galop_b200 import workloads as W
from conftest import bits

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("reduce", [g.REDUCE_ORDERED, g.REDUCE_KAHAN32])
def test_plain_schedule_matches_persistent(native, reduce):
    rng = np.random.default_rng(77)
    lens = W.log_uniform_lengths(rng, 3000, 8, 600)
    words, off = W.random_population(rng, lens, 16)
    # a block of exact copies, so that dedup leaves some programs out
    words = np.concatenate([words, words[off[10]:off[60]]])
    off = np.concatenate([off, off[-1] + off[11:61] - off[10]])
    X = rng.uniform(-2, 2, (70_000, 4)).astype(np.float32)
    y = rng.uniform(-1, 1, 70_000).astype(np.float32)
    ds = g.Dataset(X, y)
    with g.Evaluator(num_registers=16, reduce=reduce) as ev:
        fp, sp = ev.evaluate_csr(words, off, ds, with_sse=True)
        chunks = ev.stats.case_chunks
    with g.Evaluator(num_registers=16, reduce=reduce, schedule=g.SCHEDULE_PLAIN) as ev:
        fq, sq = ev.evaluate_csr(words, off, ds, with_sse=True)
        st = ev.stats
    assert st.case_chunks == 1 and st.blocks >= (len(off) - 1) // 4
    assert np.array_equal(bits(fq[-50:]), bits(fq[10:60]))
    if reduce == g.REDUCE_ORDERED:
        assert np.array_equal(bits(fp), bits(fq))
        assert np.array_equal(sp.view(np.uint64), sq.view(np.uint64))
    else:
        assert chunks > 1
        fin = np.isfinite(sp) & (fp > 0)
        assert np.all(np.abs(sq[fin] - sp[fin]) <= 1e-6 * sp[fin])
        assert np.array_equal(fp[~fin] > 0, fq[~fin] > 0)
