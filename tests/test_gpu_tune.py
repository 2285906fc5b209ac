"""The autotuner (galop_autotune): it measures every tile on a sample,
applies the fastest to the evaluator, and reuses a cached choice."""
from __future__ import annotations

import json

import numpy as np
import pytest

import galop_b200 as g
from galop_b200 import workloads as W
from conftest import bits

pytestmark = pytest.mark.gpu


def test_autotune_applies_and_caches_the_choice(native, tmp_path):
    wl = W.single_generation(seed=4, n_programs=3000, n_cases=777)
    ds = g.Dataset(wl.X, wl.y)
    cache = str(tmp_path / "tiles.jsonl")
    with g.Evaluator(num_registers=16, reduce=g.REDUCE_ORDERED) as ev:
        before = ev.evaluate_csr(wl.words, wl.offsets, ds)
        r = ev.autotune(wl.words, wl.offsets, cache=cache, sample=1024)
        assert r.from_cache == 0 and r.candidates >= 20
        assert r.sample_programs == 1024
        assert r.dispatch in (2, 3) and r.cases_per_lane in (1, 2, 4, 8) and r.warps_per_block in (2, 4, 8)
        assert r.gpops >= r.default_gpops > 0
        after = ev.evaluate_csr(wl.words, wl.offsets)
        st = ev.stats
        assert (st.cases_per_lane, st.warps_per_block) == (r.cases_per_lane, r.warps_per_block)
        # every tile computes the same thing: the choice changes speed only
        assert np.array_equal(bits(after), bits(before))
    lines = [json.loads(x) for x in open(cache)]
    assert len(lines) == 1 and lines[0]["key"] == r.key.decode()
    assert lines[0]["cases_per_lane"] == r.cases_per_lane

    with g.Evaluator(num_registers=16, reduce=g.REDUCE_ORDERED) as ev2:
        r2 = ev2.autotune(wl.words, wl.offsets, ds, cache=cache)
        assert r2.from_cache == 1 and r2.candidates == 0
        assert (r2.dispatch, r2.cases_per_lane, r2.warps_per_block) == \
            (r.dispatch, r.cases_per_lane, r.warps_per_block)
        ev2.evaluate_csr(wl.words, wl.offsets)
        assert ev2.stats.cases_per_lane == r.cases_per_lane
        # another size class (64 cases instead of 777) is a different key
        small = g.Dataset(wl.X[:64], wl.y[:64])
        r3 = ev2.autotune(wl.words, wl.offsets, small, cache=cache, sample=256, reps=1)
        assert r3.from_cache == 0 and r3.key != r.key
    assert len(open(cache).readlines()) == 2


def test_autotune_rejects_bad_input(native):
    with g.Evaluator(num_registers=8) as ev:
        words = np.zeros(4, np.uint32)
        with pytest.raises(g.GalopError) as e:
            ev.autotune(words, np.array([0, 4], np.int64))
        assert e.value.status == g.E_NO_DATASET
        ev.set_dataset(g.Dataset(np.zeros((8, 1), np.float32), np.zeros(8, np.float32)))
        with pytest.raises(g.GalopError) as e:
            ev.autotune(words, np.array([0, 3, 2], np.int64))
        assert e.value.status == g.E_INVALID
