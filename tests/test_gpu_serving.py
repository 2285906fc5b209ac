"""The serving loop (galop_server_*): continuous batching of generations
from many independent GP runs, admitted by HBM footprint."""
from __future__ import annotations

import threading

import numpy as np
import pytest

import galop_b200 as g
from galop_b200 import workloads as W
from conftest import bits

pytestmark = pytest.mark.gpu

SMALL_SLOTS = dict(slot_programs=1 << 16, slot_words=1 << 22, slot_items=1 << 18)


def _runs(seed, n_runs):
    rng = np.random.default_rng(seed)
    isa = W.IsaSpec(g.PROFILE_REF, 16)
    runs = []
    for r in range(n_runs):
        N = int(rng.choice([64, 300, 2048, 9000, 40000]))
        k = int(rng.integers(1, 9))
        ds = g.Dataset(rng.uniform(-2, 2, (N, k)).astype(np.float32), rng.uniform(-1, 1, N).astype(np.float32))
        gens = []
        for _ in range(2):
            n = int(rng.integers(1, 3000))
            words, off = W.structured_population(rng, W.uniform_lengths(rng, n, 2, 80), isa, 0.6)
            gens.append((words, off))
        runs.append((ds, gens))
    return runs


def _alone(ev, ds, words, off):
    r = g.ResidentDataset(ev, ds)
    with g.Batch(ev, [(r, off.shape[0] - 1, max(int(off[-1]), 1))]) as b:
        b.set_population(0, words, off)
        b.evaluate()
        fit = b.fitness(0)
    r.close()
    return fit


def test_results_are_the_same_alone_and_in_the_mix(native):
    runs = _runs(1, 16)
    with g.Evaluator(num_registers=16) as ev:
        with g.Server(ev, **SMALL_SLOTS) as sv:
            ids = [sv.open_run(ds) for ds, _ in runs]
            got = {}
            lock = threading.Lock()

            def client(i):
                for gen, (w, o) in enumerate(runs[i][1]):
                    rq = sv.submit(ids[i], w, o)
                    fit, info = sv.wait(rq)
                    assert info.status == 0 and info.latency_ms >= info.queued_ms >= 0
                    with lock:
                        got[(i, gen)] = (fit, info)

            threads = [threading.Thread(target=client, args=(i,)) for i in range(len(runs))]
            for t in threads:
                t.start()
            for t in threads:
                t.join()
            tot = sv.totals
            for i in ids:
                sv.close_run(i)
        assert tot.completed == 2 * len(runs) and tot.case_ops > 0
        assert max(info.batch_requests for _, info in got.values()) > 1   # requests really were batched
        for (i, gen), (fit, info) in got.items():
            w, o = runs[i][1][gen]
            assert np.array_equal(bits(fit), bits(_alone(ev, runs[i][0], w, o))), (i, gen)


def test_admission_under_a_tight_hbm_budget(native):
    """Datasets that do not all fit are admitted as memory frees up (idle
    runs' datasets are evicted); every request still completes correctly."""
    runs = _runs(2, 8)
    with g.Evaluator(num_registers=16) as ev:
        probe = g.Server(ev, **SMALL_SLOTS)
        slot_bytes = probe.totals.resident_bytes
        probe.close()
        biggest = max(((ds.N + 1023) // 1024 * 1024) * (ds.num_inputs + 1) * 4 for ds, _ in runs)
        with g.Server(ev, hbm_budget_bytes=slot_bytes + 2 * biggest, **SMALL_SLOTS) as sv:
            ids = [sv.open_run(ds) for ds, _ in runs]
            reqs = [(i, gen, sv.submit(ids[i], w, o)) for i in range(len(runs))
                    for gen, (w, o) in enumerate(runs[i][1])]
            res = {(i, gen): sv.wait(rq)[0] for i, gen, rq in reqs}
            assert sv.totals.resident_bytes <= slot_bytes + 2 * biggest
        for (i, gen), fit in res.items():
            w, o = runs[i][1][gen]
            assert np.array_equal(bits(fit), bits(_alone(ev, runs[i][0], w, o))), (i, gen)


def test_wait_timeout_keeps_the_request(native):
    runs = _runs(3, 1)
    with g.Evaluator(num_registers=16) as ev, g.Server(ev, **SMALL_SLOTS) as sv:
        rid = sv.open_run(runs[0][0])
        w, o = runs[0][1][0]
        rq = sv.submit(rid, w, o)
        try:
            fit, info = sv.wait(rq, timeout=1e-7)
        except g.GalopError as e:
            assert e.status == g.E_TIMEOUT
            fit, info = sv.wait(rq)
        assert fit.shape[0] == o.shape[0] - 1 and info.status == 0
