"""Batched evaluation (galop_batch_*): many populations, each with its own
resident dataset, in one persistent launch per generation."""
from __future__ import annotations

import numpy as np
import pytest

import galop_b200 as g
from galop_b200 import workloads as W
from conftest import bits

pytestmark = pytest.mark.gpu


def _populations(seed, specs, nr=16):
    """specs: list of (n_programs, n_cases, n_features, len_lo, len_hi)."""
    rng = np.random.default_rng(seed)
    isa = W.IsaSpec(g.PROFILE_REF, nr)
    out = []
    for n, N, k, lo, hi in specs:
        X = rng.uniform(-2, 2, (N, k)).astype(np.float32)
        y = rng.uniform(-1, 1, N).astype(np.float32)
        words, off = W.structured_population(rng, W.uniform_lengths(rng, n, lo, hi), isa, 0.6)
        out.append((g.Dataset(X, y), words, off))
    return out


SPECS = [(700, 1000, 3, 4, 60), (50, 40000, 5, 8, 120), (1500, 33, 1, 2, 30), (3, 70000, 2, 10, 40),
         (0, 100, 1, 1, 1), (900, 4096, 8, 16, 200)]


@pytest.mark.parametrize("dispatch", [2, 3])
@pytest.mark.parametrize("reduce", [g.REDUCE_KAHAN32, g.REDUCE_ORDERED])
def test_batch_matches_single_population_calls(native, reduce, dispatch):
    pops = _populations(1, SPECS)
    with g.Evaluator(num_registers=16, reduce=reduce, dispatch=dispatch) as ev:
        single = [ev.evaluate_csr(w, o, ds) if o.shape[0] > 1 else np.zeros(0, np.float32) for ds, w, o in pops]
        rds = [g.ResidentDataset(ev, ds) for ds, _, _ in pops]
        with g.Batch(ev, [(r, max(o.shape[0] - 1, 1), max(int(o[-1]), 1)) for r, (_, _, o) in zip(rds, pops)]) as b:
            for p, (_, w, o) in enumerate(pops):
                b.set_population(p, w, o)
            b.evaluate()
            b.synchronize()
            got = [b.fitness(p) for p in range(len(pops))]
            st = b.stats
    assert st.eff_instructions < st.raw_instructions
    for p, (a, want) in enumerate(zip(got, single)):
        if reduce == g.REDUCE_ORDERED:
            assert np.array_equal(bits(a), bits(want)), p
        else:
            rel = np.abs(a.astype(np.float64) - want) / np.maximum(np.abs(want.astype(np.float64)), 1e-30)
            assert rel.size == 0 or rel.max() <= 1e-6, p


def test_batch_with_intron_pass_off_matches_on(native):
    """With the intron pass off the batch interprets every raw instruction
    (the pre-pass then only marks forwarding and live-in registers); the
    fitness must equal the default batch's bit for bit (ORDERED)."""
    pops = _populations(3, SPECS)
    got = {}
    for pre in (True, False):
        with g.Evaluator(num_registers=16, reduce=g.REDUCE_ORDERED, intron_prepass=pre) as ev:
            rds = [g.ResidentDataset(ev, ds) for ds, _, _ in pops]
            with g.Batch(ev, [(r, max(o.shape[0] - 1, 1), max(int(o[-1]), 1)) for r, (_, _, o) in zip(rds, pops)]) as b:
                for p, (_, w, o) in enumerate(pops):
                    b.set_population(p, w, o)
                b.evaluate()
                b.synchronize()
                got[pre] = [b.fitness(p) for p in range(len(pops))]
                st = b.stats
        if not pre:
            assert st.eff_instructions == st.raw_instructions
    for p, (a, c) in enumerate(zip(got[True], got[False])):
        assert np.array_equal(bits(a), bits(c)), p


@pytest.mark.parametrize("dispatch", [2, 3])
def test_population_fitness_is_identical_alone_and_in_a_mix(native, dispatch):
    """Case chunking depends on a population's own case count only, so its
    fitness does not depend on what else is batched with it."""
    pops = _populations(2, SPECS)
    with g.Evaluator(num_registers=16, dispatch=dispatch) as ev:
        rds = [g.ResidentDataset(ev, ds) for ds, _, _ in pops]
        caps = [(r, max(o.shape[0] - 1, 1), max(int(o[-1]), 1)) for r, (_, _, o) in zip(rds, pops)]
        with g.Batch(ev, caps) as mix:
            for p, (_, w, o) in enumerate(pops):
                mix.set_population(p, w, o)
            mix.evaluate()
            mixed = [mix.fitness(p) for p in range(len(pops))]
        for p, (_, w, o) in enumerate(pops):
            with g.Batch(ev, [caps[p]]) as alone:
                alone.set_population(0, w, o)
                alone.evaluate()
                assert np.array_equal(bits(alone.fitness(0)), bits(mixed[p])), p


@pytest.mark.parametrize("dispatch", [2, 3])
def test_graph_replay_across_generations(native, dispatch):
    """A captured generation replays with new program contents (same counts)
    and gives the same fitness as an uncaptured evaluation."""
    rng = np.random.default_rng(3)
    pops = _populations(3, SPECS[:3])
    isa = W.IsaSpec(g.PROFILE_REF, 16)
    with g.Evaluator(num_registers=16, dispatch=dispatch) as ev:
        rds = [g.ResidentDataset(ev, ds) for ds, _, _ in pops]
        caps = [(r, o.shape[0] - 1, 2 * int(o[-1]) + 1000) for r, (_, _, o) in zip(rds, pops)]
        with g.Batch(ev, caps) as bg, g.Batch(ev, caps) as bp:
            for gen in range(3):
                gens = []
                for p, (_, _, o) in enumerate(pops):
                    n = o.shape[0] - 1
                    lens = W.uniform_lengths(rng, n, 1, 2 * int(o[-1]) // max(n, 1))
                    w, off = W.structured_population(rng, lens, isa, 0.5)
                    bg.set_population(p, w, off)
                    bp.set_population(p, w, off)
                bg.evaluate(use_graph=True)
                bp.evaluate(use_graph=False)
                for p in range(len(pops)):
                    assert np.array_equal(bits(bg.fitness(p)), bits(bp.fitness(p))), (gen, p)


def test_batch_capacity_is_enforced(native):
    pops = _populations(4, SPECS[:1])
    ds, w, o = pops[0]
    with g.Evaluator(num_registers=16) as ev:
        r = g.ResidentDataset(ev, ds)
        with g.Batch(ev, [(r, 10, 100)]) as b:
            with pytest.raises(g.GalopError) as e:
                b.set_population(0, w, o)
            assert e.value.status == g.E_CAPACITY


def test_batch_r2_objective_matches_single_population_calls(native):
    """Each population's R^2 uses its own dataset's ss_tot.  Targets are
    the first input plus noise, and every population starts with an empty
    program (its output register is that input), so R^2 > 0 occurs."""
    rng = np.random.default_rng(1)
    pops = []
    for ds, w, o in _populations(5, SPECS[:4]):
        x0 = ds.inputs[:, 0].astype(np.float64)
        y = (x0 + rng.normal(0, 0.1, x0.shape)).astype(np.float32)
        pops.append((g.Dataset(ds.inputs, y), w, np.concatenate([[0], o]).astype(np.int64)))
    with g.Evaluator(num_registers=16, reduce=g.REDUCE_ORDERED, objective=g.OBJECTIVE_R2) as ev:
        single = [ev.evaluate_csr(w, o, ds) for ds, w, o in pops]
        rds = [g.ResidentDataset(ev, ds) for ds, _, _ in pops]
        with g.Batch(ev, [(r, o.shape[0] - 1, int(o[-1])) for r, (_, _, o) in zip(rds, pops)]) as b:
            for p, (_, w, o) in enumerate(pops):
                b.set_population(p, w, o)
            b.evaluate()
            for p in range(len(pops)):
                assert np.array_equal(bits(b.fitness(p)), bits(single[p])), p
    assert all(f[0] > 0.9 for f in single)


@pytest.mark.parametrize("reduce", [g.REDUCE_KAHAN32, g.REDUCE_ORDERED])
def test_batch_copies_share_fitness_within_a_population(native, reduce):
    """Populations full of copies (identical effective code, introns apart):
    with dedup on, copies take their representative's fitness inside their
    own population; every value equals the dedup-off batch bit for bit."""
    rng = np.random.default_rng(8)
    isa = W.IsaSpec(g.PROFILE_REF, 16)
    base = _populations(9, [(40, 1000, 3, 4, 40), (25, 40000, 2, 8, 60), (60, 3000, 4, 2, 20)])
    pops = []
    for ds, w, o in base:
        progs = [w[o[i]:o[i + 1]] for i in range(len(o) - 1)]
        out = []
        for _ in range(10 * len(progs)):
            p = progs[int(rng.integers(0, len(progs)))]
            if rng.random() < 0.5:
                p = np.concatenate([p, W.encode([0], [15], [1], [2], [0])])     # an intron at the end
            out.append(p)
        pops.append((ds, np.concatenate(out).astype(np.uint32), W.csr_offsets([len(p) for p in out])))
    fits = {}
    for dd in (True, False):
        with g.Evaluator(num_registers=16, reduce=reduce, dedup=dd) as ev:
            rds = [g.ResidentDataset(ev, ds) for ds, _, _ in pops]
            with g.Batch(ev, [(r, o.shape[0] - 1, int(o[-1])) for r, (_, _, o) in zip(rds, pops)]) as b:
                for p, (_, w, o) in enumerate(pops):
                    b.set_population(p, w, o)
                b.evaluate(use_graph=dd)
                b.synchronize()
                fits[dd] = [b.fitness(p) for p in range(len(pops))]
                fits[(dd, "interp")] = b.stats.interp_instructions
    for a, c in zip(fits[True], fits[False]):
        assert np.array_equal(bits(a), bits(c))
    assert fits[(True, "interp")] < 0.3 * fits[(False, "interp")]
