"""The evolution loop on the GPU (galop_engine_*) against the reference's own
LGPEngine running on the CPU with this evaluator as its backend: same
options, same seed, same dataset -> the same history, generation for
generation (both evaluate in ORDERED mode, so fitness bits agree and every
selection and variation draw must agree for the runs to stay together)."""
from __future__ import annotations

import os
import subprocess

import numpy as np
import pytest

import galop_b200 as g
from conftest import GOLDEN, ROOT

pytestmark = pytest.mark.gpu

REF = ROOT / "oracle" / "_ref"


def host_history(exe, train, test, target, seed, tmp, env=None):
    hist = tmp / f"hist_{target}_{seed}.csv"
    subprocess.run([str(exe), str(train), str(test), target, str(seed), str(tmp / "results.csv"),
                    str(tmp / "prog.txt"), str(hist)], check=True, env=env, timeout=900,
                   stdout=subprocess.DEVNULL)
    return hist.read_text().splitlines()[1:]


def device_history(rows, target, seed):
    return [f"{target},{seed},{r.generation},{r.best_fitness:g},{r.mean_fitness:g},{r.best_length},"
            f"{r.mean_length:g}" for r in rows]


def first_difference(a, b):
    for i, (x, y) in enumerate(zip(a, b)):
        if x != y:
            return i, x, y
    return None


@pytest.mark.skipif(not (REF / "lgp_run_b200").exists(), reason="oracle/_ref/lgp_run_b200 not built")
@pytest.mark.parametrize("target,seed", [("nguyen1", 0), ("nguyen2", 1), ("nguyen3", 2)])
def test_default_config_all_generations(native, tmp_path, target, seed):
    """The reference's default configuration (P 1000, 1000 generations)."""
    train = GOLDEN / "datasets" / f"{target}_train.csv"
    want = host_history(REF / "lgp_run_b200", train, GOLDEN / "datasets" / f"{target}_test.csv", target, seed,
                        tmp_path, dict(os.environ, OMP_NUM_THREADS="1"))
    with g.Evaluator(num_registers=8, reduce=g.REDUCE_ORDERED) as ev, g.Engine(ev, seed=seed) as eng:
        got = device_history(eng.evolve(g.Dataset.from_csv(train)), target, seed)
        w, ln, f = eng.population()
    assert len(got) == len(want) == 1000
    assert first_difference(got, want) is None, first_difference(got, want)
    assert ((ln >= 1) & (ln <= 50)).all() and np.isfinite(f).all()


@pytest.mark.skipif(not (REF / "lgp_run_em_b200").exists(), reason="oracle/_ref/lgp_run_em_b200 not built")
@pytest.mark.parametrize("target,seed", [("nguyen1", 1), ("nguyen2", 2)])
def test_effective_mutation_config(native, tmp_path, target, seed):
    """GALOP_STANDARD_EM: input protection, three insert attempts and
    effective mutation (the liveness mask steers mutation and insertion)."""
    train = GOLDEN / "datasets" / f"{target}_train.csv"
    want = host_history(REF / "lgp_run_em_b200", train, GOLDEN / "datasets" / f"{target}_test.csv", target,
                        seed, tmp_path, dict(os.environ, OMP_NUM_THREADS="1"))
    with g.Evaluator(num_registers=8, input_protect=True, reduce=g.REDUCE_ORDERED) as ev, \
            g.Engine(ev, seed=seed, macro_inserts=3, effmut=1, max_generations=200) as eng:
        got = device_history(eng.evolve(g.Dataset.from_csv(train)), target, seed)
    assert len(got) == len(want) == 200
    assert first_difference(got, want) is None, first_difference(got, want)


@pytest.mark.skipif(not (REF / "lgp_run_c1_b200").exists(), reason="oracle/_ref/lgp_run_c1_b200 not built")
def test_small_problem_bj_config(native, tmp_path):
    """The 50-generation small-problem run with the BJ op set, tournament 4,
    programs up to 64 instructions and its own constants."""
    import config1 as c1
    paths = c1.write_case(tmp_path)
    want = c1.run(REF / "lgp_run_c1_b200", paths, tmp_path, "host", bj=True)[1:]
    consts = np.array(paths["constants"].read_text().split(), np.float32)
    with g.Evaluator(profile=g.PROFILE_BJ, num_registers=8, constants=consts, reduce=g.REDUCE_ORDERED) as ev, \
            g.Engine(ev, seed=0, max_program_size=64, tournament_size=4, max_generations=50) as eng:
        got = device_history(eng.evolve(g.Dataset.from_csv(paths["train"])), "c1", 0)
    assert len(got) == len(want) == 50
    assert first_difference(got, want) is None, first_difference(got, want)
