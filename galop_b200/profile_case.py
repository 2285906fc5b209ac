"""Run one workload case twice (for profiling captures of the second run).

    python -m galop_b200.profile_case [--workload single_generation|opset]
        [--programs N] [--cases N] [--dispatch D] [--k K] [--wpb W]
        [--registers NR] [--ops 0,1,2]

``single_generation``: the bench workload at a smaller population.
``opset``: 8,192 all-effective 64-instruction programs drawn from --ops
(per-op cost measurements).  Prints the stats of the second evaluation.
"""
from __future__ import annotations

import argparse
import json

import numpy as np

import galop_b200 as g
from galop_b200 import workloads as W


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--workload", default="single_generation", choices=["single_generation", "opset"])
    ap.add_argument("--programs", type=int, default=16384)
    ap.add_argument("--cases", type=int, default=4096)
    ap.add_argument("--dispatch", type=int, default=3)
    ap.add_argument("--k", type=int, default=4)
    ap.add_argument("--wpb", type=int, default=4)
    ap.add_argument("--registers", type=int, default=16)
    ap.add_argument("--ops", default="0,1,2,3,4,5,6,7")
    ap.add_argument("--reduce", type=int, default=0)
    a = ap.parse_args()
    if a.workload == "single_generation":
        wl = W.single_generation(seed=2, n_programs=a.programs, n_cases=a.cases)
        words, off, X, y, nr = wl.words, wl.offsets, wl.X, wl.y, 16
    else:
        rng = np.random.default_rng(1)
        nr = a.registers
        X = rng.uniform(-3, 3, (a.cases, min(5, nr))).astype(np.float32)
        y = rng.uniform(-1, 1, a.cases).astype(np.float32)
        ops = [int(x) for x in a.ops.split(",")]
        words, off = W.structured_population(rng, np.full(a.programs, 64), W.IsaSpec(0, nr), 1.0, ops=ops)
    with g.Evaluator(num_registers=nr, cases_per_lane=a.k, warps_per_block=a.wpb, dispatch=a.dispatch,
                     reduce=a.reduce) as ev:
        ev.set_dataset(g.Dataset(X, y))
        for _ in range(2):
            ev.evaluate_csr(words, off)
        st = ev.stats.as_dict()
    st["gpops"] = st["eff_instructions"] * st["n_cases"] / (st["interp_ms"] / 1e3) / 1e9
    print(json.dumps(st))


if __name__ == "__main__":
    main()
