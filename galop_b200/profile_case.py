"""Run one workload case twice (for profiling captures of the second run).

    python -m galop_b200.profile_case [--workload single_generation|opset]
        [--programs N] [--cases N] [--dispatch D] [--k K] [--wpb W]
        [--registers NR] [--ops 0,1,2]

``single_generation``: the bench workload at a smaller population.
``opset``: --programs all-effective 64-instruction programs drawn from
--ops (per-op cost measurements).  Prints the stats of the second
evaluation.
``lengths``: for all-effective REF programs of each fixed length in
2..1024 over --cases cases, every cases-per-lane x warps-per-block tile of
the default interpreter; prints one line per tile and the best per length.
"""
from __future__ import annotations

import argparse
import json

import numpy as np

import galop_b200 as g
from galop_b200 import workloads as W


def length_classes(n_cases: int):
    rng = np.random.default_rng(1)
    X = rng.uniform(-3, 3, (n_cases, 5)).astype(np.float32)
    y = rng.uniform(-1, 1, n_cases).astype(np.float32)
    ds = g.Dataset(X, y)
    isa = W.IsaSpec(0, 16)
    for L in (2, 4, 8, 16, 32, 64, 256, 1024):
        n = max(2048, min(65536, (1 << 24) // L // max(1, n_cases // 4096)))
        words, off = W.structured_population(rng, np.full(n, L), isa, 1.0)
        best = None
        for k in (1, 2, 4, 8):
            for wpb in (2, 4, 8):
                with g.Evaluator(num_registers=16, cases_per_lane=k, warps_per_block=wpb) as ev:
                    ev.set_dataset(ds)
                    ev.evaluate_csr(words, off)
                    ms = []
                    for _ in range(2):
                        ev.evaluate_csr(words, off)
                        ms.append(ev.stats.interp_ms)
                    gops = ev.stats.eff_instructions * n_cases / (min(ms) / 1e3) / 1e9
                r = dict(length=L, programs=n, k=k, wpb=wpb, interp_ms=round(min(ms), 3), gpops=round(gops, 1))
                print(json.dumps(r), flush=True)
                if best is None or gops > best["gpops"]:
                    best = r
        print("BEST", json.dumps(best), flush=True)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--workload", default="single_generation", choices=["single_generation", "opset", "lengths"])
    ap.add_argument("--programs", type=int, default=16384)
    ap.add_argument("--cases", type=int, default=4096)
    ap.add_argument("--dispatch", type=int, default=3)
    ap.add_argument("--k", type=int, default=4)
    ap.add_argument("--wpb", type=int, default=4)
    ap.add_argument("--registers", type=int, default=16)
    ap.add_argument("--ops", default="0,1,2,3,4,5,6,7")
    ap.add_argument("--reduce", type=int, default=0)
    a = ap.parse_args()
    if a.workload == "lengths":
        length_classes(a.cases)
        return
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
