"""The small-problem engine run (1 feature, 64 cases, 50 generations) as files for the
reference engine drivers in oracle/_ref/lgp_run_c1_*: 1 feature x ~ U[-1,1],
64 training and 64 test cases, y = a seeded random 8-effective-instruction
program of the BJ op set {+,-,*,/p,sin,cos,exp,log_p}, 8 constants
U[-5,5].  The unmodified engine draws register fields over all of its
NUM_REGISTERS = 8 registers (r0 = the input, r1..r7 calculation) and
constants over the NR-entry pool, and starts every program at
STARTING_PROGRAM_SIZE = 8 instructions (lengths then grow up to
MAX_PROGRAM_SIZE = 64); tournament 4 and 50 generations are compile-time
settings of those drivers."""
from __future__ import annotations

import os
import subprocess
from pathlib import Path

import numpy as np

from galop_b200 import workloads as W

ROOT = Path(__file__).resolve().parents[1]
REF_BIN = ROOT / "oracle" / "_ref"


def write_case(out: Path, seed: int = 0) -> dict:
    """Write train/test CSVs and the constants file; return their paths."""
    rng = np.random.default_rng(seed)
    consts = rng.uniform(-5.0, 5.0, size=8).astype(np.float32)
    isa = W.IsaSpec(W.PROFILE_BJ, 8, False, consts)
    Xtr = rng.uniform(-1.0, 1.0, size=(64, 1)).astype(np.float32)
    Xte = rng.uniform(-1.0, 1.0, size=(64, 1)).astype(np.float32)
    ytr, prog = W.regression_target(rng, Xtr, isa, 8)
    yte = W.program_outputs(prog, Xte, isa)
    out.mkdir(parents=True, exist_ok=True)
    paths = {"train": out / "c1_train.csv", "test": out / "c1_test.csv", "constants": out / "c1_constants.txt"}
    for key, X, y in (("train", Xtr, ytr), ("test", Xte, yte)):
        with open(paths[key], "w") as f:
            f.write("x,y\n")
            for a, b in zip(X[:, 0], y):
                f.write(f"{float(a):.9g},{float(b):.9g}\n")
    paths["constants"].write_text(" ".join(f"{float(c):.9g}" for c in consts) + "\n")
    return paths


def run(exe: Path, paths: dict, out: Path, tag: str, seed: int = 0, bj: bool = True) -> list[str]:
    """One 50-generation engine run; returns the history CSV lines."""
    env = dict(os.environ, OMP_NUM_THREADS="1")
    if bj:
        env["GALOP_DRIVER_PROFILE"] = "bj"
        env["GALOP_DRIVER_CONSTANTS"] = str(paths["constants"])
    hist = out / f"hist_{tag}.csv"
    subprocess.run([str(exe), str(paths["train"]), str(paths["test"]), "c1", str(seed),
                    str(out / f"results_{tag}.csv"), str(out / f"prog_{tag}.txt"), str(hist)],
                   check=True, env=env, timeout=600)
    return hist.read_text().splitlines()
