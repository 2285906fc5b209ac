"""Whole-run driver parity with the reference's throughput driver
(tests/cuda_evo_bench.cu:61-68).  galop_b200/drivers/evo_bench.cpp runs the
reference's LGPEngine (selection and variation on the host, unchanged) with
this evaluator as its backend and prints the reference's row:
name,pop,D,gens,mean_size,seconds,gpops_s,best_mse with the reference's
formats.  The row's best MSE must equal the one the same run gives with the
whole generation loop on the device (galop_engine_*), since both draw the
same random streams and see the same fitness bits."""
from __future__ import annotations

import os
import random
import re
import subprocess

import numpy as np
import pytest

import galop_b200 as g
from conftest import ROOT

pytestmark = pytest.mark.gpu

ROW = re.compile(r"^(?P<name>[a-z0-9_]+),(?P<pop>\d+),(?P<D>\d+),(?P<G>\d+),\d+\.\d{2},\d+\.\d{4},"
                 r"\d\.\d{3}e[+-]\d{2},(?P<mse>-?\d\.\d{9}e[+-]\d{2}|inf)$")


def grid_dataset(path, n_cases):
    """The reference speed grid's synthetic cell: x ~ U(-1,1) from Python's
    random seeded with 1234, y = x^4 + x^3 + x^2 + x, header "x,y"."""
    rnd = random.Random(1234)
    with open(path, "w") as f:
        f.write("x,y\n")
        for _ in range(n_cases):
            x = rnd.uniform(-1, 1)
            f.write(f"{x},{x**4 + x**3 + x**2 + x}\n")


def run_row(exe, args):
    env = dict(os.environ, OMP_NUM_THREADS=str(min(16, os.cpu_count() or 1)))
    p = subprocess.run([str(exe), *map(str, args)], capture_output=True, text=True, env=env, timeout=900)
    assert p.returncode == 0, p.stderr[-400:]
    rows = [ln for ln in p.stdout.splitlines() if ROW.match(ln)]
    assert len(rows) == 1, p.stdout
    return ROW.match(rows[0]), p.stderr


def test_whole_run_row_and_device_engine(native, tmp_path):
    exe = ROOT / "galop_b200" / "drivers" / "_bin" / "evo_b200_P10000"
    if not exe.exists():
        pytest.skip("whole-run driver not built (it compiles the reference's engine sources)")
    csv = tmp_path / "grid_D1024.csv"
    grid_dataset(csv, 1024)
    m, err = run_row(exe, [csv, 70])
    assert m["name"] == "b200" and (m["pop"], m["D"], m["G"]) == ("10000", "1024", "100")
    assert "BREAKDOWN b200:" in err
    ref_exe = ROOT / "oracle" / "_ref" / "cuda_evo_bench_P10000"
    if ref_exe.exists():
        # the reference's own driver prints the same fields with the same formats
        r, _ = run_row(ref_exe, [csv, 70, "warp"])
        assert (r["pop"], r["D"], r["G"]) == (m["pop"], m["D"], m["G"])
    ds = g.Dataset.from_csv(str(csv))
    with g.Evaluator(num_registers=8, input_protect=True) as ev, \
            g.Engine(ev, population=10000, seed=70, macro_inserts=3, max_generations=100) as eng:
        hist = eng.evolve(ds)
    best = np.float32(hist[-1].best_fitness)
    mse = np.float32(1.0) / best - np.float32(1.0) if best > 0 else np.float32(np.inf)
    assert np.float32(float(m["mse"])) == mse, (m["mse"], mse)
