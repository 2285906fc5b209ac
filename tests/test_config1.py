"""The small-problem engine run (1 feature, 64 cases, tournament 4, 50
generations) through the reference's own LGPEngine: the C restatement as
backend reproduces the reference CpuEvaluator's run byte for byte on the REF
ISA, and runs the BJ op set (EXP/LOG) to completion."""
from __future__ import annotations

import pytest

import config1 as c1

EXES = [c1.REF_BIN / f"lgp_run_c1_{b}" for b in ("cpu", "oracle")]


@pytest.mark.skipif(not all(e.exists() for e in EXES), reason="oracle/_ref/lgp_run_c1_* not built")
def test_config1_engine_runs_with_the_oracle_backend(tmp_path):
    paths = c1.write_case(tmp_path)
    cpu = c1.run(EXES[0], paths, tmp_path, "cpu", bj=False)
    orc = c1.run(EXES[1], paths, tmp_path, "oracle", bj=False)
    assert len(cpu) == 51 and cpu == orc
    bj = c1.run(EXES[1], paths, tmp_path, "oracle_bj", bj=True)
    assert len(bj) == 51
    best = [float(line.split(",")[3]) for line in bj[1:]]
    assert all(0.0 <= b <= 1.0 for b in best) and best == sorted(best)   # elitism: best never drops
