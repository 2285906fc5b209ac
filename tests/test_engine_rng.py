"""The device engine's random streams (galop_b200/csrc/engine_rng.cuh) draw
exactly what the reference engine draws: its PCG32, and libstdc++'s
uniform_int_distribution, uniform_real_distribution<float> and mt19937 as
compiled here.  Needs the reference's sources (for its PCG32) and g++."""
from __future__ import annotations

import shutil
import subprocess
from pathlib import Path

import pytest

from conftest import ROOT, reference_root

REF = reference_root()
REF_SRC = REF / "src" if REF else None


@pytest.mark.skipif(REF_SRC is None or shutil.which("g++") is None,
                    reason="needs the reference's sources and g++")
def test_engine_streams_match_reference_and_libstdcxx(tmp_path):
    exe = tmp_path / "engine_rng_check"
    subprocess.run(["g++", "-std=c++20", "-O2", "-w", f"-I{REF_SRC}", str(ROOT / "tests" / "native" /
                    "engine_rng_check.cpp"), "-o", str(exe)], check=True)
    out = subprocess.run([str(exe)], capture_output=True, text=True)
    n, bad = map(int, out.stdout.split())
    assert out.returncode == 0 and bad == 0 and n > 1_000_000, out.stdout
