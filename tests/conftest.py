"""Shared pytest setup.

Marker ``gpu``: the test runs the CUDA path on a B200 through the C ABI.
Everything unmarked runs on a CPU-only machine (oracle vs golden vectors,
host logic, ABI symbol checks).
"""
from __future__ import annotations

import subprocess
import sys
from pathlib import Path

import numpy as np
import pytest

ROOT = Path(__file__).resolve().parents[1]
GOLDEN = ROOT / "tests" / "golden"
if str(ROOT) not in sys.path:
    sys.path.insert(0, str(ROOT))


def reference_root():
    """The reference checkout: $REF, else the path oracle/Makefile built the
    checkers from (oracle/_ref/ref_path.txt); None when neither exists (the
    tests that compile against the reference's sources then skip)."""
    import os
    cands = [os.environ.get("REF")]
    rec = ROOT / "oracle" / "_ref" / "ref_path.txt"
    if rec.exists():
        cands.append(rec.read_text().strip())
    for c in cands:
        if c and (Path(c) / "src" / "EvalBackend.h").exists():
            return Path(c)
    return None


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: runs the CUDA path on a B200 (through the C ABI)")


@pytest.fixture(scope="session")
def oracle_lib():
    from oracle import oracle as orc
    if not orc.LIB.exists():
        subprocess.run(["make", "-C", str(ROOT / "oracle"), "oracle"], check=True, stdout=subprocess.DEVNULL)
    return orc


@pytest.fixture(scope="session")
def native():
    """The product library; built on demand when nvcc is available."""
    import galop_b200
    if not galop_b200.LIB_PATH.exists():
        from galop_b200 import build
        build.build()
    return galop_b200.load_library()


def load_vectors(variant: str) -> dict:
    with np.load(GOLDEN / f"vectors_{variant}.npz") as z:
        return {k: z[k] for k in z.files}


def bits(a: np.ndarray) -> np.ndarray:
    return np.ascontiguousarray(a, dtype=np.float32).view(np.uint32)


def same_bits(a, b) -> bool:
    return np.array_equal(bits(a), bits(b))
