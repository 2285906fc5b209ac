"""CSV datasets and the R^2 objective against the
reference's own loaders (load_csv_1d / load_csv_multi, src/Dataset.cpp:83-151)
and its R^2 evaluator (src/Evaluator.cpp:49-97), compiled from its sources."""
from __future__ import annotations

import numpy as np
import pytest

import galop_b200 as g
from conftest import GOLDEN, bits, load_vectors

from oracle import oracle

try:
    REF = oracle.RefLib("nr8")
except FileNotFoundError:
    REF = None
needs_ref = pytest.mark.skipif(REF is None, reason="oracle/_ref not built")

VARIANTS = {"nr8": (8, False), "nr16": (16, False), "ip16": (16, True)}


def _same_dataset(path, multi):
    want = REF.load_csv(path, multi)
    assert want is not None, path
    got = g.Dataset.from_csv(path, multi)
    X, y, ss = want
    assert got.inputs.shape == X.shape
    assert np.array_equal(bits(got.inputs), bits(X)) and np.array_equal(bits(got.targets), bits(y))
    assert got.ss_tot == ss or (np.isnan(got.ss_tot) and np.isnan(ss))


@needs_ref
@pytest.mark.parametrize("name", [f"nguyen{i}_{s}" for i in (1, 2, 3) for s in ("train", "test")])
def test_golden_csvs_read_like_the_reference(name):
    _same_dataset(GOLDEN / "datasets" / f"{name}.csv", multi=False)
    _same_dataset(GOLDEN / "datasets" / f"{name}.csv", multi=True)


@needs_ref
def test_csv_formats_read_like_the_reference(tmp_path):
    rng = np.random.default_rng(3)
    X = rng.standard_normal((300, 4)).astype(np.float32) * np.float32(1e3)
    y = rng.standard_normal(300).astype(np.float32)
    p = tmp_path / "multi.csv"
    with open(p, "w") as f:
        f.write("a,b,c,d,y\n")
        for i in range(300):
            if i % 50 == 7:
                f.write("\n")                                    # blank lines are skipped
            row = ",".join(f"{v:.9g}" for v in X[i]) + f",{y[i]:.6e}"
            f.write((" " + row if i % 3 == 0 else row) + ("\r\n" if i % 5 == 0 else "\n"))
    _same_dataset(p, multi=True)
    q = tmp_path / "one.csv"
    with open(q, "w") as f:
        f.write("x,y\n1.5,2.25\nno comma here\n\n-3,inf\n7e-3,  -1e+2\n")
    _same_dataset(q, multi=False)


@needs_ref
def test_csv_errors(tmp_path):
    cases = {"bad.csv": "x,y\n1,2\nabc,3\n", "range.csv": "x,y\n1,1e60\n"}
    for name, text in cases.items():
        p = tmp_path / name
        p.write_text(text)
        assert REF.load_csv(p, False) is None
        with pytest.raises(g.GalopError) as e:
            g.Dataset.from_csv(p)
        assert e.value.status == g.E_INVALID
    ragged = tmp_path / "ragged.csv"
    ragged.write_text("a,b,y\n1,2,3\n4,5\n")
    with pytest.raises(g.GalopError):
        g.Dataset.from_csv(ragged, multi=True)
    with pytest.raises(g.GalopError):
        g.Dataset.from_csv(tmp_path / "missing.csv")


@needs_ref
@pytest.mark.parametrize("variant", list(VARIANTS))
def test_oracle_r2_matches_reference(variant):
    """The C restatement's R^2 fitness equals the reference's
    Evaluator::evaluate_sr_r2 + r2_to_fitness bit for bit on the golden
    programs and datasets."""
    v = load_vectors(variant)
    nr, ip = VARIANTS[variant]
    ref = oracle.RefLib(variant)
    o = oracle.Oracle(oracle.PROFILE_REF, nr, ip)
    for d in ("d1", "d2", "d3", "d4"):
        X, y = v[f"{d}_X"], v[f"{d}_y"]
        ss = oracle.Oracle.ss_tot(y)
        want = ref.evaluate_csr_r2(v["words"], v["offsets"], X, y, ss)
        got = o.evaluate_csr_r2(v["words"], v["offsets"], X, y)
        assert np.array_equal(bits(got), bits(want)), d
        assert (got >= 0).all() and (got <= 1).all()
    # a constant target is degenerate: R^2 fitness 0 everywhere
    y0 = np.full_like(v["d1_y"], 3.0)
    assert not ref.evaluate_csr_r2(v["words"], v["offsets"], v["d1_X"], y0, 0.0).any()
    assert not o.evaluate_csr_r2(v["words"], v["offsets"], v["d1_X"], y0).any()
