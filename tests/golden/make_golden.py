"""Regenerate the golden fixtures in tests/golden/ from the reference itself.

Runs in a checkout that has the reference sources (the REF environment
variable names the checkout): builds oracle/_ref/ with ``make -C oracle`` (the reference's
own src/*.cpp compiled where they lie) and records what the REFERENCE CODE
computes:

* ``datasets/nguyen{1,2,3}_{train,test}.csv`` -- written by the reference's
  make_sr_dataset_1d + write_csv with tools/gen_datasets.cpp's seeds and
  sizes, and checked byte-for-byte against the reference's datasets/.
* ``histories/{hist,prog}_nguyen{1,2,3}_s{0,1,2}.*.gz`` -- 1000-generation
  golden runs of the reference's LGPEngine + CpuEvaluator, checked
  byte-for-byte against the reference's golden/ (SHA256SUMS there).
* ``vectors_{nr8,nr16,ip16}.npz`` -- random programs and datasets with the
  reference's per-case outputs (Interpreter::run_stateless), fitness
  (CpuEvaluator / Evaluator::evaluate_sr_mse) and intron masks
  (Introns::effective_mask) for each compile-time configuration.
* ``ops_ref.npz`` -- ISA::apply_op on special and random operand pairs.

Usage: python tests/golden/make_golden.py   (from the repository root)
"""
from __future__ import annotations

import gzip
import hashlib
import os
import subprocess
import sys
import tempfile
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parents[2]
sys.path.insert(0, str(ROOT))
from oracle.oracle import RefLib  # noqa: E402
from galop_b200 import workloads as W  # noqa: E402

if "REF" not in os.environ:
    sys.exit("set REF to the reference checkout (the directory holding src/ and golden/)")
REF = Path(os.environ["REF"])
OUT = Path(__file__).resolve().parent


def build():
    subprocess.run(["make", "-C", str(ROOT / "oracle"), "-j8", f"REF={REF}"], check=True,
                   stdout=subprocess.DEVNULL)


def datasets():
    d = OUT / "datasets"
    d.mkdir(exist_ok=True)
    lib = RefLib("nr8").lib
    import ctypes as C
    lib.ref_write_nguyen_csv.restype = C.c_int
    lib.ref_write_nguyen_csv.argtypes = [C.c_int, C.c_int, C.c_float, C.c_float, C.c_uint32, C.c_char_p]
    for t in (1, 2, 3):
        for split, n, seed in (("train", 32, 1234), ("test", 100, 5678)):
            p = d / f"nguyen{t}_{split}.csv"
            assert lib.ref_write_nguyen_csv(t, n, -1.0, 1.0, seed, str(p).encode()) == 0
            ref = (REF / "datasets" / p.name).read_bytes()
            assert p.read_bytes() == ref, f"{p.name} differs from the reference's datasets/"
    print("datasets: 6 files, byte-identical to the reference")


def histories():
    h = OUT / "histories"
    h.mkdir(exist_ok=True)
    tmp = Path(tempfile.mkdtemp(prefix="golden_regen_"))
    exe = ROOT / "oracle" / "_ref" / "lgp_run_cpu"
    procs = []
    env = dict(os.environ, OMP_NUM_THREADS="1")
    for t in ("nguyen1", "nguyen2", "nguyen3"):
        for s in (0, 1, 2):
            procs.append(subprocess.Popen(
                [str(exe), str(OUT / "datasets" / f"{t}_train.csv"), str(OUT / "datasets" / f"{t}_test.csv"),
                 t, str(s), str(tmp / "results.csv"), str(tmp / f"prog_{t}_s{s}.txt"),
                 str(tmp / f"hist_{t}_s{s}.csv")], env=env))
    for p in procs:
        assert p.wait() == 0
    sums = {}
    for line in (REF / "golden" / "SHA256SUMS").read_text().splitlines():
        digest, name = line.split()
        sums[name.lstrip("*").split("/")[-1]] = digest
    n = 0
    for f in sorted(tmp.glob("*_nguyen*")):
        data = f.read_bytes()
        assert data == (REF / "golden" / f.name).read_bytes(), f"{f.name} differs from golden/"
        assert hashlib.sha256(data).hexdigest() == sums[f.name]
        with gzip.GzipFile(h / (f.name + ".gz"), "wb", mtime=0) as g:
            g.write(data)
        n += 1
    print(f"histories: {n} files, byte-identical to the reference's golden/")


def special_floats():
    return np.array([0.0, -0.0, 1.0, -1.0, 0.5, 2.0, 3.14159, 1e-45, -1e-45, 1e-38, 3.4e38, -3.4e38,
                     np.inf, -np.inf, np.nan, 1e10, -1e10, 100.0, 1e5, 123456.7, -7.25, 88.7, 89.0, -104.0],
                    dtype=np.float32)


def ops_vectors():
    lib = RefLib("nr8")
    rng = np.random.default_rng(11)
    sp = special_floats()
    a = np.concatenate([np.repeat(sp, sp.size), rng.uniform(-10, 10, 2000).astype(np.float32),
                        (rng.standard_normal(2000) * 1e4).astype(np.float32),
                        rng.uniform(-1e6, 1e6, 1000).astype(np.float32)])
    b = np.concatenate([np.tile(sp, sp.size), rng.uniform(-10, 10, 2000).astype(np.float32),
                        (rng.standard_normal(2000) * 1e4).astype(np.float32),
                        rng.uniform(-1e6, 1e6, 1000).astype(np.float32)])
    out = np.empty((8, a.size), dtype=np.float32)
    for op in range(8):
        out[op] = [lib.apply_op(op, float(x), float(y)) for x, y in zip(a, b)]
    np.savez_compressed(OUT / "ops_ref.npz", a=a, b=b, out=out)
    print(f"ops: {a.size} operand pairs x 8 ops")


def vectors(variant: str, seed: int):
    lib = RefLib(variant)
    nr, maxp = lib.num_registers, lib.max_program_size
    rng = np.random.default_rng(seed)
    progs = []
    # hand-picked edge programs
    progs.append(np.zeros(0, np.uint32))                                  # empty program
    progs.append(np.array([lib.encode_manual(3, 0, 0, 1, 0)], np.uint32))  # r0 = r0 / r1 (protected)
    progs.append(np.array([lib.encode_manual(4, 0, 0, 0, 0)], np.uint32))  # r0 = sin(r0)
    progs.append(np.array([lib.encode_manual(2, nr - 1, 0, 0, 0), lib.encode_manual(0, 0, nr - 1, 1, 1)],
                          np.uint32))
    for op in range(8):                                                   # every op, reg and const src2
        for kc in (0, 1):
            progs.append(np.array([lib.encode_manual(op, 0, 0, 1 % nr, kc),
                                   lib.encode_manual(op, 1 % nr, 0, 0, kc),
                                   lib.encode_manual((op + 3) % 8, 0, 1 % nr, 0, 1 - kc)], np.uint32))
    # random programs, raw random words (masked by the reference's encoder)
    for _ in range(300):
        L = int(rng.integers(0, maxp + 1))
        raw = rng.integers(0, 2**32, size=L, dtype=np.uint64).astype(np.uint32)
        progs.append(np.array([lib.encode_from_random(int(x)) for x in raw], np.uint32))
    # unmasked random words: the decoders mask them
    for _ in range(50):
        L = int(rng.integers(1, maxp + 1))
        progs.append(rng.integers(0, 2**32, size=L, dtype=np.uint64).astype(np.uint32))
    lens = np.array([p.size for p in progs], np.int64)
    offsets = W.csr_offsets(lens)
    words = np.concatenate(progs).astype(np.uint32)

    cases = {}
    for name, n, k, lo, hi in (("d1", 100, 1, -1.0, 1.0), ("d2", 1, 1, -2.0, 2.0), ("d3", 257, 3, -3.0, 3.0),
                               ("d4", 64, min(5, nr), -10.0, 10.0)):
        X = rng.uniform(lo, hi, size=(n, k)).astype(np.float32)
        y = (rng.standard_normal(n) * 2).astype(np.float32)
        outs = np.stack([lib.case_outputs(words[offsets[i]:offsets[i + 1]], X)
                         for i in range(len(progs))]) if n else np.zeros((len(progs), 0), np.float32)
        fit, mse = lib.evaluate_csr(words, offsets, X, y, threads=1, with_mse=True)
        # dense layout through CpuEvaluator (program i at i*MAX_PROGRAM_SIZE)
        dense = np.zeros((len(progs), maxp), np.uint32)
        for i, p in enumerate(progs):
            dense[i, :p.size] = p
        fit_dense = lib.evaluate_population(dense, lens.astype(np.uint8), X, y)
        assert np.array_equal(fit.view(np.uint32), fit_dense.view(np.uint32))
        cases[name] = dict(X=X, y=y, outputs=outs, fitness=fit, mse=mse)
    masks = np.concatenate([lib.effective_mask(p) for p in progs]).astype(np.uint8) \
        if words.size else np.zeros(0, np.uint8)
    arrs = dict(words=words, offsets=offsets, masks=masks, constants=lib.constants,
                num_registers=nr, output_reg=lib.output_reg, input_protect=int(lib.input_protect),
                max_program_size=maxp)
    for name, d in cases.items():
        for key, v in d.items():
            arrs[f"{name}_{key}"] = v
    np.savez_compressed(OUT / f"vectors_{variant}.npz", **arrs)
    print(f"vectors_{variant}: {len(progs)} programs x {len(cases)} datasets")


def main():
    if not (REF / "src" / "ISA.h").exists():
        sys.exit(f"reference sources not found under {REF}")
    build()
    datasets()
    histories()
    ops_vectors()
    for i, v in enumerate(("nr8", "nr16", "ip16")):
        vectors(v, 100 + i)


if __name__ == "__main__":
    main()
