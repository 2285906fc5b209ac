"""Build recipe for the in-tree native library.

``python -m galop_b200.build`` compiles every CUDA source under
``galop_b200/csrc`` for sm_100a and links ``galop_b200/libgalop_b200.so``.
Objects go to ``galop_b200/_build`` (not committed).  nvcc cross-compiles, so
this runs on a machine without a GPU.

``csrc/dispatch_gen.cuh`` is generated: the build first renders it from
``csrc/gen_dispatch.py`` and rewrites it when the text differs, so the
compiled tables always come from the generator.

Floating-point flags matter for parity with the CPU interpreter: no
``--use_fast_math``, ``--fmad=false`` (no FMA contraction, like the
reference's ISO C++ build), IEEE division and denormals (``-prec-div=true
-ftz=false``).
"""
from __future__ import annotations

import os
import subprocess
import sys
from concurrent.futures import ThreadPoolExecutor
from pathlib import Path

PKG = Path(__file__).resolve().parent
CSRC = PKG / "csrc"
BUILD = PKG / "_build"
LIB = PKG / "libgalop_b200.so"

NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
CFLAGS = [
    "-O3", "-lineinfo", "-std=c++17", "--fmad=false", "-prec-div=true", "-prec-sqrt=true",
    "-ftz=false", "-Xcompiler", "-fPIC", "-Xcompiler", "-fvisibility=hidden",
    "-I", str(PKG.parent / "include"),
]


def sources() -> list[Path]:
    return sorted(CSRC.glob("*.cu"))


def _needs(obj: Path, src: Path) -> bool:
    if not obj.exists():
        return True
    deps = [src, *CSRC.glob("*.cuh"), PKG.parent / "include" / "galop_b200.h"]
    return any(d.stat().st_mtime > obj.stat().st_mtime for d in deps)


def _compile(src: Path, verbose: bool) -> Path:
    obj = BUILD / (src.stem + ".o")
    if not _needs(obj, src):
        return obj
    cmd = [NVCC, *ARCH, *CFLAGS, "-c", str(src), "-o", str(obj)]
    if verbose:
        cmd.insert(1, "-Xptxas=-v")
    res = subprocess.run(cmd, capture_output=True, text=True)
    if res.returncode != 0:
        raise RuntimeError(f"nvcc failed for {src.name}:\n{res.stderr}")
    if verbose and res.stderr:
        sys.stderr.write(res.stderr)
    return obj


def regenerate_dispatch() -> bool:
    """Render csrc/dispatch_gen.cuh from csrc/gen_dispatch.py; True if the
    file was stale and has been rewritten."""
    import importlib.util
    spec = importlib.util.spec_from_file_location("galop_gen_dispatch", CSRC / "gen_dispatch.py")
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    return mod.write_if_changed(CSRC / "dispatch_gen.cuh")


def build(verbose: bool = False, jobs: int | None = None) -> Path:
    BUILD.mkdir(exist_ok=True)
    regenerate_dispatch()
    srcs = sources()
    with ThreadPoolExecutor(max_workers=jobs or min(8, os.cpu_count() or 1)) as ex:
        objs = list(ex.map(lambda s: _compile(s, verbose), srcs))
    if LIB.exists() and all(o.stat().st_mtime <= LIB.stat().st_mtime for o in objs):
        return LIB
    cmd = [NVCC, *ARCH, "-shared", "-o", str(LIB), *map(str, objs), "-lcudart"]
    res = subprocess.run(cmd, capture_output=True, text=True)
    if res.returncode != 0:
        raise RuntimeError(f"link failed:\n{res.stderr}")
    return LIB


if __name__ == "__main__":
    print(build(verbose="-v" in sys.argv))
