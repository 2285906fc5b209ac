"""The C-ABI library: loads, exports every entry point include/galop_b200.h
declares, and behaves on a machine without a GPU (status codes, no crash).
No compute calls here."""
from __future__ import annotations

import ctypes as C
import os
import re
import subprocess
import sys

import pytest

from conftest import ROOT, reference_root

HEADER = ROOT / "include" / "galop_b200.h"


def declared_symbols():
    text = HEADER.read_text()
    return sorted(set(re.findall(r"GALOP_API\s+[\w\s\*]*?\b(galop_\w+)\s*\(", text)))


def test_header_declares_expected_entry_points():
    import galop_b200
    assert declared_symbols() == sorted(galop_b200.EXPORTED)


def test_library_exports_every_declared_symbol(native):
    out = subprocess.run(["nm", "-D", "--defined-only", str(ROOT / "galop_b200" / "libgalop_b200.so")],
                         capture_output=True, text=True, check=True).stdout
    exported = set(re.findall(r"\bT (galop_\w+)", out))
    missing = [s for s in declared_symbols() if s not in exported]
    assert not missing, missing
    for s in declared_symbols():
        assert getattr(native, s) is not None


def test_header_compiles_as_c_and_cpp(tmp_path):
    src = tmp_path / "t.c"
    src.write_text('#include "galop_b200.h"\nint main(void){galop_options o; return galop_options_init(&o);}\n')
    subprocess.run(["gcc", "-std=c99", "-Wall", "-Werror", "-fsyntax-only", f"-I{ROOT / 'include'}", str(src)],
                   check=True)
    subprocess.run(["g++", "-std=c++17", "-Wall", "-Werror", "-fsyntax-only", "-x", "c++",
                    f"-I{ROOT / 'include'}", str(src)], check=True)


@pytest.mark.skipif(reference_root() is None,
                    reason="the EvalBackend adapter compiles inside the reference's build")
def test_backend_adapter_compiles_against_reference_interface(tmp_path):
    src = tmp_path / "t.cpp"
    src.write_text('#include "galop_b200_backend.hpp"\n'
                   "int main(){ EvalBackend* b = nullptr; (void)b; "
                   "galop_options o = galop::B200Evaluator::options_from_config(); return o.num_registers; }\n")
    subprocess.run(["g++", "-std=c++20", "-fsyntax-only", f"-I{ROOT / 'include'}",
                    f"-I{reference_root() / 'src'}", str(src)], check=True)


def test_options_defaults_and_status_strings(native):
    import galop_b200 as g
    o = g._Options()
    assert native.galop_options_init(C.byref(o)) == 0
    assert (o.profile, o.num_registers, o.input_protect, o.reduce, o.device, o.intron_prepass) == \
        (g.PROFILE_REF, 8, 0, g.REDUCE_KAHAN32, 0, 1)
    assert native.galop_abi_version() == 2
    for code in (0, -1, -2, -3, -4, -5, -6, -7, -8):
        assert native.galop_status_string(code)
    assert native.galop_options_init(None) == g.E_INVALID


def test_create_rejects_bad_options(native):
    import galop_b200 as g
    for kw in (dict(num_registers=4), dict(num_registers=32), dict(profile=5), dict(reduce=9)):
        with pytest.raises(g.GalopError) as e:
            g.Evaluator(**kw)
        assert e.value.status in (g.E_INVALID, g.E_NO_DEVICE)


def test_no_device_is_a_status_not_a_fallback(native):
    """Without a visible GPU the library refuses with GALOP_E_NO_DEVICE; it
    never computes on the CPU."""
    code = ("import sys; sys.path.insert(0, %r)\n"
            "import galop_b200 as g\n"
            "try:\n    g.Evaluator()\nexcept g.GalopError as e:\n    print(e.status)\n"
            "else:\n    print('created')\n") % str(ROOT)
    env = dict(os.environ, CUDA_VISIBLE_DEVICES="")
    out = subprocess.run([sys.executable, "-c", code], env=env, capture_output=True, text=True, timeout=120)
    assert out.stdout.strip() == "-7", out.stdout + out.stderr


def test_missing_library_fails_loudly(tmp_path):
    import galop_b200 as g
    with pytest.raises(g.GalopError):
        g.load_library(tmp_path / "absent.so")
