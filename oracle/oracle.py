"""ctypes view of the checkers (TEST INFRASTRUCTURE ONLY).

``Oracle`` binds ``oracle/liboracle.so`` (the C restatement in oracle.c);
``RefLib`` binds ``oracle/_ref/libref_*.so`` (the reference's own evaluation
code behind ref_shim.cpp).  Only tests/, the smoke check and bench.py's CPU
baseline legs import this module; the product (galop_b200) never does.
"""
from __future__ import annotations

import ctypes as C
import subprocess
from pathlib import Path
from typing import Optional, Sequence

import numpy as np

HERE = Path(__file__).resolve().parent
LIB = HERE / "liboracle.so"
REF_DIR = HERE / "_ref"

PROFILE_REF, PROFILE_BJ = 0, 1
TRIG_LIBM, TRIG_DEVICE = 0, 1
_OP_DEVICE_TRIG = 0x100   # orc_apply_op mode flag (oracle.c ORC_OP_DEVICE_TRIG)


class OrcIsa(C.Structure):
    _fields_ = [("profile", C.c_int32), ("num_registers", C.c_int32), ("input_protect", C.c_int32),
                ("trig", C.c_int32), ("constants", C.POINTER(C.c_float))]


def build(quiet: bool = True) -> None:
    """Compile liboracle.so (and oracle/_ref when the reference is present)."""
    subprocess.run(["make", "-C", str(HERE), "-j8"], check=True,
                   stdout=subprocess.DEVNULL if quiet else None)


def _p(a, t):
    return None if a is None else a.ctypes.data_as(C.POINTER(t))


_U32, _I64, _F32, _F64, _U8 = C.c_uint32, C.c_int64, C.c_float, C.c_double, C.c_uint8


class Oracle:
    """The C restatement, configured like one evaluator context."""

    _lib: Optional[C.CDLL] = None

    def __init__(self, profile: int = PROFILE_REF, num_registers: int = 8, input_protect: bool = False,
                 constants: Optional[Sequence[float]] = None, trig: int = TRIG_LIBM):
        """trig: TRIG_LIBM (SIN/COS by the C library, as the reference) or
        TRIG_DEVICE (the device's own sine and cosine, galop_b200/csrc/trig.cuh,
        for bit-for-bit checks of GPU outputs on programs using them)."""
        lib = self.lib()
        if constants is None:
            from galop_b200 import REF_CONSTANTS_8, REF_CONSTANTS_16
            constants = REF_CONSTANTS_16 if num_registers == 16 else REF_CONSTANTS_8
        self.constants = np.ascontiguousarray(constants, dtype=np.float32)
        assert self.constants.shape == (num_registers,)
        self.isa = OrcIsa(profile, num_registers, int(bool(input_protect)), int(trig), _p(self.constants, _F32))
        self.trig = int(trig)
        self.num_registers = num_registers
        self.profile = profile
        self.input_protect = bool(input_protect)
        self.output_reg = lib.orc_output_reg(C.byref(self.isa))

    @classmethod
    def lib(cls) -> C.CDLL:
        if cls._lib is None:
            if not LIB.exists():
                build()
            lib = C.CDLL(str(LIB))
            P = C.POINTER
            sig = {
                "orc_output_reg": (C.c_int, [P(OrcIsa)]),
                "orc_decode": (C.c_int, [P(OrcIsa), C.c_uint32, P(C.c_int32)]),
                "orc_apply_op": (C.c_float, [C.c_int, C.c_int, C.c_float, C.c_float]),
                "orc_apply_op_n": (None, [C.c_int, C.c_int, P(_F32), P(_F32), _I64, P(_F32)]),
                "orc_case_outputs": (None, [P(OrcIsa), P(_U32), _I64, P(_F32), C.c_int, _I64, P(_F32)]),
                "orc_case_outputs_f64": (None, [P(OrcIsa), P(_U32), _I64, P(_F32), C.c_int, _I64, P(_F64)]),
                "orc_trace_case": (None, [P(OrcIsa), P(_U32), _I64, P(_F32), C.c_int, P(_F32)]),
                "orc_sse": (C.c_double, [P(OrcIsa), P(_U32), _I64, P(_F32), P(_F32), C.c_int, _I64]),
                "orc_evaluate_sr_mse": (C.c_float, [P(OrcIsa), P(_U32), _I64, P(_F32), P(_F32), C.c_int, _I64]),
                "orc_mse_to_fitness": (C.c_float, [C.c_float]),
                "orc_trig_accuracy": (None, [C.c_int, C.c_uint32, C.c_uint32, C.c_uint32, P(_F64)]),
                "orc_evaluate_population_csr": (None, [P(OrcIsa), P(_U32), P(_I64), _I64, P(_F32), P(_F32),
                                                       C.c_int, _I64, P(_F32), P(_F64), C.c_int]),
                "orc_evaluate_population_dense": (None, [P(OrcIsa), P(_U32), P(_U8), _I64, _I64, P(_F32),
                                                         P(_F32), C.c_int, _I64, P(_F32)]),
                "orc_case_outputs_csr": (None, [P(OrcIsa), P(_U32), P(_I64), _I64, P(_F32), C.c_int, _I64,
                                                P(_F32), C.c_int, C.c_int]),
                "orc_evaluate_population_csr_opt": (None, [P(OrcIsa), P(_U32), P(_I64), _I64, P(_F32), P(_F32),
                                                           C.c_int, _I64, P(_F32), P(_F64), C.c_int, C.c_int]),
                "orc_extract_effective_csr": (None, [P(OrcIsa), P(_U32), P(_I64), _I64, P(_I64), P(_U32),
                                                     C.c_int]),
                "orc_effective_mask": (_I64, [P(OrcIsa), P(_U32), _I64, P(_U8)]),
                "orc_extract_effective": (_I64, [P(OrcIsa), P(_U32), _I64, P(_U32)]),
                "orc_effective_lengths_csr": (None, [P(OrcIsa), P(_U32), P(_I64), _I64, P(_I64)]),
                "orc_max_threads": (C.c_int, []),
                "orc_ss_tot": (C.c_double, [P(_F32), _I64]),
                "orc_evaluate_sr_r2": (C.c_float, [P(OrcIsa), P(_U32), _I64, P(_F32), P(_F32), C.c_int, _I64,
                                                   C.c_double]),
                "orc_r2_to_fitness": (C.c_float, [C.c_float]),
                "orc_evaluate_population_csr_r2": (None, [P(OrcIsa), P(_U32), P(_I64), _I64, P(_F32), P(_F32),
                                                          C.c_int, _I64, P(_F32), C.c_int]),
            }
            for name, (res, args) in sig.items():
                fn = getattr(lib, name)
                fn.restype, fn.argtypes = res, args
            cls._lib = lib
        return cls._lib

    # --- single program --------------------------------------------------------
    def decode(self, word: int):
        out = (C.c_int32 * 5)()
        unary = self.lib().orc_decode(C.byref(self.isa), word, out)
        return tuple(out) + (unary,)

    @classmethod
    def trig_accuracy(cls, cosine: bool, lo: float, hi: float, stride: int = 1) -> dict:
        """The device's sine or cosine (galop_b200/csrc/trig.cuh, host build)
        over the non-negative floats lo <= x <= hi with bit-pattern stride
        `stride`, against the correctly rounded value and the C library."""
        out = np.zeros(7, np.float64)
        lo_b = int(np.float32(lo).view(np.uint32))
        hi_b = int(np.float32(hi).view(np.uint32))
        cls.lib().orc_trig_accuracy(int(bool(cosine)), lo_b, hi_b, stride, _p(out, _F64))
        n = int(out[0])
        return {"values": n, "max_ulp": float(out[1]), "at": float(out[2]), "correctly_rounded": int(out[3]) / n,
                "equal_to_libm": int(out[4]) / n, "over_1ulp": int(out[5]), "asymmetric": int(out[6])}

    def _op_mode(self) -> int:
        return self.profile | (_OP_DEVICE_TRIG if self.trig == TRIG_DEVICE else 0)

    def apply_op(self, op: int, a: float, b: float) -> float:
        return self.lib().orc_apply_op(self._op_mode(), op, a, b)

    def apply_op_n(self, op: int, a, b) -> np.ndarray:
        a = np.ascontiguousarray(a, dtype=np.float32)
        b = np.ascontiguousarray(b, dtype=np.float32)
        out = np.empty(a.shape[0], dtype=np.float32)
        self.lib().orc_apply_op_n(self._op_mode(), op, _p(a, _F32), _p(b, _F32), a.shape[0], _p(out, _F32))
        return out

    def case_outputs(self, prog, inputs, n_cases=None) -> np.ndarray:
        prog = np.ascontiguousarray(prog, dtype=np.uint32)
        inputs = np.ascontiguousarray(inputs, dtype=np.float32)
        k = inputs.shape[1] if inputs.ndim == 2 else 1
        n = inputs.shape[0] if n_cases is None else n_cases
        out = np.empty(n, dtype=np.float32)
        self.lib().orc_case_outputs(C.byref(self.isa), _p(prog, _U32), prog.shape[0], _p(inputs, _F32), k, n,
                                    _p(out, _F32))
        return out

    def case_outputs_f64(self, prog, inputs) -> np.ndarray:
        prog = np.ascontiguousarray(prog, dtype=np.uint32)
        inputs = np.ascontiguousarray(inputs, dtype=np.float32)
        k = inputs.shape[1]
        out = np.empty(inputs.shape[0], dtype=np.float64)
        self.lib().orc_case_outputs_f64(C.byref(self.isa), _p(prog, _U32), prog.shape[0], _p(inputs, _F32), k,
                                        inputs.shape[0], _p(out, _F64))
        return out

    def trace_case(self, prog, x) -> np.ndarray:
        prog = np.ascontiguousarray(prog, dtype=np.uint32)
        x = np.ascontiguousarray(x, dtype=np.float32)
        st = np.empty((prog.shape[0] + 1, self.num_registers), dtype=np.float32)
        self.lib().orc_trace_case(C.byref(self.isa), _p(prog, _U32), prog.shape[0], _p(x, _F32), x.shape[0],
                                  _p(st, _F32))
        return st

    def sse(self, prog, inputs, targets) -> float:
        prog = np.ascontiguousarray(prog, dtype=np.uint32)
        inputs = np.ascontiguousarray(inputs, dtype=np.float32)
        targets = np.ascontiguousarray(targets, dtype=np.float32)
        return self.lib().orc_sse(C.byref(self.isa), _p(prog, _U32), prog.shape[0], _p(inputs, _F32),
                                  _p(targets, _F32), inputs.shape[1], inputs.shape[0])

    def effective_mask(self, prog) -> np.ndarray:
        prog = np.ascontiguousarray(prog, dtype=np.uint32)
        m = np.empty(max(prog.shape[0], 1), dtype=np.uint8)
        self.lib().orc_effective_mask(C.byref(self.isa), _p(prog, _U32), prog.shape[0], _p(m, _U8))
        return m[: prog.shape[0]].astype(bool)

    # --- populations -------------------------------------------------------------
    def evaluate_csr(self, words, offsets, inputs, targets, threads: int = 0, with_sse: bool = False):
        words = np.ascontiguousarray(words, dtype=np.uint32)
        offsets = np.ascontiguousarray(offsets, dtype=np.int64)
        inputs = np.ascontiguousarray(inputs, dtype=np.float32)
        targets = np.ascontiguousarray(targets, dtype=np.float32)
        n = offsets.shape[0] - 1
        fit = np.empty(n, dtype=np.float32)
        sse = np.empty(n, dtype=np.float64)
        self.lib().orc_evaluate_population_csr(C.byref(self.isa), _p(words, _U32), _p(offsets, _I64), n,
                                               _p(inputs, _F32), _p(targets, _F32), inputs.shape[1],
                                               inputs.shape[0], _p(fit, _F32), _p(sse, _F64), threads)
        return (fit, sse) if with_sse else fit

    def case_outputs_csr(self, words, offsets, inputs, threads: int = 0, effective_only: bool = False,
                         n_cases=None) -> np.ndarray:
        """Per-case outputs of CSR programs, shape (n_programs, n_cases)."""
        words = np.ascontiguousarray(words, dtype=np.uint32)
        offsets = np.ascontiguousarray(offsets, dtype=np.int64)
        inputs = np.ascontiguousarray(inputs, dtype=np.float32)
        k = inputs.shape[1] if inputs.ndim == 2 else 1
        N = inputs.shape[0] if n_cases is None else n_cases
        n = offsets.shape[0] - 1
        out = np.empty((n, N), dtype=np.float32)
        self.lib().orc_case_outputs_csr(C.byref(self.isa), _p(words, _U32), _p(offsets, _I64), n,
                                        _p(inputs, _F32), k, N, _p(out, _F32), threads, int(effective_only))
        return out

    def evaluate_csr_opt(self, words, offsets, inputs, targets, threads: int = 0, effective_only: bool = False):
        """(fitness, double SSE) of CSR programs; see orc_evaluate_population_csr_opt."""
        words = np.ascontiguousarray(words, dtype=np.uint32)
        offsets = np.ascontiguousarray(offsets, dtype=np.int64)
        inputs = np.ascontiguousarray(inputs, dtype=np.float32)
        targets = np.ascontiguousarray(targets, dtype=np.float32)
        n = offsets.shape[0] - 1
        fit = np.empty(n, dtype=np.float32)
        sse = np.empty(n, dtype=np.float64)
        k = inputs.shape[1] if inputs.ndim == 2 else 1
        self.lib().orc_evaluate_population_csr_opt(C.byref(self.isa), _p(words, _U32), _p(offsets, _I64), n,
                                                   _p(inputs, _F32), _p(targets, _F32), k, inputs.shape[0],
                                                   _p(fit, _F32), _p(sse, _F64), threads, int(effective_only))
        return fit, sse

    def evaluate_csr_r2(self, words, offsets, inputs, targets, threads: int = 0):
        """R^2 fitness (src/Evaluator.cpp:49-97) of CSR programs."""
        words = np.ascontiguousarray(words, dtype=np.uint32)
        offsets = np.ascontiguousarray(offsets, dtype=np.int64)
        inputs = np.ascontiguousarray(inputs, dtype=np.float32)
        targets = np.ascontiguousarray(targets, dtype=np.float32)
        n = offsets.shape[0] - 1
        fit = np.empty(n, dtype=np.float32)
        self.lib().orc_evaluate_population_csr_r2(C.byref(self.isa), _p(words, _U32), _p(offsets, _I64), n,
                                                  _p(inputs, _F32), _p(targets, _F32), inputs.shape[1],
                                                  inputs.shape[0], _p(fit, _F32), threads)
        return fit

    @staticmethod
    def ss_tot(targets) -> float:
        targets = np.ascontiguousarray(targets, dtype=np.float32)
        return Oracle.lib().orc_ss_tot(_p(targets, _F32), targets.shape[0])

    def effective_lengths(self, words, offsets) -> np.ndarray:
        words = np.ascontiguousarray(words, dtype=np.uint32)
        offsets = np.ascontiguousarray(offsets, dtype=np.int64)
        n = offsets.shape[0] - 1
        out = np.empty(n, dtype=np.int64)
        self.lib().orc_effective_lengths_csr(C.byref(self.isa), _p(words, _U32), _p(offsets, _I64), n,
                                             _p(out, _I64))
        return out

    def extract_effective_csr(self, words, offsets, threads: int = 0):
        """(effective words, offsets) of every program, host-side: the
        reference's PackedEffective layout."""
        words = np.ascontiguousarray(words, dtype=np.uint32)
        offsets = np.ascontiguousarray(offsets, dtype=np.int64)
        eff = self.effective_lengths(words, offsets)
        eoff = np.zeros(eff.size + 1, dtype=np.int64)
        np.cumsum(eff, out=eoff[1:])
        out = np.empty(int(eoff[-1]), dtype=np.uint32)
        self.lib().orc_extract_effective_csr(C.byref(self.isa), _p(words, _U32), _p(offsets, _I64), eff.size,
                                             _p(eoff, _I64), _p(out, _U32), threads)
        return out, eoff

    @staticmethod
    def mse_to_fitness(mse: float) -> float:
        return Oracle.lib().orc_mse_to_fitness(mse)


class RefLib:
    """The reference's own evaluation code for one compile-time config:
    variant in {"nr8", "nr16", "ip16"}."""

    def __init__(self, variant: str = "nr8"):
        path = REF_DIR / f"libref_{variant}.so"
        if not path.exists():
            raise FileNotFoundError(f"{path} not built (make -C oracle needs the reference sources)")
        lib = C.CDLL(str(path))
        P = C.POINTER
        sig = {
            "ref_num_registers": (C.c_int, []), "ref_output_reg": (C.c_int, []),
            "ref_input_protect": (C.c_int, []), "ref_max_program_size": (C.c_int, []),
            "ref_num_contexts": (C.c_int, []), "ref_constants": (None, [P(_F32)]),
            "ref_encode_manual": (C.c_uint32, [C.c_int] * 5),
            "ref_encode_from_random": (C.c_uint32, [C.c_uint32]),
            "ref_decode": (None, [C.c_uint32, P(C.c_int)]),
            "ref_apply_op": (C.c_float, [C.c_int, C.c_float, C.c_float]),
            "ref_run_stateless": (None, [P(_U32), C.c_int, P(_F32), C.c_int, P(_F32)]),
            "ref_case_outputs": (None, [P(_U32), C.c_int, P(_F32), C.c_int, C.c_int, P(_F32)]),
            "ref_evaluate_population": (None, [P(_U32), P(_U8), P(_F32), C.c_int, P(_F32), P(_F32), C.c_int,
                                               C.c_int]),
            "ref_evaluate_csr": (None, [P(_U32), P(_I64), _I64, P(_F32), P(_F32), C.c_int, C.c_int, P(_F32),
                                        P(_F32), C.c_int]),
            "ref_effective_mask": (C.c_int, [P(_U32), C.c_int, C.c_char_p]),
            "ref_max_threads": (C.c_int, []),
            "ref_evaluate_csr_r2": (None, [P(_U32), P(_I64), _I64, P(_F32), P(_F32), C.c_int, C.c_int, C.c_double,
                                           P(_F32), P(_F32)]),
            "ref_load_csv": (C.c_int, [C.c_char_p, C.c_int, P(_I64), P(C.c_int), P(_F32), P(_F32),
                                       P(C.c_double)]),
        }
        for name, (res, args) in sig.items():
            fn = getattr(lib, name)
            fn.restype, fn.argtypes = res, args
        self.lib = lib
        self.variant = variant
        self.num_registers = lib.ref_num_registers()
        self.output_reg = lib.ref_output_reg()
        self.input_protect = bool(lib.ref_input_protect())
        self.max_program_size = lib.ref_max_program_size()
        c = np.empty(self.num_registers, dtype=np.float32)
        lib.ref_constants(_p(c, _F32))
        self.constants = c

    def encode_manual(self, op, dest, src1, src2, is_const) -> int:
        return self.lib.ref_encode_manual(op, dest, src1, src2, int(bool(is_const)))

    def encode_from_random(self, raw: int) -> int:
        return self.lib.ref_encode_from_random(raw)

    def decode(self, w: int):
        out = (C.c_int * 5)()
        self.lib.ref_decode(w, out)
        return tuple(out)

    def apply_op(self, op, a, b) -> float:
        return self.lib.ref_apply_op(op, a, b)

    def run_stateless(self, prog, inputs32) -> np.ndarray:
        prog = np.ascontiguousarray(prog, dtype=np.uint32)
        inputs32 = np.ascontiguousarray(inputs32, dtype=np.float32)
        k = inputs32.shape[1]
        out = np.empty(32, dtype=np.float32)
        self.lib.ref_run_stateless(_p(prog, _U32), prog.shape[0], _p(inputs32, _F32), k, _p(out, _F32))
        return out

    def case_outputs(self, prog, inputs) -> np.ndarray:
        prog = np.ascontiguousarray(prog, dtype=np.uint32)
        inputs = np.ascontiguousarray(inputs, dtype=np.float32)
        out = np.empty(inputs.shape[0], dtype=np.float32)
        self.lib.ref_case_outputs(_p(prog, _U32), prog.shape[0], _p(inputs, _F32), inputs.shape[1],
                                  inputs.shape[0], _p(out, _F32))
        return out

    def evaluate_population(self, instr, lengths, inputs, targets) -> np.ndarray:
        instr = np.ascontiguousarray(instr, dtype=np.uint32)
        lengths = np.ascontiguousarray(lengths, dtype=np.uint8)
        inputs = np.ascontiguousarray(inputs, dtype=np.float32)
        targets = np.ascontiguousarray(targets, dtype=np.float32)
        n = lengths.shape[0]
        assert instr.size >= n * self.max_program_size
        fit = np.empty(n, dtype=np.float32)
        self.lib.ref_evaluate_population(_p(instr, _U32), _p(lengths, _U8), _p(fit, _F32), n, _p(inputs, _F32),
                                         _p(targets, _F32), inputs.shape[0], inputs.shape[1])
        return fit

    def evaluate_csr(self, words, offsets, inputs, targets, threads: int = 1, with_mse: bool = False):
        words = np.ascontiguousarray(words, dtype=np.uint32)
        offsets = np.ascontiguousarray(offsets, dtype=np.int64)
        inputs = np.ascontiguousarray(inputs, dtype=np.float32)
        targets = np.ascontiguousarray(targets, dtype=np.float32)
        n = offsets.shape[0] - 1
        fit = np.empty(n, dtype=np.float32)
        mse = np.empty(n, dtype=np.float32)
        self.lib.ref_evaluate_csr(_p(words, _U32), _p(offsets, _I64), n, _p(inputs, _F32), _p(targets, _F32),
                                  inputs.shape[0], inputs.shape[1], _p(fit, _F32), _p(mse, _F32), threads)
        return (fit, mse) if with_mse else fit

    def evaluate_csr_r2(self, words, offsets, inputs, targets, ss_tot: float, with_r2: bool = False):
        words = np.ascontiguousarray(words, dtype=np.uint32)
        offsets = np.ascontiguousarray(offsets, dtype=np.int64)
        inputs = np.ascontiguousarray(inputs, dtype=np.float32)
        targets = np.ascontiguousarray(targets, dtype=np.float32)
        n = offsets.shape[0] - 1
        fit = np.empty(n, dtype=np.float32)
        r2 = np.empty(n, dtype=np.float32)
        self.lib.ref_evaluate_csr_r2(_p(words, _U32), _p(offsets, _I64), n, _p(inputs, _F32), _p(targets, _F32),
                                     inputs.shape[0], inputs.shape[1], ss_tot, _p(fit, _F32), _p(r2, _F32))
        return (fit, r2) if with_r2 else fit

    def load_csv(self, path, multi: bool = False):
        """The reference's load_csv_1d / load_csv_multi: (inputs (N, k),
        targets (N,), ss_tot), or None when it throws."""
        n, k, ss = _I64(0), C.c_int(0), C.c_double(0.0)
        if self.lib.ref_load_csv(str(path).encode(), int(bool(multi)), C.byref(n), C.byref(k), None, None,
                                 C.byref(ss)) != 0:
            return None
        X = np.empty((n.value, k.value), dtype=np.float32)
        y = np.empty(n.value, dtype=np.float32)
        self.lib.ref_load_csv(str(path).encode(), int(bool(multi)), C.byref(n), C.byref(k), _p(X, _F32),
                              _p(y, _F32), C.byref(ss))
        return X, y, ss.value

    def effective_mask(self, prog) -> np.ndarray:
        prog = np.ascontiguousarray(prog, dtype=np.uint32)
        m = C.create_string_buffer(max(prog.shape[0], 1))
        self.lib.ref_effective_mask(_p(prog, _U32), prog.shape[0], m)
        return np.frombuffer(m.raw[: prog.shape[0]], dtype=np.uint8).astype(bool)


class RefCuda:
    """The reference's own GPU kernel (evaluate_kernel_packed from its
    src/EvaluatorCuda.cu, built for sm_100a, 16-register configuration)."""

    def __init__(self):
        path = REF_DIR / "libref_cuda_nr16.so"
        if not path.exists():
            raise FileNotFoundError(f"{path} not built")
        lib = C.CDLL(str(path))
        lib.refcuda_evaluate_packed.restype = C.c_int
        lib.refcuda_evaluate_packed.argtypes = [C.POINTER(_U32), C.POINTER(_I64), C.c_int, C.POINTER(_F32),
                                                C.POINTER(_F32), C.c_int, C.c_int, C.c_int, C.POINTER(_F32),
                                                C.POINTER(C.c_float)]
        self.lib = lib

    def evaluate_packed(self, words, offsets, inputs, targets, reps: int = 3):
        words = np.ascontiguousarray(words, dtype=np.uint32)
        offsets = np.ascontiguousarray(offsets, dtype=np.int64)
        inputs = np.ascontiguousarray(inputs, dtype=np.float32)
        targets = np.ascontiguousarray(targets, dtype=np.float32)
        n = offsets.shape[0] - 1
        fit = np.empty(n, dtype=np.float32)
        ms = C.c_float()
        rc = self.lib.refcuda_evaluate_packed(_p(words, _U32), _p(offsets, _I64), n, _p(inputs, _F32),
                                              _p(targets, _F32), inputs.shape[0], inputs.shape[1], reps,
                                              _p(fit, _F32), C.byref(ms))
        if rc != 0:
            raise RuntimeError(f"reference kernel failed: cudaError {rc}")
        return fit, ms.value
