"""galop_b200 -- B200 fitness evaluator for Galop's linear-GP symbolic regression.

Python view of the C ABI in ``include/galop_b200.h`` (ctypes, numpy arrays,
no torch).  ``Evaluator`` mirrors the reference's evaluation backend:

* ``Evaluator.evaluate_population(instructions, lengths, fitness_out,
  n_programs, dataset)`` has the argument order and meaning of
  ``EvalBackend::evaluate_population`` (src/EvalBackend.h:11-17): program ``i``
  is ``instructions[i*stride : i*stride + lengths[i]]`` with ``stride`` the
  engine's MAX_PROGRAM_SIZE.
* ``Evaluator.evaluate_csr(words, offsets)`` takes the packed layout of
  ``evaluate_kernel_packed`` (src/eval_kernels.cuh:292-303).
* ``Dataset`` mirrors ``struct Dataset`` (src/Dataset.h:22-38): case-major
  inputs, targets, ``N``, ``num_inputs``, ``ss_tot``.

Errors raise ``GalopError`` carrying the library's status code and message
(the reference prints and calls ``exit``, src/cuda_errors.h:3-15).  The native
library must be present: there is no CPU fallback.
"""
from __future__ import annotations

import ctypes as C
import weakref
from dataclasses import dataclass, field
from pathlib import Path
from typing import Optional, Sequence

import numpy as np

_PKG = Path(__file__).resolve().parent
LIB_PATH = _PKG / "libgalop_b200.so"

PROFILE_REF, PROFILE_BJ = 0, 1
REDUCE_KAHAN32, REDUCE_FP64, REDUCE_ORDERED = 0, 1, 2
OBJECTIVE_MSE, OBJECTIVE_R2 = 0, 1
SCHEDULE_PERSISTENT, SCHEDULE_PLAIN = 0, 1

OK = 0
E_INVALID, E_CUDA, E_NOMEM, E_NO_DATASET, E_TIMEOUT, E_CAPACITY, E_NO_DEVICE, E_STATE = (
    -1, -2, -3, -4, -5, -6, -7, -8)

# The reference's constant pools (src/LGPConfig.h:159-168).
REF_CONSTANTS_8 = np.array([0.0, 1.0, -1.0, 3.14159, 0.5, 2.0, 10.0, 100.0], dtype=np.float32)
REF_CONSTANTS_16 = np.array([0.0, 1.0, -1.0, 3.14159, 0.5, 2.0, 10.0, 100.0,
                             0.1, -0.5, 0.25, 5.0, 20.0, -2.0, 0.01, 1000.0], dtype=np.float32)

# Every entry point that include/galop_b200.h declares.
EXPORTED = (
    "galop_options_init", "galop_create", "galop_destroy", "galop_last_error",
    "galop_status_string", "galop_abi_version", "galop_set_dataset", "galop_set_dataset_device",
    "galop_evaluate_population", "galop_evaluate_csr", "galop_evaluate_csr_device",
    "galop_case_outputs_csr", "galop_trace_program", "galop_effective_csr", "galop_last_stats",
    "galop_synchronize", "galop_host_alloc", "galop_host_free", "galop_device_alloc",
    "galop_device_free", "galop_memcpy_h2d", "galop_memcpy_d2h", "galop_timer_record",
    "galop_timer_elapsed", "galop_evaluate_csr_noalloc", "galop_dataset_create", "galop_dataset_destroy",
    "galop_dataset_device_bytes", "galop_batch_create", "galop_batch_destroy", "galop_batch_device_bytes",
    "galop_batch_set_population", "galop_batch_evaluate", "galop_batch_synchronize", "galop_batch_get_fitness",
    "galop_batch_last_stats", "galop_batch_stream", "galop_batch_create_pool", "galop_batch_clear",
    "galop_batch_get_fitness_all",
    "galop_batch_append", "galop_batch_population_work", "galop_server_options_init", "galop_server_create",
    "galop_server_destroy", "galop_server_open_run", "galop_server_close_run", "galop_server_submit",
    "galop_server_wait", "galop_server_stats", "galop_autotune", "galop_csv_read", "galop_csv_free",
    "galop_engine_options_init", "galop_engine_create", "galop_engine_destroy", "galop_engine_evolve",
    "galop_engine_population", "galop_engine_times_get",
)


class _Options(C.Structure):
    _fields_ = [
        ("profile", C.c_int32), ("num_registers", C.c_int32), ("input_protect", C.c_int32),
        ("reduce", C.c_int32), ("constants", C.POINTER(C.c_float)), ("device", C.c_int32),
        ("intron_prepass", C.c_int32), ("cases_per_lane", C.c_int32),
        ("warps_per_block", C.c_int32), ("dispatch", C.c_int32), ("objective", C.c_int32),
        ("dedup", C.c_int32), ("schedule", C.c_int32),
    ]


class _CsvDataset(C.Structure):
    _fields_ = [("inputs", C.POINTER(C.c_float)), ("targets", C.POINTER(C.c_float)), ("n_cases", C.c_int64),
                ("num_inputs", C.c_int32), ("reserved", C.c_int32), ("ss_tot", C.c_double)]


class _EngineOptions(C.Structure):
    _fields_ = [("population", C.c_int64), ("max_program_size", C.c_int32), ("starting_program_size", C.c_int32),
                ("max_generations", C.c_int32), ("elite_count", C.c_int32), ("tournament_size", C.c_int32),
                ("macro_inserts", C.c_int32), ("effmut", C.c_int32), ("macro_random_pos", C.c_int32),
                ("crossover_rate", C.c_float), ("micro_rate", C.c_float), ("micro_per_instr", C.c_float),
                ("effmut_rate", C.c_float), ("insert_tail_rate", C.c_float), ("delete_tail_rate", C.c_float),
                ("seed", C.c_uint32), ("reserved", C.c_int32 * 3)]


class GenerationStats(C.Structure):
    """GenerationStats (src/GenerationStats.h)."""
    _fields_ = [("generation", C.c_int32), ("best_fitness", C.c_float), ("mean_fitness", C.c_float),
                ("best_length", C.c_int32), ("mean_length", C.c_float), ("best_index", C.c_int32)]


class EngineTimes(C.Structure):
    _fields_ = [("total_s", C.c_double), ("init_s", C.c_double), ("evaluate_s", C.c_double),
                ("select_vary_s", C.c_double), ("stats_s", C.c_double), ("eff_instructions", C.c_int64)]


class TuneResult(C.Structure):
    """galop_tune_result: the tile the autotuner chose."""
    _fields_ = [("dispatch", C.c_int32), ("cases_per_lane", C.c_int32), ("warps_per_block", C.c_int32),
                ("from_cache", C.c_int32), ("candidates", C.c_int32), ("reserved0", C.c_int32),
                ("sample_programs", C.c_int64), ("gpops", C.c_double), ("default_gpops", C.c_double),
                ("key", C.c_char * 320)]

    def as_dict(self) -> dict:
        d = {name: getattr(self, name) for name, _ in self._fields_ if name != "reserved0"}
        d["key"] = self.key.decode()
        return d


class Stats(C.Structure):
    _fields_ = [
        ("n_programs", C.c_int64), ("n_cases", C.c_int64), ("raw_instructions", C.c_int64),
        ("eff_instructions", C.c_int64), ("h2d_ms", C.c_double), ("prepass_ms", C.c_double),
        ("interp_ms", C.c_double), ("finalize_ms", C.c_double), ("d2h_ms", C.c_double),
        ("total_ms", C.c_double), ("cases_per_lane", C.c_int32), ("warps_per_block", C.c_int32),
        ("blocks", C.c_int32), ("case_chunks", C.c_int32), ("kernels_launched", C.c_int32),
        ("reserved0", C.c_int32), ("interp_instructions", C.c_int64),
    ]

    def as_dict(self) -> dict:
        return {name: getattr(self, name) for name, _ in self._fields_ if name != "reserved0"}


class PopulationSpec(C.Structure):
    _fields_ = [("dataset", C.c_void_p), ("max_programs", C.c_int64), ("max_words", C.c_int64)]


class ServerOptions(C.Structure):
    _fields_ = [("hbm_budget_bytes", C.c_int64), ("slots", C.c_int32), ("max_pops_per_batch", C.c_int32),
                ("slot_programs", C.c_int64), ("slot_words", C.c_int64), ("slot_items", C.c_int64),
                ("pinned_bytes", C.c_int64)]


class RequestInfo(C.Structure):
    _fields_ = [("status", C.c_int32), ("batch_requests", C.c_int32), ("eff_instructions", C.c_int64),
                ("queued_ms", C.c_double), ("latency_ms", C.c_double), ("device_ms", C.c_double)]


class ServerTotals(C.Structure):
    _fields_ = [("completed", C.c_int64), ("batches", C.c_int64), ("pending", C.c_int64),
                ("resident_bytes", C.c_int64), ("case_ops", C.c_int64), ("device_ms", C.c_double)]


class GalopError(RuntimeError):
    def __init__(self, status: int, message: str):
        super().__init__(f"galop status {status}: {message}")
        self.status = status


_lib: Optional[C.CDLL] = None

_P = C.c_void_p
_U32P = C.POINTER(C.c_uint32)
_I64P = C.POINTER(C.c_int64)
_F32P = C.POINTER(C.c_float)
_F64P = C.POINTER(C.c_double)
_U8P = C.POINTER(C.c_uint8)


def load_library(path: Optional[Path] = None) -> C.CDLL:
    """Load libgalop_b200.so (raises if it has not been built)."""
    global _lib
    if _lib is not None and path is None:
        return _lib
    p = Path(path) if path else LIB_PATH
    if not p.exists():
        raise GalopError(E_NO_DEVICE, f"native library missing: {p} (run python -m galop_b200.build)")
    lib = C.CDLL(str(p))
    sig = {
        "galop_options_init": (C.c_int, [C.POINTER(_Options)]),
        "galop_create": (C.c_int, [C.POINTER(_Options), C.POINTER(_P)]),
        "galop_destroy": (None, [_P]),
        "galop_last_error": (C.c_char_p, [_P]),
        "galop_status_string": (C.c_char_p, [C.c_int]),
        "galop_abi_version": (C.c_int, []),
        "galop_set_dataset": (C.c_int, [_P, _F32P, _F32P, C.c_int64, C.c_int32]),
        "galop_set_dataset_device": (C.c_int, [_P, _P, _P, C.c_int64, C.c_int32]),
        "galop_evaluate_population": (C.c_int, [_P, _U32P, _U8P, C.c_int64, C.c_int64, _F32P]),
        "galop_evaluate_csr": (C.c_int, [_P, _U32P, _I64P, C.c_int64, _F32P, _F64P]),
        "galop_evaluate_csr_device": (C.c_int, [_P, _P, _P, C.c_int64, C.c_int64, _P, _P, _P]),
        "galop_case_outputs_csr": (C.c_int, [_P, _U32P, _I64P, C.c_int64, _F32P]),
        "galop_trace_program": (C.c_int, [_P, _U32P, C.c_int64, _F32P, _I64P]),
        "galop_effective_csr": (C.c_int, [_P, _U32P, _I64P, C.c_int64, _I64P, _U32P]),
        "galop_last_stats": (C.c_int, [_P, C.POINTER(Stats)]),
        "galop_csv_read": (C.c_int, [C.c_char_p, C.c_int32, C.POINTER(_CsvDataset), C.c_char_p, C.c_int32]),
        "galop_csv_free": (None, [C.POINTER(_CsvDataset)]),
        "galop_engine_options_init": (C.c_int, [C.POINTER(_EngineOptions)]),
        "galop_engine_create": (C.c_int, [_P, C.POINTER(_EngineOptions), C.POINTER(_P)]),
        "galop_engine_destroy": (C.c_int, [_P]),
        "galop_engine_evolve": (C.c_int, [_P, C.POINTER(GenerationStats), C.c_int32]),
        "galop_engine_population": (C.c_int, [_P, _U32P, _U8P, _F32P]),
        "galop_engine_times_get": (C.c_int, [_P, C.POINTER(EngineTimes)]),
        "galop_autotune": (C.c_int, [_P, _U32P, _I64P, C.c_int64, C.c_int64, C.c_int32, C.c_char_p,
                                     C.POINTER(TuneResult)]),
        "galop_synchronize": (C.c_int, [_P]),
        "galop_host_alloc": (C.c_int, [C.c_int64, C.POINTER(_P)]),
        "galop_host_free": (C.c_int, [_P]),
        "galop_device_alloc": (C.c_int, [_P, C.c_int64, C.POINTER(_P)]),
        "galop_device_free": (C.c_int, [_P, _P]),
        "galop_memcpy_h2d": (C.c_int, [_P, _P, _P, C.c_int64]),
        "galop_memcpy_d2h": (C.c_int, [_P, _P, _P, C.c_int64]),
        "galop_timer_record": (C.c_int, [_P, C.c_int32]),
        "galop_timer_elapsed": (C.c_int, [_P, C.c_int32, C.c_int32, C.POINTER(C.c_double)]),
        "galop_evaluate_csr_noalloc": (C.c_int, [C.POINTER(_Options), _P, _P, C.c_int64, C.c_int64, _P, _P,
                                                 C.c_int64, C.c_int64, C.c_int32, _P, _P, _P]),
        "galop_dataset_create": (C.c_int, [_P, _F32P, _F32P, C.c_int64, C.c_int32, C.POINTER(_P)]),
        "galop_dataset_destroy": (C.c_int, [_P]),
        "galop_dataset_device_bytes": (C.c_int64, [_P]),
        "galop_batch_create": (C.c_int, [_P, C.POINTER(PopulationSpec), C.c_int32, C.POINTER(_P)]),
        "galop_batch_destroy": (C.c_int, [_P]),
        "galop_batch_device_bytes": (C.c_int64, [_P]),
        "galop_batch_set_population": (C.c_int, [_P, C.c_int32, _U32P, _I64P, C.c_int64]),
        "galop_batch_evaluate": (C.c_int, [_P, C.c_int32]),
        "galop_batch_synchronize": (C.c_int, [_P]),
        "galop_batch_get_fitness": (C.c_int, [_P, C.c_int32, _F32P, _F64P]),
        "galop_batch_last_stats": (C.c_int, [_P, C.POINTER(Stats)]),
        "galop_batch_stream": (_P, [_P]),
        "galop_batch_create_pool": (C.c_int, [_P, C.c_int32, C.c_int64, C.c_int64, C.c_int64, C.POINTER(_P)]),
        "galop_batch_clear": (C.c_int, [_P]),
        "galop_batch_append": (C.c_int, [_P, _P, _U32P, _I64P, C.c_int64, C.POINTER(C.c_int32)]),
        "galop_batch_population_work": (C.c_int, [_P, C.c_int32, C.POINTER(C.c_int64)]),
        "galop_batch_get_fitness_all": (C.c_int, [_P, _F32P, C.POINTER(C.c_int64)]),
        "galop_server_options_init": (C.c_int, [C.POINTER(ServerOptions)]),
        "galop_server_create": (C.c_int, [_P, C.POINTER(ServerOptions), C.POINTER(_P)]),
        "galop_server_destroy": (C.c_int, [_P]),
        "galop_server_open_run": (C.c_int, [_P, _F32P, _F32P, C.c_int64, C.c_int32, C.POINTER(C.c_int32)]),
        "galop_server_close_run": (C.c_int, [_P, C.c_int32]),
        "galop_server_submit": (C.c_int, [_P, C.c_int32, _U32P, _I64P, C.c_int64, _F32P, C.POINTER(C.c_int64)]),
        "galop_server_wait": (C.c_int, [_P, C.c_int64, C.c_double, C.POINTER(RequestInfo)]),
        "galop_server_stats": (C.c_int, [_P, C.POINTER(ServerTotals)]),
    }
    for name, (res, args) in sig.items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    if path is None:
        _lib = lib
    return lib


def _ptr(a: Optional[np.ndarray], ctype):
    if a is None:
        return None
    return a.ctypes.data_as(C.POINTER(ctype))


def status_string(status: int) -> str:
    return load_library().galop_status_string(status).decode()


@dataclass
class Dataset:
    """Mirror of the reference's Dataset (src/Dataset.h:22-38).

    ``inputs`` is case-major ``(N, num_inputs)`` float32 (the reference pads the
    row count to a multiple of 32; padding rows are never evaluated, so they
    are not stored here); ``targets`` is ``(N,)`` float32.
    """
    inputs: np.ndarray
    targets: np.ndarray
    ss_tot: float = field(default=0.0)

    def __post_init__(self):
        self.inputs = np.ascontiguousarray(self.inputs, dtype=np.float32)
        if self.inputs.ndim == 1:
            self.inputs = self.inputs.reshape(-1, 1)
        self.targets = np.ascontiguousarray(self.targets, dtype=np.float32).reshape(-1)
        if self.inputs.shape[0] != self.targets.shape[0]:
            raise ValueError("inputs and targets disagree on the case count")
        # Two-pass SS_tot over the valid targets, each pass a case-order
        # double sum (cumsum accumulates sequentially) as src/Dataset.cpp:35-47.
        if self.N > 0:
            t = self.targets.astype(np.float64)
            with np.errstate(all="ignore"):
                mean = float(np.cumsum(t)[-1]) / self.N
                d = t - mean
                self.ss_tot = float(np.cumsum(d * d)[-1])

    @classmethod
    def from_csv(cls, path: str, multi: bool = False) -> "Dataset":
        """load_csv_1d / load_csv_multi (src/Dataset.cpp:83-151) through
        galop_csv_read: header line skipped, one case per non-empty line."""
        lib = load_library()
        d = _CsvDataset()
        err = C.create_string_buffer(512)
        rc = lib.galop_csv_read(str(path).encode(), int(bool(multi)), C.byref(d), err, len(err))
        if rc != OK:
            raise GalopError(rc, err.value.decode() or status_string(rc))
        try:
            n, k = int(d.n_cases), int(d.num_inputs)
            X = np.ctypeslib.as_array(d.inputs, shape=(max(n * k, 1),))[: n * k].reshape(n, k).copy()
            y = np.ctypeslib.as_array(d.targets, shape=(max(n, 1),))[:n].copy()
            ss = float(d.ss_tot)
        finally:
            lib.galop_csv_free(C.byref(d))
        ds = cls(X, y)
        ds.ss_tot = ss
        return ds

    @property
    def N(self) -> int:
        return int(self.targets.shape[0])

    @property
    def num_inputs(self) -> int:
        return int(self.inputs.shape[1])


class Evaluator:
    """One evaluator context on one GPU (replaces CudaEvaluator,
    src/EvaluatorCuda.h:11-99)."""

    def __init__(self, profile: int = PROFILE_REF, num_registers: int = 8, input_protect: bool = False,
                 reduce: int = REDUCE_KAHAN32, constants: Optional[Sequence[float]] = None,
                 device: int = 0, intron_prepass: bool = True, cases_per_lane: int = 0,
                 warps_per_block: int = 0, dispatch: Optional[int] = None, objective: int = OBJECTIVE_MSE,
                 dedup: Optional[bool] = None, schedule: int = SCHEDULE_PERSISTENT):
        self._lib = load_library()
        opt = _Options()
        self._lib.galop_options_init(C.byref(opt))
        opt.profile = profile
        opt.num_registers = num_registers
        opt.input_protect = int(bool(input_protect))
        opt.reduce = reduce
        opt.device = device
        opt.intron_prepass = int(bool(intron_prepass))
        opt.cases_per_lane = cases_per_lane
        opt.warps_per_block = warps_per_block
        if dispatch is not None:
            opt.dispatch = dispatch
        opt.objective = objective
        if dedup is not None:
            opt.dedup = int(bool(dedup))
        opt.schedule = schedule
        self.constants = None
        if constants is not None:
            self.constants = np.ascontiguousarray(constants, dtype=np.float32)
            if self.constants.shape != (num_registers,):
                raise ValueError("constant pool must have num_registers entries")
            opt.constants = _ptr(self.constants, C.c_float)
        self.options = opt
        self.num_registers = num_registers
        self.profile = profile
        self.input_protect = bool(input_protect)
        self._ctx = C.c_void_p()
        rc = self._lib.galop_create(C.byref(opt), C.byref(self._ctx))
        if rc != OK:
            raise GalopError(rc, f"galop_create failed: {status_string(rc)}")
        self._dataset_key = None
        self.dataset: Optional[Dataset] = None
        self._children = weakref.WeakSet()

    # -- lifetime -------------------------------------------------------------
    def _adopt(self, child):
        self._children.add(child)

    def close(self):
        if getattr(self, "_ctx", None) and self._ctx.value:
            # servers first (their workers use batches and datasets), then batches, then datasets
            for kind in (Server, Batch, ResidentDataset):
                for child in list(self._children):
                    if isinstance(child, kind):
                        child.close()
            self._lib.galop_destroy(self._ctx)
            self._ctx = C.c_void_p()

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    @property
    def handle(self) -> C.c_void_p:
        return self._ctx

    def _check(self, rc: int):
        if rc != OK:
            msg = self._lib.galop_last_error(self._ctx)
            raise GalopError(rc, (msg or b"").decode() or status_string(rc))

    # -- dataset ----------------------------------------------------------------
    def set_dataset(self, dataset: Dataset):
        self._check(self._lib.galop_set_dataset(self._ctx, _ptr(dataset.inputs, C.c_float),
                                                _ptr(dataset.targets, C.c_float), dataset.N,
                                                dataset.num_inputs))
        self.dataset = dataset
        self._dataset_key = (id(dataset), dataset.N, dataset.num_inputs)

    def _ensure_dataset(self, dataset: Optional[Dataset]):
        if dataset is None:
            if self.dataset is None:
                raise GalopError(E_NO_DATASET, "no dataset")
            return
        if self._dataset_key != (id(dataset), dataset.N, dataset.num_inputs) or dataset is not self.dataset:
            self.set_dataset(dataset)

    # -- evaluation -------------------------------------------------------------
    def evaluate_population(self, instructions: np.ndarray, lengths: np.ndarray,
                            fitness_out: Optional[np.ndarray] = None, n_programs: Optional[int] = None,
                            dataset: Optional[Dataset] = None, stride: Optional[int] = None) -> np.ndarray:
        """EvalBackend::evaluate_population (src/EvalBackend.h:11-17)."""
        self._ensure_dataset(dataset)
        lengths = np.ascontiguousarray(lengths, dtype=np.uint8)
        n = int(lengths.shape[0] if n_programs is None else n_programs)
        instructions = np.ascontiguousarray(instructions, dtype=np.uint32)
        if stride is None:
            stride = instructions.shape[1] if instructions.ndim == 2 else (instructions.size // max(n, 1))
        if instructions.size < n * stride:
            raise ValueError("instructions buffer shorter than n_programs * stride")
        if fitness_out is None:
            fitness_out = np.empty(n, dtype=np.float32)
        self._check(self._lib.galop_evaluate_population(self._ctx, _ptr(instructions, C.c_uint32),
                                                        _ptr(lengths, C.c_uint8), stride, n,
                                                        _ptr(fitness_out, C.c_float)))
        return fitness_out

    def evaluate_csr(self, words: np.ndarray, offsets: np.ndarray, dataset: Optional[Dataset] = None,
                     with_sse: bool = False, fitness_out: Optional[np.ndarray] = None,
                     sse_out: Optional[np.ndarray] = None):
        self._ensure_dataset(dataset)
        words = np.ascontiguousarray(words, dtype=np.uint32)
        offsets = np.ascontiguousarray(offsets, dtype=np.int64)
        n = offsets.shape[0] - 1
        fit = fitness_out if fitness_out is not None else np.empty(n, dtype=np.float32)
        sse = sse_out if sse_out is not None else (np.empty(n, dtype=np.float64) if with_sse else None)
        self._check(self._lib.galop_evaluate_csr(self._ctx, _ptr(words, C.c_uint32), _ptr(offsets, C.c_int64),
                                                 n, _ptr(fit, C.c_float), _ptr(sse, C.c_double)))
        return (fit, sse) if with_sse else fit

    def evaluate_csr_device(self, d_words: int, d_offsets: int, n_programs: int, total_words: int,
                            d_fitness: int, d_sse: int = 0, stream: int = 0):
        """Queue an evaluation of device-resident CSR programs on `stream`
        (0: the context's stream) without waiting; ``stats`` waits for it."""
        self._check(self._lib.galop_evaluate_csr_device(self._ctx, d_words, d_offsets, n_programs, total_words,
                                                        d_fitness, d_sse or None, stream or None))

    def case_outputs(self, words: np.ndarray, offsets: np.ndarray, dataset: Optional[Dataset] = None):
        self._ensure_dataset(dataset)
        words = np.ascontiguousarray(words, dtype=np.uint32)
        offsets = np.ascontiguousarray(offsets, dtype=np.int64)
        n = offsets.shape[0] - 1
        out = np.empty((n, self.dataset.N), dtype=np.float32)
        self._check(self._lib.galop_case_outputs_csr(self._ctx, _ptr(words, C.c_uint32),
                                                     _ptr(offsets, C.c_int64), n, _ptr(out, C.c_float)))
        return out

    def trace(self, program: np.ndarray, dataset: Optional[Dataset] = None) -> np.ndarray:
        """Register file after each instruction: array (L+1, NR, n_traced)."""
        self._ensure_dataset(dataset)
        program = np.ascontiguousarray(program, dtype=np.uint32)
        L = program.shape[0]
        state = np.empty(((L + 1) * self.num_registers * 1024,), dtype=np.float32)
        nt = C.c_int64(0)
        self._check(self._lib.galop_trace_program(self._ctx, _ptr(program, C.c_uint32), L,
                                                  _ptr(state, C.c_float), C.byref(nt)))
        n = nt.value
        return state[: (L + 1) * self.num_registers * n].reshape(L + 1, self.num_registers, n)

    def effective(self, words: np.ndarray, offsets: np.ndarray):
        words = np.ascontiguousarray(words, dtype=np.uint32)
        offsets = np.ascontiguousarray(offsets, dtype=np.int64)
        n = offsets.shape[0] - 1
        eff_len = np.empty(n, dtype=np.int64)
        eff_words = np.empty(max(int(offsets[-1]), 1), dtype=np.uint32)
        self._check(self._lib.galop_effective_csr(self._ctx, _ptr(words, C.c_uint32), _ptr(offsets, C.c_int64),
                                                  n, _ptr(eff_len, C.c_int64), _ptr(eff_words, C.c_uint32)))
        return eff_len, eff_words[: int(eff_len.sum())]

    @property
    def stats(self) -> Stats:
        s = Stats()
        self._check(self._lib.galop_last_stats(self._ctx, C.byref(s)))
        return s

    def autotune(self, words: np.ndarray, offsets: np.ndarray, dataset: Optional[Dataset] = None,
                 cache: Optional[str] = None, sample: int = 0, reps: int = 0) -> TuneResult:
        """galop_autotune: time every tile on a sample of this population and
        keep the fastest for this evaluator (cached in `cache`, a JSON-lines
        file, when given)."""
        self._ensure_dataset(dataset)
        words = np.ascontiguousarray(words, dtype=np.uint32)
        offsets = np.ascontiguousarray(offsets, dtype=np.int64)
        r = TuneResult()
        self._check(self._lib.galop_autotune(self._ctx, _ptr(words, C.c_uint32), _ptr(offsets, C.c_int64),
                                             offsets.shape[0] - 1, sample, reps,
                                             cache.encode() if cache else None, C.byref(r)))
        return r

    def synchronize(self):
        self._check(self._lib.galop_synchronize(self._ctx))

    def timer_record(self, slot: int):
        self._check(self._lib.galop_timer_record(self._ctx, slot))

    def timer_elapsed(self, a: int, b: int) -> float:
        ms = C.c_double()
        self._check(self._lib.galop_timer_elapsed(self._ctx, a, b, C.byref(ms)))
        return ms.value

    # -- memory helpers -------------------------------------------------------
    def device_alloc(self, nbytes: int) -> int:
        p = C.c_void_p()
        self._check(self._lib.galop_device_alloc(self._ctx, nbytes, C.byref(p)))
        return p.value or 0

    def device_free(self, p: int):
        self._check(self._lib.galop_device_free(self._ctx, p))

    def h2d(self, dst: int, src: np.ndarray):
        self._check(self._lib.galop_memcpy_h2d(self._ctx, dst, src.ctypes.data, src.nbytes))

    def d2h(self, dst: np.ndarray, src: int):
        self._check(self._lib.galop_memcpy_d2h(self._ctx, dst.ctypes.data, src, dst.nbytes))


class PinnedArray:
    """numpy view over page-locked host memory from galop_host_alloc."""

    def __init__(self, shape, dtype):
        self._lib = load_library()
        dtype = np.dtype(dtype)
        nbytes = int(np.prod(shape)) * dtype.itemsize
        p = C.c_void_p()
        rc = self._lib.galop_host_alloc(nbytes, C.byref(p))
        if rc != OK:
            raise GalopError(rc, "galop_host_alloc failed")
        self._p = p
        buf = (C.c_char * max(nbytes, 1)).from_address(p.value)
        self.array = np.frombuffer(buf, dtype=dtype, count=int(np.prod(shape))).reshape(shape)

    def free(self):
        if self._p and self._p.value:
            self.array = None
            self._lib.galop_host_free(self._p)
            self._p = C.c_void_p()

    def __del__(self):
        try:
            self.free()
        except Exception:
            pass


def csr_from_dense(instructions: np.ndarray, lengths: np.ndarray, stride: int):
    """Pack the engine's dense layout into CSR (the reference's host pack,
    src/EvaluatorCuda.cu:335-373)."""
    lengths = np.asarray(lengths, dtype=np.int64)
    offsets = np.zeros(lengths.shape[0] + 1, dtype=np.int64)
    np.cumsum(lengths, out=offsets[1:])
    flat = np.asarray(instructions, dtype=np.uint32).reshape(-1)
    idx = (np.repeat(np.arange(lengths.shape[0], dtype=np.int64) * stride, lengths)
           + (np.arange(offsets[-1], dtype=np.int64) - np.repeat(offsets[:-1], lengths)))
    return flat[idx], offsets


class ResidentDataset:
    """A dataset kept on the device (galop_dataset_create); usable by
    several batches of the same evaluator."""

    def __init__(self, evaluator: "Evaluator", dataset: Dataset):
        self.evaluator = evaluator
        self.dataset = dataset
        self._h = C.c_void_p()
        evaluator._adopt(self)
        evaluator._check(evaluator._lib.galop_dataset_create(
            evaluator.handle, _ptr(dataset.inputs, C.c_float), _ptr(dataset.targets, C.c_float), dataset.N,
            dataset.num_inputs, C.byref(self._h)))

    @property
    def handle(self):
        return self._h

    @property
    def device_bytes(self) -> int:
        return int(self.evaluator._lib.galop_dataset_device_bytes(self._h))

    def close(self):
        if self._h and self._h.value:
            self.evaluator._lib.galop_dataset_destroy(self._h)
            self._h = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class Batch:
    """Several populations evaluated by one persistent launch per generation
    (galop_batch_*).  ``specs``: (ResidentDataset, max_programs, max_words)."""

    def __init__(self, evaluator: "Evaluator", specs):
        self.evaluator = evaluator
        self.specs = list(specs)
        arr = (PopulationSpec * len(self.specs))()
        for i, (ds, mp, mw) in enumerate(self.specs):
            arr[i] = PopulationSpec(ds.handle.value, int(mp), int(mw))
        self._h = C.c_void_p()
        evaluator._adopt(self)
        self._n = [0] * len(self.specs)
        evaluator._check(evaluator._lib.galop_batch_create(evaluator.handle, arr, len(self.specs), C.byref(self._h)))

    def _check(self, rc):
        self.evaluator._check(rc)

    @property
    def device_bytes(self) -> int:
        return int(self.evaluator._lib.galop_batch_device_bytes(self._h))

    def set_population(self, pop: int, words: np.ndarray, offsets: np.ndarray):
        words = np.ascontiguousarray(words, dtype=np.uint32)
        offsets = np.ascontiguousarray(offsets, dtype=np.int64)
        self._keep = getattr(self, "_keep", {})
        self._keep[pop] = (words, offsets)      # host buffers must live until the copy is done
        self._check(self.evaluator._lib.galop_batch_set_population(
            self._h, pop, _ptr(words, C.c_uint32), _ptr(offsets, C.c_int64), offsets.shape[0] - 1))
        self._n[pop] = offsets.shape[0] - 1

    def evaluate(self, use_graph: bool = False):
        self._check(self.evaluator._lib.galop_batch_evaluate(self._h, int(bool(use_graph))))

    def synchronize(self):
        self._check(self.evaluator._lib.galop_batch_synchronize(self._h))
        self._keep = {}

    def fitness(self, pop: int, with_sse: bool = False):
        n = self._n[pop]
        fit = np.empty(n, dtype=np.float32)
        sse = np.empty(n, dtype=np.float64) if with_sse else None
        self._check(self.evaluator._lib.galop_batch_get_fitness(self._h, pop, _ptr(fit, C.c_float),
                                                                _ptr(sse, C.c_double)))
        return (fit, sse) if with_sse else fit

    @property
    def stats(self) -> Stats:
        s = Stats()
        self._check(self.evaluator._lib.galop_batch_last_stats(self._h, C.byref(s)))
        return s

    def close(self):
        if self._h and self._h.value:
            self.evaluator._lib.galop_batch_destroy(self._h)
            self._h = C.c_void_p()

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class Server:
    """Continuous-batching evaluation for many GP runs (galop_server_*).

    ``open_run(dataset)`` registers a run; ``submit(run, words, offsets)``
    queues one generation and returns a request id; ``wait(id)`` returns its
    fitness and a RequestInfo (latency, batch size, ...)."""

    def __init__(self, evaluator: "Evaluator", **options):
        self.evaluator = evaluator
        lib = evaluator._lib
        o = ServerOptions()
        lib.galop_server_options_init(C.byref(o))
        for k, v in options.items():
            setattr(o, k, v)
        self.options = o
        self._h = C.c_void_p()
        evaluator._adopt(self)
        evaluator._check(lib.galop_server_create(evaluator.handle, C.byref(o), C.byref(self._h)))
        self._out = {}

    def open_run(self, dataset: Dataset) -> int:
        rid = C.c_int32()
        self.evaluator._check(self.evaluator._lib.galop_server_open_run(
            self._h, _ptr(dataset.inputs, C.c_float), _ptr(dataset.targets, C.c_float), dataset.N,
            dataset.num_inputs, C.byref(rid)))
        return rid.value

    def close_run(self, run_id: int):
        self.evaluator._check(self.evaluator._lib.galop_server_close_run(self._h, run_id))

    def submit(self, run_id: int, words: np.ndarray, offsets: np.ndarray) -> int:
        words = np.ascontiguousarray(words, dtype=np.uint32)
        offsets = np.ascontiguousarray(offsets, dtype=np.int64)
        out = np.empty(offsets.shape[0] - 1, dtype=np.float32)
        rq = C.c_int64()
        rc = self.evaluator._lib.galop_server_submit(self._h, run_id, _ptr(words, C.c_uint32),
                                                     _ptr(offsets, C.c_int64), offsets.shape[0] - 1,
                                                     _ptr(out, C.c_float), C.byref(rq))
        if rc != OK:
            raise GalopError(rc, "galop_server_submit failed")
        self._out[rq.value] = out
        return rq.value

    def wait(self, request_id: int, timeout: float = 0.0):
        info = RequestInfo()
        rc = self.evaluator._lib.galop_server_wait(self._h, request_id, timeout, C.byref(info))
        if rc == E_TIMEOUT:
            raise GalopError(rc, "timed out")
        if rc != OK:
            self._out.pop(request_id, None)
            raise GalopError(rc, "request failed")
        return self._out.pop(request_id), info

    @property
    def totals(self) -> ServerTotals:
        t = ServerTotals()
        self.evaluator._check(self.evaluator._lib.galop_server_stats(self._h, C.byref(t)))
        return t

    def close(self):
        if self._h and self._h.value:
            self.evaluator._lib.galop_server_destroy(self._h)
            self._h = C.c_void_p()

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class Engine:
    """LGPEngine::evolve_sr with the population resident on the GPU
    (galop_engine_*).  Keyword arguments are galop_engine_options fields;
    the defaults are the reference's default LGPConfig.  The ISA, constants
    and reduction are the evaluator's."""

    def __init__(self, ev: "Evaluator", **options):
        self._ev = ev
        self._lib = ev._lib
        o = _EngineOptions()
        self._lib.galop_engine_options_init(C.byref(o))
        if "population" in options and "elite_count" not in options:
            options["elite_count"] = int(np.float32(options["population"]) * np.float32(0.1))
        for k, v in options.items():
            if not hasattr(o, k):
                raise TypeError(f"unknown engine option {k}")
            setattr(o, k, v)
        self.options = o
        self._h = C.c_void_p()
        ev._check(self._lib.galop_engine_create(ev.handle, C.byref(o), C.byref(self._h)))

    def evolve(self, dataset: Optional[Dataset] = None):
        """Run init + max_generations; returns the history as a list of
        GenerationStats rows."""
        self._ev._ensure_dataset(dataset)
        hist = (GenerationStats * self.options.max_generations)()
        self._ev._check(self._lib.galop_engine_evolve(self._h, hist, len(hist)))
        return list(hist)

    def population(self):
        P, L = int(self.options.population), int(self.options.max_program_size)
        w = np.empty(P * L, np.uint32)
        ln = np.empty(P, np.uint8)
        f = np.empty(P, np.float32)
        self._ev._check(self._lib.galop_engine_population(self._h, _ptr(w, C.c_uint32), _ptr(ln, C.c_uint8),
                                                          _ptr(f, C.c_float)))
        return w.reshape(P, L), ln, f

    @property
    def times(self) -> EngineTimes:
        t = EngineTimes()
        self._lib.galop_engine_times_get(self._h, C.byref(t))
        return t

    def close(self):
        if getattr(self, "_h", None) and self._h.value:
            self._lib.galop_engine_destroy(self._h)
            self._h = C.c_void_p()

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
