#!/usr/bin/env python3
"""Throughput of population fitness evaluation on B200.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl b200|reference]

Workload (one step = one generation's evaluation of the whole population):
2^20 seeded random LGP programs, lengths U[16,256] with ~40% introns by
construction, 5 input features U[-3,3], 4,096 fitness cases, target = a
seeded random 16-effective-instruction program + N(0, 0.01^2); reference ISA,
16 registers.  Synthetic data of the reference's shapes (no datasets ship).

Metric: GPop/s = (effective instructions x fitness cases) / second, whole job.
``value``: population resident in HBM when the clock starts (intron pre-pass,
interpreter and fitness reduction on the device).  ``e2e``: the same through
the host-pointer C call (galop_evaluate_csr): H2D of the raw population from
pinned memory, pre-pass, interpretation, D2H of fitness, every step.

Multi-GPU (torchrun, one rank per GPU): every rank evaluates its own
population of the same size on the shared dataset (programs are independent,
so there is no collective on the data path; torch.distributed is used only for
the barrier and the max-over-ranks of the timings).  ``--impl reference``
times the reference's own CPU evaluator (Evaluator::evaluate_sr_mse built from
its sources, OpenMP over programs on every host core) on a bounded sample of
the same workload.
"""
from __future__ import annotations

import argparse
import ctypes
import json
import os
import statistics
import subprocess
import sys
import tempfile
import time
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))

METRIC = "GPop/s (eff. instr x cases/s) vs FP32-issue roofline; p50/p99 eval latency"
UNIT = "GPop/s"
WORKLOAD = ("single generation: 2^20 random programs, L~U[16,256] (~40% introns by construction), "
            "5 features U[-3,3], 4096 cases, target = random 16-effective-instruction program + N(0,0.01^2), "
            "reference ISA with 16 registers")


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="b200", choices=["b200", "reference"])
    ap.add_argument("--programs", type=int, default=1 << 20)
    ap.add_argument("--cases", type=int, default=4096)
    ap.add_argument("--cases-per-lane", type=int, default=0)
    ap.add_argument("--warps-per-block", type=int, default=0)
    ap.add_argument("--reduce", type=int, default=0)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--cpu-seconds", type=float, default=12.0)
    ap.add_argument("--workload", default="single", choices=["single", "batch", "serve", "stream", "evo", "capacity"],
                    help="single: the headline single-generation workload; batch: many populations in one "
                         "persistent launch per generation (graph replay) vs one plain launch per population; "
                         "serve: continuous batching of Poisson-arriving GP runs; stream: 2^20-case dataset; "
                         "evo: a whole 100-generation run of the reference engine with this backend, beside "
                         "the reference's own whole-run benchmark on the same GPU; capacity: the largest "
                         "device-resident population that evaluates, and its footprint per program")
    ap.add_argument("--evo-pop", type=int, default=100000, choices=[10000, 100000, 1000000])
    ap.add_argument("--evo-cases", type=int, default=1024)
    ap.add_argument("--evo-seed", type=int, default=70)
    ap.add_argument("--scale", type=float, default=1.0 / 32,
                    help="population-size scale of the batch/serve/stream workloads")
    return ap.parse_args()


class Dist:
    """torch.distributed plumbing (barrier, max) when launched by torchrun."""

    def __init__(self):
        self.world = int(os.environ.get("WORLD_SIZE", "1"))
        self.rank = int(os.environ.get("RANK", "0"))
        self.local = int(os.environ.get("LOCAL_RANK", "0"))
        self.pg = None
        if self.world > 1:
            import datetime
            import torch
            import torch.distributed as dist
            torch.cuda.set_device(self.local)
            dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=600))
            self.torch, self.dist = torch, dist

    def barrier(self):
        if self.world > 1:
            self.dist.barrier(device_ids=[self.local])

    def max(self, x: float) -> float:
        if self.world == 1:
            return x
        t = self.torch.tensor([x], dtype=self.torch.float64, device=f"cuda:{self.local}")
        self.dist.all_reduce(t, op=self.dist.ReduceOp.MAX)
        return float(t.item())

    def sum(self, x: float) -> float:
        if self.world == 1:
            return x
        t = self.torch.tensor([x], dtype=self.torch.float64, device=f"cuda:{self.local}")
        self.dist.all_reduce(t, op=self.dist.ReduceOp.SUM)
        return float(t.item())

    def close(self):
        if self.world > 1:
            self.dist.destroy_process_group()


class ClockSampler:
    """nvidia-smi clocks and throttle reasons while the timed region runs."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu: int):
        self.gpu = gpu
        self.proc = None
        self.f = tempfile.NamedTemporaryFile("w+", suffix=".csv", delete=False)

    def start(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.gpu), f"--query-gpu={self.FIELDS}",
                                          "--format=csv,noheader,nounits", "-lms", "100"], stdout=self.f,
                                         stderr=subprocess.DEVNULL)
        except OSError:
            self.proc = None

    def stop(self) -> dict:
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        self.proc.wait(timeout=10)
        self.f.flush()
        self.f.seek(0)
        rows = [r.split(", ") for r in self.f.read().strip().splitlines() if r.strip()]
        os.unlink(self.f.name)
        sm, smax, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for r in rows:
            try:
                sm.append(float(r[1]))
                smax.append(float(r[2]))
                for name, v in zip(names, r[5:9]):
                    if v.strip().lower().startswith("active"):
                        reasons.add(name)
            except (ValueError, IndexError):
                continue
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(smax) if smax else None,
                "reasons": sorted(reasons), "samples": len(sm)}


def load_workload(n_programs: int, n_cases: int, seed: int):
    from galop_b200 import workloads as W
    return W.single_generation(seed=seed, n_programs=n_programs, n_cases=n_cases)


def measured_peaks() -> dict:
    p = ROOT / "MEASURED_PEAKS.json"
    if p.exists():
        return json.loads(p.read_text())
    return {}


def profile_summary() -> dict:
    """Kernel name and DRAM bytes per interpreter launch from the committed
    ncu summary."""
    p = ROOT / "profiles" / "interp_single_generation.json"
    if p.exists():
        try:
            return json.loads(p.read_text())
        except (ValueError, OSError):
            return {}
    return {}


def fp32_issue_peak(device: int, peaks: dict):
    """SMs x 128 FP32 lanes x the measured maximum SM clock, in G lane-ops/s."""
    sm_count = 148
    try:
        import ctypes
        cudart = ctypes.CDLL("libcudart.so")
        v = ctypes.c_int()
        if cudart.cudaDeviceGetAttribute(ctypes.byref(v), 16, device) == 0:
            sm_count = v.value
    except OSError:
        pass
    sm_max = float(peaks.get("sm_max_mhz", 1965.0))
    return sm_count * 128 * sm_max * 1e6 / 1e9, sm_count, sm_max


def hbm_view(traffic, kernel_ms: float, peaks: dict):
    """DRAM bytes per launch over the launch time, against the measured
    copy bandwidth (or the fallback figure when no measurement exists)."""
    if not traffic or kernel_ms <= 0:
        return None
    peak = float(peaks.get("hbm_gbs", 6650.0))
    achieved = traffic / (kernel_ms / 1e3) / 1e9
    return {"achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak,
            "peak_source": "hbm_gbs of MEASURED_PEAKS.json" if "hbm_gbs" in peaks else "fallback"}


def profile_traffic():
    return profile_summary().get("dram_bytes_per_launch_full")


def cpu_reference_rate(wl, seconds: float, threads: int):
    """The reference's CPU evaluator (libref_nr16: Evaluator::evaluate_sr_mse
    + mse_to_fitness, OpenMP over programs) on successive batches of the
    workload until `seconds` of wall time; effective-instruction GPop/s."""
    from oracle.oracle import Oracle, RefLib
    kind = "reference"
    try:
        ref = RefLib("nr16")
        evaluate = lambda w, o: ref.evaluate_csr(w, o, wl.X, wl.y, threads=threads)  # noqa: E731
    except (FileNotFoundError, OSError):
        kind = "port"
        orc = Oracle(0, 16)
        evaluate = lambda w, o: orc.evaluate_csr(w, o, wl.X, wl.y, threads=threads)  # noqa: E731
    orc = Oracle(0, 16)
    batch = 256
    done_progs, ops, t_total = 0, 0.0, 0.0
    start = 0
    while t_total < seconds:
        if start >= wl.n_programs:
            start = 0
        idx = np.arange(start, min(start + batch, wl.n_programs))
        sub = wl.subsample(idx)
        eff = orc.effective_lengths(sub.words, sub.offsets)
        t0 = time.perf_counter()
        evaluate(sub.words, sub.offsets)
        t_total += time.perf_counter() - t0
        ops += float(eff.sum()) * wl.n_cases
        done_progs += idx.size
        start += batch
    rate = ops / t_total / 1e9
    return rate, kind, done_progs, t_total


def run_reference(args, dist: Dist):
    if dist.rank != 0:
        return
    threads = os.cpu_count() or 1
    wl = load_workload(min(args.programs, 16384), args.cases, 2)
    per_step = max(2.0, args.cpu_seconds / max(args.steps, 1))
    for _ in range(max(args.warmup, 0)):
        cpu_reference_rate(wl, 0.5, threads)
    rates, secs, progs = [], [], 0
    kind = "reference"
    for _ in range(args.steps):
        r, kind, n, t = cpu_reference_rate(wl, per_step, threads)
        rates.append(r)
        secs.append(t)
        progs = n
    value = float(np.mean(rates))
    line = {
        "metric": METRIC, "value": value, "unit": UNIT, "impl": "reference", "n_gpus": args.gpus,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1000 * float(np.mean(secs)),
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
        "data": "synthetic (seeded)",
        "config": {"workload": WORKLOAD, "programs_per_step": progs, "cases": args.cases,
                   "sample": f"first {progs} programs of the same workload per step"},
        "cpu_baseline": {"value": value, "unit": UNIT, "cores": threads, "kind": kind,
                         "sample": f"{progs} programs x {args.cases} cases per step, ~{per_step:.0f} s each"},
        "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


def run_b200(args, dist: Dist):
    import galop_b200 as g

    wl = load_workload(args.programs, args.cases, 2 + dist.rank)
    ds = g.Dataset(wl.X, wl.y)
    ev = g.Evaluator(num_registers=16, device=dist.local if dist.world > 1 else 0, reduce=args.reduce,
                     cases_per_lane=args.cases_per_lane, warps_per_block=args.warps_per_block)
    ev.set_dataset(ds)
    n = wl.n_programs
    words = np.ascontiguousarray(wl.words)
    offsets = np.ascontiguousarray(wl.offsets)

    # ---- device-resident population: the `value` leg -------------------------
    d_words = ev.device_alloc(words.nbytes)
    d_off = ev.device_alloc(offsets.nbytes)
    d_fit = ev.device_alloc(4 * n)
    d_sse = ev.device_alloc(8 * n)
    ev.h2d(d_words, words)
    ev.h2d(d_off, offsets)

    def step_device():
        ev.evaluate_csr_device(d_words, d_off, n, int(offsets[-1]), d_fit, d_sse)
        ev.synchronize()
        st = ev.stats
        return st

    for _ in range(args.warmup):
        step_device()
    # counts of one evaluation (identical every step)
    fit_check = ev.evaluate_csr(words, offsets)
    st0 = ev.stats
    eff_instr, raw_instr = st0.eff_instructions, st0.raw_instructions
    interp_instr = st0.interp_instructions

    clocks = ClockSampler(dist.local)
    dist.barrier()
    ev.synchronize()
    clocks.start()
    ev.timer_record(0)
    interp_ms, launches = [], 0
    for _ in range(args.steps):
        st = step_device()
        interp_ms.append(st.interp_ms)
        launches += st.kernels_launched
    ev.timer_record(1)
    ms_total = ev.timer_elapsed(0, 1)
    clock = clocks.stop()
    dist.barrier()
    ms_total_max = dist.max(ms_total)
    ops_rank = float(eff_instr) * wl.n_cases * args.steps
    ops_all = dist.sum(ops_rank)
    value = ops_all / (ms_total_max / 1e3) / 1e9

    # ---- end to end through the host-pointer C call ---------------------------
    pin_w = g.PinnedArray(words.shape, np.uint32)
    pin_o = g.PinnedArray(offsets.shape, np.int64)
    pin_f = g.PinnedArray((n,), np.float32)
    pin_w.array[:] = words
    pin_o.array[:] = offsets
    ev.evaluate_csr(pin_w.array, pin_o.array, fitness_out=pin_f.array)   # warm the host path
    dist.barrier()
    ev.synchronize()
    ev.timer_record(2)
    e2e_launches = 0
    for _ in range(args.steps):
        ev.evaluate_csr(pin_w.array, pin_o.array, fitness_out=pin_f.array)
        e2e_launches += ev.stats.kernels_launched
    ev.timer_record(3)
    e2e_ms = dist.max(ev.timer_elapsed(2, 3))
    e2e_value = ops_all / (e2e_ms / 1e3) / 1e9
    assert np.array_equal(pin_f.array.view(np.uint32), fit_check.view(np.uint32))

    # ---- roofline of the interpreter (FP32 issue) -------------------------------
    peaks = measured_peaks()
    peak_gops, sm_count, sm_max = fp32_issue_peak(dist.local if dist.world > 1 else 0, peaks)
    interp_avg_ms = float(np.mean(interp_ms))
    achieved = eff_instr * wl.n_cases / (interp_avg_ms / 1e3) / 1e9

    # ---- the reference's own GPU kernel on the same B200 (a sample) ------------
    ref_gpu = None
    if dist.rank == 0 and dist.world == 1 and not args.no_cpu_baseline:
        try:
            from oracle.oracle import Oracle, RefCuda
            m = min(n, 4096)
            sub = wl.subsample(np.arange(m))
            _, kms = RefCuda().evaluate_packed(sub.words, sub.offsets, wl.X, wl.y, reps=1)
            eff = float(Oracle(0, 16).effective_lengths(sub.words, sub.offsets).sum())
            ref_gpu = {"value": eff * wl.n_cases / (kms / 1e3) / 1e9, "unit": UNIT,
                       "raw_gpops": float(sub.offsets[-1]) * wl.n_cases / (kms / 1e3) / 1e9,
                       "kernel_ms": kms, "sample": f"first {m} programs x {wl.n_cases} cases",
                       "kernel": "evaluate_kernel_packed from the reference's src/EvaluatorCuda.cu, sm_100a"}
        except (FileNotFoundError, OSError, RuntimeError) as e:
            ref_gpu = {"unavailable": str(e)}

    cpu = None
    if dist.rank == 0 and dist.world == 1 and not args.no_cpu_baseline:
        threads = os.cpu_count() or 1
        rate, kind, progs, secs = cpu_reference_rate(wl, args.cpu_seconds, threads)
        # the reference's CpuEvaluator as shipped is serial (src/EvaluatorCpu.cpp:7-15)
        rate1, _, progs1, secs1 = cpu_reference_rate(wl, 3.0, 1)
        cpu = {"value": rate, "unit": UNIT, "cores": threads, "kind": kind,
               "sample": f"first {progs} programs of the workload x {wl.n_cases} cases ({secs:.1f} s wall, "
                         f"OpenMP over programs)",
               "one_core": {"value": rate1, "unit": UNIT, "cores": 1,
                            "sample": f"first {progs1} programs x {wl.n_cases} cases ({secs1:.1f} s)"}}

    if dist.rank == 0:
        line = {
            "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": dist.world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": ms_total_max / args.steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic (seeded)",
            "config": {"workload": WORKLOAD, "programs_per_gpu": n, "cases": wl.n_cases,
                       "raw_instructions_per_gpu": raw_instr, "effective_instructions_per_gpu": eff_instr,
                       "interpreted_instructions_per_gpu": interp_instr,
                       "cases_per_lane": st0.cases_per_lane, "warps_per_block": st0.warps_per_block,
                       "reduce": ["kahan32", "fp64", "ordered"][args.reduce],
                       "l2": "inputs larger than L2 (raw population %.2f GB per GPU)" % (words.nbytes / 1e9),
                       "parallelism": f"programs sharded, {dist.world} rank(s), no data-path collective"},
            "e2e": {"value": e2e_value, "unit": UNIT, "h2d_bytes_per_step": int(words.nbytes + offsets.nbytes),
                    "d2h_bytes_per_step": int(4 * n), "ms_per_step": e2e_ms / args.steps},
            "gpu_launches": launches,
            "raw_gpops": value * raw_instr / max(eff_instr, 1),
            "roofline": {"bound": "fp32_issue", "achieved": achieved, "peak": peak_gops, "unit": UNIT,
                         "frac": achieved / peak_gops, "traffic": profile_traffic(),
                         "kernel": profile_summary().get("kernel", "interp_wide_kernel"), "kernel_ms": interp_avg_ms,
                         "peak_source": f"{sm_count} SMs x 128 FP32 lanes x {sm_max:.0f} MHz "
                                        f"(sm_max_mhz of MEASURED_PEAKS.json)",
                         "ops_per_launch": float(eff_instr) * wl.n_cases,
                         # instructions the interpreter actually runs per case: the effective ones
                         # minus those evaluated once per program (every operand case-independent)
                         "interpreted_ops_per_launch": float(interp_instr) * wl.n_cases,
                         "interpreted_achieved": interp_instr * wl.n_cases / (interp_avg_ms / 1e3) / 1e9,
                         # the same kernel read against HBM (it streams each program once)
                         "hbm_view": hbm_view(profile_traffic(), interp_avg_ms, peaks),
                         "issue_slots_active": profile_summary().get("issue_slots_active")},
            "clocks": clock,
            "latency_ms": {"p50": float(np.percentile(interp_ms, 50)), "p99": float(np.percentile(interp_ms, 99))},
        }
        if cpu:
            line["cpu_baseline"] = cpu
        if ref_gpu:
            line["reference_gpu_same_b200"] = ref_gpu
        print(json.dumps(line), flush=True)
    for d in (d_words, d_off, d_fit, d_sse):
        ev.device_free(d)
    pin_w.free()
    pin_o.free()
    pin_f.free()
    ev.close()


def run_batch(args):
    """Many populations of uneven sizes and lengths on one shared dataset,
    one persistent launch per generation replayed from a CUDA graph; the
    plain form (one launch per population, no intron pass) timed beside it,
    and the compensated-FP32 fitness compared with the FP64 case-order sum."""
    import galop_b200 as g
    from galop_b200 import workloads as W
    n_cases = args.cases if args.cases != 4096 else 1 << 16
    lo, hi = max(8, int(1000 * args.scale)), max(64, int((1 << 20) * args.scale))
    isa, X, y, pops = W.many_populations(n_cases=n_cases, size_lo=lo, size_hi=hi)
    ds = g.Dataset(X, y)
    ev = g.Evaluator(num_registers=16)
    # Tile from the autotuner, measured on a sample of all populations together.
    all_words = np.concatenate([w for w, _ in pops])
    all_off = np.concatenate([[0]] + [o[1:] + base for (_, o), base in
                                      zip(pops, np.cumsum([0] + [int(o[-1]) for _, o in pops[:-1]]))])
    tune = ev.autotune(all_words, all_off.astype(np.int64), ds, cache=os.environ.get("GALOP_TUNE_CACHE"))
    rd = g.ResidentDataset(ev, ds)
    caps = [(rd, o.shape[0] - 1, int(o[-1])) for _, o in pops]
    b = g.Batch(ev, caps)

    def generation(use_graph):
        for p_, (w, o) in enumerate(pops):
            b.set_population(p_, w, o)
        b.evaluate(use_graph=use_graph)
        b.synchronize()
        return b.stats

    for _ in range(args.warmup):
        generation(True)
    dev_ms, wall = [], time.perf_counter()
    for _ in range(args.steps):
        dev_ms.append(generation(True).total_ms)
    wall = (time.perf_counter() - wall) * 1e3 / args.steps
    st = b.stats
    eff_total = 0
    for p_ in range(len(pops)):
        e = ctypes.c_int64()
        ev._check(ev._lib.galop_batch_population_work(b._h, p_, ctypes.byref(e)))
        eff_total += e.value
    ops = float(eff_total) * n_cases
    batched = ops / (np.mean(dev_ms) / 1e3) / 1e9
    fit_k = [b.fitness(p_) for p_ in range(len(pops))]
    b.close()
    # FP64 case-order reference of the same outputs
    ev_o = g.Evaluator(num_registers=16, reduce=g.REDUCE_ORDERED)
    rd_o = g.ResidentDataset(ev_o, ds)
    bo = g.Batch(ev_o, [(rd_o, c[1], c[2]) for c in caps])
    for p_, (w, o) in enumerate(pops):
        bo.set_population(p_, w, o)
    bo.evaluate()
    bo.synchronize()
    fit_o = [bo.fitness(p_) for p_ in range(len(pops))]
    bo.close()
    ev_o.close()
    fk = np.concatenate(fit_k).astype(np.float64)
    fo = np.concatenate(fit_o).astype(np.float64)
    nz = fo > 0
    rel = float(np.max(np.abs(fk[nz] - fo[nz]) / fo[nz])) if nz.any() else 0.0
    zero_mismatch = int(np.sum((fo > 0) != (fk > 0)))
    # plain: one launch per population, raw programs (no intron pass), per generation
    ev_p = g.Evaluator(num_registers=16, intron_prepass=False)
    ev_p.set_dataset(ds)
    plain_ms = 0.0
    for w, o in pops:
        ev_p.evaluate_csr(w, o)
        plain_ms += ev_p.stats.prepass_ms + ev_p.stats.interp_ms + ev_p.stats.finalize_ms
    ev_p.close()
    plain = ops / (plain_ms / 1e3) / 1e9
    line = {
        "metric": METRIC, "value": batched, "unit": UNIT, "workload": "batch", "n_gpus": 1,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": float(np.mean(dev_ms)),
        "wall_ms_per_generation": wall, "higher_is_better": True, "dtype": "f32", "data": "synthetic (seeded)",
        "config": {"workload": f"{len(pops)} populations, sizes log-uniform [{lo},{hi}] (x{args.scale:g} of "
                               f"[1000, 2^20]), lengths log-uniform [8,2048], one shared dataset of {n_cases} cases "
                               "x 4 features N(0,10^2), targets ~1e4 + N(0,1); generations replayed from a CUDA graph",
                   "programs": int(sum(c[1] for c in caps)), "raw_instructions": int(sum(c[2] for c in caps)),
                   "effective_instructions": int(eff_total)},
        "plain_per_population_gpops": plain, "speedup_vs_plain": batched / plain,
        "fitness_rel_err_kahan32_vs_fp64_case_order": rel,
        "fitness_zero_mismatches": zero_mismatch,
        "kernels_per_generation": st.kernels_launched,
        "autotune": {k: v for k, v in tune.as_dict().items() if k != "key"},
    }
    peak_gops, sm_count, sm_max = fp32_issue_peak(0, measured_peaks())
    line["roofline"] = {"bound": "fp32_issue", "achieved": batched, "peak": peak_gops, "unit": UNIT,
                        "frac": batched / peak_gops, "traffic": None,
                        "scope": "whole generation (pre-pass, interpreter, finalize), device time",
                        "peak_source": f"{sm_count} SMs x 128 FP32 lanes x {sm_max:.0f} MHz "
                                       f"(sm_max_mhz of MEASURED_PEAKS.json)"}
    rd.close()
    ev.close()
    print(json.dumps(line), flush=True)


def run_serve(args):
    """256 independent GP runs arriving as a Poisson process (mean 2 ms),
    each with its own dataset; every run submits its generations one after
    the other through the continuous-batching server."""
    import threading
    import galop_b200 as g
    from galop_b200 import workloads as W
    cases_hi = max(1024, int((1 << 20) * args.scale * 2))
    pop_hi = max(1024, int((1 << 18) * args.scale * 2))
    isa, runs = W.serving_runs(n_runs=256, cases_hi=cases_hi, pop_hi=pop_hi, generations=3)
    ev = g.Evaluator(num_registers=16)
    sv = g.Server(ev, hbm_budget_bytes=int(150e9), slots=4, slot_programs=1 << 20, slot_words=1 << 27,
                  slot_items=1 << 23)
    rng = np.random.default_rng(9)
    arrivals = np.cumsum(rng.exponential(2e-3, size=len(runs)))
    lat, queued, sizes = [], [], []
    lock = threading.Lock()
    t0 = time.perf_counter()

    def client(i):
        X, y, gens = runs[i]
        delay = t0 + arrivals[i] - time.perf_counter()
        if delay > 0:
            time.sleep(delay)
        rid = sv.open_run(g.Dataset(X, y))
        for w, o in gens:
            rq = sv.submit(rid, w, o)
            _, info = sv.wait(rq)
            with lock:
                lat.append(info.latency_ms)
                queued.append(info.queued_ms)
                sizes.append(info.batch_requests)
        sv.close_run(rid)

    threads = [threading.Thread(target=client, args=(i,)) for i in range(len(runs))]
    for t in threads:
        t.start()
    for t in threads:
        t.join()
    wall = time.perf_counter() - t0
    tot = sv.totals
    sv.close()
    ev.close()
    line = {
        "metric": METRIC, "value": tot.case_ops / wall / 1e9, "unit": UNIT, "workload": "serve",
        "n_gpus": 1, "higher_is_better": True, "dtype": "f32", "data": "synthetic (seeded)",
        "latency_ms": {"p50": float(np.percentile(lat, 50)), "p99": float(np.percentile(lat, 99)),
                       "mean": float(np.mean(lat))},
        "queued_ms": {"p50": float(np.percentile(queued, 50)), "p99": float(np.percentile(queued, 99))},
        "requests": len(lat), "batches": int(tot.batches), "mean_batch_requests": float(np.mean(sizes)),
        # sum of the batches' own device times over wall time: above 1 when
        # batches in different slots overlap on the device
        "batch_device_time_over_wall": tot.device_ms / 1e3 / wall, "wall_s": wall,
        "config": {"workload": f"256 GP runs, Poisson arrivals (mean 2 ms), 3 generations each; cases "
                               f"log-uniform [256,{cases_hi}], 1-8 features; populations log-uniform "
                               f"[1000,{pop_hi}], lengths U[8,512]; HBM admission cap 150 GB; 4 batches in flight"},
    }
    print(json.dumps(line), flush=True)


def run_stream(args):
    """2^20 fitness cases x 8 features (32 MiB + 4 MiB resident), programs
    log-uniform [32,1024], the intron pre-pass on; a sample of the 2^22
    programs."""
    import galop_b200 as g
    from galop_b200 import workloads as W
    n = max(1024, int((1 << 22) * args.scale / 8))
    wl = W.hbm_streaming(n_programs=n, n_cases=1 << 20)
    ev = g.Evaluator(num_registers=16)
    ev.set_dataset(g.Dataset(wl.X, wl.y))
    for _ in range(args.warmup):
        ev.evaluate_csr(wl.words, wl.offsets)
    ms = []
    for _ in range(args.steps):
        ev.evaluate_csr(wl.words, wl.offsets)
        ms.append(ev.stats.interp_ms + ev.stats.prepass_ms + ev.stats.finalize_ms)
    st = ev.stats
    ev.close()
    ops = float(st.eff_instructions) * wl.n_cases
    line = {"metric": METRIC, "value": ops / (np.mean(ms) / 1e3) / 1e9, "unit": UNIT, "workload": "stream",
            "n_gpus": 1, "steps": args.steps, "warmup": args.warmup, "ms_per_step": float(np.mean(ms)),
            "higher_is_better": True, "dtype": "f32", "data": "synthetic (seeded)",
            "config": {"workload": wl.description, "programs": n, "raw_instructions": st.raw_instructions,
                       "effective_instructions": st.eff_instructions, "case_chunks": st.case_chunks}}
    print(json.dumps(line), flush=True)


def evo_dataset(path: Path, n_cases: int):
    """The reference speed grid's synthetic cell: x ~ U(-1,1) from Python's
    random seeded with 1234, y = x^4 + x^3 + x^2 + x, header "x,y"."""
    import random
    rnd = random.Random(1234)
    with open(path, "w") as f:
        f.write("x,y\n")
        for _ in range(n_cases):
            x = rnd.uniform(-1, 1)
            f.write(f"{x},{x**4 + x**3 + x**2 + x}\n")


def parse_evo(out: str, err: str, name: str) -> dict:
    row = next(line for line in out.splitlines() if line.startswith(name + ","))
    f = row.split(",")
    r = {"pop": int(f[1]), "cases": int(f[2]), "generations": int(f[3]), "mean_length": float(f[4]),
         "seconds": float(f[5]), "raw_gpops": float(f[6]) / 1e9, "best_mse": float(f[7])}
    for line in err.splitlines():
        if line.startswith("BREAKDOWN"):
            e = line.split("eval=")[1].split("s")[0]
            r["eval_seconds"] = float(e)
    return r


def run_evo(args):
    """A whole evolutionary run (GALOP_STANDARD settings, 100 generations) three
    ways on the same cell and seed: the whole generation on the GPU
    (galop_engine_*, the value), the reference's LGPEngine on the host with
    this backend, and the reference's own whole-run benchmark (its
    CudaEvaluator, warp strategy, built for sm_100a)."""
    P, D, seed = args.evo_pop, args.evo_cases, args.evo_seed
    ours_bin = ROOT / "galop_b200" / "drivers" / "_bin" / f"evo_b200_P{P}"
    with tempfile.TemporaryDirectory() as td:
        csv = Path(td) / f"grid_D{D}.csv"
        evo_dataset(csv, D)
        env = dict(os.environ, OMP_NUM_THREADS=str(min(16, os.cpu_count() or 1)))
        p = subprocess.run([str(ours_bin), str(csv), str(seed)], capture_output=True, text=True, env=env,
                           timeout=3000)
        if p.returncode != 0:
            raise RuntimeError(f"{ours_bin.name} failed: {p.stderr[-400:]}")
        ours = parse_evo(p.stdout, p.stderr, "b200")
        ref = None
        if not args.no_cpu_baseline:
            # baseline leg: the reference's own whole-run benchmark, same GPU
            ref_bin = ROOT / "oracle" / "_ref" / f"cuda_evo_bench_P{P}"
            if ref_bin.exists():
                q = subprocess.run([str(ref_bin), str(csv), str(seed), "warp"], capture_output=True, text=True,
                                   env=env, timeout=3000)
                ref = parse_evo(q.stdout, q.stderr, "warp") if q.returncode == 0 else \
                    {"unavailable": q.stderr[-300:]}
            else:
                ref = {"unavailable": f"{ref_bin.name} not built"}
        # the same run with the whole generation on the GPU (galop_engine_*)
        import galop_b200 as g
        ds = g.Dataset.from_csv(csv)
        with g.Evaluator(num_registers=8, input_protect=True) as ev, \
                g.Engine(ev, population=P, seed=seed, macro_inserts=3, max_generations=100) as eng:
            t0 = time.perf_counter()
            hist = eng.evolve(ds)
            wall = time.perf_counter() - t0
            tm = eng.times
        ops = sum(float(P) * r.mean_length * D for r in hist)
        best = max(r.best_fitness for r in hist[-1:])
        device = {"pop": P, "cases": D, "generations": len(hist), "mean_length": float(np.mean([r.mean_length
                                                                                             for r in hist])),
                  "seconds": wall, "raw_gpops": ops / wall / 1e9,
                  "best_mse": (1.0 / best - 1.0) if best > 0 else float("inf"),
                  "init_seconds": tm.init_s, "eval_seconds": tm.evaluate_s, "select_vary_seconds": tm.select_vary_s,
                  "stats_seconds": tm.stats_s}
    line = {"metric": "raw GPop/s of a whole 100-generation run (P x mean length x D per generation / wall s)",
            "value": device["raw_gpops"], "unit": "GPop/s", "workload": "evo", "n_gpus": 1,
            "higher_is_better": True, "dtype": "f32", "data": "synthetic (seeded; the reference speed grid's cell)",
            "config": {"workload": f"GALOP_STANDARD engine settings, P={P}, D={D}, 100 generations, seed {seed}; "
                                   "value = the generation loop on the GPU (galop_engine)"},
            "device_engine": device, "host_engine_b200_backend": ours, "reference_whole_run_same_b200": ref}
    if ref and "seconds" in ref:
        line["speedup_vs_reference_whole_run"] = ref["seconds"] / device["seconds"]
        line["speedup_host_engine_vs_reference"] = ref["seconds"] / ours["seconds"]
    print(json.dumps(line), flush=True)


def run_capacity(args):
    """Largest device-resident population that evaluates (SURVEY §8(f) item 2,
    after tests/cuda_capacity.cu): random-word programs of 30 instructions
    (the reference probe's evolved shape; ~16% effective), 8 registers, a
    32-case dataset, populations generated on the device (no host copy).
    The footprint per program is measured on 2^22 programs (caller's words,
    offsets and fitness plus the evaluator's buffers), the largest population
    that fits in 92% of the free memory (and in int32 program indices) is
    then allocated and evaluated once as the proof, and twice more timed."""
    import torch
    import galop_b200 as g
    L, D = 30, 32
    rng = np.random.default_rng(1234)
    x = rng.uniform(-1, 1, (D, 1)).astype(np.float32)
    y = (x[:, 0] ** 3 + x[:, 0] ** 2 + x[:, 0]).astype(np.float32)
    ds = g.Dataset(x, y)
    dev = torch.device("cuda", 0)
    free0, total_mem = torch.cuda.mem_get_info(dev)
    rows = []

    def population(P):
        gen = torch.Generator(device=dev)
        gen.manual_seed(7)
        w = torch.randint(-2**31, 2**31 - 1, (P * L,), dtype=torch.int32, device=dev, generator=gen)
        off = torch.arange(P + 1, dtype=torch.int64, device=dev) * L
        fit = torch.empty(P, dtype=torch.float32, device=dev)
        return w, off, fit

    # dispatch 3 with dedup (the default), without it (its per-program sort
    # buffers are the price of interpreting identical programs once), and the
    # 4-byte micro-op interpreter
    for dispatch, dedup in ((3, True), (3, False), (2, False)):
        # footprint per program from a 2^22-program population
        P0 = 1 << 22
        torch.cuda.synchronize()
        before = torch.cuda.mem_get_info(dev)[0]
        ev = g.Evaluator(num_registers=8, dispatch=dispatch, dedup=dedup)
        ev.set_dataset(ds)
        w, off, fit = population(P0)
        ev.evaluate_csr_device(w.data_ptr(), off.data_ptr(), P0, P0 * L, fit.data_ptr())
        ev.synchronize()
        used = before - torch.cuda.mem_get_info(dev)[0]
        per_prog = used / P0
        del w, off, fit
        ev.close()
        torch.cuda.empty_cache()
        free_now = torch.cuda.mem_get_info(dev)[0]
        P = int(min(2**31 - 1, 0.92 * free_now / per_prog))
        row = {"dispatch": dispatch, "dedup": dedup, "bytes_per_program": round(per_prog, 1), "max_programs": P}
        for attempt in range(3):
            try:
                ev = g.Evaluator(num_registers=8, dispatch=dispatch, dedup=dedup)
                ev.set_dataset(ds)
                w, off, fit = population(P)
                ev.evaluate_csr_device(w.data_ptr(), off.data_ptr(), P, P * L, fit.data_ptr())   # the proof
                ev.synchronize()
                ms = []
                for _ in range(2):
                    ev.evaluate_csr_device(w.data_ptr(), off.data_ptr(), P, P * L, fit.data_ptr())
                    st = ev.stats
                    ms.append(st.prepass_ms + st.interp_ms + st.finalize_ms)
                st = ev.stats
                row.update({"max_programs": P, "evaluated": True, "eval_ms": min(ms),
                            "device_used_gb": round((free0 - torch.cuda.mem_get_info(dev)[0]) / 1e9, 1),
                            "raw_gpops": float(P) * L * D / (min(ms) / 1e3) / 1e9,
                            "eff_fraction": st.eff_instructions / max(st.raw_instructions, 1)})
                del w, off, fit
                ev.close()
                torch.cuda.empty_cache()
                break
            except (g.GalopError, torch.OutOfMemoryError) as e:
                row.setdefault("retries", []).append(f"P={P}: {e}")
                try:
                    del w, off, fit
                except NameError:
                    pass
                try:
                    ev.close()
                except Exception:
                    pass
                torch.cuda.empty_cache()
                P = int(P * 0.85)
        rows.append(row)
    line = {"metric": "largest device-resident population evaluated (programs)",
            "value": max(r["max_programs"] for r in rows if r.get("evaluated")), "unit": "programs",
            "workload": "capacity", "n_gpus": 1, "higher_is_better": True, "dtype": "f32",
            "data": "synthetic (random words generated on the device)",
            "config": {"workload": f"programs of {L} random words, 8 registers, {D} cases, intron pass on; "
                                   f"device memory {total_mem / 1e9:.1f} GB, free at start {free0 / 1e9:.1f} GB"},
            "by_dispatch": rows}
    print(json.dumps(line), flush=True)


def main():
    args = parse()
    dist = Dist()
    try:
        if args.impl == "reference":
            run_reference(args, dist)
        elif args.workload == "batch":
            run_batch(args)
        elif args.workload == "serve":
            run_serve(args)
        elif args.workload == "stream":
            run_stream(args)
        elif args.workload == "evo":
            run_evo(args)
        elif args.workload == "capacity":
            run_capacity(args)
        else:
            run_b200(args, dist)
    finally:
        dist.close()


if __name__ == "__main__":
    main()
