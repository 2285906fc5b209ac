#!/usr/bin/env python3
"""Throughput of population fitness evaluation on B200.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl b200|reference]

Headline workload (the HBM-streaming configuration at full size): a
population of 2^22 seeded random LGP programs, lengths log-uniform in
[32,1024] (uniform random words, ~10% effective), resident in HBM; 8 input
features U[-1,1] over 2^20 fitness cases (32 MiB + 4 MiB); target = a seeded
random 24-effective-instruction program; reference ISA, 16 registers; the
intron pre-pass on.  One step evaluates the next batch of 2^18 programs of
the population (16 steps = one generation); one whole-population call (all
2^22 programs) is timed beside the steps.  Synthetic data of the reference's
shapes (no datasets ship).

Metric: GPop/s = (effective instructions x fitness cases) / second, whole job.
``value``: population resident in HBM when the clock starts (intron pre-pass,
interpreter and fitness reduction on the device).  ``e2e``: the same through
the host-pointer C call (galop_evaluate_csr): H2D of the step's raw programs
from pinned memory, pre-pass, interpretation, D2H of fitness, every step.

Beside the headline the line carries: the single-generation configuration
(2^20 programs, 4,096 cases) measured the same way, the reference's own GPU
kernel on that configuration's whole population (raw words and host-stripped
effective words, as its Packed and PackedEffective layouts), the batching
configuration at a stated scale with all 2^22 cases (persistent batched
launch against one plain launch per population), and the reference's CPU
evaluator timed on the host's cores.

Multi-GPU (torchrun, one rank per GPU): every rank evaluates its own
population of the same size on the shared dataset (programs are independent,
so there is no collective on the data path; torch.distributed is used only for
the barrier and the max-over-ranks of the timings).  ``--impl reference``
times the reference's own CPU evaluator (Evaluator::evaluate_sr_mse built from
its sources, OpenMP over programs on every host core) on bounded samples of
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
WORKLOAD = ("HBM-streaming configuration at full size: population of 2^22 random programs resident in HBM, "
            "L log-uniform [32,1024], 8 features U[-1,1], 2^20 cases (32 MiB + 4 MiB), target = random "
            "24-effective-instruction program, reference ISA with 16 registers, intron pre-pass on; one step "
            "evaluates the next 2^18-program batch of the population (16 steps = one generation)")
SINGLE_WORKLOAD = ("single generation: 2^20 random programs, L~U[16,256] (~40% introns by construction), "
                   "5 features U[-3,3], 4096 cases, target = random 16-effective-instruction program + "
                   "N(0,0.01^2), reference ISA with 16 registers")


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="b200", choices=["b200", "reference"])
    ap.add_argument("--programs", type=int, default=1 << 22, help="population of the headline workload")
    ap.add_argument("--batch-programs", type=int, default=1 << 18, help="programs evaluated per step")
    ap.add_argument("--cases", type=int, default=1 << 20)
    ap.add_argument("--cases-per-lane", type=int, default=0)
    ap.add_argument("--warps-per-block", type=int, default=0)
    ap.add_argument("--reduce", type=int, default=0)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-extras", action="store_true",
                    help="headline only: skip the single-generation, batching and reference-GPU keys")
    ap.add_argument("--cpu-seconds", type=float, default=12.0)
    ap.add_argument("--workload", default="generation",
                    choices=["generation", "single", "batch", "serve", "evo", "capacity", "lengths"],
                    help="generation: the headline (HBM-streaming configuration at full size); single: "
                         "the single-generation configuration alone; batch: many populations in one "
                         "persistent launch per generation (graph replay) vs one plain launch per population; "
                         "serve: continuous batching of Poisson-arriving GP runs; evo: a whole 100-generation "
                         "run of the reference engine with this backend, beside the reference's own whole-run "
                         "benchmark on the same GPU; capacity: the largest device-resident population that "
                         "evaluates, and its footprint per program; lengths: every tile on populations of "
                         "one fixed program length per class")
    ap.add_argument("--evo-pop", type=int, default=100000, choices=[10000, 100000, 1000000])
    ap.add_argument("--evo-cases", type=int, default=1024)
    ap.add_argument("--evo-seed", type=int, default=70)
    ap.add_argument("--scale", type=float, default=1.0 / 64,
                    help="population-size scale of the batch workload (the serve workload runs at full size)")
    ap.add_argument("--batch-generations", type=int, default=3)
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


def measured_peaks() -> dict:
    p = ROOT / "MEASURED_PEAKS.json"
    if p.exists():
        return json.loads(p.read_text())
    return {}


def profile_summary(name: str) -> dict:
    """Figures of a committed ncu summary (profiles/<name>.json)."""
    p = ROOT / "profiles" / f"{name}.json"
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
        cudart = ctypes.CDLL("libcudart.so")
        v = ctypes.c_int()
        if cudart.cudaDeviceGetAttribute(ctypes.byref(v), 16, device) == 0:
            sm_count = v.value
    except OSError:
        pass
    sm_max = float(peaks.get("sm_max_mhz", 1965.0))
    src = "sm_max_mhz of MEASURED_PEAKS.json" if "sm_max_mhz" in peaks else "fallback clock 1965 MHz"
    return sm_count * 128 * sm_max * 1e6 / 1e9, sm_count, sm_max, src


def hbm_view(traffic, kernel_ms: float, peaks: dict):
    """DRAM bytes per launch over the launch time, against the measured
    copy bandwidth (or the fallback figure when no measurement exists)."""
    if not traffic or kernel_ms <= 0:
        return None
    peak = float(peaks.get("hbm_gbs", 6650.0))
    achieved = traffic / (kernel_ms / 1e3) / 1e9
    return {"achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak,
            "peak_source": "hbm_gbs of MEASURED_PEAKS.json" if "hbm_gbs" in peaks else "fallback 6650 GB/s"}


def roofline(eff_instr: float, interp_instr: float, n_cases: int, kernel_ms: float, device: int, prof: dict,
             programs_per_launch: int) -> dict:
    """The interpreter against the FP32-issue roofline (1 op = 1 effective
    instruction x 1 case); DRAM traffic from the committed ncu capture,
    scaled from its program count to this launch's."""
    peaks = measured_peaks()
    peak, sm_count, sm_max, src = fp32_issue_peak(device, peaks)
    achieved = eff_instr * n_cases / (kernel_ms / 1e3) / 1e9
    traffic = None
    if prof.get("dram_bytes") and prof.get("programs"):
        traffic = float(prof["dram_bytes"]) * programs_per_launch / float(prof["programs"])
    return {"bound": "fp32_issue", "achieved": achieved, "peak": peak, "unit": UNIT, "frac": achieved / peak,
            "traffic": traffic, "kernel": prof.get("kernel", "interp_wide_kernel"), "kernel_ms": kernel_ms,
            "peak_source": f"{sm_count} SMs x 128 FP32 lanes x {sm_max:.0f} MHz ({src})",
            "ops_per_launch": float(eff_instr) * n_cases,
            # instructions the interpreter actually runs per case: the effective ones minus
            # those evaluated once per program (every operand case-independent) and the copies
            # of programs interpreted once
            "interpreted_ops_per_launch": float(interp_instr) * n_cases,
            "interpreted_achieved": interp_instr * n_cases / (kernel_ms / 1e3) / 1e9,
            "hbm_view": hbm_view(traffic, kernel_ms, peaks),
            "issue_slots_active": prof.get("issue_slots_active"),
            "achieved_occupancy": prof.get("achieved_occupancy"),
            "profile_note": prof.get("captured"),
            "traffic_source": (f"ncu capture of {prof.get('programs')} programs x {prof.get('cases')} cases, "
                               f"scaled to {programs_per_launch} programs") if traffic else None}


def cpu_reference_rate(wl, seconds: float, threads: int, batch: int = 0):
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
    if batch <= 0:
        # a few programs per thread and about a second of work per call
        raw_per_prog = float(wl.offsets[-1]) / max(wl.n_programs, 1)
        batch = int(threads * max(4, min(256, 4e8 / max(raw_per_prog * wl.n_cases, 1.0))))
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


def headline_workload(args, seed: int, prefix=None):
    from galop_b200 import workloads as W
    return W.hbm_streaming(seed=seed, n_programs=args.programs, n_cases=args.cases, prefix_programs=prefix)


def run_reference(args, dist: Dist):
    if dist.rank != 0:
        return
    threads = os.cpu_count() or 1
    if args.workload == "single":
        from galop_b200 import workloads as W
        wl = W.single_generation(seed=2, n_programs=16384, n_cases=4096)
        workload, cases = SINGLE_WORKLOAD, 4096
    else:
        wl = headline_workload(args, 3, prefix=4096)
        workload, cases = WORKLOAD, args.cases
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
        "config": {"workload": workload, "programs_per_step": progs, "cases": cases,
                   "sample": f"the first {progs} programs of the same population per step"},
        "cpu_baseline": {"value": value, "unit": UNIT, "cores": threads, "kind": kind,
                         "sample": f"{progs} programs x {cases} cases per step, ~{per_step:.0f} s each"},
        "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


def batches_of(offsets: np.ndarray, batch: int):
    """[(lo, hi, offsets rebased to 0)] program ranges of `batch` programs."""
    n = offsets.shape[0] - 1
    out = []
    for lo in range(0, n, batch):
        hi = min(n, lo + batch)
        out.append((lo, hi, np.ascontiguousarray(offsets[lo:hi + 1] - offsets[lo])))
    return out


def cpu_baseline_leg(wl, args) -> dict:
    threads = os.cpu_count() or 1
    rate, kind, progs, secs = cpu_reference_rate(wl, args.cpu_seconds, threads)
    # the reference's CpuEvaluator as shipped is serial (src/EvaluatorCpu.cpp:7-15)
    rate1, _, progs1, secs1 = cpu_reference_rate(wl, 3.0, 1)
    return {"value": rate, "unit": UNIT, "cores": threads, "kind": kind,
            "sample": f"the first {progs} programs of the population x {wl.n_cases} cases ({secs:.1f} s wall, "
                      f"OpenMP over programs)",
            "one_core": {"value": rate1, "unit": UNIT, "cores": 1,
                         "sample": f"the first {progs1} programs x {wl.n_cases} cases ({secs1:.1f} s)"}}


def run_generation(args, dist: Dist):
    """The headline: the HBM-streaming configuration at full size."""
    import galop_b200 as g

    dev = dist.local if dist.world > 1 else 0
    wl = headline_workload(args, 3 + dist.rank)
    n = wl.n_programs
    words, offsets = wl.words, wl.offsets
    pop_bytes = words.nbytes
    B = min(args.batch_programs, n)
    bats = batches_of(offsets, B)
    ev = g.Evaluator(num_registers=16, device=dev, reduce=args.reduce, cases_per_lane=args.cases_per_lane,
                     warps_per_block=args.warps_per_block)
    ev.set_dataset(g.Dataset(wl.X, wl.y))

    # ---- device-resident population: the `value` leg -------------------------
    d_words = ev.device_alloc(words.nbytes)
    ev.h2d(d_words, words)
    d_off_all = ev.device_alloc(offsets.nbytes)
    ev.h2d(d_off_all, offsets)
    d_boff = []
    for lo, hi, o in bats:
        d = ev.device_alloc(o.nbytes)
        ev.h2d(d, o)
        d_boff.append(d)
    d_fit = ev.device_alloc(4 * n)
    d_sse = ev.device_alloc(8 * n)

    def step_device(i):
        b = i % len(bats)
        lo, hi, o = bats[b]
        ev.evaluate_csr_device(d_words + 4 * int(offsets[lo]), d_boff[b], hi - lo, int(o[-1]), d_fit + 4 * lo,
                               d_sse + 8 * lo)
        return ev.stats

    for i in range(args.warmup):
        step_device(i)
    clocks = ClockSampler(dev)
    dist.barrier()
    ev.synchronize()
    clocks.start()
    ev.timer_record(0)
    per_step = []
    for i in range(args.steps):
        st = step_device(args.warmup + i)
        per_step.append((st.eff_instructions, st.interp_instructions, st.raw_instructions, st.interp_ms,
                         st.total_ms, st.kernels_launched, st.n_programs))
    ev.timer_record(1)
    ms_total = ev.timer_elapsed(0, 1)
    clock = clocks.stop()
    dist.barrier()
    ms_total_max = dist.max(ms_total)
    eff_sum = float(sum(r[0] for r in per_step))
    ops_all = dist.sum(eff_sum * wl.n_cases)
    value = ops_all / (ms_total_max / 1e3) / 1e9
    launches = int(sum(r[5] for r in per_step))

    # ---- one whole generation: all programs in one call ----------------------
    ev.evaluate_csr_device(d_words, d_off_all, n, int(offsets[-1]), d_fit, d_sse)
    stg = ev.stats
    full_fit = np.empty(n, np.float32)
    ev.d2h(full_fit, d_fit)
    generation = {"programs": n, "ms": stg.total_ms,
                  "value": stg.eff_instructions * wl.n_cases / (stg.total_ms / 1e3) / 1e9, "unit": UNIT,
                  "interp_ms": stg.interp_ms, "raw_instructions": stg.raw_instructions,
                  "effective_instructions": stg.eff_instructions,
                  "interpreted_instructions": stg.interp_instructions}

    # ---- end to end through the host-pointer C call ---------------------------
    pin_w = g.PinnedArray(words.shape, np.uint32)
    pin_w.array[:] = words
    pin_o = [g.PinnedArray(o.shape, np.int64) for _, _, o in bats]
    for p_, (_, _, o) in zip(pin_o, bats):
        p_.array[:] = o
    pin_f = g.PinnedArray((B,), np.float32)

    def step_host(i):
        b = i % len(bats)
        lo, hi, o = bats[b]
        ev.evaluate_csr(pin_w.array[offsets[lo]:offsets[hi]], pin_o[b].array, fitness_out=pin_f.array[:hi - lo])
        return b, hi - lo, int(o[-1])

    step_host(0)   # warm the host path (and its copy stream)
    dist.barrier()
    ev.synchronize()
    ev.timer_record(2)
    e2e_wall, h2d_bytes, d2h_bytes = [], 0, 0
    check = None
    for i in range(args.steps):
        t0 = time.perf_counter()
        b, m, nw = step_host(args.warmup + i)
        e2e_wall.append((time.perf_counter() - t0) * 1e3)
        h2d_bytes += 4 * nw + 8 * (m + 1)
        d2h_bytes += 4 * m
        if check is None:
            lo = bats[b][0]
            check = bool(np.array_equal(pin_f.array[:m].view(np.uint32), full_fit[lo:lo + m].view(np.uint32)))
    ev.timer_record(3)
    e2e_ms = dist.max(ev.timer_elapsed(2, 3))
    e2e_value = ops_all / (e2e_ms / 1e3) / 1e9
    assert check, "host-pointer fitness differs from the device-resident call's"

    kernel_ms = float(sum(r[3] for r in per_step))
    interp_sum = float(sum(r[1] for r in per_step))
    raw_sum = float(sum(r[2] for r in per_step))
    roof = roofline(eff_sum / args.steps, interp_sum / args.steps, wl.n_cases, kernel_ms / args.steps, dev,
                    profile_summary("interp_hbm_streaming"), B)
    cpu = None
    extras = {}
    if dist.rank == 0 and dist.world == 1 and not args.no_cpu_baseline:
        cpu = cpu_baseline_leg(wl, args)
    for d in [d_words, d_off_all, d_fit, d_sse] + d_boff:
        ev.device_free(d)
    for p_ in [pin_w, pin_f] + pin_o:
        p_.free()
    ev.close()
    n_cases = wl.n_cases
    del wl, words, offsets
    if dist.rank == 0 and dist.world == 1 and not args.no_extras:
        extras["single_generation"] = single_generation_leg(args)
        extras["batching"] = batching_leg(args)

    if dist.rank == 0:
        total_ms = [r[4] for r in per_step]
        line = {
            "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": dist.world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": ms_total_max / args.steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic (seeded)",
            "config": {"workload": WORKLOAD, "population_per_gpu": n, "programs_per_step": B,
                       "steps_per_generation": len(bats), "cases": n_cases,
                       "raw_instructions_per_step": raw_sum / args.steps,
                       "effective_instructions_per_step": eff_sum / args.steps,
                       "interpreted_instructions_per_step": interp_sum / args.steps,
                       "reduce": ["kahan32", "fp64", "ordered"][args.reduce],
                       "l2": "inputs larger than L2 (the population's raw words are %.2f GB per GPU, each "
                             "step's batch %.2f GB); the 36 MB dataset itself fits in L2" %
                             (pop_bytes / 1e9, 4.0 * raw_sum / args.steps / 1e9),
                       "parallelism": f"programs sharded, {dist.world} rank(s), no data-path collective"},
            "e2e": {"value": e2e_value, "unit": UNIT, "h2d_bytes_per_step": int(h2d_bytes / args.steps),
                    "d2h_bytes_per_step": int(d2h_bytes / args.steps), "ms_per_step": e2e_ms / args.steps,
                    "latency_ms": {"p50": float(np.percentile(e2e_wall, 50)),
                                   "p99": float(np.percentile(e2e_wall, 99))}},
            "gpu_launches": launches,
            "raw_gpops": value * raw_sum / max(eff_sum, 1.0),
            "roofline": roof,
            "clocks": clock,
            # one evaluation call (pre-pass through finalize) on the device, per step
            "latency_ms": {"p50": float(np.percentile(total_ms, 50)), "p99": float(np.percentile(total_ms, 99)),
                           "scope": "device time of one evaluate call of 2^18 programs x 2^20 cases"},
            "generation": generation,
        }
        if cpu:
            line["cpu_baseline"] = cpu
        line.update(extras)
        print(json.dumps(line), flush=True)


def single_generation_leg(args) -> dict:
    """The single-generation configuration (2^20 programs x 4,096 cases),
    device-resident, beside the reference's own GPU kernel on the same whole
    population."""
    import galop_b200 as g
    from galop_b200 import workloads as W
    wl = W.single_generation(seed=2, n_programs=1 << 20, n_cases=4096)
    n = wl.n_programs
    out = {"workload": SINGLE_WORKLOAD}
    with g.Evaluator(num_registers=16) as ev:
        ev.set_dataset(g.Dataset(wl.X, wl.y))
        d_w, d_o = ev.device_alloc(wl.words.nbytes), ev.device_alloc(wl.offsets.nbytes)
        d_f = ev.device_alloc(4 * n)
        ev.h2d(d_w, wl.words)
        ev.h2d(d_o, wl.offsets)
        for _ in range(2):
            ev.evaluate_csr_device(d_w, d_o, n, int(wl.offsets[-1]), d_f)
            ev.stats
        ms, interp = [], []
        for _ in range(5):
            ev.evaluate_csr_device(d_w, d_o, n, int(wl.offsets[-1]), d_f)
            st = ev.stats
            ms.append(st.total_ms)
            interp.append(st.interp_ms)
        for d in (d_w, d_o, d_f):
            ev.device_free(d)
    out.update({"value": st.eff_instructions * 4096 / (np.mean(ms) / 1e3) / 1e9, "unit": UNIT,
                "ms_per_generation": float(np.mean(ms)),
                "roofline": roofline(st.eff_instructions, st.interp_instructions, 4096, float(np.mean(interp)), 0,
                                     profile_summary("interp_single_generation"), n),
                "effective_instructions": st.eff_instructions, "interpreted_instructions": st.interp_instructions,
                "raw_instructions": st.raw_instructions})
    try:
        from oracle.oracle import Oracle, RefCuda
        ref = RefCuda()
        _, kms_raw = ref.evaluate_packed(wl.words, wl.offsets, wl.X, wl.y, reps=3)
        ew, eo = Oracle(0, 16).extract_effective_csr(wl.words, wl.offsets)
        _, kms_eff = ref.evaluate_packed(ew, eo, wl.X, wl.y, reps=3)
        eff = float(eo[-1]) * 4096
        out["reference_gpu_same_b200"] = {
            "kernel": "evaluate_kernel_packed from the reference's src/EvaluatorCuda.cu, sm_100a, launched as "
                      "tests/cuda_capacity.cu:119-132 does (grid ceil(n/8) x 256)",
            "sample": f"the whole population ({n} programs x 4096 cases), mean of 3 launches after one warm-up",
            "packed_raw_words": {"kernel_ms": kms_raw, "value": eff / (kms_raw / 1e3) / 1e9, "unit": UNIT,
                                 "raw_gpops": float(wl.offsets[-1]) * 4096 / (kms_raw / 1e3) / 1e9},
            "packed_effective_words": {"kernel_ms": kms_eff, "value": eff / (kms_eff / 1e3) / 1e9, "unit": UNIT,
                                       "note": "introns stripped on the host first, as its PackedEffective "
                                               "layout (src/EvaluatorCuda.cu:374-422)"},
            "ours_over_best_reference": out["value"] / (eff / (min(kms_raw, kms_eff) / 1e3) / 1e9)}
    except (FileNotFoundError, OSError, RuntimeError) as e:
        out["reference_gpu_same_b200"] = {"unavailable": str(e)}
    return out


def batching_leg(args) -> dict:
    """The batching configuration: 64 populations of uneven sizes (log-uniform
    [1k, 2^20] x scale) and lengths (log-uniform [8,2048]) on one shared
    dataset of 2^22 cases x 4 features N(0, 10^2) with targets ~1e4 + N(0,1).
    The batched form evaluates every population in one persistent launch per
    generation, replayed from a CUDA graph; the plain form launches one
    warp-per-individual grid per population (one warp per program over all
    cases, program order, no work queue, no case chunking) with the same
    intron pass, folding and dedup.  KAHAN32 fitness is compared with the
    FP64 case-order sum of the same outputs."""
    import galop_b200 as g
    from galop_b200 import workloads as W
    n_cases = 1 << 22
    lo, hi = max(8, int(1000 * args.scale)), max(64, int((1 << 20) * args.scale))
    isa, X, y, pops = W.many_populations(n_cases=n_cases, size_lo=lo, size_hi=hi)
    ds = g.Dataset(X, y)
    gens = max(1, args.batch_generations)
    ev = g.Evaluator(num_registers=16)
    all_words = np.concatenate([w for w, _ in pops])
    all_off = np.concatenate([[0]] + [o[1:] + base for (_, o), base in
                                      zip(pops, np.cumsum([0] + [int(o[-1]) for _, o in pops[:-1]]))])
    # tile from the autotuner, on a sample of all populations together
    tune = ev.autotune(all_words, all_off.astype(np.int64), ds, cache=os.environ.get("GALOP_TUNE_CACHE"),
                       sample=2048)
    rd = g.ResidentDataset(ev, ds)
    caps = [(rd, o.shape[0] - 1, int(o[-1])) for _, o in pops]
    b = g.Batch(ev, caps)

    def generation(use_graph):
        for p_, (w, o) in enumerate(pops):
            b.set_population(p_, w, o)
        b.evaluate(use_graph=use_graph)
        b.synchronize()
        return b.stats

    generation(True)
    dev_ms, t0 = [], time.perf_counter()
    for _ in range(gens):
        dev_ms.append(generation(True).total_ms)
    wall = (time.perf_counter() - t0) * 1e3 / gens
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
    rd.close()
    # FP64 case-order sum of the same outputs
    ev_o = g.Evaluator(num_registers=16, reduce=g.REDUCE_ORDERED)
    rd_o = g.ResidentDataset(ev_o, ds)
    bo = g.Batch(ev_o, [(rd_o, c[1], c[2]) for c in caps])
    for p_, (w, o) in enumerate(pops):
        bo.set_population(p_, w, o)
    bo.evaluate()
    bo.synchronize()
    fit_o = [bo.fitness(p_) for p_ in range(len(pops))]
    bo.close()
    rd_o.close()
    ev_o.close()
    fk = np.concatenate(fit_k).astype(np.float64)
    fo = np.concatenate(fit_o).astype(np.float64)
    nz = fo > 0
    rel = float(np.max(np.abs(fk[nz] - fo[nz]) / fo[nz])) if nz.any() else 0.0
    zero_mismatch = int(np.sum((fo > 0) != (fk > 0)))
    # plain: one warp-per-individual launch per population, same pre-pass
    ev_p = g.Evaluator(num_registers=16, schedule=g.SCHEDULE_PLAIN, cases_per_lane=tune.cases_per_lane,
                       warps_per_block=tune.warps_per_block)
    ev_p.set_dataset(ds)
    plain_ms = 0.0
    fit_p = []
    for w, o in pops:
        fit_p.append(ev_p.evaluate_csr(w, o))
        plain_ms += ev_p.stats.prepass_ms + ev_p.stats.interp_ms + ev_p.stats.finalize_ms
    ev_p.close()
    ev.close()
    fp = np.concatenate(fit_p).astype(np.float64)
    nzk = fk > 0
    plain = ops / (plain_ms / 1e3) / 1e9
    peak, sm_count, sm_max, src = fp32_issue_peak(0, measured_peaks())
    return {
        "workload": f"batching configuration at population scale {args.scale:g}: {len(pops)} populations, sizes "
                    f"log-uniform [{lo},{hi}] (x{args.scale:g} of [1000, 2^20]), lengths log-uniform [8,2048], "
                    f"one shared dataset of {n_cases} cases x 4 features N(0,10^2), targets ~1e4 + N(0,1); "
                    f"{gens} generations replayed from a CUDA graph",
        "value": batched, "unit": UNIT, "ms_per_generation": float(np.mean(dev_ms)),
        "wall_ms_per_generation": wall, "generations": gens,
        "programs": int(sum(c[1] for c in caps)), "raw_instructions": int(sum(c[2] for c in caps)),
        "effective_instructions": int(eff_total),
        "plain_per_population": {"value": plain, "unit": UNIT, "ms_per_generation": plain_ms,
                                 "launch": "one grid per population: one warp per program over all cases, "
                                           "program order, no work queue, no case chunking; intron pass, "
                                           "folding and dedup as the batched form"},
        "speedup_vs_plain": batched / plain,
        "plain_fitness_rel_err_vs_batched": float(np.max(np.abs(fp[nzk] - fk[nzk]) / fk[nzk])) if nzk.any() else 0.0,
        "fitness_rel_err_kahan32_vs_fp64_case_order": rel,
        "fitness_zero_mismatches": zero_mismatch,
        "kernels_per_generation": st.kernels_launched,
        "autotune": {k: v for k, v in tune.as_dict().items() if k != "key"},
        "roofline": {"bound": "fp32_issue", "achieved": batched, "peak": peak, "unit": UNIT,
                     "frac": batched / peak, "scope": "whole generation (pre-pass, interpreter, finalize), device time",
                     "peak_source": f"{sm_count} SMs x 128 FP32 lanes x {sm_max:.0f} MHz ({src})"},
    }


def run_batch(args):
    out = batching_leg(args)
    line = {"metric": METRIC, "value": out["value"], "unit": UNIT, "workload": "batch", "n_gpus": 1,
            "higher_is_better": True, "dtype": "f32", "data": "synthetic (seeded)",
            "config": {"workload": out["workload"]}, **{k: v for k, v in out.items() if k not in ("value", "unit")}}
    print(json.dumps(line), flush=True)


def run_serve(args):
    """The serving configuration at its stated distributions: 256
    independent GP runs arriving as a Poisson process (mean 2 ms), each with
    its own seeded dataset (cases log-uniform [256, 2^20], 1-8 features) and
    population (log-uniform [1k, 2^18] programs, lengths U[8,512]); every run
    submits two generations one after the other (the second a variation of
    the first: 10% of its words redrawn) through the continuous-batching
    server, admission capped at 150 GB of HBM.  A run's data are generated
    when it arrives and dropped when it finishes."""
    import threading
    import galop_b200 as g
    from galop_b200 import workloads as W
    specs = W.serving_run_specs(n_runs=256)
    ev = g.Evaluator(num_registers=16)
    sv = g.Server(ev, hbm_budget_bytes=int(150e9), slots=4, slot_programs=1 << 20, slot_words=1 << 27,
                  slot_items=1 << 25, pinned_bytes=4 << 30)
    rng = np.random.default_rng(9)
    arrivals = np.cumsum(rng.exponential(2e-3, size=len(specs)))
    lat, queued, sizes, peak = [], [], [], [0]
    lock = threading.Lock()
    errors = []
    t0 = time.perf_counter()

    def client(i):
        try:
            delay = t0 + arrivals[i] - time.perf_counter()
            if delay > 0:
                time.sleep(delay)
            X, y, (w, o) = W.serving_run_data(specs[i])
            rid = sv.open_run(g.Dataset(X, y))
            for gen in range(2):
                if gen:
                    W.vary_words(np.random.default_rng(specs[i]["seed"] + gen), w, 0.1, 16)
                rq = sv.submit(rid, w, o)
                _, info = sv.wait(rq)
                with lock:
                    lat.append(info.latency_ms)
                    queued.append(info.queued_ms)
                    sizes.append(info.batch_requests)
                    peak[0] = max(peak[0], sv.totals.resident_bytes)
            sv.close_run(rid)
        except Exception as e:  # reported in the line
            with lock:
                errors.append(f"run {i}: {e}")

    threads = [threading.Thread(target=client, args=(i,)) for i in range(len(specs))]
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
                       "mean": float(np.mean(lat)),
                       "scope": "submit -> fitness in the caller's buffer, per generation of one run"},
        "queued_ms": {"p50": float(np.percentile(queued, 50)), "p99": float(np.percentile(queued, 99))},
        "requests": len(lat), "batches": int(tot.batches), "mean_batch_requests": float(np.mean(sizes)),
        # sum of the batches' own device times over wall time: above 1 when
        # batches in different slots overlap on the device
        "batch_device_time_over_wall": tot.device_ms / 1e3 / wall, "wall_s": wall,
        "device_busy_s": tot.device_ms / 1e3, "peak_resident_gb": peak[0] / 1e9,
        "errors": errors[:5],
        "config": {"workload": "256 GP runs, Poisson arrivals (mean 2 ms), 2 generations each; cases "
                               "log-uniform [256, 2^20], 1-8 features U[-1,1]; populations log-uniform "
                               "[1000, 2^18], lengths U[8,512]; HBM admission cap 150 GB; 4 batches in flight"},
    }
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
    """Largest device-resident population that evaluates (the capacity probe of
    the reference's tests/cuda_capacity.cu): random-word programs of 30 instructions
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
        # torch generates on its (legacy default) stream; the device call runs
        # on the evaluator's own non-blocking stream, so wait for the data
        torch.cuda.synchronize()
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
        st0 = ev.stats
        used = before - torch.cuda.mem_get_info(dev)[0]
        # At this size the device call sizes its micro-op buffer for the raw
        # words (no wait); at the largest population it sizes it exactly
        # (the raw-sized buffer would exceed half the free memory), so the
        # footprint is extrapolated with the exact size.
        per_uop = 16 if dispatch == 3 else 4
        used += (st0.eff_instructions - P0 * L) * per_uop
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


def run_lengths(args):
    """Every tile (cases per lane 1/2/4/8 x warps per block 2/4/8) on
    populations of all-effective programs of one fixed length per class,
    at 4,096 and 65,536 cases: does the best tile depend on the length?
    One JSON line per (cases, length) with the rate of every tile (effective
    GPop/s of the interpreter launches, best of two calls)."""
    import galop_b200 as g
    from galop_b200 import workloads as W
    isa = W.IsaSpec(g.PROFILE_REF, 16)
    for n_cases in (4096, 65536):
        rng = np.random.default_rng(7)
        X = rng.uniform(-3, 3, (n_cases, 5)).astype(np.float32)
        y = np.sin(X[:, 0]).astype(np.float32)
        ds = g.Dataset(X, y)
        for L in (2, 4, 8, 16, 32, 64, 256, 1024):
            n = int(min(65536, max(2048, 2**31 // (L * n_cases))))
            words, off = W.structured_population(rng, np.full(n, L), isa, 1.0)
            rates = {}
            for k in (1, 2, 4, 8):
                for wpb in (2, 4, 8):
                    with g.Evaluator(num_registers=16, cases_per_lane=k, warps_per_block=wpb) as ev:
                        ev.set_dataset(ds)
                        ev.evaluate_csr(words, off)
                        ms = []
                        for _ in range(2):
                            ev.evaluate_csr(words, off)
                            ms.append(ev.stats.interp_ms)
                        eff = ev.stats.eff_instructions
                    rates[f"K{k}_w{wpb}"] = round(eff * n_cases / (min(ms) / 1e3) / 1e9, 1)
            best = max(rates, key=rates.get)
            print(json.dumps({"workload": "lengths", "cases": n_cases, "length": L, "programs": n,
                              "best_tile": best, "best_gpops": rates[best], "gpops": rates}), flush=True)


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
        elif args.workload == "evo":
            run_evo(args)
        elif args.workload == "capacity":
            run_capacity(args)
        elif args.workload == "lengths":
            run_lengths(args)
        elif args.workload == "single":
            line = {"metric": METRIC, "unit": UNIT, "n_gpus": 1, "higher_is_better": True, "dtype": "f32",
                    "data": "synthetic (seeded)", **single_generation_leg(args)}
            print(json.dumps(line), flush=True)
        else:
            run_generation(args, dist)
    finally:
        dist.close()


if __name__ == "__main__":
    main()
