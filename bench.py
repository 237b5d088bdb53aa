#!/usr/bin/env python
"""Benchmark: generations/s of the plain NSGA-III codon-design loop on B200.

Workload (one step = one generation): one synthetic protein of L=1000 amino
acids (+ stop), m=8 CDSs per solution, population N=1024, mutation probability
0.02, four objectives (min CAI, min pairwise Hamming distance, GC3 deviation,
longest hairpin stem), Das-Dennis M=4 p=8 (165 reference points); a full design
job is 500 generations (designs/s = generations/s / 500).

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

Multi-GPU: one independent replica per rank (its own seed, no data-path
collective); `value` = generations of all ranks / the slowest rank's time.
The reference arm times whole generations of the CPU restatement of the
reference algorithm (the oracle; the reference itself has no CPU
implementation) on all host threads, with inputs the oracle generates itself.
"""
from __future__ import annotations

import argparse
import csv
import importlib.util
import io
import json
import math
import os
import statistics
import subprocess
import sys
import time
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parent
L_AA, M_CDS, POP, PM, P_REF, G_JOB, SEED = 1000, 8, 1024, 0.02, 8, 500, 2024
# objective set of the plain workload: 1 = the four objectives (default), 0 = the reference's six
# (then p follows the reference's rule from N: p = 7, 792 points); set by --objectives
OBJ_SET, P_USE, M_OBJ = 1, P_REF, 4
# string objective: 0 = the reference's hairpin stem (default), 1 = longest repeated/common substring
SL_KIND = 0
WORKLOAD = (f"plain NSGA-III, one synthetic protein L={L_AA} aa (+stop), m={M_CDS} CDSs, N={POP}, Pm={PM}, "
            f"4 objectives, Das-Dennis M=4 p={P_REF} (165 points), design job = {G_JOB} generations")


def set_workload(shape: str | None, six: bool, lrcs: bool = False):
    """Plain workload other than the default: --shape L,m,N,p (p = 0: the reference's rule
    from N), the reference's six objectives, and/or the longest repeated/common substring
    as the string objective."""
    global L_AA, M_CDS, POP, P_REF, G_JOB, OBJ_SET, P_USE, M_OBJ, WORKLOAD, SL_KIND
    if shape:
        v = [int(x) for x in shape.split(",")]
        L_AA, M_CDS, POP, P_REF = v[:4]
        if len(v) > 4:
            G_JOB = v[4]
    OBJ_SET, M_OBJ = (0, 6) if six else (1, 4)
    P_USE = 0 if six and not shape else P_REF
    p, R = P_USE, None
    if p <= 0:   # the reference's rule (src/main.cu:564-576): largest p with C(M+p-1, p) <= N
        p = 1
        while math.comb(M_OBJ + p - 1, p) <= POP:
            p += 1
        p -= 1
    R = math.comb(M_OBJ + p - 1, p)
    SL_KIND = 1 if lrcs else 0
    WORKLOAD = (f"plain NSGA-III, one synthetic protein L={L_AA} aa (+stop), m={M_CDS} CDSs, N={POP}, Pm={PM}, "
                f"{'the reference' + chr(39) + 's 6' if six else '4'} objectives"
                f"{' (string objective: longest repeated/common substring)' if lrcs else ''}, Das-Dennis M={M_OBJ} "
                f"p={p} ({R} points), design job = {G_JOB} generations")
METRIC = "generations/s"
L2_FLUSH_BYTES = 256 << 20
# The string-objective kernel (k_sl) per flavour, from one ncu capture of one launch each
# (the committed k_sl profile summaries give the commands and these same numbers): warp
# instructions issued, ALU-pipe warp instructions, shared-memory data-pipe wavefronts,
# thread instructions and DRAM bytes of the launch, the scans (CDSs, LRCS CDS pairs) it ran
# and their counted cells, and the percentages ncu reported.  The seeded first pass does
# work linear in the CDS length per scan, so the roofline scales the counts by the scans a
# timed generation ran.  `source` is the sha256 prefix of the kernel's source section
# (pe_eval.cu from the k_sl banner on) at the capture; a host test fails when the source
# changes without a new capture.
SL_NCU = {
    "hairpin": {"workload": "L=1000 m=8 N=1024, generation 1 (2311 CDSs scanned)",
                "scans": 2311, "cells": 10389102811, "warp_inst": 31266336, "alu_warp_inst": 11443642,
                "smem_wavefronts": 4298609, "thread_inst": 902922790, "dram_bytes": 2336000,
                "issue_pct": 65.40, "alu_pct": 46.42, "smem_pct": 28.82, "source": "47194a0c7b06c89a"},
    "lrcs": {"workload": "L=3000 m=4 N=4096, generation 1 (18320 CDS pairs scanned)",
             "scans": 18320, "cells": 1250515745682, "warp_inst": 1456922853, "alu_warp_inst": 611990996,
             "smem_wavefronts": 156125635, "thread_inst": 41066332937, "dram_bytes": 31110656,
             "issue_pct": 45.90, "alu_pct": 38.43, "smem_pct": 19.38, "source": "47194a0c7b06c89a"},
}
SM_COUNT, ISSUE_WARP_INST_PER_SM_CLK, SMEM_WAVEFRONTS_PER_SM_CLK, ALU_WARP_INST_PER_SM_CLK = 148, 4, 1, 2
# kernels one generation launches (one CUDA graph replay): k_variation, k_sl, k_dominance,
# k_fronts, k_select, k_assoc, k_niche
KERNELS_PER_GENERATION = 7


def load_pkg():
    spec = importlib.util.spec_from_file_location("pe_b200", ROOT / "protein_encoding_v2_nsga-iii_b200" / "__init__.py")
    mod = importlib.util.module_from_spec(spec)
    sys.modules["pe_b200"] = mod
    spec.loader.exec_module(mod)
    return mod


def hairpin_cells_per_cds(n: int) -> int:
    """Counted cells of the stem scan for one CDS of n nucleotides: the upper-triangle
    pairs (r, c) with c - r >= 5 over all anti-diagonals."""
    k = n - 5
    return k * (k + 1) // 2 if k > 0 else 0


def roofline(scans: float, cells: float, sl_seconds: float, clocks: dict, kind: str = "hairpin") -> dict:
    """Roofline of the string-objective scan (integer work on shared-memory tables: a
    table join of 6- or 7-nucleotide words, then the runs it finds measured on bit planes)
    on its three candidate bounds: instruction issue (4 warp instructions per SM per clock),
    the ALU pipe (2 per SM per clock) and the shared-memory data pipe (1 wavefront per SM per
    clock), each x 148 SMs x the SM clock sampled during the timed region.  Achieved = the
    launch's count (ncu, scaled to the scans run) / the launch time measured here.  The
    headline figures are those of the unit with the largest fraction; the others are
    reported beside them."""
    c = SL_NCU[kind]
    scale = scans / c["scans"]
    hz = (clocks.get("sm_mhz") or 1965.0) * 1e6
    src = "(ncu peak_sustained) x 148 SMs at the sampled SM clock"
    units = {}
    for name, count, per_clk, unit, what in (
            ("issue", "warp_inst", ISSUE_WARP_INST_PER_SM_CLK, "G warp-inst/s", "instruction issue 4 warp-inst/SM/clk"),
            ("alu", "alu_warp_inst", ALU_WARP_INST_PER_SM_CLK, "G ALU warp-inst/s", "ALU pipe 2 warp-inst/SM/clk"),
            ("smem", "smem_wavefronts", SMEM_WAVEFRONTS_PER_SM_CLK, "G wavefronts/s",
             "shared-memory data pipe 1 wavefront/SM/clk")):
        achieved = c[count] * scale / sl_seconds / 1e9
        peak = SM_COUNT * per_clk * hz / 1e9
        units[name] = {"achieved": achieved, "peak": peak, "frac": achieved / peak, "unit": unit,
                       "peak_source": f"{what} {src}"}
    bound = max(units, key=lambda k: units[k]["frac"])
    head = units[bound]
    name = "k_sl (hairpin-stem scan)" if kind == "hairpin" else "k_sl (longest repeated/common substring scan)"
    out = {"bound": bound, "kernel": name, "unit": head["unit"], "achieved": head["achieved"],
           "peak": head["peak"], "frac": head["frac"], "traffic": c["dram_bytes"] * scale,
           "peak_source": head["peak_source"] + "; MEASURED_PEAKS.json has no integer or issue peak"}
    for k, v in units.items():
        if k != bound:
            out[k] = {kk: vv for kk, vv in v.items() if kk != "peak_source"}
    out.update({"algorithmic_bytes_per_launch": c["dram_bytes"] * scale,
                "scans_per_launch": scans, "cells_per_launch": cells, "cells_per_s": cells / sl_seconds,
                "counted_cells": "cells of the scans run (unchanged CDSs keep their parents' results)",
                "warp_inst_per_scan": c["warp_inst"] / c["scans"],
                "lane_ops_per_cell": c["thread_inst"] / c["cells"],
                "ncu_pct_of_peak": {"issue": c["issue_pct"], "alu_pipe": c["alu_pct"], "smem_wavefronts": c["smem_pct"]},
                "instruction_count": f"ncu, {c['workload']}; scaled by scans"})
    return out


class ClockSampler:
    """nvidia-smi clocks / throttle reasons sampled every 20 ms while timing.

    A reader thread timestamps every row.  Entering waits (up to 5 s) for the first
    row, so sampling is running when the timed region starts; leaving waits for one
    more row, so the region is covered even when it is shorter than the sampling
    period.  The summary uses the rows from 25 ms before the region to 25 ms after."""

    QUERY = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,clocks_event_reasons.hw_slowdown,"
             "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
             "clocks_event_reasons.sw_power_cap")

    def __init__(self, index: int):
        self.index = index
        self.proc = None
        self.rows = []
        self.t0 = self.t1 = None

    def _read(self):
        for line in self.proc.stdout:
            r = next(csv.reader(io.StringIO(line)), [])
            if len(r) >= 9:
                self.rows.append((time.perf_counter(), [x.strip() for x in r]))

    def _wait_rows(self, n: int, limit_s: float):
        end = time.perf_counter() + limit_s
        while len(self.rows) < n and time.perf_counter() < end and self.proc.poll() is None:
            time.sleep(0.002)

    def __enter__(self):
        import threading
        try:
            self.proc = subprocess.Popen(["nvidia-smi", f"--id={self.index}", f"--query-gpu={self.QUERY}",
                                          "--format=csv,noheader,nounits", "-lms", "20"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True, bufsize=1)
        except OSError:
            self.proc = None
        if self.proc is not None:
            self.thread = threading.Thread(target=self._read, daemon=True)
            self.thread.start()
            self._wait_rows(1, 5.0)
        self.t0 = time.perf_counter()
        return self

    def __exit__(self, *a):
        self.t1 = time.perf_counter()
        if self.proc is None:
            return
        self._wait_rows(len(self.rows) + 1, 1.0)
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
            self.proc.wait()
        self.thread.join(timeout=2)

    def summary(self):
        if not self.rows or self.t0 is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unavailable"], "samples": 0}
        lo, hi = self.t0 - 0.025, (self.t1 or self.t0) + 0.025
        rows = [r for t, r in self.rows if lo <= t <= hi] or [self.rows[-1][1]]
        sm = [float(r[1]) for r in rows if r[1].replace(".", "").isdigit()]
        mx = [float(r[2]) for r in rows if r[2].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[i] for r in rows for i, v in enumerate(r[5:9]) if v.lower() == "active"})
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": reasons, "samples": len(rows), "timed_region_s": round((self.t1 or self.t0) - self.t0, 4)}


def dist_setup():
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return world, rank, local


def host_threads() -> int:
    try:
        return len(os.sched_getaffinity(0))
    except AttributeError:
        return os.cpu_count() or 1


# the same dict in both arms: the workload, not how an arm times it
def config_dict(world: int) -> dict:
    return {"workload": WORKLOAD, "global_batch": POP * world, "parallelism": f"replicas{world}",
            "l2": "GPU arm: L2 flushed between timed steps (256 MiB write, untimed); CPU arm: no device cache"}


def oracle_problem(orc):
    """The plain workload's protein, codon table and problem, built by the oracle alone
    (the engine library is not loaded)."""
    aa = orc.synthetic_protein(L_AA, SEED)
    table = orc.dirichlet_table(SEED)
    return orc.Problem(aa, table, M_CDS, POP, PM, objset=OBJ_SET, p=P_USE, seed=SEED, slkind=SL_KIND)


def time_oracle_generations(run, steps: int, threads: int) -> list[float]:
    """Seconds of each of `steps` whole oracle generations (mutation + evaluation of all N
    offspring with every objective, then selection on the 2N set; src/main.cu:708-728)."""
    out = []
    for _ in range(steps):
        t0 = time.perf_counter()
        run.generation(threads)
        out.append(time.perf_counter() - t0)
    return out


def run_reference(args, world, rank):
    """The reference arm: whole generations of the CPU restatement of the reference
    algorithm on all host threads.  Rank 0 alone runs it."""
    if rank != 0:
        return
    sys.path.insert(0, str(ROOT / "oracle"))
    import pe_oracle as orc
    threads = host_threads()
    prob = oracle_problem(orc)
    run = orc.Run(prob)
    t_init = time.perf_counter()
    run.init(threads)
    t_init = time.perf_counter() - t_init
    time_oracle_generations(run, args.warmup, threads)
    t0 = time.perf_counter()
    secs = time_oracle_generations(run, args.steps, threads)
    wall = time.perf_counter() - t0
    run.close()
    total = sum(secs)
    value = args.steps / total
    sample = (f"{args.steps} whole generations of the workload (after {args.warmup} untimed ones and the "
              f"initial population, {t_init:.1f} s): mutation and full evaluation of all {POP} offspring, "
              f"selection on the {2 * POP}-solution set; {threads} threads")
    line = {"metric": METRIC, "value": value, "unit": "generations/s", "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": 1000.0 * total / args.steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "u32", "data": "synthetic", "impl": "reference",
            "config": config_dict(world), "designs_per_s": value / G_JOB,
            "cpu_baseline": {"value": value, "unit": "generations/s", "cores": threads, "kind": "port",
                             "sample": sample},
            "e2e": {"value": value, "unit": "generations/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
            "step_s": [round(x, 3) for x in secs], "wall_s": wall}
    print(json.dumps(line), flush=True)


def cpu_baseline_one_generation(pe_state, extremes, generation: int) -> dict:
    """The oracle on this host: one whole generation started from the engine's current
    population (bit-identical to the oracle's own state at that generation)."""
    sys.path.insert(0, str(ROOT / "oracle"))
    import pe_oracle as orc
    threads = host_threads()
    run = orc.Run(oracle_problem(orc))
    ids, obj, objidx, pql, surv = pe_state
    run.set_state(ids, obj, objidx, pql, surv, extremes, generation)
    sec = time_oracle_generations(run, 1, threads)[0]
    run.close()
    return {"value": 1.0 / sec, "unit": "generations/s", "cores": threads, "kind": "port",
            "sample": f"one whole generation (mutation and full evaluation of all {POP} offspring, selection on "
                      f"the {2 * POP}-solution set) started from the GPU run's population at generation "
                      f"{generation}; {threads} threads; {sec:.1f} s"}


# The reference's own CUDA build (compiled unmodified from its sources) did not
# terminate on this workload's protein on a B200: 10 generations under a 90 s limit
# and 100 generations under a 150 s limit were both killed at the limit.  Code that
# hung is not run again, so the line records that instead of a rate.
REFERENCE_CUDA_UNAVAILABLE = ("the reference's CUDA build (src/main.cu compiled unmodified for sm_100a) did not "
                              "terminate on this workload's protein on a B200 (10 generations: killed at a 90 s "
                              "limit; 100 generations: killed at 150 s); it is not run again")


def run_ours(args, world, rank, local):
    import torch
    pe = load_pkg()
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    if world > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120), device_id=dev)
    stream = torch.cuda.Stream(device=dev)
    aa = pe.synthetic_protein(L_AA, SEED)
    table = pe.dirichlet_table(SEED)
    eng = pe.Engine(aa, table, M_CDS, POP, PM, objectives=OBJ_SET, ref_p=P_USE, seed=SEED + rank,
                    sl_threads=args.sl_threads, stream=stream.cuda_stream, sl_kind=SL_KIND)
    eng.init()
    eng.set_profiling(True)
    for _ in range(args.warmup):
        eng.step(1)
    eng.synchronize()
    scans0, cells0 = eng.scan_count(), eng.scan_cells()
    flush = torch.empty(L2_FLUSH_BYTES, dtype=torch.uint8, device=dev)
    ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(args.steps)]
    stage = np.zeros((args.steps, 3))
    if world > 1:
        torch.distributed.barrier()
    torch.cuda.synchronize(dev)
    with ClockSampler(local) as clk:
        t_wall = time.perf_counter()
        for k in range(args.steps):
            with torch.cuda.stream(stream):
                flush.zero_()                       # L2 flush between timed steps (not timed)
                ev[k][0].record(stream)
                eng.step(1)
                ev[k][1].record(stream)
            eng.synchronize()
            stage[k] = eng.stage_times()
        torch.cuda.synchronize(dev)
        t_wall = time.perf_counter() - t_wall
    if world > 1:
        torch.distributed.barrier()
    step_ms = [a.elapsed_time(b) for a, b in ev]
    total_s = sum(step_ms) / 1000.0
    replicas = load_pkg_module("replicas")
    max_s = replicas.max_over_ranks(total_s, dev)
    value = world * args.steps / max_s
    stage_ms = stage.mean(axis=0)
    # stage times per window of 5 timed generations (early generations are front-heavy)
    windows = [{"generations": [args.warmup + w, args.warmup + min(w + 5, args.steps) - 1],
                "variation_eval": float(stage[w:w + 5, 0].mean()), "hairpin_scan": float(stage[w:w + 5, 1].mean()),
                "selection": float(stage[w:w + 5, 2].mean())} for w in range(0, args.steps, 5)]
    # a child's CDS (LRCS: CDS pair) that its mutation left unchanged keeps its parent's
    # result: the string-objective work is the cells of the scans actually run
    cells = (eng.scan_cells() - cells0) / args.steps
    scans = (eng.scan_count() - scans0) / args.steps
    sl_s = stage_ms[1] / 1000.0

    # end-to-end through the public API with host buffers: every rank runs whole design jobs
    # (G_JOB generations) on its GPU; the whole-job rate uses the slowest rank (three jobs, the median)
    G_E2E, E2E_JOBS = G_JOB, 3
    # the per-generation objective reads go to page-locked host memory, queued behind
    # each generation (a ring of two buffers: the host could read one while the other
    # fills); the job waits once, at its end
    obj_ring = [torch.empty((2 * POP, M_OBJ), dtype=torch.float32, pin_memory=True) for _ in range(2)]
    obj_host = obj_ring[0].numpy()
    if world > 1:
        torch.distributed.barrier()
    torch.cuda.synchronize(dev)
    job_s = []
    for job in range(E2E_JOBS):
        t0 = time.perf_counter()
        e2 = pe.Engine(aa, table, M_CDS, POP, PM, objectives=OBJ_SET, ref_p=P_USE, seed=SEED + 7 + rank + 1000 * job,
                       sl_threads=args.sl_threads, sl_kind=SL_KIND)
        e2.init()
        for g in range(G_E2E):
            e2.step(1)
            e2.read_objectives_async(obj_ring[g & 1].data_ptr())  # this generation's objectives to the host
        final = e2.population()                 # waits for the generations and the reads
        e2.close()
        job_s.append(time.perf_counter() - t0)
    e2e_s = replicas.max_over_ranks(statistics.median(job_s), dev)
    h2d = aa.nbytes + 4 * (64 * 4 + 61 * 61 + 12)
    d2h = obj_host.nbytes + sum(a.nbytes for a in final) / G_E2E

    line = None
    if rank == 0:
        # CPU baseline: the oracle on this host, bounded sample (N=1 only)
        cpu, ref_cuda = None, None
        if world == 1 and not args.no_cpu_baseline:
            # extreme points only steer the normalisation: the survivors' first M objective
            # vectors give the timed generation the same work
            state = eng.population()
            ext = state[1][state[4][:M_OBJ]]
            cpu = cpu_baseline_one_generation(state, ext, eng.generation)
        if world == 1:
            ref_cuda = {"unavailable": REFERENCE_CUDA_UNAVAILABLE}

        peaks = {}
        try:
            peaks = json.loads((ROOT / "MEASURED_PEAKS.json").read_text())
        except Exception:
            pass
        clocks = clk.summary()
        line = {
            "metric": METRIC, "value": value, "unit": "generations/s", "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": 1000.0 * max_s / args.steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "u32", "data": "synthetic",
            "config": config_dict(world),
            "designs_per_s": value / G_JOB,
            "stage_ms": {"variation_eval": stage_ms[0], "hairpin_scan": stage_ms[1], "selection": stage_ms[2]},
            "stage_ms_windows": windows,
            "roofline": roofline(scans, cells, sl_s, clocks, "lrcs" if SL_KIND else "hairpin"),
            "clocks": clocks,
            "e2e": {"value": world * G_E2E / e2e_s, "unit": "generations/s", "h2d_bytes_per_step": world * h2d / G_E2E,
                    "d2h_bytes_per_step": world * d2h,
                    "designs_per_s": world / e2e_s,
                    "job": f"per rank: create + init + {G_E2E} generations (a whole design job) + per-generation "
                           f"objective reads (queued into page-locked host memory behind each generation) + "
                           f"final population read, median of {E2E_JOBS} jobs; all ranks / slowest rank",
                    "rank0_job_s": [round(x, 5) for x in job_s]},
            "gpu_launches": KERNELS_PER_GENERATION * args.steps,
            "wall_s": t_wall,
            "peaks_file": {k: peaks.get(k) for k in ("hbm_gbs", "bf16_tflops", "sm_max_mhz")},
        }
        if cpu:
            line["cpu_baseline"] = cpu
        if ref_cuda:
            line["ref_cuda"] = ref_cuda
        print(json.dumps(line), flush=True)
    eng.close()
    if world > 1:
        torch.distributed.destroy_process_group()


def batched_jobs(master_seed: int, count: int = 64):
    """64 independent proteins: L log-uniform in [100, 3000] aa, m from {2, 4, 8},
    per-instance seeds from the master seed (SplitMix64)."""
    x = master_seed
    jobs = []
    for j in range(count):
        x = (x + 0x9E3779B97F4A7C15) & 0xFFFFFFFFFFFFFFFF
        z = x
        z = ((z ^ (z >> 30)) * 0xBF58476D1CE4E5B9) & 0xFFFFFFFFFFFFFFFF
        z = ((z ^ (z >> 27)) * 0x94D049BB133111EB) & 0xFFFFFFFFFFFFFFFF
        z ^= z >> 31
        u = ((z >> 11) + 0.5) / float(1 << 53)
        L = int(round(100 * (3000 / 100) ** u))
        m = (2, 4, 8)[(z >> 3) % 3]
        jobs.append((L, m, z))
    return jobs


def run_batched(args, world: int = 1, rank: int = 0, local: int = 0):
    """Config 4: 64 design jobs (N=512, 300 generations) as one batch.  On N GPUs the
    jobs are sharded across the ranks by estimated stem-scan cells (longest first onto
    the least-loaded rank; no data-path collective), each rank runs its shard as one
    batch, the time is the slowest rank's and every job's result is gathered on rank 0.
    At N=1 the same jobs also run one at a time (the plain per-protein form)."""
    import torch
    pe = load_pkg()
    rep = load_pkg_module("replicas")
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    if world > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=600), device_id=dev)
    G = args.generations or 300
    jobs = batched_jobs(SEED)
    N, pm = 512, 0.02
    costs = [N * m * hairpin_cells_per_cds(3 * (L + 1)) for L, m, _ in jobs]
    mine = rep.shard_jobs(costs, world)[rank]

    def make(j):
        L, m, seed = jobs[j]
        e = pe.Engine(pe.synthetic_protein(L, seed), pe.dirichlet_table(seed), m, N, pm, objectives=pe.OBJ_BASE4,
                      seed=seed)
        e.init()
        return e

    cells = sum(costs) * G
    t_plain = None
    if world == 1:
        # one at a time (the plain per-protein form)
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        for j in range(len(jobs)):
            e = make(j)
            e.step(G)
            e.synchronize()
            e.close()
        t_plain = time.perf_counter() - t0
        # the same batch with the batch's stem scans queued (one wave per length class)
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        engines = [make(j) for j in mine]
        with pe.Batch(engines) as b:
            b.set_scan_queue(True)
            b.step(G)
            b.synchronize()
        for e in engines:
            e.close()
        t_queued = time.perf_counter() - t0
    # this rank's shard together (create + init + generations), a graph branch per member
    if world > 1:
        torch.distributed.barrier()
    with ClockSampler(local) as clk:
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        engines = [make(j) for j in mine]
        if engines:
            with pe.Batch(engines) as b:
                b.step(G)
                b.synchronize()
        t_rank = time.perf_counter() - t0
    results = {}
    for j, e in zip(mine, engines):
        surv = e.survivor_objectives()
        results[j] = {"rank": rank, "scan_cells": e.scan_cells(),
                      "hv": float(load_pkg_module("server").front_hypervolume(pe, surv, pe.OBJ_BASE4))}
        e.close()
    t_batch = rep.max_over_ranks(t_rank, dev)
    results = rep.gather_results(results)
    if rank == 0:
        assert sorted(results) == list(range(len(jobs)))
        scanned_cells = sum(r["scan_cells"] for r in results.values())
        line = {"metric": "designs/s", "value": len(jobs) / t_batch, "unit": "designs/s", "n_gpus": world,
                "steps": G, "warmup": 0, "ms_per_step": 1000.0 * t_batch / G, "higher_is_better": True,
                "scaling": "strong" if world > 1 else "weak", "vs_baseline": None, "dtype": "u32",
                "data": "synthetic",
                "config": {"workload": f"batched: {len(jobs)} proteins, L log-uniform [100, 3000], m in {{2,4,8}}, "
                                       f"N={N}, Pm={pm}, 4 objectives, {G} generations, one graph launch per 2 "
                                       f"generations for all instances of a rank, a branch per instance",
                           "parallelism": f"job shards over {world} GPU(s) by stem-scan cells"},
                "stem_cells_per_s": scanned_cells / t_batch, "stem_cells_scanned_of_all": scanned_cells / cells,
                "mean_final_hv": float(np.mean([r["hv"] for r in results.values()])),
                "timing": "wall clock per mode, each including create + init + all generations; N>1: slowest rank",
                "clocks": clk.summary()}
        if t_plain is not None:
            line["plain_designs_per_s"] = len(jobs) / t_plain
            line["batched_over_plain"] = t_plain / t_batch
            line["queued_scans_designs_per_s"] = len(jobs) / t_queued
            line["queued_over_branches"] = t_batch / t_queued
        print(json.dumps(line), flush=True)
    if world > 1:
        torch.distributed.destroy_process_group()


def served_jobs(pe, srv_mod, master_seed: int, count: int, rate: float):
    """Design requests of the served workload: Poisson arrivals at `rate` jobs/s,
    L log-uniform in [50, 5000] aa, m uniform in [2, 10], N uniform in
    {256, 512, 1024, 2048}, generation budget uniform in [200, 1000], stall 50."""
    rng = np.random.default_rng(master_seed)
    t, jobs = 0.0, []
    for j in range(count):
        t += rng.exponential(1.0 / rate)
        L = int(round(50 * 100.0 ** rng.random()))
        m = int(rng.integers(2, 11))
        N = int(rng.choice([256, 512, 1024, 2048]))
        G = int(rng.integers(200, 1001))
        seed = int(rng.integers(1, 1 << 62))
        jobs.append(srv_mod.Job(pe.synthetic_protein(L, seed), pe.dirichlet_table(seed), m, N, G, seed,
                                objectives=pe.OBJ_BASE4, mutation_prob=PM, stall=50, arrival=t))
    return jobs


def run_served(args):
    """Config 5: Poisson arrivals of design jobs served by the library's serving core
    (pe_server_*: continuous batching, footprint admission, stall retirement), against
    the plain form (the same core with one resident job at a time, in arrival order) on
    the first --plain-jobs jobs of the same stream, whose results must equal the served
    ones."""
    import copy

    import torch
    pe = load_pkg()
    srv_mod = load_pkg_module("server")
    torch.cuda.set_device(0)
    count = args.jobs
    base = served_jobs(pe, srv_mod, SEED, count, 20.0)
    free, _ = torch.cuda.mem_get_info()
    budget = int(free * 0.8)
    lines = {}
    n_plain = min(count, args.plain_jobs)
    modes = (("served", base, 16, True, "shortest"), ("plain", base[:n_plain], 1, False, "arrival"))
    for mode, jobset, max_active, prio, order in modes:
        jobs = [copy.copy(j) for j in jobset]
        srv = srv_mod.NativeServer(pe, memory_budget=budget, max_active=max_active, tick=10, hv_every=25,
                                   priority=prio, order=order, max_wait=60.0)
        with ClockSampler(0) as clk:
            done = srv.run(jobs)
        stats = srv.stats()
        srv.close()
        st = srv_mod.latency_stats(done)
        st["peak_active"], st["peak_gb"] = stats.peak_active, stats.peak_used_bytes / 1e9
        st["generations"] = sum(j.generations_run for j in done)
        st["mean_hv"] = float(np.mean([j.hv for j in done if j.hv is not None]))
        st["clocks"] = clk.summary()
        st["hv"] = {int(round(j.arrival * 1e9)): j.hv for j in done}
        lines[mode] = st
        if st["failed"]:
            raise RuntimeError(f"{st['failed']} jobs failed: " + "; ".join(j.error for j in done if j.error))
    s, p = lines["served"], lines["plain"]
    same_hv = all(s["hv"][k] == v for k, v in p["hv"].items())
    line = {"metric": "designs/s", "value": s["designs_per_s"], "unit": "designs/s", "n_gpus": 1,
            "steps": count, "warmup": 0, "ms_per_step": 1000.0 * s["span_s"] / count, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "u32", "data": "synthetic",
            "config": {"workload": f"served: {count} Poisson arrivals at 20 jobs/s"
                                   f"{'' if count == 2000 else f' (the first {count} of the 2000-job stream)'}, "
                                   "L log-uniform [50, 5000], m U[2,10], N in {256,512,1024,2048}, G U[200,1000], "
                                   "stop on hypervolume stall over 50 generations (checked every 25), "
                                   "4 objectives, Pm=0.02"},
            "p50_s": s["p50_s"], "p99_s": s["p99_s"], "mean_s": s["mean_s"],
            "plain_jobs": n_plain, "plain_p50_s": p["p50_s"], "plain_p99_s": p["p99_s"],
            "plain_designs_per_s": p["designs_per_s"],
            "served_over_plain_designs_per_s": s["designs_per_s"] / p["designs_per_s"],
            "stalled_jobs": s["stalled"], "generations": s["generations"], "mean_final_hv": s["mean_hv"],
            "same_results_as_plain": same_hv, "peak_resident_jobs": s["peak_active"],
            "peak_device_gb": s["peak_gb"], "memory_budget_gb": budget / 1e9,
            "policy": "C++ serving core: up to 16 resident jobs, shortest estimated work admitted first (a job "
                      "waiting over 60 s goes first), stream priority by estimated work; plain = the same core "
                      "with one resident job at a time in arrival order",
            "timing": "wall clock from each arrival to its result on the host",
            "clocks": s["clocks"], "plain_clocks": p["clocks"]}
    print(json.dumps(line), flush=True)


def load_pkg_module(stem: str):
    name = f"pe_b200_{stem}"
    if name not in sys.modules:
        spec = importlib.util.spec_from_file_location(name, ROOT / "protein_encoding_v2_nsga-iii_b200" / f"{stem}.py")
        mod = importlib.util.module_from_spec(spec)
        sys.modules[name] = mod
        spec.loader.exec_module(mod)
    return sys.modules[name]


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--workload", choices=["plain", "batched", "served"], default="plain")
    ap.add_argument("--generations", type=int, default=0, help="generations per job (batched)")
    ap.add_argument("--jobs", type=int, default=2000, help="design requests in the served workload")
    ap.add_argument("--plain-jobs", type=int, default=200,
                    help="served workload: jobs of the stream also run one at a time (the plain form)")
    ap.add_argument("--shape", default=None, help="plain workload L,m,N,p[,G] instead of 1000,8,1024,8,500 "
                    "(p=0: the reference's rule from N; G: generations of a design job)")
    ap.add_argument("--string", choices=["hairpin", "lrcs"], default="hairpin",
                    help="string objective of the plain workload: the reference's hairpin stem or the longest "
                         "repeated/common substring")
    ap.add_argument("--objectives", choices=["base4", "ref6"], default="base4",
                    help="objective set of the plain workload (ref6: the reference's six, p by its rule)")
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=None,
                    help="timed generations (default 500; 3 for --impl reference, whose CPU generations take ~20 s)")
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--no-cpu-baseline", action="store_true",
                    help="skip the CPU baseline (one whole oracle generation: minutes at the long-sequence shapes)")
    ap.add_argument("--sl-threads", type=int, default=0, choices=[0, 64, 128, 256],
                    help="stem-scan CTA size (0: timed per instance at init); a fixed size keeps a run "
                         "under a profiler, which slows every launch, on the kernels a plain run picks")
    ap.add_argument("--profile-case", action="store_true",
                    help="only build the bench instance, init and run --profile-gens generations (for ncu captures)")
    ap.add_argument("--profile-gens", type=int, default=2,
                    help="generations of --profile-case (e.g. 60 to capture a steady-state selection)")
    args = ap.parse_args()
    if args.steps is None:
        args.steps = 3 if args.impl == "reference" else 500
    if args.objectives == "ref6" or args.shape or args.string == "lrcs":
        set_workload(args.shape, args.objectives == "ref6", args.string == "lrcs")
    world, rank, local = dist_setup()
    if args.workload == "batched":
        run_batched(args, world, rank, local)
        return
    if args.workload == "served":
        run_served(args)
        return
    if args.profile_case:
        pe = load_pkg()
        # the stem-scan CTA size is fixed at the one the bench instance's tuning picks (128
        # threads), so the launches are the same with and without a profiler: the initial
        # scan, then one scan per generation
        eng = pe.Engine(pe.synthetic_protein(L_AA, SEED), pe.dirichlet_table(SEED), M_CDS, POP, PM,
                        objectives=OBJ_SET, ref_p=P_USE, seed=SEED, sl_threads=args.sl_threads or 128,
                        sl_kind=SL_KIND)
        eng.init()
        scans, cells = [eng.scan_count()], [eng.scan_cells()]
        for _ in range(args.profile_gens):
            eng.step(1)
            scans.append(eng.scan_count())
            cells.append(eng.scan_cells())
        eng.close()
        print(json.dumps({"scans_per_launch": [scans[0]] + [b - a for a, b in zip(scans, scans[1:])],
                          "cells_per_launch": [cells[0]] + [b - a for a, b in zip(cells, cells[1:])]}))
        return
    if args.impl == "reference":
        run_reference(args, world, rank)
    else:
        run_ours(args, world, rank, local)


if __name__ == "__main__":
    main()
