#!/usr/bin/env python
"""Equal-hypervolume check of whole runs: the reference's own CUDA build
(oracle/_ref/Protein_NSGA3, compiled unmodified by `make -C oracle ref`) against
this engine's command line, at the same settings, several runs each.

Test infrastructure: it runs the reference binary as the checker and prints one
JSON line (medians, spreads and their ratio).  Both programs use the reference's
six objectives, its codon table and its reference-point rule, and write the
final 2N set normalised as src/main.cu:789-844 does; the hypervolume of each
file is computed here with the oracle's exact hypervolume (reference point all
ones), and the value each program printed is recorded beside it.

The reference seeds itself from time() in seconds (src/main.cu:469,525), so its
runs are spaced by more than a second; this engine's runs use seeds 1..runs.
Every run has a wall-clock limit; the script stops at the first run that fails
or overruns it and reports what it has.

    python oracle/equal_hv.py [--L 1000] [--N 1024] [--G 100] [--m 8] [--pm 0.02] [--runs 10]
"""
from __future__ import annotations

import argparse
import json
import re
import shutil
import statistics
import subprocess
import sys
import tempfile
import time
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
REF = HERE / "_ref"
CLI = HERE.parent / "protein_encoding_v2_nsga-iii_b200" / "lib" / "pe_nsga3"
AMINO = "ACDEFGHIKLMNPQRSTVWY"
sys.path.insert(0, str(HERE))
import pe_oracle as orc  # noqa: E402


def printed(text: str, key: str):
    m = re.search(key + r"\s*:\s*([0-9.eE+-]+)", text)
    return float(m.group(1)) if m else None


def file_hv(path: Path) -> float:
    pts = np.loadtxt(path, dtype=np.float64, ndmin=2)
    return orc.hypervolume(pts, np.ones(pts.shape[1]))


def spread(v):
    if not v:
        return {}
    q = np.percentile(v, [25, 50, 75])
    return {"median": float(q[1]), "min": float(min(v)), "max": float(max(v)), "q1": float(q[0]), "q3": float(q[2])}


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--L", type=int, default=1000, help="synthetic protein length (amino acids, before the stop)")
    ap.add_argument("--protein-seed", type=int, default=2024)
    ap.add_argument("--N", type=int, default=1024)
    ap.add_argument("--G", type=int, default=100)
    ap.add_argument("--m", type=int, default=8)
    ap.add_argument("--pm", type=float, default=0.02)
    ap.add_argument("--runs", type=int, default=10)
    ap.add_argument("--timeout", type=int, default=120, help="wall-clock limit per run, seconds")
    ap.add_argument("--out", default=None, help="also write the JSON line to this file")
    a = ap.parse_args()
    aa = orc.synthetic_protein(a.L, a.protein_seed)[:-1]
    work = Path(tempfile.mkdtemp(prefix="equal_hv_"))
    fasta = work / "protein.fasta.txt"
    fasta.write_text(">synthetic\n" + "".join(AMINO[int(x)] for x in aa) + "\n")
    args = [str(fasta), str(a.N), str(a.G), str(a.m), str(a.pm)]
    res = {"L": a.L, "protein_seed": a.protein_seed, "N": a.N, "G": a.G, "m": a.m, "pm": a.pm, "runs": a.runs,
           "timeout_s": a.timeout, "reference": [], "engine": [], "failure": None}
    try:
        for r in range(a.runs):
            for who in ("reference", "engine"):
                d = Path(tempfile.mkdtemp(dir=work))
                if who == "reference":
                    shutil.copy(REF / "hv", d / "hv")
                    cmd = [str((REF / "Protein_NSGA3").resolve())] + args
                else:
                    cmd = [str(CLI)] + args + ["--seed", str(r + 1), "--out", str(d)]
                t0 = time.time()
                try:
                    out = subprocess.run(cmd, cwd=d, capture_output=True, text=True, timeout=a.timeout)
                except subprocess.TimeoutExpired:
                    res["failure"] = f"{who} run {r + 1} exceeded {a.timeout} s"
                    raise StopIteration
                wall = time.time() - t0
                if out.returncode != 0 or not (d / "Normalized_value_quality_computation.txt").exists():
                    res["failure"] = (f"{who} run {r + 1} exit {out.returncode}: "
                                      f"{out.stdout[-300:]} {out.stderr[-300:]}")
                    raise StopIteration
                lookups = out.stdout.count("findIndexAmongSynonymousCodons Function failure")
                res[who].append({"hv": file_hv(d / "Normalized_value_quality_computation.txt"),
                                 "hv_printed": printed(out.stdout, "Hypervolume"),
                                 "generation_s": printed(out.stdout, "Generation cycles time"),
                                 "init_s": printed(out.stdout, "Initialization time"), "wall_s": wall,
                                 "lookup_failure_prints": lookups})
                if who == "reference":
                    time.sleep(max(0.0, 1.1 - (time.time() - t0)))   # a new time() seed for the next run
    except StopIteration:
        pass
    finally:
        shutil.rmtree(work, ignore_errors=True)
    ref_hv = [x["hv"] for x in res["reference"]]
    eng_hv = [x["hv"] for x in res["engine"]]
    res["reference_hv"] = spread(ref_hv)
    res["engine_hv"] = spread(eng_hv)
    if ref_hv and eng_hv:
        res["engine_over_reference_median_hv"] = statistics.median(eng_hv) / statistics.median(ref_hv)
        rg = [x["generation_s"] for x in res["reference"] if x["generation_s"]]
        eg = [x["generation_s"] for x in res["engine"] if x["generation_s"]]
        if rg and eg:
            res["reference_generations_per_s"] = a.G / statistics.median(rg)
            res["engine_generations_per_s"] = a.G / statistics.median(eg)
    line = json.dumps(res)
    print(line, flush=True)
    if a.out:
        Path(a.out).write_text(line + "\n")
    return 0 if res["failure"] is None else 1


if __name__ == "__main__":
    sys.exit(main())
