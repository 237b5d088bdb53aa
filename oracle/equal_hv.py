#!/usr/bin/env python
"""Quality check at equal settings: normalised hypervolume of whole runs of the
reference's own CUDA build (oracle/_ref/Protein_NSGA3, built by `make -C oracle
ref`) and of this engine's command line, on one of the reference's sample
proteins, each run several times.  Test infrastructure: it runs the reference
binary as the checker and prints one JSON line.

The reference seeds itself from time() in seconds, so its runs are spaced by
more than a second; this engine's runs use seeds 1..runs.  Both use the
reference's six objectives, codon table and reference-point rule, and report the
hypervolume of the final 2N set normalised as src/main.cu:820-858 does.

    python oracle/equal_hv.py [--protein Q5VZP5] [--N 100] [--G 100] [--m 2] [--pm 0.1] [--runs 10]
"""
import argparse
import json
import re
import shutil
import statistics
import subprocess
import tempfile
import time
from pathlib import Path

HERE = Path(__file__).resolve().parent
REF = HERE / "_ref"
CLI = HERE.parent / "protein_encoding_v2_nsga-iii_b200" / "lib" / "pe_nsga3"


def hv_of(text: str) -> float:
    return float(re.search(r"Hypervolume\s*:\s*([0-9.eE+-]+)", text).group(1))


def gen_time(text: str) -> float:
    return float(re.search(r"Generation cycles time\s*:\s*([0-9.eE+-]+)", text).group(1))


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--protein", default="Q5VZP5")
    ap.add_argument("--N", type=int, default=100)
    ap.add_argument("--G", type=int, default=100)
    ap.add_argument("--m", type=int, default=2)
    ap.add_argument("--pm", type=float, default=0.1)
    ap.add_argument("--runs", type=int, default=10)
    ap.add_argument("--timeout", type=int, default=300)
    a = ap.parse_args()
    fasta = REF / "fasta" / f"{a.protein}.fasta.txt"
    args = [str(fasta.resolve()), str(a.N), str(a.G), str(a.m), str(a.pm)]
    ref_hv, ref_t, our_hv, our_t = [], [], [], []
    for r in range(a.runs):
        with tempfile.TemporaryDirectory() as d:
            shutil.copy(REF / "hv", Path(d) / "hv")
            t0 = time.time()
            out = subprocess.run([str((REF / "Protein_NSGA3").resolve())] + args, cwd=d, capture_output=True, text=True,
                                 timeout=a.timeout)
            if out.returncode != 0:
                raise SystemExit(f"reference run failed: {out.stdout[-500:]} {out.stderr[-500:]}")
            ref_hv.append(hv_of(out.stdout))
            ref_t.append(gen_time(out.stdout))
            time.sleep(max(0.0, 1.1 - (time.time() - t0)))   # a new time() seed for the next run
        with tempfile.TemporaryDirectory() as d:
            out = subprocess.run([str(CLI)] + args + ["--seed", str(r + 1), "--out", d], capture_output=True, text=True,
                                 timeout=a.timeout)
            if out.returncode != 0:
                raise SystemExit(f"engine run failed: {out.stderr[-500:]}")
            our_hv.append(hv_of(out.stdout))
            our_t.append(gen_time(out.stdout))
    med_ref, med_our = statistics.median(ref_hv), statistics.median(our_hv)
    print(json.dumps({"protein": a.protein, "N": a.N, "G": a.G, "m": a.m, "pm": a.pm, "runs": a.runs,
                      "reference_hv": ref_hv, "engine_hv": our_hv,
                      "median_reference": med_ref, "median_engine": med_our, "engine_over_reference": med_our / med_ref,
                      "reference_gen_s_median": statistics.median(ref_t), "engine_gen_s_median": statistics.median(our_t)}))


if __name__ == "__main__":
    main()
