"""Extract the reference's codon table (include/info.cuh:6-54) into
data/ref_codon_table.txt (next to this script), the text format read by pe_load_codon_table.

Run where the reference sources are available, giving their directory (or
PE_REFERENCE_DIR):
    python protein_encoding_v2_nsga-iii_b200/data/make_ref_table.py <reference dir>
The table is data (genetic code, relative-adaptiveness weights, codon-pair
scores); the weights are evaluated as the C float expressions they are written as.
"""
import re
import sys
from pathlib import Path

import numpy as np


def main(ref_root: str):
    src = (Path(ref_root) / "include" / "info.cuh").read_text()
    active = src.split("#if 0")[0]
    amino = re.search(r"aminoacids\[21\]\s*=\s*\{([^}]*)\}", active).group(1)
    amino = [c for c in re.findall(r"'(.)'", amino)]
    start = [int(x) for x in re.search(r"codons_start_idx\[21\]\s*=\s*\{([^}]*)\}", active).group(1).split(",")]
    count = [int(x) for x in re.search(r"syn_codons_num\[21\]\s*=\s*\{([^}]*)\}", active).group(1).split(",")]
    cod = re.search(r'codons\[[^\]]*\]\s*=\s*"(.*?)";', active, re.S).group(1)
    cod = re.sub(r"\\\s*\n", "", cod).replace("\n", "")
    assert len(cod) == 192, len(cod)
    wtxt = re.search(r"codons_weight\[[^\]]*\]\s*=\s*\{(.*?)\};", active, re.S).group(1)
    weights = []
    for term in wtxt.split(","):
        term = term.strip()
        if not term:
            continue
        m = re.fullmatch(r"(\d+)\s*/\s*([\d.]+)f", term)
        if m:
            weights.append(np.float32(np.float32(int(m.group(1))) / np.float32(float(m.group(2)))))
        else:
            weights.append(np.float32(float(term.rstrip("f"))))
    assert len(weights) == 64
    cps = re.search(r"cps\[[^\]]*\]\s*=\s*\{(.*?)\};", active, re.S).group(1)
    cps = [np.float32(float(x.strip().rstrip("f"))) for x in cps.split(",") if x.strip()]
    assert len(cps) == 61 * 61
    gc = float(re.search(r"ref_GC_percent\s*=\s*([\d.]+)f", active).group(1))
    gc3 = float(re.search(r"ref_GC3_percent\s*=\s*([\d.]+)f", active).group(1))
    aa_of = []
    for a, (s, k) in enumerate(zip(start, count)):
        assert s == len(aa_of)
        aa_of += [amino[a]] * k
    out = ["# reference codon table (include/info.cuh:6-54): codon amino weight, in id order"]
    for i in range(64):
        out.append(f"{cod[3*i:3*i+3]} {aa_of[i]} {float(weights[i]):.9g}")
    out.append(f"gc3 {gc3:.9g}")
    out.append(f"gc {gc:.9g}")
    out.append("cps")
    for r in range(61):
        out.append(" ".join(f"{float(v):.9g}" for v in cps[61 * r:61 * r + 61]))
    dst = Path(__file__).resolve().parent / "ref_codon_table.txt"
    dst.write_text("\n".join(out) + "\n")
    print("wrote", dst)


if __name__ == "__main__":
    import os
    src = sys.argv[1] if len(sys.argv) > 1 else os.environ.get("PE_REFERENCE_DIR")
    if not src:
        sys.exit("usage: make_ref_table.py <reference source directory> (or set PE_REFERENCE_DIR)")
    main(src)
