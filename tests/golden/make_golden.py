"""Golden vectors from the reference's own device functions.

    python tests/golden/make_golden.py jobs  <dir>   # write harness inputs (CPU)
    python tests/golden/make_golden.py run   <dir>   # run oracle/_ref/ref_harness on each (needs a GPU)
    python tests/golden/make_golden.py collect <dir> # pack inputs + outputs into tests/golden/ref_*.npz

The harness (oracle/ref_harness.cu, built by `make -C oracle ref`) compiles the
reference's evaluators (include/utils.cuh), non-dominated sort, normalisation
and association (include/sorting.cuh) and Das-Dennis generator unmodified.
Inputs are seeded: synthetic proteins, the reference FASTA B7KHU9 (embedded
below as its amino-acid string), random solutions and objective vectors.
"""
from __future__ import annotations

import importlib.util
import json
import struct
import subprocess
import sys
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parents[2]
GOLDEN = Path(__file__).resolve().parent
HARNESS = ROOT / "oracle" / "_ref" / "ref_harness"

# Protein_FASTA/B7KHU9.fasta.txt sequence (38 aa), stop appended by the loader
B7KHU9 = "MIEPLVLGLVMGLVPITLAGLFVAAYLQYKRGNQLNLD"
AMINO = "ACDEFGHIKLMNPQRSTVWYZ"
NT = "ACGU"


def _pkg():
    spec = importlib.util.spec_from_file_location("pe_b200", ROOT / "protein_encoding_v2_nsga-iii_b200" / "__init__.py")
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    return mod


def _oracle():
    sys.path.insert(0, str(ROOT / "oracle"))
    import pe_oracle
    return pe_oracle


def random_solutions(rng, aa, tab, m, n):
    ids = np.zeros((n, m, len(aa)), np.uint8)
    start, count = tab["start"], tab["count"]
    for i in range(n):
        for c in range(m):
            ids[i, c] = start[aa] + (rng.random(len(aa)) * count[aa]).astype(np.int64)
    return ids


def to_chars(ids, tab):
    cod = ["".join(NT[b] for b in tab["nt"][c]) for c in range(64)]
    return "".join(cod[c] for c in ids.reshape(-1)).encode()


def eval_cases(pe):
    """(name, aa, table arrays, custom_table_flag, ids)"""
    ref_tab = pe.load_codon_table(ROOT / "protein_encoding_v2_nsga-iii_b200" / "data" / "ref_codon_table.txt").arrays()
    dir_tab = pe.dirichlet_table(11).arrays()
    rng = np.random.default_rng(2024)
    cases = []
    aa = np.array([AMINO.index(c) for c in B7KHU9] + [20], np.int8)
    ids = random_solutions(rng, aa, ref_tab, 3, 24)
    ids[0] = ref_tab["start"][aa] + ref_tab["count"][aa] - 1     # highest-weight codons everywhere
    ids[1, 1] = ids[1, 0]                                         # duplicated CDS (HD = 0, ties)
    ids[2, 2] = ids[2, 0]
    cases.append(("b7khu9_m3", aa, ref_tab, 0, ids))
    aa = pe.synthetic_protein(200, 101)
    cases.append(("syn200_m2", aa, ref_tab, 0, random_solutions(rng, aa, ref_tab, 2, 24)))
    for L in (2, 3, 4, 6):
        aa = pe.synthetic_protein(L, 200 + L)
        cases.append((f"tiny{L + 1}_m2", aa, ref_tab, 0, random_solutions(rng, aa, ref_tab, 2, 16)))
    aa = pe.synthetic_protein(1000, 303)
    cases.append(("syn1000_m8", aa, ref_tab, 0, random_solutions(rng, aa, ref_tab, 8, 4)))
    aa = pe.synthetic_protein(100, 404)
    cases.append(("dirichlet100_m4", aa, dir_tab, 1, random_solutions(rng, aa, dir_tab, 4, 24)))
    return cases


def select_cases(pe, orc):
    rng = np.random.default_rng(77)
    out = []
    for N in (16, 50, 100):
        obj = rng.random((2 * N, 6)).astype(np.float32)
        obj[:, 0] = -0.5 - 0.5 * obj[:, 0]
        ext = obj[:6].copy()
        out.append((f"uniform_N{N}", N, obj, ext))
    # objective vectors of evaluated random populations (duplicates included)
    tab = pe.load_codon_table(ROOT / "protein_encoding_v2_nsga-iii_b200" / "data" / "ref_codon_table.txt").arrays()
    aa = pe.synthetic_protein(60, 505)
    N = 40
    prob = orc.Problem(aa, tab, 3, N, 0.05, objset=0)
    ids = random_solutions(rng, aa, tab, 3, 2 * N)
    ids[N:N + 10] = ids[:10]
    obj, _, _ = prob.evaluate(ids)
    out.append(("evaluated_N40", N, obj.astype(np.float32), obj[:6].copy()))
    return out


DD_CASES = [(4, 6), (4, 8), (6, 4), (6, 5), (3, 12), (5, 3), (6, 1)]


def cmd_jobs(d: Path):
    pe = _pkg()
    orc = _oracle()
    d.mkdir(parents=True, exist_ok=True)
    meta = {"eval": [], "select": [], "dd": []}
    for name, aa, tab, custom, ids in eval_cases(pe):
        L, m, n = len(aa), ids.shape[1], ids.shape[0]
        b = bytearray(b"PEH1") + struct.pack("<iiiii", 1, L, m, n, custom)
        if custom:
            cod = "".join("".join(NT[x] for x in tab["nt"][c]) for c in range(64)).encode()
            b += cod + np.asarray(tab["weight"], np.float32).tobytes() + np.asarray(tab["start"], np.int8).tobytes()
            b += np.asarray(tab["count"], np.int8).tobytes() + np.asarray(tab["cps"], np.float32).tobytes()
        b += np.asarray(aa, np.int8).tobytes() + to_chars(ids, tab)
        (d / f"eval_{name}.job").write_bytes(b)
        np.savez(d / f"eval_{name}.in.npz", aa=aa, ids=ids, custom=custom,
                 **{f"tab_{k}": np.asarray(v) for k, v in tab.items()})
        meta["eval"].append(name)
    for name, N, obj, ext in select_cases(pe, orc):
        p = 3
        b = bytearray(b"PEH1") + struct.pack("<iii", 2, N, p) + np.asarray(ext, np.float32).tobytes()
        b += np.asarray(obj, np.float32).tobytes()
        (d / f"select_{name}.job").write_bytes(b)
        np.savez(d / f"select_{name}.in.npz", N=N, p=p, obj=obj, ext=ext)
        meta["select"].append(name)
    for M, p in DD_CASES:
        (d / f"dd_{M}_{p}.job").write_bytes(b"PEH1" + struct.pack("<iii", 3, M, p))
        meta["dd"].append([M, p])
    (d / "meta.json").write_text(json.dumps(meta))
    print("jobs written to", d)


def cmd_run(d: Path):
    rc = 0
    for job in sorted(d.glob("*.job")):
        out = job.with_suffix(".out")
        r = subprocess.run([str(HARNESS), str(job), str(out)], capture_output=True, text=True, timeout=600)
        print(job.name, "rc", r.returncode, r.stderr.strip()[:200])
        rc |= r.returncode
    sys.exit(rc)


def cmd_collect(d: Path):
    meta = json.loads((d / "meta.json").read_text())
    for name in meta["eval"]:
        inp = dict(np.load(d / f"eval_{name}.in.npz"))
        raw = (d / f"eval_{name}.job").read_bytes()
        n = inp["ids"].shape[0]
        rec = np.dtype([("obj", "<f4", 6), ("objidx", "i1", 12), ("pql", "<i4", 3), ("slw", "<i4")])
        out = np.frombuffer((d / f"eval_{name}.out").read_bytes(), rec, count=n)
        np.savez_compressed(GOLDEN / f"ref_eval_{name}.npz", **inp, ref_obj=out["obj"], ref_objidx=out["objidx"],
                            ref_pql=out["pql"], ref_slw=out["slw"])
        del raw
    for name in meta["select"]:
        inp = dict(np.load(d / f"select_{name}.in.npz"))
        N, p = int(inp["N"]), int(inp["p"])
        N2 = 2 * N
        from math import comb
        R = comb(6 + p - 1, p)
        raw = np.frombuffer((d / f"select_{name}.out").read_bytes(), np.uint8)
        o = 0

        def take(dt, cnt):
            nonlocal o
            a = np.frombuffer(raw[o:o + np.dtype(dt).itemsize * cnt].tobytes(), dt)
            o += np.dtype(dt).itemsize * cnt
            return a
        flags = take("<i4", 4)
        rcount = take("<i4", N2)
        srt = take("<i4", N2)
        ideal, worst, nadir = take("<f4", 6), take("<f4", 6), take("<f4", 6)
        ext = take("<f4", 36)
        dist = take("<f4", N2)
        inc = take("<i4", R)
        np.savez_compressed(GOLDEN / f"ref_select_{name}.npz", **inp, ref_flags=flags, ref_front_count=rcount,
                            ref_sorted=srt, ref_ideal=ideal, ref_worst=worst, ref_nadir=nadir, ref_ext=ext,
                            ref_dist=dist, ref_included=inc)
    dd = {}
    for M, p in meta["dd"]:
        raw = (d / f"dd_{M}_{p}.out").read_bytes()
        R = struct.unpack("<i", raw[:4])[0]
        dd[f"M{M}_p{p}"] = np.frombuffer(raw[4:], "<f4").reshape(R, M)
    np.savez_compressed(GOLDEN / "ref_das_dennis.npz", **dd)
    print("fixtures written to", GOLDEN)


if __name__ == "__main__":
    cmd, d = sys.argv[1], Path(sys.argv[2])
    {"jobs": cmd_jobs, "run": cmd_run, "collect": cmd_collect}[cmd](d)
