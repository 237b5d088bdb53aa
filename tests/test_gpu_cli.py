"""The command line (`lib/pe_nsga3`, the reference's `Protein_NSGA3 <fasta> <N> <G> <m> <Pm>`
surface): FASTA in, Result.txt and the normalised-objective file out, in the
reference's formats (src/main.cu:491-523, 789-858), with the same populations as
the library run with the same seed."""
import subprocess

import numpy as np
import pytest

from conftest import ROOT

pytestmark = pytest.mark.gpu

IDEAL4, NADIR4 = np.array([1.0, 0.4, 0.0, 0.0], np.float32), np.array([0.0, 0.0, 0.6, 1.0], np.float32)


def test_cli_matches_library(pe, gpu, tmp_path):
    L, N, G, m, pm, seed = 60, 32, 10, 2, 0.05, 5
    aa = pe.synthetic_protein(L, 77)
    fasta = tmp_path / "p.fasta"
    letters = "".join(pe.AMINO[i] for i in aa[:-1])
    fasta.write_text(">sp|TEST|synthetic\n" + "\n".join(letters[k:k + 60] for k in range(0, L, 60)) + "\n")
    assert np.array_equal(pe.parse_fasta(fasta), aa)
    cli = ROOT / "protein_encoding_v2_nsga-iii_b200" / "lib" / "pe_nsga3"
    out = subprocess.run([str(cli), str(fasta), str(N), str(G), str(m), str(pm), "--seed", str(seed),
                          "--objectives", "base4", "--dirichlet", str(seed), "--out", str(tmp_path)],
                         capture_output=True, text=True, timeout=120)
    assert out.returncode == 0, out.stderr
    tab = pe.dirichlet_table(seed)
    with pe.Engine(aa, tab, m, N, pm, objectives=pe.OBJ_BASE4, seed=seed) as e:
        e.init()
        e.step(G)
        ids, obj, objidx, _, _ = e.population()
    codons = tab.codon_strings()
    names = ["mCAI", "mHD", "MGC", "MSL"]
    pos = obj.copy()
    pos[:, :2] *= -1.0
    lines = []
    for i in range(2 * N):
        lines.append(f"{i + 1} Solutions")
        for j in range(m):
            lines.append(f"{j + 1} CDS : " + "".join(codons[c] for c in ids[i, j]))
        lines.append("")
        lines.append(f" {i + 1} Solution")
        for k, nm in enumerate(names):
            ix = objidx[i, 2 * k:2 * k + 2]
            pre = f"{ix[0]} {ix[1]}" if nm == "mHD" else f"{ix[0]}"
            lines.append(f"{pre}\t{nm} : {float(pos[i, k]):f}")
    assert (tmp_path / "Result.txt").read_text() == "\n".join(lines) + "\n"
    norm = (pos - IDEAL4) / (NADIR4 - IDEAL4)
    norm = np.where(norm >= 1.0, np.float32(0.999999), norm)
    norm = np.where(norm < 0.0, np.float32(0.0), norm).astype(np.float32)
    got = np.loadtxt(tmp_path / "Normalized_value_quality_computation.txt")
    assert got.shape == (2 * N, 4) and np.allclose(got, norm, atol=1e-6)
    hv = pe.hypervolume(norm.astype(np.float64), np.ones(4))
    line = [x for x in out.stdout.splitlines() if x.startswith("Hypervolume")][0]
    assert abs(float(line.split(":")[1]) - hv) < 1e-6
