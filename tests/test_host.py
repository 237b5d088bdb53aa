"""Host-side pieces that need no GPU: library exports, input builders, hypervolume."""
import ctypes
import math

import numpy as np
import pytest

from conftest import GOLDEN, ROOT

B7KHU9 = "MIEPLVLGLVMGLVPITLAGLFVAAYLQYKRGNQLNLD"


def test_library_exports_every_declared_symbol(pe):
    names = pe.declared_symbols()
    assert len(names) == 43 and "pe_step" in names and "pe_batch_step" in names and "pe_hypervolume" in names and "pe_instance_bytes" in names
    lib = pe.lib()
    for n in names:
        assert hasattr(lib, n), n
    assert b"sm_100a" in lib.pe_version()


def test_cli_built():
    assert (ROOT / "protein_encoding_v2_nsga-iii_b200" / "lib" / "pe_nsga3").exists()


def test_create_without_device_fails_loudly(pe, cuda_ok):
    if cuda_ok:
        pytest.skip("a CUDA device is present")
    with pytest.raises(pe.PeError) as e:
        pe.Engine(pe.synthetic_protein(20, 1), pe.dirichlet_table(1), 2, 8, 0.05)
    assert e.value.code == 7


def write_fasta(path, seq, width=60, trailing_newline=True):
    lines = [">sp|TEST|header line"] + [seq[i:i + width] for i in range(0, len(seq), width)]
    path.write_text("\n".join(lines) + ("\n" if trailing_newline else ""))


@pytest.mark.parametrize("trailing", [True, False])
def test_fasta_loader(pe, tmp_path, trailing):
    f = tmp_path / "p.fasta"
    write_fasta(f, B7KHU9, 13, trailing)
    aa = pe.parse_fasta(f)
    assert "".join(pe.AMINO[a] for a in aa) == B7KHU9 + "Z"


def test_fasta_rejects_unknown_letters(pe, tmp_path):
    f = tmp_path / "bad.fasta"
    write_fasta(f, "MKB*X")
    with pytest.raises(pe.PeError):
        pe.parse_fasta(f)


def test_synthetic_protein(pe):
    a = pe.synthetic_protein(5000, 7)
    assert len(a) == 5001 and a[-1] == 20 and a[:-1].min() >= 0 and a[:-1].max() <= 19
    assert np.array_equal(a, pe.synthetic_protein(5000, 7))
    assert not np.array_equal(a, pe.synthetic_protein(5000, 8))
    counts = np.bincount(a[:-1], minlength=20)
    assert counts.min() > 180 and counts.max() < 330


def test_dirichlet_table(pe):
    t = pe.dirichlet_table(3).arrays()
    ref = pe.load_codon_table(ROOT / "protein_encoding_v2_nsga-iii_b200" / "data" / "ref_codon_table.txt").arrays()
    # same genetic code grouping as the reference
    assert np.array_equal(t["start"], ref["start"]) and np.array_equal(t["count"], ref["count"])
    code = lambda tab: [sorted("".join("ACGU"[b] for b in tab["nt"][tab["start"][a] + j]) for j in range(tab["count"][a]))
                        for a in range(21)]
    assert code(t) == code(ref)
    for a in range(21):
        s, k = t["start"][a], t["count"][a]
        w = t["weight"][s:s + k]
        assert w[-1] == 1.0 and (np.diff(w) >= 0).all() and (w > 0).all()
    assert not np.array_equal(t["weight"], pe.dirichlet_table(4).arrays()["weight"])


def test_reference_table_file(pe):
    t = pe.load_codon_table(ROOT / "protein_encoding_v2_nsga-iii_b200" / "data" / "ref_codon_table.txt").arrays()
    # include/info.cuh:9-10
    assert t["start"].tolist() == [0, 4, 6, 8, 10, 12, 16, 18, 21, 23, 29, 30, 32, 36, 38, 44, 50, 54, 58, 59, 61]
    assert t["count"].tolist() == [4, 2, 2, 2, 2, 4, 2, 3, 2, 6, 1, 2, 4, 2, 6, 6, 4, 4, 1, 2, 3]
    assert t["weight"][2] == np.float32(7223) / np.float32(135063.0)
    assert abs(t["ref_gc3"] - 0.381) < 1e-7 and abs(t["ref_gc"] - 0.3977) < 1e-7
    # include/info.cuh:54 (61x61 codon-pair scores; long lines must parse whole)
    cps = t["cps"]
    assert cps[:3].tolist() == [np.float32(0.007921), np.float32(0.060698), np.float32(-0.159742)]
    assert np.abs(cps).max() < 1.0 and np.count_nonzero(cps) > 3600


def test_reference_points_match_oracle(pe, orc):
    for M, p in [(4, 6), (4, 8), (6, 4), (6, 3)]:
        assert np.array_equal(pe.reference_points(M, p), orc.das_dennis(M, p))


def test_hypervolume_known_answer(pe, orc):
    # the reference's sample output; its `hv -r "1 1 1 1 1 1"` prints 0.121643
    pts = np.loadtxt(GOLDEN / "sample_normalized_N100.txt")
    hv = pe.hypervolume(pts, np.ones(6))
    assert abs(hv - 0.121643) < 5e-7
    assert abs(orc.hypervolume(pts, np.ones(6)) - hv) < 1e-12


@pytest.mark.parametrize("d", [2, 3, 4, 5])
def test_hypervolume_vs_oracle(pe, orc, d):
    rng = np.random.default_rng(d)
    for trial in range(5):
        pts = rng.random((40, d))
        pts[:5] = pts[5:10]  # duplicates
        a, b = pe.hypervolume(pts, np.ones(d)), orc.hypervolume(pts, np.ones(d))
        assert abs(a - b) < 1e-12 * max(1.0, abs(b))
    # coordinates on a coarse grid: equal x / y / z values, points on the boundary of others' boxes
    for trial in range(5):
        pts = rng.integers(0, 6, (60, d)) / 6.0
        a, b = pe.hypervolume(pts, np.ones(d)), orc.hypervolume(pts, np.ones(d))
        assert abs(a - b) < 1e-12 * max(1.0, abs(b))
    # single point and box volume
    assert abs(pe.hypervolume(np.full((1, d), 0.5), np.ones(d)) - 0.5 ** d) < 1e-15


def test_hypervolume_front_sized(pe, orc):
    # a 4-objective front of 300 mutually non-dominated points (the served stall check's shape)
    rng = np.random.default_rng(11)
    x = rng.random((300, 4))
    x /= np.linalg.norm(x, axis=1, keepdims=True) * 1.2
    a, b = pe.hypervolume(x, np.ones(4)), orc.hypervolume(x, np.ones(4))
    assert abs(a - b) < 1e-12 * b


def test_instance_bytes_host(pe):
    base = pe.instance_bytes(1001, 8, 1024, pe.OBJ_BASE4, ref_p=8)
    assert base % 512 == 0 and 30 << 20 < base < 200 << 20
    assert pe.instance_bytes(2001, 8, 1024, pe.OBJ_BASE4, ref_p=8) > base
    assert pe.instance_bytes(1001, 8, 2048, pe.OBJ_BASE4, ref_p=8) > base
    assert pe.instance_bytes(1001, 8, 1024, pe.OBJ_REF6) > base          # R = 792 reference points
    with pytest.raises(pe.PeError):
        pe.instance_bytes(2, 8, 1024)


def test_sl_threads_must_be_a_supported_size(pe):
    with pytest.raises(pe.PeError):
        pe.Engine(pe.synthetic_protein(40, 1), pe.dirichlet_table(1), 2, 8, 0.05, sl_threads=96)
