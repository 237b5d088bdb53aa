"""The string scan's two first passes give the same runs.

The seeded pass looks up T's 8-nucleotide words in a table and measures only the
runs that start at an equal word; the band scan visits every counted cell.  Whole
runs with each must be identical bit for bit (populations, objectives, stems), on
random-like proteins, where the seeded pass decides every CDS, and on
low-complexity ones, where its table chains grow long and it hands CDSs to the
band scan (counted by pe_scan_fallbacks)."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def run(pe, aa, tab, m, N, gens, kind, method, seed):
    with pe.Engine(aa, tab, m, N, 0.05, objectives=1, seed=seed, sl_kind=kind) as eng:
        eng.set_scan_method(method)
        eng.init()
        eng.step(gens)
        return eng.population(), eng.scan_count(), eng.scan_fallbacks()


def assert_same(a, b):
    for k, (u, v) in enumerate(zip(a, b)):
        u, v = np.asarray(u), np.asarray(v)
        if u.dtype.kind == "f":
            u, v = u.view(np.uint32), v.view(np.uint32)
        assert np.array_equal(u, v), f"population field {k} differs"


@pytest.mark.parametrize("kind", ["hairpin", "lrcs"])
@pytest.mark.parametrize("L,m,N", [(400, 3, 32), (1000, 2, 16), (90, 4, 32)])
def test_random_protein_seeded_equals_band(pe, gpu, kind, L, m, N):
    k = pe.SL_HAIRPIN if kind == "hairpin" else pe.SL_LRCS
    aa = pe.synthetic_protein(L, 40 + L)
    tab = pe.dirichlet_table(L + m)
    pop0, scans0, fb0 = run(pe, aa, tab, m, N, 6, k, 0, 5)
    pop1, scans1, fb1 = run(pe, aa, tab, m, N, 6, k, 1, 5)
    assert_same(pop0, pop1)
    assert scans0 == scans1 > 0
    assert fb0 == 0           # random-like CDSs: short chains, no hand-over
    assert fb1 == 0           # the band scan alone never counts one


@pytest.mark.parametrize("kind", ["hairpin", "lrcs"])
def test_low_complexity_equal(pe, gpu, kind):
    """K/F proteins (codons AAA/AAG, UUU/UUC): few distinct words, long chains."""
    k = pe.SL_HAIRPIN if kind == "hairpin" else pe.SL_LRCS
    K, F = pe.AMINO.index("K"), pe.AMINO.index("F")
    rng = np.random.default_rng(8)
    aa = np.append(rng.choice([K, F], 500).astype(np.int8), np.int8(20))
    tab = pe.dirichlet_table(9)
    pop0, scans0, fb0 = run(pe, aa, tab, 3, 32, 4, k, 0, 6)
    pop1, scans1, fb1 = run(pe, aa, tab, 3, 32, 4, k, 1, 6)
    assert_same(pop0, pop1)
    assert scans0 == scans1 and fb0 <= scans0 and fb1 == 0


def test_one_codon_protein_hands_over(pe, gpu):
    """M/W only (one codon each): every CDS is the same, so each LRCS pair's words
    repeat every 6 nucleotides and every chain holds a sixth of the CDS: the seeded
    pass gives up on every scan and the band scan answers."""
    M_, W_ = pe.AMINO.index("M"), pe.AMINO.index("W")
    aa = np.array([M_, W_] * 200 + [20], np.int8)
    tab = pe.dirichlet_table(4)
    pop0, scans0, fb0 = run(pe, aa, tab, 3, 16, 3, pe.SL_LRCS, 0, 2)
    pop1, scans1, fb1 = run(pe, aa, tab, 3, 16, 3, pe.SL_LRCS, 1, 2)
    assert_same(pop0, pop1)
    assert scans0 == scans1 and fb0 == scans0 > 0 and fb1 == 0


def test_scan_method_argument(pe, gpu):
    aa = pe.synthetic_protein(60, 3)
    with pe.Engine(aa, pe.dirichlet_table(3), 2, 16, 0.05, objectives=1) as eng:
        with pytest.raises(pe.PeError):
            eng.set_scan_method(2)
        eng.set_scan_method(1)
        eng.set_scan_method(0)
