"""Longest-stem objective (calMaximumSL, include/utils.cuh:712-888) on long and
structured CDSs: the engine's two-pass scan against the oracle's serial
anti-diagonal sweep, bit for bit (value, CDS index, p, q, length)."""
import numpy as np
import pytest

from test_gpu_parity import rand_ids, same

pytestmark = pytest.mark.gpu


def check(pe, orc, aa, tabc, ids):
    """Both first passes (seeded word table, band scan) against the oracle; returns the
    engine's result and the seeded run's hand-overs to the band scan."""
    tab = tabc.arrays()
    m = ids.shape[1]
    o = orc.Problem(aa, tab, m, 8, 0.05, objset=1, p=2).evaluate(ids)
    handed = []
    for method in (0, 1):
        with pe.Engine(aa, tabc, m, 8, 0.05, objectives=1, ref_p=2) as eng:
            eng.set_scan_method(method)
            g = eng.evaluate(ids)
            handed.append(eng.scan_fallbacks())
        for what, u, v in zip(("obj", "objidx", "pql"), g, o):
            assert same(u, v), f"scan method {method}, {what}: gpu {u[:4]} oracle {v[:4]}"
    assert handed[1] == 0
    return g, handed[0]


@pytest.mark.parametrize("L,m,n", [(51, 3, 16), (151, 2, 12), (400, 3, 6), (1001, 8, 3), (2001, 2, 2), (3334, 2, 1)])
def test_random_cds(pe, orc, gpu, L, m, n):
    tabc = pe.dirichlet_table(L)
    aa = pe.synthetic_protein(L - 1, 1000 + L)
    ids = rand_ids(np.random.default_rng(L), aa, tabc.arrays(), m, n)
    g, handed = check(pe, orc, aa, tabc, ids)
    if L >= 400:
        assert (g[2][:, 2] >= 8).all()      # the first pass decides these
    assert handed == 0                      # random-like CDSs: the seeded pass never gives up


def test_long_perfect_hairpin(pe, orc, gpu):
    """AAA..A UUU..U: one stem of about half the CDS (runs far past 32 rows and
    across many segments), next to solutions with shorter designed stems."""
    tabc = pe.dirichlet_table(3)
    tab = tabc.arrays()
    K, F = pe.AMINO.index("K"), pe.AMINO.index("F")
    aa = np.array([K] * 300 + [F] * 300 + [20], np.int8)
    nt = tab["nt"]
    aaa = [c for c in range(64) if list(nt[c]) == [0, 0, 0]][0]
    uuu = [c for c in range(64) if list(nt[c]) == [3, 3, 3]][0]
    ids = rand_ids(np.random.default_rng(9), aa, tab, 3, 6)
    ids[0, 0, :300], ids[0, 0, 300:600] = aaa, uuu
    ids[1, 2, 100:300], ids[1, 2, 300:500] = aaa, uuu
    ids[2, 1, 290:300], ids[2, 1, 300:310] = aaa, uuu
    g, handed = check(pe, orc, aa, tabc, ids)
    assert g[2][0, 2] > 800
    assert handed > 0                       # the AAA..A UUU..U CDSs: long chains, band scan


def test_low_complexity_many_runs(pe, orc, gpu):
    """Only A/U/G codons from K and F: runs of >= 8 pairs everywhere, so most
    rows take the exact path."""
    tabc = pe.dirichlet_table(5)
    K, F = pe.AMINO.index("K"), pe.AMINO.index("F")
    rng = np.random.default_rng(4)
    aa = np.append(rng.choice([K, F], 700).astype(np.int8), np.int8(20))
    ids = rand_ids(rng, aa, tabc.arrays(), 4, 4)
    check(pe, orc, aa, tabc, ids)


def test_stem_near_every_edge(pe, orc, gpu):
    """Designed stems of length 8..12 at the start, the end and the middle of
    the CDS and at the loop limit: first and last bands, first rows, the
    hypotenuse of the counted triangle."""
    tabc = pe.dirichlet_table(6)
    tab = tabc.arrays()
    K, F = pe.AMINO.index("K"), pe.AMINO.index("F")
    E = pe.AMINO.index("E")                                 # K, E: purine codons, nothing pairs
    rng = np.random.default_rng(8)
    base = rng.choice([K, E], 500).astype(np.int8)
    nt = tab["nt"]
    aaa = [c for c in range(64) if list(nt[c]) == [0, 0, 0]][0]
    uuu = [c for c in range(64) if list(nt[c]) == [3, 3, 3]][0]
    cases = []
    for (i0, i1, w) in [(0, 496, 3), (0, 10, 3), (240, 245, 4), (247, 250, 2), (100, 400, 4), (490, 496, 1)]:
        aa = base.copy()
        aa[i0:i0 + w] = K
        aa[i1:i1 + w] = F                                   # a stem of 3w pairs (w = 1: none reaches 8)
        cases.append(np.append(aa, np.int8(20)))
    for aa in cases:
        ids = rand_ids(rng, aa, tab, 2, 3)
        ids[:, :, aa == K] = aaa
        ids[:, :, aa == F] = uuu
        check(pe, orc, aa, tabc, ids)


def test_cta_size_does_not_change_results(pe, gpu):
    """The hairpin-scan CTA size (forced, or picked by timing at init) changes speed only."""
    aa = pe.synthetic_protein(400, 12)
    tab = pe.dirichlet_table(12)
    pops = []
    for nt in (0, 64, 128, 256):
        with pe.Engine(aa, tab, 4, 96, 0.05, seed=12, sl_threads=nt) as e:
            e.init()
            assert e.sl_threads in (64, 128, 256) and (nt == 0 or e.sl_threads == nt)
            e.step(4)
            pops.append(e.population())
    for p in pops[1:]:
        for x, y in zip(p, pops[0]):
            assert np.array_equal(np.asarray(x).view(np.uint8), np.asarray(y).view(np.uint8))
