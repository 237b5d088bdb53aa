"""The longest repeated/common substring flavour of the string objective (LRCS) on
the GPU against the oracle, bit for bit: values, CDS pairs and (p, q, length).

The reference only names this objective (MLRCS, src/auto_execution_experiments.py:
45, 215), so its parity is pinned to the oracle's own definition (checked against
a dynamic-programming restatement in test_oracle_lrcs.py).  Cases: random
synonymous designs (long cross-CDS runs on the aligned diagonal), identical CDSs
(a common substring of the whole CDS), low-complexity proteins (self repeats
everywhere), designs short enough that no run reaches 8 (the exact word scan),
planted repeats at the CDS ends, and whole runs where children keep their
parents' pair results."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def rand_ids(rng, aa, tab, m, n):
    ids = np.zeros((n, m, len(aa)), np.uint8)
    for i in range(n):
        for c in range(m):
            ids[i, c] = tab["start"][aa] + (rng.random(len(aa)) * tab["count"][aa]).astype(np.int64)
    return ids


def same(a, b):
    a, b = np.asarray(a), np.asarray(b)
    if a.dtype.kind == "f":
        return np.array_equal(a.view(np.uint32), b.view(np.uint32))
    return np.array_equal(a, b)


def check_eval(pe, orc, aa, tabc, ids, objset=1):
    m = ids.shape[1]
    tab = tabc.arrays()
    o = orc.Problem(aa, tab, m, 8, 0.05, objset=objset, p=2, slkind=1).evaluate(ids)
    for method in (0, 1):  # seeded word table, band scan
        with pe.Engine(aa, tabc, m, 8, 0.05, objectives=objset, ref_p=2, sl_kind=pe.SL_LRCS) as eng:
            eng.set_scan_method(method)
            g = eng.evaluate(ids)
        for what, a, b in zip(("obj", "objidx", "pql"), g, o):
            ok = np.all((a == b) if a.dtype.kind != "f" else (a.view(np.uint32) == b.view(np.uint32)), axis=1)
            bad = np.flatnonzero(~ok)
            assert len(bad) == 0, (f"scan method {method}, {what} differs for solutions {bad[:5]}: "
                                   f"gpu {a[bad[0]]} oracle {b[bad[0]]}")


@pytest.mark.parametrize("L,m,n", [(201, 2, 64), (120, 4, 48), (1001, 8, 6), (33, 10, 32), (12, 3, 48), (5, 2, 32)])
def test_lrcs_random_designs(pe, orc, gpu, L, m, n):
    tabc = pe.dirichlet_table(L + m)
    tab = tabc.arrays()
    aa = pe.synthetic_protein(L - 1, 7 * L + m)
    rng = np.random.default_rng(L * 31 + m)
    ids = rand_ids(rng, aa, tab, m, n)
    ids[0] = tab["start"][aa] + tab["count"][aa] - 1      # every CDS the same: the common run is the whole CDS
    ids[1, 1] = ids[1, 0]                                  # two identical CDSs
    check_eval(pe, orc, aa, tabc, ids)


def test_lrcs_low_complexity_and_planted_ends(pe, orc, gpu):
    tabc = pe.dirichlet_table(5)
    tab = tabc.arrays()
    K, F, M_, W_ = (pe.AMINO.index(x) for x in "KFMW")
    # one-codon amino acids only (M, W): every CDS is the same and self-repeats are periodic
    aa = np.array([M_, W_] * 40 + [20], np.int8)
    rng = np.random.default_rng(3)
    check_eval(pe, orc, aa, tabc, rand_ids(rng, aa, tab, 3, 16))
    # two-letter protein (K/F): long self repeats on many diagonals
    aa = np.array(([K] * 7 + [F] * 5) * 30 + [20], np.int8)
    ids = rand_ids(rng, aa, tab, 4, 24)
    # plant the first 40 codons of CDS 0 at the end of CDS 3 in some solutions
    for i in range(0, 24, 3):
        ids[i, 3, -41:-1] = ids[i, 0, :40]
    check_eval(pe, orc, aa, tabc, ids)


def test_lrcs_reference_six_objectives(pe, orc, ref_table, gpu):
    tab = ref_table.arrays()
    aa = pe.synthetic_protein(150, 11)
    rng = np.random.default_rng(11)
    check_eval(pe, orc, aa, ref_table, rand_ids(rng, aa, tab, 5, 40), objset=0)


def test_lrcs_long_sequence_shape(pe, orc, gpu):
    """L = 3000 amino acids (9003 nucleotides per CDS), m = 4: the long-sequence
    configuration's CDS length, a few solutions."""
    tabc = pe.dirichlet_table(3)
    tab = tabc.arrays()
    aa = pe.synthetic_protein(3000, 3)
    rng = np.random.default_rng(3)
    ids = rand_ids(rng, aa, tab, 4, 3)
    ids[2, 3] = ids[2, 1]
    check_eval(pe, orc, aa, tabc, ids)


@pytest.mark.parametrize("L,m,N,G,objset", [(61, 3, 32, 8, 1), (150, 4, 48, 6, 1), (90, 5, 40, 5, 0)])
def test_lrcs_whole_run_bit_exact(pe, orc, ref_table, gpu, L, m, N, G, objset):
    tabc = ref_table if objset == 0 else pe.dirichlet_table(L)
    tab = tabc.arrays()
    aa = pe.synthetic_protein(L - 1, 500 + L)
    seed = 0xBEEF + L
    # a high mutation probability so the LRCS operator changes codons often
    with pe.Engine(aa, tabc, m, N, 0.3, objectives=objset, ref_p=3, seed=seed, sl_kind=pe.SL_LRCS) as eng:
        run = orc.Run(orc.Problem(aa, tab, m, N, 0.3, objset=objset, p=3, seed=seed, slkind=1))
        eng.init()
        run.init()
        for g in range(G + 1):
            gs = eng.population()
            os_ = run.state()
            for k, what in enumerate(("codons", "obj", "objidx", "pql", "survivors")):
                assert same(gs[k], os_[k]), f"generation {g}: {what} differ"
            if g < G:
                eng.step(1)
                run.generation()
        run.close()


def test_lrcs_incremental_pairs_equal_full_evaluation(pe, gpu):
    """After some generations (children reuse their parents' pair results), every
    solution re-evaluated from scratch gives the same objectives."""
    tabc = pe.dirichlet_table(8)
    aa = pe.synthetic_protein(400, 8)
    with pe.Engine(aa, tabc, 6, 64, 0.02, objectives=1, ref_p=3, seed=8, sl_kind=pe.SL_LRCS) as eng:
        eng.init()
        eng.step(7)
        ids, obj, objidx, pql, _ = eng.population()
        o2, i2, p2 = eng.evaluate(ids)
    assert same(obj, o2) and same(objidx, i2) and same(pql, p2)


def test_scan_cells_count_the_scans(pe, gpu):
    tabc = pe.dirichlet_table(2)
    aa = pe.synthetic_protein(120, 2)
    n = 3 * len(aa)
    with pe.Engine(aa, tabc, 3, 32, 0.05, objectives=1, ref_p=3, seed=2) as eng:
        eng.init()
        eng.step(3)
        assert eng.scan_cells() == eng.scan_count() * (n - 5) * (n - 4) // 2
    with pe.Engine(aa, tabc, 3, 32, 0.05, objectives=1, ref_p=3, seed=2, sl_kind=pe.SL_LRCS, sl_threads=128) as eng:
        eng.init()
        # the initial population scans every pair: 3 self pairs and 3 cross pairs per solution
        assert eng.scan_count() == 32 * 6
        assert eng.scan_cells() == 32 * (3 * n * (n - 1) // 2 + 3 * n * n)
