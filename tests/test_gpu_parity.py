"""CUDA engine vs the CPU oracle, through the C ABI.  Integer/index outputs and
every float are compared bit for bit: the engine and the oracle execute the same
IEEE operations in the same order (fixed-point log sums for CAI, --fmad=false)."""
import numpy as np
import pytest

from conftest import ROOT

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


EVAL_CASES = [
    # name, L (incl. stop), m, n, objset, gcmode, table
    ("ref6_L40_m3", 40, 3, 64, 0, 0, "ref"),
    ("base4_L201_m2", 201, 2, 96, 1, 0, "dir"),
    ("base4_gcall_L120_m4", 120, 4, 64, 1, 1, "dir"),
    ("ref6_L1001_m8", 1001, 8, 6, 0, 0, "ref"),
    ("ref6_tiny3", 3, 2, 48, 0, 0, "ref"),
    ("ref6_tiny4", 4, 3, 48, 0, 0, "ref"),
    ("base4_tiny6", 6, 2, 48, 1, 0, "dir"),
    ("base4_L33_m10", 33, 10, 64, 1, 0, "dir"),
]


def tables(pe, which, ref_table):
    return ref_table if which == "ref" else pe.dirichlet_table(17)


@pytest.mark.parametrize("name,L,m,n,objset,gcmode,tabname", EVAL_CASES)
def test_evaluators_match_oracle(pe, orc, ref_table, gpu, name, L, m, n, objset, gcmode, tabname):
    tabc = tables(pe, tabname, ref_table)
    tab = tabc.arrays()
    rng = np.random.default_rng(abs(hash(name)) % (1 << 31))
    aa = pe.synthetic_protein(L - 1, L * 7 + m)
    ids = rand_ids(rng, aa, tab, m, n)
    ids[0] = tab["start"][aa] + tab["count"][aa] - 1      # highest-weight codons
    ids[1, 1] = ids[1, 0]                                  # duplicate CDS: ties everywhere
    with pe.Engine(aa, tabc, m, 8, 0.05, objectives=objset, gc_mode=gcmode, ref_p=2) as eng:
        g = eng.evaluate(ids)
    o = orc.Problem(aa, tab, m, 8, 0.05, objset=objset, gcmode=gcmode, p=2).evaluate(ids)
    for what, a, b in zip(("obj", "objidx", "pql"), g, o):
        bad = np.flatnonzero(~np.all((a == b) if a.dtype.kind != "f" else (a.view(np.uint32) == b.view(np.uint32)),
                                     axis=1))
        assert len(bad) == 0, f"{what} differs for solutions {bad[:5]}: gpu {a[bad[0]]} oracle {b[bad[0]]}"


def test_hairpin_stems_long_and_absent(pe, orc, gpu):
    """Solutions with long designed stems and with no pairing at all."""
    tabc = pe.dirichlet_table(23)
    tab = tabc.arrays()
    # protein of K (AAA/AAG) and F (UUU/UUC): A-U pairing only; plus stop
    Kidx, Fidx = pe.AMINO.index("K"), pe.AMINO.index("F")
    aa = np.array([Kidx] * 30 + [Fidx] * 30 + [20], np.int8)
    rng = np.random.default_rng(5)
    ids = rand_ids(rng, aa, tab, 2, 32)
    aa2 = np.array([Kidx] * 25 + [20], np.int8)   # only A/G: no complementary pair except stop codon bases
    ids2 = rand_ids(rng, aa2, tab, 3, 32)
    for a, x in ((aa, ids), (aa2, ids2)):
        m = x.shape[1]
        with pe.Engine(a, tabc, m, 8, 0.05, objectives=1, ref_p=2) as eng:
            g = eng.evaluate(x)
        o = orc.Problem(a, tab, m, 8, 0.05, objset=1, p=2).evaluate(x)
        for u, v in zip(g, o):
            assert same(u, v)


@pytest.mark.parametrize("objset,gen,pm", [(0, 0, 0.3), (0, 1, 0.3), (1, 5, 0.3), (1, 2, 1.0), (0, 3, 0.0)])
def test_mutation_matches_oracle(pe, orc, ref_table, gpu, objset, gen, pm):
    tabc = ref_table if objset == 0 else pe.dirichlet_table(31)
    tab = tabc.arrays()
    L, m, n = 90, 4, 300
    rng = np.random.default_rng(gen * 13 + objset)
    aa = pe.synthetic_protein(L - 1, 77 + gen)
    ids = rand_ids(rng, aa, tab, m, n)
    prob = orc.Problem(aa, tab, m, 8, pm, objset=objset, p=2)
    pobj, pobjidx, ppql = prob.evaluate(ids)
    idx = (np.arange(n) * 7 + 3).astype(np.int32)
    with pe.Engine(aa, tabc, m, 8, pm, objectives=objset, ref_p=2) as eng:
        gc, gops = eng.mutate(gen, idx, ids, pobj, pobjidx, ppql)
    oc, oops, _, _, _ = prob.mutate(gen, idx, ids, pobj, pobjidx, ppql)
    assert np.array_equal(gops, oops)
    assert np.array_equal(gc, oc)
    # every child stays a synonymous encoding of the protein
    aa_of = np.repeat(np.arange(21), tab["count"])
    assert (aa_of[gc] == aa[None, None, :]).all()
    assert len(set(gops.tolist())) == (7 if objset == 0 else 5)


def select_inputs(rng, N, M):
    obj = rng.random((2 * N, M)).astype(np.float32)
    obj[5:15] = obj[20:30]                                 # duplicates
    obj[40:44, 0] = obj[45, 0] + np.float32(5e-7)          # inside the 1e-6 equality band
    obj[50:54, 1] = obj[55, 1] + np.float32(2e-6)          # just outside
    return obj


@pytest.mark.parametrize("N,M,p", [(32, 4, 4), (64, 4, 6), (100, 6, 3), (512, 4, 8), (1024, 4, 8),
                                   (2048, 6, 0), (4096, 4, 0)])
def test_selection_matches_oracle(pe, orc, gpu, N, M, p):
    objset = 0 if M == 6 else 1
    tabc = pe.dirichlet_table(3)
    aa = pe.synthetic_protein(20, 1)
    rng = np.random.default_rng(N + M)
    for trial in range(3):
        obj = select_inputs(rng, N, M)
        if trial == 2:
            obj = np.round(obj * 4) / 4                    # many fronts, many ties
        ext = obj[:M].copy()
        with pe.Engine(aa, tabc, 2, N, 0.05, objectives=objset, ref_p=p) as eng:
            gs, gf, ge, gi = eng.select(9 + trial, obj, ext)
        os_, of, oe, oi = orc.Problem(aa, tabc.arrays(), 2, N, 0.05, objset=objset, p=p).select(9 + trial, obj, ext)
        assert np.array_equal(gf, of), "front assignment"
        assert (gi.rank_count, gi.last_front_size, gi.n_fronts, gi.cut, gi.hyp_exception) == \
            (oi.rank_count, oi.last_front_size, oi.n_fronts, oi.cut, oi.hyp_exception)
        assert same(ge, oe), "extreme points"
        for k in range(M):
            assert same(np.float32(gi.nadir[k]), np.float32(oi.nadir[k]))
        assert np.array_equal(gs, os_), "survivors"
        assert len(set(gs.tolist())) == N


RUNS = [
    # name, L incl stop, m, N, G, objset, table, p
    ("base4_L201_m2_N128", 201, 2, 128, 12, 1, "dir", 6),
    ("ref6_L39_m3_N64", 39, 3, 64, 12, 0, "ref", 0),
    ("base4_L61_m5_N50", 61, 5, 50, 12, 1, "dir", 0),
]


@pytest.mark.parametrize("name,L,m,N,G,objset,tabname,p", RUNS)
def test_whole_run_bit_exact(pe, orc, ref_table, gpu, name, L, m, N, G, objset, tabname, p):
    tabc = tables(pe, tabname, ref_table)
    tab = tabc.arrays()
    aa = pe.synthetic_protein(L - 1, 1000 + L)
    seed = 0xC0FFEE + L
    with pe.Engine(aa, tabc, m, N, 0.05, objectives=objset, ref_p=p, seed=seed) as eng:
        run = orc.Run(orc.Problem(aa, tab, m, N, 0.05, objset=objset, p=p, seed=seed))
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


def test_full_size_generation(pe, orc, gpu):
    """L=1000, m=8, N=1024, p=8: determinism, validity, and oracle checks on sampled offspring."""
    tabc = pe.dirichlet_table(1)
    tab = tabc.arrays()
    aa = pe.synthetic_protein(1000, 42)
    pops = []
    for rep in range(2):
        with pe.Engine(aa, tabc, 8, 1024, 0.02, objectives=1, ref_p=8, seed=99) as eng:
            eng.init()
            eng.step(3)
            pops.append(eng.population())
    for k in range(5):
        assert same(pops[0][k], pops[1][k])
    ids, obj, objidx, pql, surv = pops[0]
    aa_of = np.repeat(np.arange(21), tab["count"])
    assert (aa_of[ids] == aa[None, None, :]).all()
    assert len(set(surv.tolist())) == 1024
    prob = orc.Problem(aa, tab, 8, 1024, 0.02, objset=1, p=8)
    pick = np.array([1024, 1500, 2047])
    o = prob.evaluate(ids[pick])
    for a, b in zip((obj[pick], objidx[pick], pql[pick]), o):
        assert same(a, b)


def test_unchanged_cds_keeps_parent_stem(pe, orc, gpu):
    """A child's CDS that its mutation left unchanged keeps its parent's stem result
    instead of being scanned again: fewer scans than CDSs, and every solution's
    objectives still equal a fresh evaluation by the oracle."""
    tabc = pe.dirichlet_table(6)
    tab = tabc.arrays()
    aa = pe.synthetic_protein(119, 8)
    N, m, G = 64, 8, 6
    with pe.Engine(aa, tabc, m, N, 0.02, objectives=1, ref_p=4, seed=11, sl_threads=128) as eng:
        eng.init()
        assert eng.scan_count() == N * m
        eng.step(G)
        per_gen = (eng.scan_count() - N * m) / G
        ids, obj, objidx, pql, surv = eng.population()
    assert 0 < per_gen < 0.7 * N * m
    o = orc.Problem(aa, tab, m, N, 0.02, objset=1, p=4).evaluate(ids)
    for a, b in zip((obj, objidx, pql), o):
        assert same(a, b)


def test_long_protein_large_population_fits(pe, gpu):
    """L=3000, m=4, N=4096 with the reference's p rule (4060 reference points): the
    selection and stem-scan kernels' shared memory still fits one CTA, and a
    generation keeps N distinct survivors."""
    tabc = pe.dirichlet_table(4)
    aa = pe.synthetic_protein(3000, 5)
    with pe.Engine(aa, tabc, 4, 4096, 0.02, objectives=1, ref_p=0, seed=3) as eng:
        assert eng.R == 4060
        eng.init()
        eng.step(2)
        surv = eng.population()[4]
        assert len(set(surv.tolist())) == 4096


def test_population_of_one_and_errors(pe, gpu):
    tabc = pe.dirichlet_table(2)
    aa = pe.synthetic_protein(30, 3)
    with pe.Engine(aa, tabc, 2, 1, 0.1, objectives=1, ref_p=1) as eng:
        eng.init()
        eng.step(3)
        ids, obj, _, _, surv = eng.population()
        assert surv.tolist() in ([0], [1])
    with pytest.raises(pe.PeError):
        pe.Engine(aa, tabc, 2, 2, 0.1, objectives=1, ref_p=0)   # reference rule needs N >= M
    with pytest.raises(pe.PeError):
        pe.Engine(aa, tabc, 1, 8, 0.1)                            # m must be >= 2
    with pytest.raises(pe.PeError):
        pe.Engine(aa[:2], tabc, 2, 8, 0.1)                        # too short
    with pe.Engine(aa, tabc, 2, 8, 0.1, objectives=1) as eng:
        with pytest.raises(pe.PeError) as e:
            eng.step(1)                                           # before init
        assert e.value.code == 5
