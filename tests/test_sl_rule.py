"""The closed-form hairpin-stem rule used by the CUDA scan, against the oracle's
literal single-thread transcription of calMaximumSL (include/utils.cuh:712-888).

Rule: per CDS, the longest run of pairing cells over the counted cells
r in [max(0, d-n+1), floor((d-5)/2)] of every anti-diagonal d; the solution's
stem is the largest CDS index reaching the maximum L, on its smallest such d;
there (p, q) is the outermost stem of exactly L pairs closed on both sides,
else the run cut at the loop limit."""
import numpy as np
import pytest


def rule(cds_nt):
    res = []
    for s in cds_nt:
        n = len(s)
        best, bestd = 0, 1 << 30
        for d in range(2 * n - 1):
            rlo, rhi = max(0, d - (n - 1)), (d - 5) // 2
            run = db = 0
            for r in range(rlo, rhi + 1):
                run = run + 1 if (s[r] ^ s[d - r]) == 3 else 0
                db = max(db, run)
            if db > best or (db == best and d < bestd):
                best, bestd = db, d
        res.append((best, bestd))
    Lb, cb, d = -1, 0, 0
    for c, (b, dd) in enumerate(res):
        if b >= Lb:
            Lb, cb, d = b, c, dd
    if Lb <= 0:
        return 0, 0, 0, 0
    s = cds_nt[cb]
    n = len(s)
    rlo, rhi = max(0, d - (n - 1)), (d - 5) // 2
    run, first, cut = 0, -1, False
    for r in range(rlo, rhi + 2):
        on = (s[r] ^ s[d - r]) == 3
        if r <= rhi:
            if on:
                run += 1
            else:
                if run == Lb and first < 0:
                    first = r - run
                run = 0
        elif run == Lb:
            if not on and first < 0:
                first = r - run
            cut = cut or on
    if first >= 0:
        return Lb, first, d - (first + Lb - 1), cb
    assert cut
    return Lb, rhi - Lb + 1, d - rhi, cb


@pytest.mark.parametrize("seed", range(6))
def test_rule_matches_serial_sweep(pe, orc, seed):
    rng = np.random.default_rng(seed)
    tab = pe.dirichlet_table(seed + 3).arrays()
    for trial in range(60):
        L = int(rng.integers(3, 22))
        m = int(rng.integers(2, 4))
        aa = pe.synthetic_protein(L - 1, int(rng.integers(1 << 30)))
        ids = np.stack([tab["start"][aa] + (rng.random(L) * tab["count"][aa]).astype(np.int64) for _ in range(m)])
        if trial % 3 == 0:
            ids[1] = ids[0]
        prob = orc.Problem(aa, tab, m, 4, 0.05, objset=1)
        obj, objidx, pql = prob.evaluate(ids[None].astype(np.uint8))
        nt = [np.asarray(tab["nt"])[ids[c]].reshape(-1) for c in range(m)]
        got = (int(pql[0, 2]), int(pql[0, 0]), int(pql[0, 1]), int(objidx[0, 6]))
        assert rule(nt) == got
