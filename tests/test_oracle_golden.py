"""The oracle against the reference's own device functions (CPU).

Fixtures tests/golden/ref_*.npz hold inputs and the outputs of the reference's
evaluators, non-dominated sort / normalisation / association and Das-Dennis
generator, produced on a B200 by oracle/ref_harness (see make_golden.py).

Tolerances: the reference builds with -use_fast_math and multiplies CAI factors
in float, so its CAI carries up to ~2L'*2^-24 relative error; counts divided by
lengths carry <= 2 ulp.  Counts themselves (hidden stops, mismatches, GC3,
stem length), argmin/argmax indices, fronts and ideal/worst values must agree
exactly."""
import math
from pathlib import Path

import numpy as np
import pytest

from conftest import GOLDEN

EVAL = sorted(GOLDEN.glob("ref_eval_*.npz"))
SELECT = sorted(GOLDEN.glob("ref_select_*.npz"))
ULP2 = 2.5e-7


def table_from(z):
    return {k[4:]: (z[k].item() if z[k].ndim == 0 else z[k]) for k in z.files if k.startswith("tab_")}


def test_fixtures_present():
    assert len(EVAL) >= 8 and len(SELECT) >= 4 and (GOLDEN / "ref_das_dennis.npz").exists()


def fp64_cai(tab, aa, ids):
    """CAI of each CDS in FP64 (product of w^(1/L'), include/utils.cuh:271-337)."""
    w = np.asarray(tab["weight"], np.float64)
    L = len(aa)
    return np.exp(np.log(w[ids]).sum(axis=-1) / L)


@pytest.mark.parametrize("path", EVAL, ids=[p.stem for p in EVAL])
def test_evaluators_vs_reference(orc, path):
    z = np.load(path)
    aa, ids = z["aa"], z["ids"]
    tab = table_from(z)
    n, m, L = ids.shape
    prob = orc.Problem(aa, tab, m, 8, 0.05, objset=0, p=1)
    obj, objidx, pql = prob.evaluate(ids)
    robj, ridx, rpql, rslw = z["ref_obj"], z["ref_objidx"], z["ref_pql"], z["ref_slw"]
    n_nt = 3 * L
    # CAI: oracle within 1e-6 of FP64; reference within its float-product error
    cai64 = fp64_cai(tab, aa, ids).min(axis=1)
    assert np.all(np.abs(-obj[:, 0] - cai64) <= 1e-6 * cai64)
    assert np.all(np.abs(obj[:, 0] - robj[:, 0]) <= 2 * L * 2 ** -24 * np.abs(robj[:, 0]) + 1e-7)
    # CBP: float sums in the reference
    assert np.all(np.abs(obj[:, 1] - robj[:, 1]) <= 1e-5 * (1 + np.abs(robj[:, 1])))
    # count-valued objectives: same counts, values within 2 ulp
    for k, den in ((2, L - 1), (3, n_nt)):
        assert np.all(np.abs(obj[:, k] - robj[:, k]) <= ULP2 * np.maximum(1e-30, np.abs(robj[:, k])) + 1e-9), k
        assert np.array_equal(np.rint(-obj[:, k] * den), np.rint(-robj[:, k] * den)), k
    # GC3 deviation |cnt/L' - 0.381|: the quotient carries the division error, so compare
    # the GC3 counts behind the values and bound the value absolutely
    ref3 = float(np.float32(tab["ref_gc3"]))
    def gc3_count(v, direction):
        return np.rint((ref3 - np.where(direction == 1, v, -v)) * L)
    assert np.array_equal(gc3_count(obj[:, 4], objidx[:, 9]), gc3_count(robj[:, 4], ridx[:, 9]))
    assert np.all(np.abs(obj[:, 4] - robj[:, 4]) <= 2.5e-7)
    # indices: CAI, CBP, HSC, HD pair, GC3 cds + direction
    for col in (0, 2, 4, 6, 7, 8, 9):
        assert np.array_equal(objidx[:, col], ridx[:, col]), col
    cbp_same = objidx[:, 2] == ridx[:, 2]
    assert cbp_same.mean() >= 0.95
    # hairpin stem: same length; the reference's (p, q, cds) is one of the maximal stems
    wrote = rslw.astype(bool)
    assert np.array_equal(pql[wrote, 2], rpql[wrote, 2])
    assert np.all(pql[~wrote, 2] == 0)
    K = (n_nt - 4) // 2
    assert np.all(np.abs(obj[wrote, 5] - robj[wrote, 5]) <= ULP2 * np.abs(robj[wrote, 5]) + 1e-9)
    nt = np.asarray(tab["nt"])
    for i in np.flatnonzero(wrote):
        p, q, l = rpql[i]
        c = ridx[i, 10]
        s = nt[ids[i, c]].reshape(-1)
        assert q - (p + l - 1) > 4
        assert all((s[p + t] ^ s[q + l - 1 - t]) == 3 for t in range(l))
    # oracle's own pick is a maximal stem too
    for i in np.flatnonzero(pql[:, 2] > 0):
        p, q, l = pql[i]
        s = nt[ids[i, objidx[i, 10]]].reshape(-1)
        assert q - (p + l - 1) > 4 and all((s[p + t] ^ s[q + l - 1 - t]) == 3 for t in range(l))
    assert K > 0


@pytest.mark.parametrize("path", SELECT, ids=[p.stem for p in SELECT])
def test_selection_vs_reference(orc, path):
    z = np.load(path)
    N, p = int(z["N"]), int(z["p"])
    obj, ext = z["obj"], z["ext"]
    tab = {"nt": np.zeros((64, 3)), "weight": np.ones(64), "cps": np.zeros(3721), "start": np.zeros(21),
           "count": np.ones(21), "ref_gc3": 0.381, "ref_gc": 0.3977}
    prob = orc.Problem(np.zeros(5, np.int8), tab, 2, N, 0.0, objset=0, p=p)
    surv, front, ext_o, info = prob.select(0, obj, ext)
    flags = z["ref_flags"]
    assert info.rank_count == flags[0]
    assert info.n_fronts - 1 == flags[1]
    assert info.cut == flags[2]
    assert info.hyp_exception == flags[3]
    # fronts: same sizes; same members for every front the reference's niching does not
    # overwrite in its sorted array (it lists each front in atomic order)
    counts = z["ref_front_count"]
    srt = z["ref_sorted"]
    off = 0
    for f in range(info.n_fronts):
        assert counts[f] == np.count_nonzero(front == f), f
        if f < info.n_fronts - 1 or info.cut:
            members = set(srt[off:off + counts[f]].tolist())
            assert members == set(np.flatnonzero(front == f).tolist()), f
        off += counts[f]
    assert np.array_equal(np.float32(info.ideal)[:6], z["ref_ideal"])
    assert np.array_equal(np.float32(info.worst)[:6], z["ref_worst"])
    assert np.array_equal(ext_o.reshape(-1), z["ref_ext"])
    if info.hyp_exception:
        assert np.array_equal(np.float32(info.nadir)[:6], z["ref_nadir"])
    else:
        assert np.allclose(np.float32(info.nadir)[:6], z["ref_nadir"], rtol=1e-5)
    if not info.cut:
        # association: distances of every solution in fronts 0..last and niche counts
        ideal, nadir = np.float32(info.ideal)[:6], np.float32(info.nadir)[:6]
        ranked = np.flatnonzero(front >= 0)
        refpts = orc.das_dennis(6, p)
        f = (obj[ranked] - ideal) / (nadir - ideal)
        num = f @ refpts.T
        den = (refpts * refpts).sum(1)
        kk = num / den
        d = np.sqrt(((kk[:, :, None] * refpts[None] - f[:, None, :]) ** 2).sum(-1))
        assert np.allclose(d.min(1), z["ref_dist"][ranked], rtol=2e-5, atol=1e-6)
        last = front == info.n_fronts - 1
        earlier = ranked[~last[ranked]]
        rho = (np.bincount(d[~last[ranked]].argmin(1), minlength=len(refpts)) if len(earlier)
               else np.zeros(len(refpts), np.int64))
        # the reference's counts include its own niche picks (+1 per pick, sorting.cuh:1244,1262)
        inc = z["ref_included"].astype(np.int64)
        picks = inc - rho
        assert (picks >= 0).all()
        assert picks.sum() >= N - len(earlier)
        cand = np.bincount(d[last[ranked]].argmin(1), minlength=len(refpts))
        assert (picks <= cand).all()


def test_das_dennis_vs_reference(orc):
    z = np.load(GOLDEN / "ref_das_dennis.npz")
    for key in z.files:
        M, p = (int(x[1:]) for x in key.split("_"))
        ours = orc.das_dennis(M, p)
        ref = z[key]
        assert ours.shape == ref.shape
        assert np.array_equal(np.rint(ours * p), np.rint(ref * p))
        assert np.allclose(ours, ref, rtol=3e-7, atol=0)
