"""The oracle's own synthetic inputs and state loading (CPU).

The CPU baseline builds its workload without loading the engine library, so the
oracle restates the engine's generators; these must agree draw for draw."""
import numpy as np
import pytest


@pytest.mark.parametrize("seed", [0, 1, 2024, 2**63 + 5])
def test_synthetic_inputs_match_the_engine(pe, orc, seed):
    assert np.array_equal(orc.synthetic_protein(1000, seed), pe.synthetic_protein(1000, seed))
    want = pe.dirichlet_table(seed).arrays()
    got = orc.dirichlet_table(seed)
    for k in ("nt", "weight", "cps", "start", "count"):
        assert np.array_equal(np.asarray(got[k]), np.asarray(want[k])), k
    assert got["ref_gc3"] == want["ref_gc3"] and got["ref_gc"] == want["ref_gc"]


def test_dirichlet_weights_ascend_inside_groups(orc):
    t = orc.dirichlet_table(7)
    for a in range(21):
        s, k = int(t["start"][a]), int(t["count"][a])
        w = t["weight"][s:s + k]
        assert np.all(np.diff(w) >= 0) and w[-1] == 1.0


def test_set_state_continues_a_run(orc):
    aa = orc.synthetic_protein(40, 3)
    tab = orc.dirichlet_table(3)
    prob = orc.Problem(aa, tab, 3, 24, 0.05, objset=1, p=3, seed=9)
    a = orc.Run(prob)
    a.init()
    a.generation()
    a.generation()
    ids, obj, objidx, pql, surv, ext, gen = a.state()
    b = orc.Run(prob)
    b.set_state(ids, obj, objidx, pql, surv, ext, gen)
    a.generation()
    b.generation()
    for x, y in zip(a.state(), b.state()):
        assert np.array_equal(np.asarray(x), np.asarray(y))
    a.close()
    b.close()
