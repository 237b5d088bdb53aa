"""The oracle's mutation operators against the behaviour the reference's code
specifies, in distribution (CPU).

The reference draws from per-thread XORWOW streams (src/main.cu:35), so its exact
children cannot be reproduced; the CUDA engine equals the oracle bit for bit, and
these tests pin the oracle's stochastic half to the rules of include/mutation.cuh
and the dispatch of src/main.cu:172-211, each checked over many seeded children:

* the operator is uniform over the 7 types (six objectives) or the 5 kept with
  four objectives (src/main.cu:174-177);
* mutationRandom (:16-63): each position whose amino acid has k > 1 codons changes
  with probability Pm, to one of the other k-1 codons uniformly;
* mutationCAI (:65-142, SELECT_UPPER_RANDOM): only the CDS with the lowest CAI,
  each position with probability Pm, to a uniformly drawn higher-index
  (higher-weight) codon; positions already at the best codon stay;
* mutationCBP / mutationHSC (:144-388): only their worst CDS, only positions of
  the generation's parity, with probability 2Pm (CBP: position 0 .. L-2);
* mutationHD (:390-534): only the first CDS of the closest pair;
* mutationGC3 (:536-653): only the CDS farthest from the GC3 target, each change
  moving its third nucleotide towards the target (GC_UP: to G/C, GC_DOWN: away);
* mutationSL (:775-969): at most one codon, in the CDS holding the stem.
Bounds are five standard deviations wide, so the seeded tests are stable."""
import math

import numpy as np
import pytest

NT_GC = {1, 2}  # C, G


def _population(orc, objset, L=120, m=4, n=24, pm=0.05, seed=5):
    aa = orc.synthetic_protein(L, seed)
    tab = orc.dirichlet_table(seed)
    prob = orc.Problem(aa, tab, m, 64, pm, objset=objset, p=3, seed=seed)
    parents = np.stack([prob.gen_solution(i) for i in range(n)])
    obj, objidx, pql = prob.evaluate(parents)
    return prob, tab, parents, obj, objidx, pql


def _children(prob, parents, obj, objidx, pql, gens, reps):
    """children of every parent, `reps` offspring indices each, over several generations"""
    out = []
    n = parents.shape[0]
    for g in gens:
        for r in range(reps):
            idx = np.arange(n, dtype=np.int32) + r * n
            child, ops, _, _, _ = prob.mutate(g, idx, parents, obj, objidx, pql)
            for i in range(n):
                out.append((g, i, int(ops[i]), child[i]))
    return out


def _within(x, n, p, sig=5.0):
    mu, sd = n * p, math.sqrt(max(n * p * (1 - p), 1e-12))
    return abs(x - mu) <= sig * sd + 1


@pytest.mark.parametrize("objset,kinds", [(0, 7), (1, 5)])
def test_operator_choice_is_uniform(orc, objset, kinds):
    prob, tab, parents, obj, objidx, pql = _population(orc, objset)
    res = _children(prob, parents, obj, objidx, pql, range(4), 20)
    ops = np.array([o for _, _, o, _ in res])
    allowed = list(range(7)) if objset == 0 else [0, 1, 4, 5, 6]
    assert set(np.unique(ops)) == set(allowed)
    for o in allowed:
        assert _within(int((ops == o).sum()), len(ops), 1.0 / kinds)


def test_random_operator(orc):
    prob, tab, parents, obj, objidx, pql = _population(orc, 1, pm=0.05)
    start, count = np.asarray(tab["start"]), np.asarray(tab["count"])
    aa = prob.aa
    multi = count[aa] > 1
    trials = changed = 0
    moves = {}
    for g, i, op, child in _children(prob, parents, obj, objidx, pql, range(12), 40):
        if op != 0:
            continue
        diff = child != parents[i]
        assert not diff[:, ~multi].any()                      # single-codon amino acids never change
        trials += int(multi.sum()) * prob.m
        changed += int(diff.sum())
        for c, a in zip(*np.nonzero(diff)):
            k, s0 = int(count[aa[a]]), int(start[aa[a]])
            new, old = int(child[c, a]) - s0, int(parents[i][c, a]) - s0
            assert 0 <= new < k and new != old                # a different synonymous codon
            moves.setdefault(k, []).append((new - old) % k - 1)   # 0 .. k-2: which of the others
    assert trials > 0 and _within(changed, trials, 0.05)
    # the other codons are drawn uniformly
    checked = 0
    for k, offs in moves.items():
        if k >= 3 and len(offs) >= 80:
            for v in range(k - 1):
                assert _within(offs.count(v), len(offs), 1.0 / (k - 1))
            checked += 1
    assert checked >= 1


def test_cai_operator_moves_up_in_the_worst_cds(orc):
    prob, tab, parents, obj, objidx, pql = _population(orc, 1, pm=0.2)
    start, count = np.asarray(tab["start"]), np.asarray(tab["count"])
    aa = prob.aa
    slot = 0
    ups = {}
    trials = changed = 0
    for g, i, op, child in _children(prob, parents, obj, objidx, pql, range(6), 30):
        if op != 1:
            continue
        c = int(objidx[i][2 * slot])
        diff = child != parents[i]
        assert not np.delete(diff, c, axis=0).any()          # only the lowest-CAI CDS
        for a in range(prob.L):
            k, s0 = int(count[aa[a]]), int(start[aa[a]])
            old = int(parents[i][c, a]) - s0
            if k > 1 and old < k - 1:
                trials += 1
            if diff[c, a]:
                new = int(child[c, a]) - s0
                assert new > old                             # SELECT_UPPER_RANDOM: a higher index
                changed += 1
                ups.setdefault((k, old), []).append(new)
    assert _within(changed, trials, 0.2)
    # uniform over the higher indices, e.g. from the lowest of four codons: 1, 2, 3 equally
    for (k, old), news in ups.items():
        if len(news) >= 60:
            for v in range(old + 1, k):
                assert _within(news.count(v), len(news), 1.0 / (k - 1 - old))


def test_cbp_hsc_operators_use_parity_and_twice_pm(orc):
    prob, tab, parents, obj, objidx, pql = _population(orc, 0, pm=0.1)
    count = np.asarray(tab["count"])
    aa = prob.aa
    for op, kind_slot in ((2, 1), (3, 2)):
        hits = eligible = 0
        for g, i, o, child in _children(prob, parents, obj, objidx, pql, range(6), 40):
            if o != op:
                continue
            c = int(objidx[i][2 * kind_slot])
            diff = child != parents[i]
            assert not np.delete(diff, c, axis=0).any()
            pos = np.nonzero(diff[c])[0]
            assert all(p % 2 == g % 2 for p in pos)           # positions of the generation's parity
            if op == 2:
                assert all(p <= prob.L - 2 for p in pos)
            last = prob.L - 2 if op == 2 else prob.L - 1
            eligible += sum(1 for a in range(g % 2, last + 1, 2) if count[aa[a]] > 1)
            hits += len(pos)
        # a position is tried with probability 2 Pm; a try changes the codon only when a
        # synonym improves the local score, so the changes stay below 2 Pm of the positions
        assert 0 < hits and (hits - eligible * 0.2) <= 5 * math.sqrt(eligible * 0.2 * 0.8) + 1


def test_hd_gc_sl_operators_touch_their_cds(orc):
    prob, tab, parents, obj, objidx, pql = _population(orc, 1, pm=0.3)
    nt = np.asarray(tab["nt"])
    seen = set()
    for g, i, op, child in _children(prob, parents, obj, objidx, pql, range(6), 30):
        diff = child != parents[i]
        if op == 4:        # HD slot 1: the first CDS of the closest pair
            c = int(objidx[i][2])
            assert not np.delete(diff, c, axis=0).any()
        elif op == 5:      # GC slot 2: the farthest CDS, third nucleotide towards the target
            c, d = int(objidx[i][4]), int(objidx[i][5])
            assert not np.delete(diff, c, axis=0).any()
            for a in np.nonzero(diff[c])[0]:
                before = int(nt[parents[i][c, a]][2]) in NT_GC
                after = int(nt[child[c, a]][2]) in NT_GC
                assert (after and not before) if d == 1 else (before and not after)
        elif op == 6:      # SL slot 3: at most one codon, in the stem's CDS
            c = int(objidx[i][6])
            assert int(diff.sum()) <= 1 and not np.delete(diff, c, axis=0).any()
        if diff.any():
            seen.add(op)
    assert {4, 5} <= seen
