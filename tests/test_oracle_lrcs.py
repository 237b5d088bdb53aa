"""The oracle's longest repeated/common substring (LRCS flavour of the string
objective), checked against a plain dynamic-programming restatement (CPU).

The reference only names this objective (MLRCS, src/auto_execution_experiments.py:45,
215), so the oracle defines it; these tests pin that definition: the longest run
of identical nucleotides on one diagonal of CDS a against CDS b (a < b: any
diagonal; a == b: diagonals delta >= 1), first pair, then smallest delta, then
smallest start."""
import numpy as np
import pytest


def dp_pair(sa, sb, self_pair):
    n = len(sa)
    best = (0, 0, 0)
    for delta in range(1 if self_pair else -(n - 1), n):
        run = 0
        for r in range(max(0, -delta), min(n - 1, n - 1 - delta) + 1):
            if sa[r] == sb[r + delta]:
                run += 1
                if run > best[0]:
                    best = (run, delta, r - run + 1)
            else:
                run = 0
    return best


def lcs_length(sa, sb):
    """classic longest-common-substring table (no positions): a second check of the length"""
    n, m = len(sa), len(sb)
    prev = [0] * (m + 1)
    best = 0
    for i in range(1, n + 1):
        cur = [0] * (m + 1)
        for j in range(1, m + 1):
            if sa[i - 1] == sb[j - 1]:
                cur[j] = prev[j - 1] + 1
                best = max(best, cur[j])
        prev = cur
    return best


def lrs_length(s):
    n = len(s)
    best = 0
    for i in range(n):
        for j in range(i + 1, n):
            k = 0
            while j + k < n and s[i + k] == s[j + k]:
                k += 1
            best = max(best, k)
    return best


@pytest.mark.parametrize("seed,n,alphabet", [(1, 40, 4), (2, 61, 2), (3, 90, 4), (4, 33, 1)])
def test_pairs_match_dynamic_programming(orc, seed, n, alphabet):
    rng = np.random.default_rng(seed)
    a = rng.integers(0, alphabet, n).astype(np.uint8)
    b = a.copy()
    b[rng.integers(0, n, n // 5)] = rng.integers(0, 4, n // 5)
    for sa, sb, self_pair in ((a, b, False), (a, a, True), (b, a, False)):
        got = orc.lrcs_pair(sa, sb, self_pair)
        assert got == dp_pair(sa, sb, self_pair)
        assert got[0] == (lrs_length(sa) if self_pair else lcs_length(sa, sb))


def test_whole_solution_record_order(orc):
    rng = np.random.default_rng(9)
    n, m = 48, 4
    nt = rng.integers(0, 4, (m, n)).astype(np.uint8)
    # plant the same 12-nt block in CDS 1 and CDS 3 and a 12-nt repeat inside CDS 2
    blk = rng.integers(0, 4, 12).astype(np.uint8)
    nt[1, 5:17] = blk
    nt[3, 20:32] = blk
    nt[2, 0:12] = blk[::-1]
    nt[2, 30:42] = blk[::-1]
    L, p, q, a, b = orc.lrcs(nt)
    want = (0, 0, 0, 0, 0)
    for x in range(m):
        for y in range(x, m):
            r = dp_pair(nt[x], nt[y], x == y)
            if r[0] > want[0]:
                want = (r[0], r[2], r[2] + r[1], x, y)
    assert (L, p, q, a, b) == want
    assert L >= 12 and (a, b) in ((1, 3), (2, 2))


def test_lrcs_objective_in_evaluation(orc):
    aa = orc.synthetic_protein(30, 4)
    tab = orc.dirichlet_table(4)
    prob = orc.Problem(aa, tab, 3, 8, 0.05, objset=1, p=3, seed=1, slkind=1)
    ids = np.stack([prob.gen_solution(i) for i in range(4)])
    obj, objidx, pql = prob.evaluate(ids)
    nt = np.asarray(tab["nt"])[ids].reshape(4, 3, -1)
    n = nt.shape[2]
    for i in range(4):
        L, p, q, a, b = orc.lrcs(nt[i])
        assert obj[i, 3] == np.float32(L) / np.float32(n)
        assert tuple(objidx[i, 6:8]) == (a, b) and tuple(pql[i]) == (p, q, L)
