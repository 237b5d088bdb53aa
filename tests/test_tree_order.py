"""The extreme-point search replaces the reference's tree reduction (findMinValue:
level 1 pairs position t with t + B/2, each later level of h slots pairs slot t
with t + h/2, an odd h first folding slot h-1 into slot 0, a pair keeping its
first slot on equal values) by a minimum over (value, tree order).  This checks
that characterisation on the host, for every B up to 300 and many value draws:
the tree's winner is the lowest value and, among equal values, the position with
the smallest tree key (the same key the selection kernel computes)."""
import numpy as np


def tree_key(p, B):
    # choice made at each level (0 first slot, 1 the folded odd slot, 2 the other),
    # root level in the highest bits; None for a position level 1 leaves out
    h = B >> 1
    if p >= 2 * h:
        return None
    slot = p if p < h else p - h
    key = 0 if p < h else 2
    lvl = 1
    while h > 1:
        hn = h >> 1
        if slot < hn:
            d = 0
        elif slot < 2 * hn:
            d, slot = 2, slot - hn
        else:
            d, slot = 1, 0
        key |= d << (2 * lvl)
        lvl += 1
        h = hn
    return key


def tree_argmin(vals):
    B = len(vals)
    h = B // 2
    tb, tx = [None] * h, [None] * h
    for t in range(h):
        v0, v1 = vals[t], vals[t + h]
        tb[t], tx[t] = (v1, t + h) if v1 < v0 else (v0, t)
    while h > 1:
        odd, hp = h & 1, h - 1
        h >>= 1

        def pair(t, u):
            if tb[u] < tb[t]:
                tb[t], tx[t] = tb[u], tx[u]
        if odd:
            pair(0, hp)
        for t in range(h):
            pair(t, t + h)
    return tx[0]


def test_tree_winner_is_first_in_value_then_tree_order():
    rng = np.random.default_rng(7)
    for B in range(2, 301):
        keys = [tree_key(p, B) for p in range(B)]
        live = [p for p in range(B) if keys[p] is not None]
        assert len(set(keys[p] for p in live)) == len(live)  # a total order
        for _ in range(12):
            vals = rng.integers(0, 3, B).tolist()  # many ties
            expect = min(live, key=lambda p: (vals[p], keys[p]))
            assert tree_argmin(vals) == expect
