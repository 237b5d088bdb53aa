"""The seeded first pass of the string scan, restated in Python, against the
exhaustive rule: every counted run of >= 8 pairing cells is found exactly once.

The kernel (k_sl, sl_seed_scan) looks up S's words of K nucleotides at rows that
are multiples of t = 9 - K in a table of T's words at every position; an equal word
(e, e + delta) whose row e+K-1 is counted is measured: the run's start is found by
walking back at most t-1 rows (a word whose t rows below all pair is dropped: the
word t rows lower owns the run), and the run is followed to its end and clipped to
the diagonal's counted range.  This file checks that rule, for the hairpin's
(K=6, t=3) and LRCS's (K=7, t=2), against the full scan of every anti-diagonal
(hairpin, the rule of include/utils.cuh:712-888 as restated by the oracle) and
against the oracle's own LRCS pair search, whenever the longest run reaches 8."""
import numpy as np
import pytest


def full_hairpin(s):
    """(longest run, smallest anti-diagonal) over the counted cells."""
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
    return best, bestd


def seeded(S, T, lrcs, self_pair, K):
    """The seeded pass's (longest, smallest key) over the runs it measures."""
    n, t = len(S), 9 - K
    if not lrcs:
        dlo, dhi = -(n - 6), n - 6
    else:
        dlo, dhi = (1 if self_pair else -(n - 1)), n - 1
    table = {}
    for i in range(n - K + 1):
        table.setdefault(tuple(T[i:i + K]), []).append(i)

    def rows(delta):
        r_lo = max(0, -delta)
        r_hi = (n - 6 - delta) >> 1 if not lrcs else min(n - 1, n - 1 - delta)
        return r_lo, r_hi

    best, bestd = 0, 1 << 30
    for e in range(0, n - K + 1, t):
        for j in table.get(tuple(S[e:e + K]), []):
            delta = j - e
            r_lo, r_hi = rows(delta)
            if not (dlo <= delta <= dhi and e + K - 1 <= r_hi):
                continue
            st = e
            while st > e - t and st - 1 >= r_lo and S[st - 1] == T[st - 1 + delta]:
                st -= 1
            if st == e - t or st + 7 > r_hi:
                continue
            last = e + K - 1
            while last < r_hi and S[last + 1] == T[last + 1 + delta]:
                last += 1
            L = min(last, r_hi) - st + 1
            key = n - 1 - delta if not lrcs else delta + n
            if L > best or (L == best and key < bestd):
                best, bestd = L, key
    return best, bestd


def sequences(rng, count, lo, hi):
    out = []
    for k in range(count):
        n = int(rng.integers(lo, hi))
        kind = k % 3
        if kind == 0:
            s = rng.integers(0, 4, n).astype(np.uint8)
        elif kind == 1:      # a planted stem of 7 .. 19 pairs
            s = rng.integers(0, 4, n).astype(np.uint8)
            L = int(rng.integers(7, 20))
            if n > 2 * L + 20:
                a = int(rng.integers(0, n - 2 * L - 10))
                b = int(rng.integers(a + L + 4, n - L))
                s[b:b + L] = s[a:a + L][::-1] ^ 3
        else:                # low complexity: a unit and its reverse complement repeated
            unit = rng.integers(0, 4, int(rng.integers(1, 5))).astype(np.uint8)
            s = np.resize(np.concatenate([unit, unit[::-1] ^ 3]), n).astype(np.uint8)
            s[rng.integers(0, n, 3)] = rng.integers(0, 4, 3)
        out.append(s)
    return out


@pytest.mark.parametrize("K", [6, 7])
def test_hairpin_seeded_rule_equals_full_scan(K):
    rng = np.random.default_rng(100 + K)
    for s in sequences(rng, 90, 20, 160):
        T = (s[::-1] ^ 3).astype(np.uint8)
        want = full_hairpin(s)
        got = seeded(s, T, False, True, K)
        if want[0] >= 8:
            assert got == want, (len(s), want, got)
        else:
            assert got[0] < 8      # the exact word scan decides these


@pytest.mark.parametrize("K", [6, 7])
def test_lrcs_seeded_rule_equals_oracle(orc, K):
    rng = np.random.default_rng(200 + K)
    for k in range(120):
        n = int(rng.integers(20, 150))
        self_pair = k % 2 == 0
        sa = rng.integers(0, 4, n).astype(np.uint8)
        sb = sa.copy() if self_pair else rng.integers(0, 4, n).astype(np.uint8)
        if k % 3 == 1 and n > 40:   # a planted common substring
            L = int(rng.integers(7, 16))
            a, b = int(rng.integers(0, n - L)), int(rng.integers(0, n - L))
            sb[b:b + L] = sa[a:a + L]
            if self_pair:
                sa = sb.copy()
        if k % 5 == 4:              # periodic CDSs: runs on many diagonals
            sa = np.resize(np.array([0, 1, 2], np.uint8), n)
            sb = sa.copy() if self_pair else np.resize(np.array([1, 2, 0], np.uint8), n)
        length, delta, _ = orc.lrcs_pair(sa, sb, self_pair)
        got_len, got_key = seeded(sa, sb, True, self_pair, K)
        if length >= 8:
            assert (got_len, got_key - n) == (length, delta), (n, self_pair, length, delta, got_len, got_key - n)
        else:
            assert got_len < 8
