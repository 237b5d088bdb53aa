"""Known-answer tests of the oracle's building blocks (CPU)."""
import math

import numpy as np
import pytest

# Random123 known-answer vectors for Philox4x32-10 (kat_vectors, Salmon et al.)
PHILOX_KAT = [
    ((0, 0, 0, 0), (0, 0), (0x6627E8D5, 0xE169C58D, 0xBC57AC4C, 0x9B00DBD8)),
    ((0xFFFFFFFF,) * 4, (0xFFFFFFFF,) * 2, (0x408F276D, 0x41C83B0E, 0xA20BC7C6, 0x6D5451FD)),
    ((0x243F6A88, 0x85A308D3, 0x13198A2E, 0x03707344), (0xA4093822, 0x299F31D0),
     (0xD16CFE09, 0x94FDCCEB, 0x5001E420, 0x24126EA1)),
]


@pytest.mark.parametrize("ctr,key,expect", PHILOX_KAT)
def test_philox_kat(orc, ctr, key, expect):
    assert tuple(int(x) for x in orc.philox(ctr, key)) == expect


def test_draw_layout(orc):
    # word j of stream (tag, gen, idx, pos) = philox(ctr=(tag, gen, idx, 8*pos + j/4), key=seed)[j % 4]
    seed = 0x1234_5678_9ABC_DEF0
    key = (seed & 0xFFFFFFFF, seed >> 32)
    for j in range(8):
        w = orc.philox((3, 7, 11, 8 * 5 + j // 4), key)[j % 4]
        assert orc.lib().or_draw(seed, 3, 7, 11, 5, j) == w


def test_det_exp(orc):
    xs = np.concatenate([np.linspace(-700, 0, 20001), -np.logspace(-12, 2, 2001)])
    worst = max(abs(orc.det_exp(x) - math.exp(x)) / math.exp(x) for x in xs)
    assert worst < 5e-16


def test_auto_p_rule(orc):
    # largest p with C(M+p-1, p) <= N (src/main.cu:564-576)
    for M, N in [(6, 100), (4, 128), (4, 1024), (6, 2048), (4, 4096)]:
        p = orc.lib().or_auto_p(M, N)
        assert math.comb(M + p - 1, p) <= N < math.comb(M + p, p + 1)


@pytest.mark.parametrize("M,p", [(4, 6), (4, 8), (6, 4), (3, 12), (5, 3), (6, 1)])
def test_das_dennis_lattice(orc, M, p):
    pts = orc.das_dennis(M, p)
    assert pts.shape == (math.comb(M + p - 1, p), M)
    counts = np.rint(pts * p).astype(int)
    assert (counts.sum(axis=1) == p).all()
    assert len({tuple(r) for r in counts}) == len(counts)
    # rank order: multisets of {1..M} in lexicographic order = counts in reverse lexicographic order
    keys = [tuple(-c for c in r) for r in counts]
    assert keys == sorted(keys)
