"""The FP64 operation count of a prolongation box-pair (carpet_b200.bo.fp64_ops),
which the bench divides by a phase's time for its FP64 roofline, checked
against a point-by-point enumeration of what a separable evaluation needs
(CPU only)."""
import itertools
import random

import pytest

from carpet_b200.bo import fp64_ops


def enumerate_ops(reg, srcbbox, order, ntl):
    """walks every fine point: the x-pass values it reads (fine x, coarse y,
    coarse z), the y-pass values (fine x, fine y, coarse z), then counts the
    odd positions among them -- the taps -- and the time combination"""
    lo1, hi1 = -(order // 2), order // 2 + 1
    soff = [(reg[d] - srcbbox[d]) // reg[6 + d] for d in range(3)]
    n = [(reg[3 + d] - reg[d]) // reg[6 + d] + 1 for d in range(3)]

    def window(s):
        return range((s >> 1) + lo1, (s >> 1) + hi1 + 1) if s & 1 else [s >> 1]

    xvals, yvals = set(), set()
    for i, j, k in itertools.product(*(range(m) for m in n)):
        sx, sy, sz = soff[0] + i, soff[1] + j, soff[2] + k
        for cz in window(sz):
            yvals.add((sx, sy, cz))
            for cy in window(sy):
                xvals.add((sx, cy, cz))
    taps = sum(1 for v in xvals if v[0] & 1) + sum(1 for v in yvals if v[1] & 1)
    taps += n[0] * n[1] * sum(1 for k in range(n[2]) if (soff[2] + k) & 1)
    ops = ntl * taps * (2 * order + 1)
    if ntl > 1:
        ops += (2 * ntl - 1) * n[0] * n[1] * n[2]
    return ops


@pytest.mark.parametrize("seed", range(12))
def test_fp64_ops_matches_enumeration(seed):
    rng = random.Random(seed)
    order = rng.choice([1, 3, 5])
    ntl = rng.choice([1, 2, 3])
    src = [rng.randrange(-8, 8) * 2 for _ in range(3)]
    lo = [s + rng.randrange(2 * order + 2, 2 * order + 12) for s in src]
    hi = [a + rng.randrange(0, 9) * 2 for a in lo]
    reg = lo + hi + [2, 2, 2]
    srcbbox = src + [s + 200 for s in src] + [4, 4, 4]
    # fine indices: (lo - src) / 2 in fine units
    assert fp64_ops("prolong", ntl, reg, srcbbox, order) == enumerate_ops(reg, srcbbox, order, ntl)


def test_fp64_ops_copies_and_injection_have_no_arithmetic():
    reg = [0, 0, 0, 10, 10, 10, 2, 2, 2]
    assert fp64_ops("sync", 1, reg, reg) == 0
    assert fp64_ops("restrict", 1, reg, reg) == 0
