"""The transfer phases of one coarse Berger-Oliger step (pure Python).

Carpet's evolution loop (Carpet/src/Evolve.cc:44-121, with CallEvol
369-454 and CallRestrict 456-583) runs, for every iteration of the finest
level, each level whose step begins -- cycle its timelevels, prolongate its
boundary from the next coarser level at its new time (with time
interpolation when that time falls between coarse timelevels), sync its
ghost zones -- and then, coarsest last, every level aligned at the end of
the iteration receives the restriction from the next finer level followed
by a sync.  This module lists those transfer phases; it needs neither the
library nor a GPU, so the CPU reference driver and the device driver
(``carpet_b200.amr.BergerOliger``) replay the same order.

A phase key is ``(kind, level, rotations, ntl)``:

* ``("prolong", l, (rot_l, rot_{l-1}), ntl)``: boundary prolongation into
  level l from level l-1, ``ntl`` = 3 when the fine time falls between the
  coarse timelevels (quadratic time interpolation), 1 when it coincides
  with the coarse TL0;
* ``("sync", l, (rot_l,), 1)``: ghost-zone sync of level l;
* ``("restrict", l, (rot_l, rot_{l+1}), 1)``: restriction into level l from
  level l+1.

``rot_l`` counts level l's timelevel cycles modulo ``ntl`` (ggf::cycle_all,
CarpetLib/src/ggf.cc:248-267): pool ``(tl - rot_l) % ntl`` holds timelevel tl.
"""
from __future__ import annotations

from typing import List, Tuple

# coarsest time step of the benchmark hierarchies: dyadic, so that the time
# weights of every coarse step are the same bits and a replayed graph is exact
DT_COARSE = 1.0 / 64


def step_phases(nlevels: int, ntl: int, rot: List[int]) -> List[Tuple]:
    """the phases of one coarse step; advances ``rot`` (one entry per level)
    in place"""
    L = nlevels
    nit = 2 ** (L - 1)
    keys = []
    for it in range(1, nit + 1):
        for l in range(L):
            every = 2 ** (L - 1 - l)
            if (it - 1) % every == 0:
                rot[l] = (rot[l] + 1) % ntl  # cycle_all
                if l > 0:
                    # odd substeps of level l fall between coarse times
                    sub = ((it - 1) // every) % 2
                    n = 3 if sub == 0 else 1
                    keys.append(("prolong", l, (rot[l], rot[l - 1]), n))
                keys.append(("sync", l, (rot[l],), 1))
        for l in range(L - 2, -1, -1):
            if it % (2 ** (L - 1 - l)) == 0:
                keys.append(("restrict", l, (rot[l], rot[l + 1]), 1))
                keys.append(("sync", l, (rot[l],), 1))
    return keys


def pool_index(rot: int, tl: int, ntl: int) -> int:
    """the pool holding timelevel ``tl`` of a level rotated ``rot`` times"""
    return (tl - rot) % ntl


def prolong_times(ntl: int):
    """(coarse timelevel times, fine time) of a boundary prolongation: the
    coarse timelevels sit at 0, -dt, -2dt; the fine level is half a coarse
    step back (between timelevels) or on TL0"""
    times = [0.0, -DT_COARSE, -2 * DT_COARSE]
    return times, (-DT_COARSE / 2 if ntl > 1 else 0.0)


def phase_pairs(h, key):
    """the box-pairs of a phase and its (destination, source) levels"""
    kind, l, _, _ = key
    if kind == "sync":
        return h.sync[l], l, l
    if kind == "prolong":
        return h.prolong[l], l, l - 1
    return h.restrict[l + 1], l, l + 1


def stencil_points(reg, srcbbox, order: int = 5) -> int:
    """coarse points a vertex-centred prolongation of region ``reg`` reads
    from a source array with bbox ``srcbbox``: per axis, the union of the
    windows of the region's first two and last two fine points"""
    lo1, hi1 = -(order // 2), order // 2 + 1
    n = 1
    for d in range(3):
        soff = (reg[d] - srcbbox[d]) // reg[6 + d]
        m = (reg[3 + d] - reg[d]) // reg[6 + d] + 1
        cs = [(soff + i) for i in range(min(2, m))] + [(soff + i) for i in range(max(0, m - 2), m)]
        lo = min((s >> 1) + (lo1 if s & 1 else 0) for s in cs)
        hi = max((s >> 1) + (hi1 if s & 1 else 0) for s in cs)
        n *= hi - lo + 1
    return n


def fp64_ops(kind: str, ntl: int, reg, srcbbox, order: int = 5) -> int:
    """the double-precision operations a bit-exact, separable evaluation of
    one vertex-centred prolongation box-pair cannot avoid, in the exact mode
    (every product and every sum its own rounding, as prolongate_3d_rf2.cc
    computes them without contraction): a (order + 1)-tap sum costs order + 1
    multiplies and order adds; the x pass evaluates every odd fine x on every
    coarse (y, z) the region's windows touch, the y pass every odd fine y on
    every coarse z, the z pass every odd fine z; even fine points are copies.
    Time interpolation adds ntl multiplies and ntl - 1 adds per fine point.
    Copies and injection have no arithmetic (0)."""
    if kind != "prolong":
        return 0
    lo1, hi1 = -(order // 2), order // 2 + 1
    m, odd, coarse = [], [], []
    for d in range(3):
        soff = (reg[d] - srcbbox[d]) // reg[6 + d]
        n = (reg[3 + d] - reg[d]) // reg[6 + d] + 1
        m.append(n)
        odd.append(sum(1 for i in range(n) if (soff + i) & 1))
        cs = [soff + i for i in range(min(2, n))] + [soff + i for i in range(max(0, n - 2), n)]
        lo = min((s >> 1) + (lo1 if s & 1 else 0) for s in cs)
        hi = max((s >> 1) + (hi1 if s & 1 else 0) for s in cs)
        coarse.append(hi - lo + 1)
    taps = (odd[0] * coarse[1] * coarse[2] + m[0] * odd[1] * coarse[2] + m[0] * m[1] * odd[2])
    ops = ntl * taps * (2 * (order + 1) - 1)
    if ntl > 1:
        ops += (2 * ntl - 1) * m[0] * m[1] * m[2]
    return ops


def algorithmic_bytes(kind: str, ntl: int, dstbox, srcbox, order: int = 5) -> int:
    """the algorithmic bytes of one box-pair: copy 16 B per destination
    point, injection 16 B per coarse point, prolongation 8 B per fine point
    plus 8 B per coarse point its stencil reads per timelevel"""
    from .hierarchy import npoints
    if kind in ("sync", "restrict"):
        return 16 * npoints(dstbox)
    return 8 * npoints(dstbox) + ntl * 8 * stencil_points(dstbox, srcbox, order)


def step_totals(h, keys, order: int = 5):
    """(algorithmic bytes, destination points) of the phases for one grid
    function"""
    from .hierarchy import npoints
    b = p = 0
    for key in keys:
        kind, _, _, ntl = key
        pairs, _, _ = phase_pairs(h, key)
        b += sum(algorithmic_bytes(kind, ntl, q.dstbox, q.srcbox, order) for q in pairs)
        p += sum(npoints(q.dstbox) for q in pairs)
    return b, p


def workload_totals(h, ngf: int, ntl: int = 3, order: int = 5):
    """algorithmic bytes and destination points of one coarse step of ngf
    grid functions (the average of the three timelevel-rotation variants)"""
    L = len(h.levels)
    rot = [0] * L
    tb = tp = 0
    for _ in range(3):
        b, p = step_totals(h, step_phases(L, ntl, rot), order)
        tb, tp = tb + b, tp + p
    return tb * ngf / 3, tp * ngf / 3
