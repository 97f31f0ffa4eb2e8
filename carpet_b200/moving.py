"""Moving-box hierarchies: regridding and the fill of newly refined regions.

The host side of CarpetLib's regrid for the transfer path (CarpetLib/src/
dh.cc: the old-to-new schedules ``fast_old2new_sync_sendrecv`` and
``fast_old2new_ref_prol_sendrecv``, 1717-1830, consumed by
``ggf::recompose_fill``, CarpetLib/src/ggf.cc:160-246): when the refined
regions move, every component of a refined level is refilled, level by level
from coarse to fine and for every timelevel -- from the old level's data
where the old level's interior covered the point (a copy), and by
prolongation from the (already refilled) next coarser level elsewhere.

``MovingSpec`` describes the moving-box workload: a coarse level covering the
domain and ``nlevels - 1`` refined levels, each made of two boxes centred on
two points that orbit the domain centre at ``radius`` times the domain width
(opposite each other, one revolution per ``steps_per_rev`` coarse steps); a
level's boxes are nested in the next coarser level's boxes around the same
centres.  Every box is split into components.

``build`` gives the hierarchy (with its sync / boundary-prolongation /
restriction schedules) at a coarse step; ``old2new`` the fill schedule of one
refined level between two hierarchies; ``Regrid`` builds the device batches
of a whole regrid, which run as one CUDA graph.
"""
from __future__ import annotations

import math
from dataclasses import dataclass
from typing import Dict, List, Optional, Tuple

from . import hierarchy as H
from .hierarchy import Box, Hierarchy, Level, Pair, empty, grow, intersect, mkbox, npoints, subtract
from .transfer import Batch, Graph


@dataclass
class MovingSpec:
    nlevels: int = 8
    n0: int = 257            # coarse-level points per axis
    nbox: int = 161          # points per axis of every refined box
    parts0: Tuple[int, int, int] = (4, 2, 2)
    parts: Tuple[int, int, int] = (2, 2, 2)
    ghost: int = 3
    buffer: int = 9
    order: int = 5
    radius: float = 0.3      # orbit radius / domain width
    steps_per_rev: int = 256
    regrid_every: int = 8


def centres(spec: MovingSpec, step: int):
    """the two region centres at a coarse step, in finest-stride index units"""
    s0 = 2 ** (spec.nlevels - 1)
    L = (spec.n0 - 1) * s0
    th = 2 * math.pi * step / spec.steps_per_rev
    out = []
    for a in (th, th + math.pi):
        out.append((L / 2 + spec.radius * L * math.cos(a), L / 2 + spec.radius * L * math.sin(a), L / 2))
    return out


def _sub_level(lev: Level, box: Box, comps) -> Level:
    return Level(lev.stride, box, comps)


def build(spec: MovingSpec, step: int, native: bool = True) -> Hierarchy:
    """the hierarchy at a coarse step; schedules from the library's C++
    (``native``) or from the Python restatement (the tests compare both)"""
    s0 = 2 ** (spec.nlevels - 1)
    box0 = mkbox((0, 0, 0), ((spec.n0 - 1) * s0,) * 3, (s0,) * 3)
    levels = [H.build_level(box0, spec.parts0, spec.ghost)]
    boxes: List[List[Box]] = [[box0]]
    owners: List[List[Tuple[int, int]]] = [[(0, len(levels[0].comps))]]  # comp range per box
    cs_ = centres(spec, step)
    for l in range(1, spec.nlevels):
        s = s0 >> l
        cs = 2 * s
        half = (spec.nbox - 1) // 2 * s
        bl, comps, rng = [], [], []
        for c in cs_:
            lo = [int(round((c[d] - half) / cs)) * cs for d in range(3)]
            up = [lo[d] + (spec.nbox - 1) * s for d in range(3)]
            b = mkbox(lo, up, (s,) * 3)
            sub = H.build_level(b, spec.parts, spec.ghost)
            rng.append((len(comps), len(comps) + len(sub.comps)))
            comps += sub.comps
            bl.append(b)
        levels.append(Level(s, bl[0], comps))
        boxes.append(bl)
        owners.append(rng)
    h = Hierarchy(levels, spec.ghost, spec.buffer, spec.order)
    h.boxes, h.owners = boxes, owners
    if native:
        from . import sched
        for l, lev in enumerate(levels):
            h.sync[l] = sched.sync(lev.comps)
            if l > 0:
                c = levels[l - 1].comps
                h.prolong[l] = sched.prolong(boxes[l], lev.comps, c, spec.ghost, spec.buffer, spec.order)
                h.restrict[l] = sched.restrict(boxes[l], lev.comps, c, spec.ghost, spec.buffer)
        check(h)
        return h
    for l, lev in enumerate(levels):
        h.sync[l] = H._sync_pairs(lev)
        if l == 0:
            continue
        h.prolong[l], h.restrict[l] = [], []
        for b, (c0, c1) in zip(boxes[l], owners[l]):
            sub = _sub_level(lev, b, lev.comps[c0:c1])
            for p in H._prolong_pairs(sub, levels[l - 1], spec.ghost, spec.buffer, spec.order):
                h.prolong[l].append(Pair(p.dst_comp + c0, p.src_comp, p.dstbox, p.srcbox))
            for p in H._restrict_pairs(levels[l - 1], sub, spec.ghost, spec.buffer):
                h.restrict[l].append(Pair(p.dst_comp, p.src_comp + c0, p.dstbox, p.srcbox))
    check(h)
    return h


def check(h: Hierarchy):
    """each schedule writes every destination point exactly once"""
    for l, lev in enumerate(h.levels):
        want = sum(npoints(c.exterior) - npoints(c.interior) for c in lev.comps)
        assert sum(npoints(p.dstbox) for p in h.sync[l]) == want, ("sync", l)
        if l > 0:
            w = h.ghost + h.buffer
            shell = sum(npoints(b) - npoints(grow(b, (-w,) * 3, (-w,) * 3)) for b in h.boxes[l])
            assert sum(npoints(p.dstbox) for p in h.prolong[l]) == shell, ("prolongation", l)
        for sched in (h.sync[l], h.prolong.get(l, [])):
            by: Dict[int, List[Box]] = {}
            for p in sched:
                by.setdefault(p.dst_comp, []).append(p.dstbox)
            for bs in by.values():
                for i in range(len(bs)):
                    for j in range(i + 1, len(bs)):
                        assert empty(intersect(bs[i], bs[j])), ("overlap", l)


def _minus_all(a: Box, cut: List[Box]) -> List[Box]:
    parts = [a]
    for c in cut:
        nxt = []
        for p in parts:
            nxt += subtract(p, c)
        parts = nxt
    return parts


def old2new(old: Hierarchy, new: Hierarchy, l: int, native: bool = True):
    """the fill of refined level l of ``new``: copy pairs (dst: new component,
    src: old component of level l) over the old interiors, and prolongation
    pairs (src: component of level l-1 of ``new``) for the rest of every new
    component's exterior; C++ (``native``) or the Python restatement"""
    assert l > 0
    if native:
        from . import sched
        copies, prols = sched.old2new(new.levels[l].comps, old.levels[l].comps, new.levels[l - 1].comps,
                                      new.order)
        want = sum(npoints(cm.exterior) for cm in new.levels[l].comps)
        assert sum(npoints(p.dstbox) for p in copies + prols) == want, ("old2new coverage", l)
        return copies, prols
    lnew, lold, coarse = new.levels[l], old.levels[l], new.levels[l - 1]
    cs = coarse.stride
    copies, prols = [], []
    for c, comp in enumerate(lnew.comps):
        for c2, oc in enumerate(lold.comps):
            r = intersect(comp.exterior, oc.interior)
            if not empty(r):
                copies.append(Pair(c, c2, r, r))
        for piece in _minus_all(comp.exterior, [oc.interior for oc in lold.comps]):
            for c3, cc in enumerate(coarse.comps):
                ci = cc.interior
                own = mkbox(ci[:3], [ci[3 + d] + cs - lnew.stride for d in range(3)], (lnew.stride,) * 3)
                r = intersect(piece, own)
                if empty(r):
                    continue
                send = grow(H.coarsen_cover(r, cs), (new.order // 2,) * 3, (new.order // 2,) * 3)
                assert all(send[d] >= cc.exterior[d] and send[3 + d] <= cc.exterior[3 + d]
                           for d in range(3)), "fill stencil leaves the coarse component"
                prols.append(Pair(c, c3, r, send))
    want = sum(npoints(cm.exterior) for cm in lnew.comps)
    assert sum(npoints(p.dstbox) for p in copies + prols) == want, ("old2new coverage", l)
    return copies, prols


class Regrid:
    """The device fill of one regrid: for every refined level (coarse to fine)
    and timelevel, one batch of the old-to-new copies and the prolongations
    from the next coarser level (one timelevel, no time interpolation), all
    captured in one CUDA graph.  ``old_tl(l, tl)`` / ``new_tl(l, tl)`` give the
    device arrays ([gf][comp] of Data) of timelevel tl of level l (the coarse
    level, which does not move, is shared: ``new_tl(0, tl)``)."""

    def __init__(self, old: Hierarchy, new: Hierarchy, ngf: int, ntl: int, old_tl, new_tl):
        self.batches: List[Batch] = []
        self.pairs = 0
        for l in range(1, len(new.levels)):
            copies, prols = old2new(old, new, l)
            for tl in range(ntl):
                b = Batch()
                dst, src_old = new_tl(l, tl), old_tl(l, tl)
                src_coarse = new_tl(l - 1, tl)
                b.add_many([(dst[g][p.dst_comp], [src_old[g][p.src_comp]], p.dstbox, p.srcbox)
                            for g in range(ngf) for p in copies], [0.0], 0.0, 1, 0)
                b.add_many([(dst[g][p.dst_comp], [src_coarse[g][p.src_comp]], p.dstbox, p.srcbox)
                            for g in range(ngf) for p in prols], [0.0], 0.0, new.order, 0)
                self.pairs += ngf * (len(copies) + len(prols))
                self.batches.append(b)

    def upload(self, autotune: bool = False, stream=None):
        for b in self.batches:
            if autotune:
                b.autotune(2, stream)
            else:
                b.upload(stream)

    def stats(self):
        tot = dict(pairs=0, points=0, bytes=0, kernels=0)
        for b in self.batches:
            s = b.stats()
            for k in ("pairs", "points", "bytes"):
                tot[k] += s[k]
            tot["kernels"] += b.kernels()
        return tot

    def run(self, stream=None):
        for b in self.batches:
            b.launch(stream)

    def graph(self, stream) -> Graph:
        g = Graph()
        with g.capture(stream):
            self.run(stream)
        return g
