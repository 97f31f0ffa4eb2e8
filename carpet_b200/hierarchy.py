"""Nested vertex-centred AMR hierarchies and their box-pair schedules.

The host-side producer of the send/recv box lists that CarpetLib's ``dh``
builds at regrid time (CarpetLib/src/dh.cc: sync 837-894, boundary
prolongation 896-977, restriction 981-1088), for the regular hierarchies of
the benchmark workloads: each level is one box split into components, each
finer level nested inside the next coarser one with refinement factor 2.

Per component (CarpetLib/src/dh.cc:300-542):
* ``interior``: the component's share of the level box (a partition);
* ``exterior``: the interior grown by ``ghost`` points on sides that face
  another component of the level (the inter-component ghost zones);
* the level's outer ``ghost + buffer`` layers (levels > 0) are filled by
  prolongation from the coarser level (outer boundary + buffer zones);
* restriction overwrites the coarse points under the fine level's active
  region (the level box without its ghost and buffer layers).

Every destination point of each schedule is covered exactly once; the
builders check it (the role of the ASSERT_c checks of dh.cc:825-831,
971-973, 1080-1082).
"""
from __future__ import annotations

import itertools
from dataclasses import dataclass, field
from typing import Dict, List, Tuple

Box = Tuple[int, ...]  # (lo x,y,z, up x,y,z, stride x,y,z)


def mkbox(lo, up, st) -> Box:
    return tuple(int(v) for v in (*lo, *up, *st))


def empty(b: Box) -> bool:
    return any(b[d] > b[3 + d] for d in range(3))


def size(b: Box):
    return tuple(0 if empty(b) else (b[3 + d] - b[d]) // b[6 + d] + 1 for d in range(3))


def npoints(b: Box) -> int:
    s = size(b)
    return s[0] * s[1] * s[2]


def intersect(a: Box, b: Box) -> Box:
    assert a[6:] == b[6:]
    lo = [max(a[d], b[d]) for d in range(3)]
    up = [min(a[3 + d], b[3 + d]) for d in range(3)]
    return mkbox(lo, up, a[6:])


def grow(b: Box, lo, up) -> Box:
    """bbox::expand by multiples of the stride (bbox.cc:180-191)"""
    return mkbox([b[d] - lo[d] * b[6 + d] for d in range(3)],
                 [b[3 + d] + up[d] * b[6 + d] for d in range(3)], b[6:])


def subtract(a: Box, b: Box) -> List[Box]:
    """a minus b as disjoint boxes (z slabs, then y, then x)"""
    c = intersect(a, b)
    if empty(c):
        return [] if empty(a) else [a]
    out, rest = [], list(a)
    for d in (2, 1, 0):
        st = a[6 + d]
        if rest[d] < c[d]:
            lo, up = list(rest[:3]), list(rest[3:6])
            up[d] = c[d] - st
            out.append(mkbox(lo, up, a[6:]))
        if rest[3 + d] > c[3 + d]:
            lo, up = list(rest[:3]), list(rest[3:6])
            lo[d] = c[3 + d] + st
            out.append(mkbox(lo, up, a[6:]))
        rest[d], rest[3 + d] = c[d], c[3 + d]
    return out


def coarsen_cover(b: Box, cs: int) -> Box:
    """the smallest coarse-stride box containing b (bbox::expanded_for)"""
    lo = [(b[d] // cs) * cs for d in range(3)]
    up = [-((-b[3 + d]) // cs) * cs for d in range(3)]
    return mkbox(lo, up, (cs,) * 3)


def coarsen_inside(b: Box, cs: int) -> Box:
    """the largest coarse-stride box inside b (bbox::contracted_for)"""
    lo = [-((-b[d]) // cs) * cs for d in range(3)]
    up = [(b[3 + d] // cs) * cs for d in range(3)]
    return mkbox(lo, up, (cs,) * 3)


@dataclass
class Component:
    interior: Box
    exterior: Box


@dataclass
class Level:
    stride: int
    box: Box
    comps: List[Component]


@dataclass
class Pair:
    """one sendrecv_pseudoregion_t (CarpetLib/src/region.hh:97-106)"""
    dst_comp: int
    src_comp: int
    dstbox: Box  # recv region, destination stride
    srcbox: Box  # send region, source stride


@dataclass
class Hierarchy:
    levels: List[Level]
    ghost: int
    buffer: int
    order: int
    sync: Dict[int, List[Pair]] = field(default_factory=dict)
    prolong: Dict[int, List[Pair]] = field(default_factory=dict)   # level l <- l-1
    restrict: Dict[int, List[Pair]] = field(default_factory=dict)  # level l-1 <- l


def split(box: Box, parts) -> List[Box]:
    """split a box into parts[0] x parts[1] x parts[2] near-equal pieces"""
    cuts = []
    for d in range(3):
        n = size(box)[d]
        st = box[6 + d]
        edges = [box[d] + (n * i // parts[d]) * st for i in range(parts[d] + 1)]
        cuts.append([(edges[i], edges[i + 1] - st) for i in range(parts[d])])
    out = []
    for (zl, zu) in cuts[2]:
        for (yl, yu) in cuts[1]:
            for (xl, xu) in cuts[0]:
                out.append(mkbox((xl, yl, zl), (xu, yu, zu), box[6:]))
    return out


def build_level(box: Box, parts, ghost: int) -> Level:
    comps = []
    for inter in split(box, parts):
        lo = [ghost if inter[d] > box[d] else 0 for d in range(3)]
        up = [ghost if inter[3 + d] < box[3 + d] else 0 for d in range(3)]
        comps.append(Component(inter, grow(inter, lo, up)))
    return Level(box[6], box, comps)


def nested(nlevels: int, npoints, parts=(2, 2, 2), ghost=3, buffer=9, order=5,
           origin=(0, 0, 0), native: bool = True, schedule: str = "regular") -> Hierarchy:
    """``nlevels`` vertex-centred levels of ``npoints`` points per axis each
    (an int or one per axis, each 1 mod 4), each level covering the central
    half of the next coarser one; ``parts`` splits every level into
    components (one (px, py, pz) for all levels, or a list of one per level).

    ``schedule``: "regular" -- this module's region lists for box
    hierarchies (the C++ ``cgx_sched_*`` with ``native``, else the Python
    restatement); "dh" -- CarpetLib's own region algebra for the same
    arrays (``carpet_b200.dh``: internal ghost points in a refined level's
    outer ghost layer are boundary-prolongated rather than synced, and
    restriction also fills the coarse ghost zones), which needs the levels
    properly nested (every refined level inside the next coarser level's
    active region with its stencils)."""
    n = (npoints,) * 3 if isinstance(npoints, int) else tuple(npoints)
    assert all((m - 1) % 4 == 0 for m in n)
    st0 = 2 ** (nlevels - 1)
    lo = list(origin)
    levels = []
    for l in range(nlevels):
        st = st0 >> l
        box = mkbox(lo, [lo[d] + (n[d] - 1) * st for d in range(3)], (st,) * 3)
        lp = parts[l] if isinstance(parts[0], (tuple, list)) else parts
        levels.append(build_level(box, lp, ghost))
        # next level: the central half, (n-1)/4 coarse points in
        lo = [lo[d] + ((n[d] - 1) // 4) * st for d in range(3)]
    h = Hierarchy(levels, ghost, buffer, order)
    if schedule == "dh":
        from . import dh
        doms, ints = dh.from_nested(h)
        g = (dh.schedule if native else dh.schedule_py)(doms, ints, ghost, buffer, order)
        for l in range(nlevels):
            assert [c.exterior for c in g.levels[l].comps] == [c.exterior for c in h.levels[l].comps]
        h.sync, h.prolong, h.restrict = g.sync, g.prolong, g.restrict
        return h
    if schedule != "regular":
        raise ValueError(f"unknown schedule {schedule!r}")
    globals()["schedule"](h, native)
    return h


def _sync_pairs(lev: Level) -> List[Pair]:
    """dh.cc:837-894: ghost zones of c from the interiors of the others"""
    pairs = []
    for c, comp in enumerate(lev.comps):
        ghosts = subtract(comp.exterior, comp.interior)
        for g in ghosts:
            for c2, comp2 in enumerate(lev.comps):
                if c2 == c:
                    continue
                r = intersect(g, comp2.interior)
                if not empty(r):
                    pairs.append(Pair(c, c2, r, r))
    return pairs


def _prolong_pairs(fine: Level, coarse: Level, ghost: int, buffer: int, order: int) -> List[Pair]:
    """dh.cc:896-977: the fine level's outer ghost+buffer shell, each fine
    point from the coarse component that owns the coarse point at or below
    it; the send box is that region's coarse cover grown by the stencil
    size order/2 (dh.cc:119-122, 805-806)."""
    cs = coarse.stride
    w = ghost + buffer
    shell = subtract(fine.box, grow(fine.box, (-w,) * 3, (-w,) * 3))
    pairs = []
    for c, comp in enumerate(fine.comps):
        for s in shell:
            piece = intersect(s, comp.interior)
            if empty(piece):
                continue
            for c2, comp2 in enumerate(coarse.comps):
                ci = comp2.interior
                own = mkbox(ci[:3], [ci[3 + d] + cs - fine.stride for d in range(3)],
                            (fine.stride,) * 3)
                r = intersect(piece, own)
                if empty(r):
                    continue
                send = grow(coarsen_cover(r, cs), (order // 2,) * 3, (order // 2,) * 3)
                assert all(send[d] >= comp2.exterior[d] and send[3 + d] <= comp2.exterior[3 + d]
                           for d in range(3)), "stencil leaves the coarse component"
                pairs.append(Pair(c, c2, r, send))
    return pairs


def _restrict_pairs(coarse: Level, fine: Level, ghost: int, buffer: int) -> List[Pair]:
    """dh.cc:981-1088: coarse interior points under the fine active region"""
    cs = coarse.stride
    w = ghost + buffer
    active = grow(fine.box, (-w,) * 3, (-w,) * 3)
    pairs = []
    for c2, comp2 in enumerate(coarse.comps):
        for c, comp in enumerate(fine.comps):
            region = coarsen_inside(intersect(active, comp.interior), cs)
            r = intersect(region, comp2.interior)
            if empty(r):
                continue
            send = mkbox(r[:3], r[3:6], (fine.stride,) * 3)
            pairs.append(Pair(c2, c, r, send))
    return pairs


def schedule(h: Hierarchy, native: bool = True):
    """the sync / boundary-prolongation / restriction lists of every level,
    built by the library's C++ schedules (``native``) or by the Python
    restatement in this module (``_sync_pairs`` ...), which the tests compare"""
    if native:
        from . import sched
    for l, lev in enumerate(h.levels):
        h.sync[l] = sched.sync(lev.comps) if native else _sync_pairs(lev)
        if l > 0:
            c = h.levels[l - 1]
            if native:
                h.prolong[l] = sched.prolong([lev.box], lev.comps, c.comps, h.ghost, h.buffer, h.order)
                h.restrict[l] = sched.restrict([lev.box], lev.comps, c.comps, h.ghost, h.buffer)
            else:
                h.prolong[l] = _prolong_pairs(lev, c, h.ghost, h.buffer, h.order)
                h.restrict[l] = _restrict_pairs(c, lev, h.ghost, h.buffer)
    check_coverage(h)


def _points(b: Box):
    s = size(b)
    for k in range(s[2]):
        for j in range(s[1]):
            for i in range(s[0]):
                yield (b[0] + i * b[6], b[1] + j * b[7], b[2] + k * b[8])


def check_coverage(h: Hierarchy, max_points: int = 3_000_000):
    """every destination point of a schedule is written exactly once"""
    for l, lev in enumerate(h.levels):
        # sync: exactly the ghost zones of each component
        want = sum(npoints(comp.exterior) - npoints(comp.interior) for comp in lev.comps)
        got = sum(npoints(p.dstbox) for p in h.sync[l])
        assert got == want, ("sync coverage", l, got, want)
        if l > 0:
            w = h.ghost + h.buffer
            shell = npoints(lev.box) - npoints(grow(lev.box, (-w,) * 3, (-w,) * 3))
            got = sum(npoints(p.dstbox) for p in h.prolong[l])
            assert got == shell, ("prolongation coverage", l, got, shell)
    # disjointness of the destination boxes per component (counts above
    # then imply exact covering); explicit point sets for small hierarchies
    for l, lev in enumerate(h.levels):
        for sched in (h.sync.get(l, []), h.prolong.get(l, [])):
            by = {}
            for p in sched:
                by.setdefault(p.dst_comp, []).append(p.dstbox)
            for boxes in by.values():
                for a, b in itertools.combinations(boxes, 2):
                    assert empty(intersect(a, b)), ("overlap", l, a, b)
