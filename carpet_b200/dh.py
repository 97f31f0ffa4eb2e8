"""Python face of the library's dh schedule producer (cgx_dh_* in
include/cgx.h): the region algebra of CarpetLib's dh::regrid
(CarpetLib/src/dh.cc:300-1088) for arbitrary vertex-centred component sets,
computed in C++.

``schedule(levels, ...)`` takes per level its domain box (the whole domain
at the level's stride) and its component interiors, and returns a
``carpet_b200.hierarchy.Hierarchy`` whose components carry the derived
interiors/exteriors and whose ``sync`` / ``prolong`` / ``restrict`` lists are
the dh send/recv lists.  ``from_nested`` gives the dh description of a
nested hierarchy built by ``carpet_b200.hierarchy.nested``: the same arrays,
with the refined levels' outer ghost layer outside the component interiors,
as Carpet's regridders place it.
"""
from __future__ import annotations

import ctypes as C
from typing import List, Sequence, Tuple

import numpy as np

from .hierarchy import Box, Component, Hierarchy, Level, Pair, grow, mkbox

SYNC, BNDPROL, RESTRICT = 0, 1, 2


def _library():
    """the C++ producer's entry points (the library is loaded on first use,
    so that the Python restatement below runs without it)"""
    from . import _lib
    lib = _lib.lib
    if not getattr(lib, "_dh_bound", False):
        lib.cgx_dh_create.argtypes = [C.POINTER(C.c_void_p), C.c_int, C.c_void_p, C.c_void_p, C.c_void_p,
                                      C.c_int, C.c_int, C.c_int, C.c_int, C.c_int]
        lib.cgx_dh_destroy.argtypes = [C.c_void_p]
        lib.cgx_dh_exteriors.argtypes = [C.c_void_p, C.c_int, C.c_void_p]
        lib.cgx_dh_pairs.argtypes = [C.c_void_p, C.c_int, C.c_int, C.POINTER(_lib.cgx_pair_box), C.c_int,
                                     C.POINTER(C.c_int)]
        lib._dh_bound = True
    return _lib, lib


def _pairs(h, level, kind) -> List[Pair]:
    _lib, lib = _library()
    check = _lib.check
    n = C.c_int()
    rc = lib.cgx_dh_pairs(h, level, kind, None, 0, C.byref(n))
    out = (_lib.cgx_pair_box * max(1, n.value))()
    check(lib.cgx_dh_pairs(h, level, kind, out, n.value, C.byref(n)))
    del rc
    return [Pair(out[i].dst_comp, out[i].src_comp, tuple(out[i].dstbox), tuple(out[i].srcbox))
            for i in range(n.value)]


def schedule(domains: Sequence[Box], interiors: Sequence[Sequence[Box]], ghost: int, buffer: int,
             order: int, boundary_width: int = 0, restrict_into_ghosts: bool = True) -> Hierarchy:
    """the dh regions and send/recv lists of a hierarchy given by its
    levels' domains and component interiors"""
    L = len(domains)
    dom = np.ascontiguousarray(np.array(domains, dtype=np.int32).reshape(L, 9))
    nc = np.array([len(i) for i in interiors], dtype=np.int32)
    intr = np.ascontiguousarray(np.array([b for i in interiors for b in i], dtype=np.int32).reshape(-1, 9))
    vp = lambda a: a.ctypes.data_as(C.c_void_p)  # noqa: E731
    _lib, lib = _library()
    check = _lib.check
    h = C.c_void_p()
    check(lib.cgx_dh_create(C.byref(h), L, vp(dom), vp(nc), vp(intr), ghost, buffer, boundary_width, order,
                            int(restrict_into_ghosts)))
    try:
        levels = []
        for l in range(L):
            ext = np.zeros((max(1, len(interiors[l])), 9), dtype=np.int32)
            check(lib.cgx_dh_exteriors(h, l, vp(ext)))
            comps = [Component(tuple(int(x) for x in interiors[l][c]), tuple(int(x) for x in ext[c]))
                     for c in range(len(interiors[l]))]
            levels.append(Level(domains[l][6], tuple(domains[l]), comps))
        hier = Hierarchy(levels, ghost, buffer, order)
        for l in range(L):
            hier.sync[l] = _pairs(h, l, SYNC)
            if l > 0:
                hier.prolong[l] = _pairs(h, l, BNDPROL)
            if l < L - 1:
                hier.restrict[l + 1] = _pairs(h, l, RESTRICT)
        return hier
    finally:
        lib.cgx_dh_destroy(h)


def from_nested(h: Hierarchy) -> Tuple[List[Box], List[List[Box]]]:
    """(domains, interiors) of a nested hierarchy in dh's terms: the domain of
    every level is the coarsest level's box at that level's stride; a refined
    level's component interiors leave out its outer ghost layer (Carpet's
    ghost zones at the refined region's boundary), so that the derived
    exteriors are the nested hierarchy's arrays"""
    d0 = h.levels[0].box
    domains, interiors = [], []
    for l, lev in enumerate(h.levels):
        s = lev.stride
        domains.append(mkbox(d0[:3], d0[3:6], (s,) * 3))
        if l == 0:
            interiors.append([c.interior for c in lev.comps])
            continue
        b = lev.box
        out = []
        for c in lev.comps:
            lo = [h.ghost if c.interior[d] == b[d] else 0 for d in range(3)]
            up = [h.ghost if c.interior[3 + d] == b[3 + d] else 0 for d in range(3)]
            out.append(grow(c.interior, [-x for x in lo], [-x for x in up]))
        interiors.append(out)
    return domains, interiors


# ------------------------------------------------------------------ Python
# A restatement of cgx_dh.cu in Python, box for box: the same region algebra
# in the same order, so the two give identical pair lists (the tests compare
# them); used where the library must not be loaded (the host reference
# driver of the benchmark).

def _isect(a: Box, b: Box) -> Box:
    return mkbox([max(a[d], b[d]) for d in range(3)], [min(a[3 + d], b[3 + d]) for d in range(3)], a[6:])


def _empty(b: Box) -> bool:
    return any(b[d] > b[3 + d] for d in range(3))


def _expand(b: Box, lo, up) -> Box:
    return mkbox([b[d] - lo[d] * b[6 + d] for d in range(3)], [b[3 + d] + up[d] * b[6 + d] for d in range(3)],
                 b[6:])


def _expanded_for(b: Box, l: Box) -> Box:
    """bbox::expanded_for (CarpetLib/src/bbox.cc:210-219)"""
    lo, up, st = [], [], []
    for d in range(3):
        s = l[6 + d]
        st.append(s)
        if _empty(b):
            lo.append(l[d])
            up.append(l[d] - s)
            continue
        lo.append(b[d] - (b[d] - l[d]) % s)
        up.append(b[3 + d] + (s - (b[3 + d] - l[d]) % s) % s)
    return mkbox(lo, up, st)


def _contracted_for(b: Box, l: Box) -> Box:
    """bbox::contracted_for (CarpetLib/src/bbox.cc:223-232)"""
    lo, up, st = [], [], []
    for d in range(3):
        s = l[6 + d]
        st.append(s)
        if _empty(b):
            lo.append(l[d])
            up.append(l[d] - s)
            continue
        lo.append(b[d] + (s - (b[d] - l[d]) % s) % s)
        up.append(b[3 + d] - (b[3 + d] - l[d]) % s)
    return mkbox(lo, up, st)


def _minus_into(a: Box, b: Box, out: list):
    c = _isect(a, b)
    if _empty(c):
        if not _empty(a):
            out.append(a)
        return
    rest = list(a)
    for d in (2, 1, 0):
        st = a[6 + d]
        if rest[d] < c[d]:
            s = list(rest)
            s[3 + d] = c[d] - st
            out.append(tuple(s))
        if rest[3 + d] > c[3 + d]:
            s = list(rest)
            s[d] = c[3 + d] + st
            out.append(tuple(s))
        rest[d], rest[3 + d] = c[d], c[3 + d]


class BSet:
    """disjoint boxes of one stride (the role of bboxset), as in cgx_dh.cu"""

    def __init__(self, v=None):
        self.v = list(v or [])

    @staticmethod
    def of(b: Box) -> "BSet":
        return BSet([] if _empty(b) else [b])

    def empty(self) -> bool:
        return not self.v

    def minus(self, other) -> "BSet":
        if isinstance(other, BSet):
            r = self
            for b in other.v:
                r = r.minus(b)
            return r
        out = []
        for a in self.v:
            _minus_into(a, other, out)
        return BSet(out)

    def isect(self, other) -> "BSet":
        if isinstance(other, BSet):
            out = []
            for b in other.v:
                out += self.isect(b).v
            return BSet(out)
        out = []
        for a in self.v:
            c = _isect(a, other)
            if not _empty(c):
                out.append(c)
        return BSet(out)

    def add(self, other):
        if isinstance(other, BSet):
            for b in other.v:
                self.add(b)
            return
        if _empty(other):
            return
        self.v += BSet([other]).minus(self).v

    def expanded(self, n: int) -> "BSet":
        r = BSet()
        for b in self.v:
            r.add(_expand(b, (n,) * 3, (n,) * 3))
        return r

    def expanded_for(self, l: Box) -> "BSet":
        r = BSet()
        for b in self.v:
            r.add(_expanded_for(b, l))
        return r

    def contracted_for(self, l: Box) -> "BSet":
        r = BSet()
        for b in self.v:
            r.add(_contracted_for(b, l))
        return r

    def normalized(self) -> "BSet":
        """boxes continuing each other along one axis (equal extents in the
        other two) merged until none do, in cgx_dh.cu's order"""
        w = list(self.v)
        changed = True
        while changed:
            changed = False
            for d in range(3):
                i = 0
                while i < len(w):
                    j = i + 1
                    while j < len(w):
                        a, b = w[i], w[j]
                        same = all(a[e] == b[e] and a[3 + e] == b[3 + e] for e in range(3) if e != d)
                        if same and (a[3 + d] + a[6 + d] == b[d] or b[3 + d] + b[6 + d] == a[d]):
                            m = list(a)
                            m[d], m[3 + d] = min(a[d], b[d]), max(a[3 + d], b[3 + d])
                            w[i] = tuple(m)
                            del w[j]
                            changed = True
                        else:
                            j += 1
                    i += 1
        return BSet(w)


def _contains(outer: Box, b: Box) -> bool:
    return _empty(b) or all(b[d] >= outer[d] and b[3 + d] <= outer[3 + d] for d in range(3))


def schedule_py(domains: Sequence[Box], interiors: Sequence[Sequence[Box]], ghost: int, buffer: int,
                order: int, boundary_width: int = 0, restrict_into_ghosts: bool = True) -> Hierarchy:
    """``schedule`` restated in Python (no library); raises ValueError where
    the C++ returns CGX_EINVAL"""
    bw = boundary_width
    L = len(domains)
    lv = []
    for l in range(L):
        D = tuple(domains[l])
        comps = []
        allowned = BSet()
        for c, intr in enumerate(interiors[l]):
            intr = tuple(intr)
            gl = [0 if intr[d] == D[d] else ghost for d in range(3)]
            gu = [0 if intr[3 + d] == D[3 + d] else ghost for d in range(3)]
            bl = [-bw if intr[d] == D[d] else 0 for d in range(3)]
            bu = [-bw if intr[3 + d] == D[3 + d] else 0 for d in range(3)]
            extr = _expand(intr, gl, gu)
            if not _contains(D, intr) or not _contains(D, extr):
                raise ValueError(f"dh: the interior/exterior must be contained in the domain ({l}, {c})")
            k = dict(intr=intr, extr=extr, ghosts=BSet.of(extr).minus(intr), comm=_expand(extr, bl, bu),
                     owned=_expand(intr, bl, bu), sync=BSet())
            comps.append(k)
            allowned.add(k["owned"])
        notowned = BSet.of(_expand(D, (-bw,) * 3, (-bw,) * 3)).minus(allowned)
        notactive = notowned.expanded(buffer)
        allbuffers = allowned.isect(notactive)
        allactive = allowned.minus(notactive)
        for k in comps:
            k["buffers"] = allbuffers.isect(k["owned"])
            k["active"] = allactive.isect(k["owned"])
        lv.append(dict(D=D, comps=comps, allactive=allactive, sync=[], bndprol=[], restrict=[]))
    for l in range(L):
        F = lv[l]
        for c, k in enumerate(F["comps"]):
            need = k["ghosts"]
            for cc, o in enumerate(F["comps"]):
                if need.empty():
                    break
                ovlp = need.isect(o["intr"]).normalized()
                if cc == c and not ovlp.empty():
                    raise ValueError("dh: A region may not synchronise from itself")
                for r in ovlp.v:
                    F["sync"].append(Pair(c, cc, r, r))
                need = need.minus(ovlp)
                k["sync"].add(ovlp)
        if l == 0:
            continue
        Cl = lv[l - 1]
        for c, k in enumerate(F["comps"]):
            need = k["ghosts"].minus(k["sync"]).isect(k["comm"])
            need.add(k["buffers"])
            for cc, o in enumerate(Cl["comps"]):
                if need.empty():
                    break
                eoa = o["active"].expanded_for(k["intr"]).expanded(2)
                ovlp = need.isect(eoa).normalized()
                for r in ovlp.v:
                    send = _expand(_expanded_for(r, o["intr"]), (order // 2,) * 3, (order // 2,) * 3)
                    if not _contains(o["extr"], send):
                        raise ValueError("dh: Boundary prolongation: Send region must be contained in exterior")
                    F["bndprol"].append(Pair(c, cc, r, send))
                need = need.minus(ovlp)
            if not need.empty():
                raise ValueError("dh: Synchronisation and boundary prolongation: All points must have been received")
        allrestricted = F["allactive"].contracted_for(Cl["D"])
        for oc, o in enumerate(Cl["comps"]):
            need = allrestricted.isect(o["extr"] if restrict_into_ghosts else o["intr"])
            if not need.isect(o["buffers"]).empty():
                raise ValueError("dh: Cannot restrict into buffer zones")
            for c, k in enumerate(F["comps"]):
                if need.empty():
                    break
                ovlp = need.isect(BSet.of(_contracted_for(k["extr"], Cl["D"]))).normalized()
                for r in ovlp.v:
                    send = _expanded_for(r, k["extr"])
                    if not _contains(k["extr"], send):
                        raise ValueError("dh: Refinement restriction: Send region must be contained in exterior")
                    Cl["restrict"].append(Pair(oc, c, r, send))
                need = need.minus(ovlp)
            if not need.empty():
                raise ValueError("dh: Refinement restriction: All points must have been received")
    levels = []
    for l in range(L):
        comps = [Component(k["intr"], k["extr"]) for k in lv[l]["comps"]]
        levels.append(Level(domains[l][6], tuple(domains[l]), comps))
    hier = Hierarchy(levels, ghost, buffer, order)
    for l in range(L):
        hier.sync[l] = lv[l]["sync"]
        if l > 0:
            hier.prolong[l] = lv[l]["bndprol"]
        if l < L - 1:
            hier.restrict[l + 1] = lv[l]["restrict"]
    return hier
