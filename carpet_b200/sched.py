"""Python face of the library's host schedules (cgx_sched_* in
csrc/cgx_sched.cu): the dh send/recv region lists of box hierarchies as
``Pair`` lists, computed in C++."""
from __future__ import annotations

import ctypes as C
from typing import List, Sequence

import numpy as np

from . import _lib
from ._lib import check, lib


def _boxes(bs: Sequence[Sequence[int]]):
    a = np.ascontiguousarray(np.array(list(bs), dtype=np.int32).reshape(-1, 9))
    return a, a.ctypes.data_as(C.c_void_p)


def _call(fn, *args, cap=1024):
    """runs a schedule call, growing the output until it fits"""
    while True:
        out = (_lib.cgx_pair_box * cap)()
        n = C.c_int()
        rc = fn(*args, out, cap, C.byref(n))
        if rc == _lib.OK or n.value <= cap:
            check(rc)
            return out, n.value
        cap = n.value


def _pairs(out, n):
    from .hierarchy import Pair
    return [Pair(out[i].dst_comp, out[i].src_comp, tuple(out[i].dstbox), tuple(out[i].srcbox))
            for i in range(n)]


def sync(comps) -> list:
    ia, ip = _boxes([c.interior for c in comps])
    ea, ep = _boxes([c.exterior for c in comps])
    return _pairs(*_call(lib.cgx_sched_sync, len(comps), ip, ep))


def prolong(fboxes, fcomps, ccomps, ghost: int, buffer: int, order: int) -> list:
    ba, bp = _boxes(fboxes)
    fa, fp = _boxes([c.interior for c in fcomps])
    ia, ip = _boxes([c.interior for c in ccomps])
    ea, ep = _boxes([c.exterior for c in ccomps])
    return _pairs(*_call(lib.cgx_sched_prolong, len(fboxes), bp, len(fcomps), fp, len(ccomps), ip, ep,
                         ghost, buffer, order))


def restrict(fboxes, fcomps, ccomps, ghost: int, buffer: int) -> list:
    ba, bp = _boxes(fboxes)
    fa, fp = _boxes([c.interior for c in fcomps])
    ia, ip = _boxes([c.interior for c in ccomps])
    return _pairs(*_call(lib.cgx_sched_restrict, len(fboxes), bp, len(fcomps), fp, len(ccomps), ip,
                         ghost, buffer))


def old2new(new_comps, old_comps, ccomps, order: int):
    na, np_ = _boxes([c.exterior for c in new_comps])
    oa, op = _boxes([c.interior for c in old_comps])
    ia, ip = _boxes([c.interior for c in ccomps])
    ea, ep = _boxes([c.exterior for c in ccomps])
    cap = 4096
    while True:
        co = (_lib.cgx_pair_box * cap)()
        po = (_lib.cgx_pair_box * cap)()
        nc, npr = C.c_int(), C.c_int()
        rc = lib.cgx_sched_old2new(len(new_comps), np_, len(old_comps), op, len(ccomps), ip, ep, order,
                                   co, cap, C.byref(nc), po, cap, C.byref(npr))
        if rc == _lib.OK or max(nc.value, npr.value) <= cap:
            check(rc)
            return _pairs(co, nc.value), _pairs(po, npr.value)
        cap = max(nc.value, npr.value)
