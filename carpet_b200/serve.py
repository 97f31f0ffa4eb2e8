"""The served form: an ensemble of small AMR hierarchies behind a request
server (cgx_server_* in include/cgx.h).

``Ensemble`` builds independent vertex-centred hierarchies, admits each
against the server's HBM budget before allocating its grid functions, and
defines one server operation per (hierarchy, transfer, level): the ghost sync
of a level, the boundary prolongation of a level from the next coarser one
(order-5 Lagrange with 3-timelevel time interpolation) and the restriction of
a level from the next finer one.  With ``regrid`` each hierarchy also gets a
regrid-fill operation: its finest level moved by two coarse points in x,
filled for every timelevel from the old level where that covered the point
and by order-5 prolongation from the next coarser level elsewhere -- the
transfers of ``ggf::recompose_fill`` (CarpetLib/src/ggf.cc:175-215) over the
old-to-new schedules of ``dh`` (CarpetLib/src/dh.cc:1717-1830).
Hierarchies the budget refuses wait in ``pending`` and ``admit_pending``
admits them later (also while the server runs) once ``retire`` has
released memory.  ``poisson_trace`` draws a request stream;
``Server.replay`` feeds it to the C++ worker at the drawn arrival times.
"""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass
from typing import Dict, List, Tuple

import numpy as np

from . import _lib
from ._lib import check, lib
from .amr import Storage, storage_bytes
from .hierarchy import nested
from .transfer import OP_LAGRANGE, VERTEX, Batch

SERVE_BATCHED, SERVE_PLAIN = 0, 1


class Report(C.Structure):
    _fields_ = [("requests", C.c_int64), ("launches", C.c_int64), ("fine_points", C.c_int64),
                ("hbm_used", C.c_int64), ("p50_ms", C.c_double), ("p99_ms", C.c_double),
                ("mean_ms", C.c_double), ("makespan_s", C.c_double),
                ("points_per_s", C.c_double), ("mean_batch", C.c_double),
                ("bytes", C.c_int64), ("bytes_per_s", C.c_double)]


lib.cgx_server_create.argtypes = [C.POINTER(C.c_void_p), C.c_int, C.c_int64, C.c_int, C.c_int64,
                                  C.c_int64]
for _f in ("cgx_server_destroy", "cgx_server_start", "cgx_server_drain"):
    getattr(lib, _f).argtypes = [C.c_void_p]
lib.cgx_server_admit.argtypes = [C.c_void_p, C.c_int64]
lib.cgx_server_set_config.argtypes = [C.c_void_p, C.c_int, C.c_int]
lib.cgx_server_release.argtypes = [C.c_void_p, C.c_int64]
lib.cgx_server_define_op.argtypes = [C.c_void_p, C.c_int, C.c_void_p, C.POINTER(C.c_int)]
lib.cgx_server_submit.argtypes = [C.c_void_p, C.c_int, C.POINTER(C.c_int64)]
lib.cgx_server_replay.argtypes = [C.c_void_p, C.POINTER(C.c_int), C.POINTER(C.c_double), C.c_int]
lib.cgx_server_stats.argtypes = [C.c_void_p, C.POINTER(Report)]
lib.cgx_server_latencies.argtypes = [C.c_void_p, C.POINTER(C.c_double), C.c_int64]


class Server:
    def __init__(self, mode=SERVE_BATCHED, hbm_budget=150 * 10**9, max_pairs=65536,
                 max_tiles=1 << 22, max_requests=1 << 20):
        h = C.c_void_p()
        check(lib.cgx_server_create(C.byref(h), mode, int(hbm_budget), max_pairs, max_tiles,
                                    max_requests))
        self.h, self.mode = h, mode

    def close(self):
        if self.h:
            lib.cgx_server_destroy(self.h)
            self.h = None

    __del__ = close

    def set_config(self, config: int, variant: int = -1):
        """tile configuration of the TMA prolongation variants (all: -1) for
        operations defined from now on"""
        check(lib.cgx_server_set_config(self.h, variant, config))

    def admit(self, nbytes: int) -> bool:
        rc = lib.cgx_server_admit(self.h, int(nbytes))
        if rc == _lib.ENOMEM:
            return False
        check(rc)
        return True

    def release(self, nbytes: int):
        check(lib.cgx_server_release(self.h, int(nbytes)))

    def define(self, hier: int, batch: Batch) -> int:
        op = C.c_int()
        check(lib.cgx_server_define_op(self.h, hier, batch.h, C.byref(op)))
        return op.value

    def submit(self, op: int):
        """one request now (starts the worker if it is not running)"""
        check(lib.cgx_server_start(self.h))
        check(lib.cgx_server_submit(self.h, op, None))

    def start(self):
        check(lib.cgx_server_start(self.h))

    def replay(self, ops, arrivals):
        n = len(ops)
        a = (C.c_int * n)(*[int(x) for x in ops])
        t = (C.c_double * n)(*[float(x) for x in arrivals])
        check(lib.cgx_server_replay(self.h, a, t, n))

    def drain(self):
        check(lib.cgx_server_drain(self.h))

    def report(self) -> Dict[str, float]:
        r = Report()
        check(lib.cgx_server_stats(self.h, C.byref(r)))
        return {f: getattr(r, f) for f, _ in Report._fields_}


@dataclass
class Member:
    hier: object
    storage: Storage
    nbytes: int
    moved: object = None          # the regrid-fill target: hierarchy with the moved finest level
    moved_storage: Storage = None  # its finest level's arrays (coarser levels shared)
    retired: bool = False


class Ensemble:
    """Independent 3-level hierarchies with per-axis coarse sizes drawn from
    U{lo..hi} (rounded up to 1 mod 4), 2 components per level."""

    KINDS = ("sync", "prolong", "restrict", "regrid")

    def __init__(self, server: Server, nhier=64, size_range=(24, 64), ngf=4, ntl=3, nlevels=3,
                 ghost=3, buffer=3, order=5, seed=0, fill_seed=1, regrid=False):
        rng = np.random.default_rng(seed)
        self.server, self.order, self.regrid = server, order, regrid
        self.ngf, self.ntl, self.fill_seed = ngf, ntl, fill_seed
        self.members: List[Member] = []
        self.pending: List[Tuple[object, int]] = []  # (hierarchy, bytes) the budget refused so far
        self.ops: Dict[Tuple[int, str, int], int] = {}
        for hid in range(nhier):
            n = [int(((int(rng.integers(size_range[0], size_range[1] + 1)) - 1 + 3) // 4) * 4 + 1)
                 for _ in range(3)]
            h = nested(nlevels, n, parts=(2, 1, 1), ghost=ghost, buffer=buffer, order=order)
            nbytes = storage_bytes(h, ngf, ntl)
            if regrid:
                nbytes += self._moved_bytes(h)
            if not server.admit(nbytes):
                self.pending.append((h, nbytes))
                continue
            self._add(h, nbytes)
        self.ops = self.define(server)

    @property
    def deferred(self) -> int:
        return len(self.pending)

    def _moved(self, h):
        """h with its finest level moved by two coarse points in x"""
        from .hierarchy import Hierarchy, build_level, mkbox
        L = len(h.levels)
        fine = h.levels[L - 1]
        cs = h.levels[L - 2].stride
        b = fine.box
        nb = mkbox((b[0] + 2 * cs, b[1], b[2]), (b[3] + 2 * cs, b[4], b[5]), b[6:])
        lev = build_level(nb, (2, 1, 1), h.ghost)
        return Hierarchy(h.levels[:L - 1] + [lev], h.ghost, h.buffer, h.order)

    def _moved_bytes(self, h) -> int:
        mv = self._moved(h)
        one = storage_bytes(mv, self.ngf, self.ntl) - storage_bytes(
            type(mv)(mv.levels[:-1], mv.ghost, mv.buffer, mv.order), self.ngf, self.ntl)
        return one

    def _add(self, h, nbytes) -> int:
        st = Storage(h, self.ngf, self.ntl)
        mem = Member(h, st, nbytes)
        if self.regrid:
            mem.moved = self._moved(h)
            L = len(h.levels)
            mem.moved_storage = Storage(mem.moved, self.ngf, self.ntl, share=st,
                                        shared_levels=tuple(range(L - 1)))
        self.members.append(mem)
        m = len(self.members) - 1
        fill_random(st, self.fill_seed + m)
        if mem.moved_storage is not None:
            fill_random_level(mem.moved_storage, len(h.levels) - 1, self.fill_seed + 1000 + m)
        return m

    def define(self, server: Server) -> Dict[Tuple[int, str, int], int]:
        """register every (hierarchy, transfer, level) operation with a server;
        returns the operation ids"""
        ops: Dict[Tuple[int, str, int], int] = {}
        for m, mem in enumerate(self.members):
            if not mem.retired:
                self._define(server, ops, m, mem)
        return ops

    def retire(self, m: int):
        """release hierarchy m's memory from the budget (its operations must
        not be submitted any more)"""
        mem = self.members[m]
        if mem.retired:
            return
        self.server.release(mem.nbytes)
        mem.retired = True
        mem.storage = mem.moved_storage = None

    def admit_pending(self, servers=()):
        """admit the waiting hierarchies that now fit the budget (also while
        the servers run), define their operations on this ensemble's server
        (into ``ops``) and on every server of ``servers``; returns (the new
        members' indices, [their operation ids on each of ``servers``])"""
        new, keep = [], []
        for h, nbytes in self.pending:
            if self.server.admit(nbytes):
                new.append(self._add(h, nbytes))
            else:
                keep.append((h, nbytes))
        self.pending = keep
        extra = []
        for m in new:
            self._define(self.server, self.ops, m, self.members[m])
        for sv in servers:
            d = {}
            for m in new:
                self._define(sv, d, m, self.members[m])
            extra.append(d)
        return new, extra

    def _define(self, server: Server, ops, m: int, mem: Member):
        h, st = mem.hier, mem.storage
        L = len(h.levels)
        dtc = 1.0 / 64
        times = [0.0, -dtc, -2 * dtc]
        for l in range(L):
            b = Batch()
            arrs = st.data[l][0]
            for g in range(st.ngf):
                for p in h.sync[l]:
                    b.add(arrs[g][p.dst_comp], [arrs[g][p.src_comp]], [0.0], p.dstbox, p.srcbox,
                          0.0, 1, 0, op=OP_LAGRANGE, cent=VERTEX)
            ops[(m, "sync", l)] = server.define(m, b)
        for l in range(1, L):
            b = Batch()
            dst = st.data[l][0]
            srcs = [st.data[l - 1][t] for t in range(st.ntl)]
            for g in range(st.ngf):
                for p in h.prolong[l]:
                    b.add(dst[g][p.dst_comp], [s[g][p.src_comp] for s in srcs], times, p.dstbox,
                          p.srcbox, -dtc / 2, self.order, 2, op=OP_LAGRANGE, cent=VERTEX)
            ops[(m, "prolong", l)] = server.define(m, b)
        for l in range(L - 1):
            b = Batch()
            dst, src = st.data[l][0], st.data[l + 1][0]
            for g in range(st.ngf):
                for p in h.restrict[l + 1]:
                    b.add(dst[g][p.dst_comp], [src[g][p.src_comp]], [0.0], p.dstbox, p.srcbox, 0.0,
                          self.order, 0, op=OP_LAGRANGE, cent=VERTEX)
            ops[(m, "restrict", l)] = server.define(m, b)
        if mem.moved is not None:
            ops[(m, "regrid", L - 1)] = server.define(m, self.regrid_batch(mem))

    def regrid_batch(self, mem: Member) -> Batch:
        """the regrid fill of the moved finest level, every timelevel: copies
        from the old finest level over its interiors, order-5 prolongation
        (one timelevel) from the next coarser level elsewhere"""
        from .moving import old2new
        h, mv = mem.hier, mem.moved
        l = len(h.levels) - 1
        copies, prols = old2new(h, mv, l)
        b = Batch()
        for tl in range(self.ntl):
            dst = mem.moved_storage.data[l][tl]
            old = mem.storage.data[l][tl]
            coarse = mem.storage.data[l - 1][tl]
            b.add_many([(dst[g][p.dst_comp], [old[g][p.src_comp]], p.dstbox, p.srcbox)
                        for g in range(self.ngf) for p in copies], [0.0], 0.0, 1, 0)
            b.add_many([(dst[g][p.dst_comp], [coarse[g][p.src_comp]], p.dstbox, p.srcbox)
                        for g in range(self.ngf) for p in prols], [0.0], 0.0, self.order, 0)
        return b

    def snapshot(self):
        out = []
        for mem in self.members:
            if mem.retired:
                continue
            out += [[p.clone() for p in lp] for lp in mem.storage.pools]
            if mem.moved_storage is not None:
                out.append([p.clone() for p in mem.moved_storage.pools[-1]])
        return out

    def restore(self, snap):
        it = iter(snap)
        for mem in self.members:
            if mem.retired:
                continue
            pools = list(mem.storage.pools)
            if mem.moved_storage is not None:
                pools.append(mem.moved_storage.pools[-1])
            for lp in pools:
                src = next(it)
                for p, q in zip(lp, src):
                    p.copy_(q)

    def state(self, m: int):
        """every device array of hierarchy m (for comparisons)"""
        mem = self.members[m]
        out = [p for lp in mem.storage.pools for p in lp]
        if mem.moved_storage is not None:
            out += list(mem.moved_storage.pools[-1])
        return out

    def close(self):
        for m, mem in enumerate(self.members):
            if not mem.retired:
                self.server.release(mem.nbytes)
        self.members = []


def fill_random(st: Storage, seed: int):
    import torch
    gen = torch.Generator(device="cuda").manual_seed(seed)
    for lp in st.pools:
        for p in lp:
            p.copy_(torch.randn(p.shape, generator=gen, device="cuda", dtype=torch.float64))


def fill_random_level(st: Storage, l: int, seed: int):
    import torch
    gen = torch.Generator(device="cuda").manual_seed(seed)
    for p in st.pools[l]:
        p.copy_(torch.randn(p.shape, generator=gen, device="cuda", dtype=torch.float64))


def request_key(ens: Ensemble, m: int, k: int, rng):
    """the request of kind k (0 sync, 1 prolong, 2 restrict, 3 regrid fill)
    for hierarchy m, at a uniformly chosen level"""
    L = len(ens.members[m].hier.levels)
    if k == 0:
        return (m, "sync", int(rng.integers(0, L)))
    if k == 1:
        return (m, "prolong", int(rng.integers(1, L)))
    if k == 2:
        return (m, "restrict", int(rng.integers(0, L - 1)))
    return (m, "regrid", L - 1)


def poisson_trace(ens: Ensemble, rate: float, n: int, seed=0, mix=(0.60, 0.25, 0.15)):
    """n requests with exponential inter-arrival times at ``rate`` per second:
    sync / prolongation / restriction (/ regrid fill, with a fourth entry) in
    proportions ``mix``, a uniformly chosen live hierarchy and level.
    Returns (keys, arrival times); map keys to a server's operation ids with
    ``ops_for``."""
    rng = np.random.default_rng(seed)
    arr = np.cumsum(rng.exponential(1.0 / rate, n))
    arr -= arr[0]
    live = [m for m, mem in enumerate(ens.members) if not mem.retired]
    ops = []
    for i in range(n):
        m = live[int(rng.integers(0, len(live)))]
        k = int(rng.choice(len(mix), p=mix))
        ops.append(request_key(ens, m, k, rng))
    return ops, arr


def ops_for(op_ids: Dict[Tuple[int, str, int], int], keys):
    return [op_ids[k] for k in keys]


def main(argv=None):
    """``python -m carpet_b200.serve``: drive one served ensemble (64
    hierarchies as in the benchmark) with a Poisson stream, or with every
    request submitted at once (``--rate 0``: the closed-loop saturation
    point), and print the server's report as one JSON line"""
    import argparse
    import json

    import torch
    p = argparse.ArgumentParser(prog="python -m carpet_b200.serve")
    p.add_argument("--requests", type=int, default=20000)
    p.add_argument("--rate", type=float, default=0.0, help="requests/s; 0: all at once")
    p.add_argument("--plain", action="store_true", help="the plain per-box server")
    p.add_argument("--tile-config", type=int, default=1)
    p.add_argument("--hierarchies", type=int, default=64)
    a = p.parse_args(argv)
    warm = Server(mode=SERVE_BATCHED)
    ens = Ensemble(warm, nhier=a.hierarchies, size_range=(24, 64), seed=42, regrid=True)
    wk, wa = poisson_trace(ens, 1e4, 200, seed=1)  # warm-up: module loading, kernel attributes
    warm.replay(ops_for(ens.ops, wk), wa)
    warm.drain()
    sv = Server(mode=SERVE_PLAIN if a.plain else SERVE_BATCHED)
    if not a.plain:
        sv.set_config(a.tile_config)
    op_ids = ens.define(sv)
    torch.cuda.synchronize()
    keys, arr = poisson_trace(ens, a.rate if a.rate > 0 else 1e5, a.requests, seed=99)
    sv.replay(ops_for(op_ids, keys), arr if a.rate > 0 else [0.0] * len(keys))
    sv.drain()
    r = sv.report()
    r["gbs"] = r["bytes_per_s"] / 1e9
    r["us_per_launch"] = 1e6 * r["makespan_s"] / max(1, r["launches"])
    print(json.dumps({k: (round(v, 6) if isinstance(v, float) else v) for k, v in r.items()}))
    sv.close()
    warm.close()


if __name__ == "__main__":
    main()
