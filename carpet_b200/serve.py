"""The served form: an ensemble of small AMR hierarchies behind a request
server (cgx_server_* in include/cgx.h).

``Ensemble`` builds independent vertex-centred hierarchies, admits each
against the server's HBM budget before allocating its grid functions, and
defines one server operation per (hierarchy, transfer, level): the ghost sync
of a level, the boundary prolongation of a level from the next coarser one
(order-5 Lagrange with 3-timelevel time interpolation) and the restriction of
a level from the next finer one.  ``poisson_trace`` draws a request stream;
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
                ("points_per_s", C.c_double), ("mean_batch", C.c_double)]


lib.cgx_server_create.argtypes = [C.POINTER(C.c_void_p), C.c_int, C.c_int64, C.c_int, C.c_int64,
                                  C.c_int64]
for _f in ("cgx_server_destroy", "cgx_server_start", "cgx_server_drain"):
    getattr(lib, _f).argtypes = [C.c_void_p]
lib.cgx_server_admit.argtypes = [C.c_void_p, C.c_int64]
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


class Ensemble:
    """Independent 3-level hierarchies with per-axis coarse sizes drawn from
    U{lo..hi} (rounded up to 1 mod 4), 2 components per level."""

    KINDS = ("sync", "prolong", "restrict")

    def __init__(self, server: Server, nhier=64, size_range=(24, 64), ngf=4, ntl=3, nlevels=3,
                 ghost=3, buffer=3, order=5, seed=0, fill_seed=1):
        rng = np.random.default_rng(seed)
        self.server, self.order = server, order
        self.members: List[Member] = []
        self.deferred = 0
        self.ops: Dict[Tuple[int, str, int], int] = {}
        for hid in range(nhier):
            n = [int(((int(rng.integers(size_range[0], size_range[1] + 1)) - 1 + 3) // 4) * 4 + 1)
                 for _ in range(3)]
            h = nested(nlevels, n, parts=(2, 1, 1), ghost=ghost, buffer=buffer, order=order)
            nbytes = storage_bytes(h, ngf, ntl)
            if not server.admit(nbytes):
                self.deferred += 1
                continue
            st = Storage(h, ngf, ntl)
            self.members.append(Member(h, st, nbytes))
        for m, mem in enumerate(self.members):
            fill_random(mem.storage, fill_seed + m)
        self.ops = self.define(server)

    def define(self, server: Server) -> Dict[Tuple[int, str, int], int]:
        """register every (hierarchy, transfer, level) operation with a server;
        returns the operation ids"""
        ops: Dict[Tuple[int, str, int], int] = {}
        for m, mem in enumerate(self.members):
            self._define(server, ops, m, mem)
        return ops

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

    def snapshot(self):
        return [[p.clone() for p in lp] for mem in self.members for lp in mem.storage.pools]

    def restore(self, snap):
        it = iter(snap)
        for mem in self.members:
            for lp in mem.storage.pools:
                src = next(it)
                for p, q in zip(lp, src):
                    p.copy_(q)

    def close(self):
        for mem in self.members:
            self.server.release(mem.nbytes)
        self.members = []


def fill_random(st: Storage, seed: int):
    import torch
    gen = torch.Generator(device="cuda").manual_seed(seed)
    for lp in st.pools:
        for p in lp:
            p.copy_(torch.randn(p.shape, generator=gen, device="cuda", dtype=torch.float64))


def poisson_trace(ens: Ensemble, rate: float, n: int, seed=0, mix=(0.60, 0.25, 0.15)):
    """n requests with exponential inter-arrival times at ``rate`` per second:
    sync / prolongation / restriction in proportions ``mix``, a uniformly
    chosen hierarchy and level.  Returns (keys, arrival times); map keys to a
    server's operation ids with ``ops_for``."""
    rng = np.random.default_rng(seed)
    arr = np.cumsum(rng.exponential(1.0 / rate, n))
    arr -= arr[0]
    ops = []
    M = len(ens.members)
    for i in range(n):
        m = int(rng.integers(0, M))
        k = int(rng.choice(3, p=mix))
        L = len(ens.members[m].hier.levels)
        if k == 0:
            key = (m, "sync", int(rng.integers(0, L)))
        elif k == 1:
            key = (m, "prolong", int(rng.integers(1, L)))
        else:
            key = (m, "restrict", int(rng.integers(0, L - 1)))
        ops.append(key)
    return ops, arr


def ops_for(op_ids: Dict[Tuple[int, str, int], int], keys):
    return [op_ids[k] for k in keys]
