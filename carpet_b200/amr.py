"""Device-resident grid functions of a hierarchy and a Berger-Oliger driver.

``Storage`` holds, for every level, ``ngf`` grid functions x ``ntl``
timelevels x components, as ``Data`` arrays carved out of one device pool
per (level, timelevel) -- the layout a CarpetLib ``ggf`` keeps as
``storage[ml][rl][lc][tl]`` (CarpetLib/src/ggf.hh), packed so that a
timelevel of a whole level is one contiguous block.  Cycling timelevels
(ggf::cycle_all, CarpetLib/src/ggf.cc:248-267) is a rotation of which pool
plays TL0/TL1/TL2, never a copy.

``BergerOliger`` replays the transfer calls of one coarse Berger-Oliger
step in Carpet's order (Carpet/src/Evolve.cc:44-121 with CallEvol
369-454 and CallRestrict 456-583): every iteration of the finest level,
each level whose step begins evolves -- cycle, boundary prolongation from
the next coarser level at its new time (with time interpolation when the
time falls between coarse timelevels), ghost sync -- and every level
aligned at the end of the iteration receives the restriction from the next
finer level followed by a sync.  The evolution itself (the right-hand
side) is not part of the transfer path and is not run.

Each such phase is one batch of box-pairs over all grid functions, run by
the persistent kernel; a whole coarse step can be captured as a CUDA graph.
Grid functions never exchange data, so with ``groups`` > 1 the grid
functions are split into that many groups whose phase chains run on
separate streams: each group keeps the reference's call order, and one
group's kernels fill the SMs that another group's kernel leaves idle while
its last tiles drain.
"""
from __future__ import annotations

from dataclasses import dataclass
from typing import Dict, List, Optional, Tuple

import numpy as np
import torch

from .hierarchy import Hierarchy, npoints, size
from .transfer import OP_LAGRANGE, VERTEX, Batch, Chain, Data, Graph, _arrays, _stream
from . import _lib, bo
import ctypes as C


def _padded(ext_box):
    nx, ny, nz = size(ext_box)
    return nx + (nx & 1), ny, nz


def storage_bytes(h: Hierarchy, ngf: int, ntl: int) -> int:
    """device bytes a Storage of this hierarchy allocates"""
    n = 0
    for lev in h.levels:
        per = 0
        for c in lev.comps:
            px, py, pz = _padded(c.exterior)
            per += ((px * py * pz + 31) // 32) * 32
        n += ntl * ngf * per * 8
    return n


class Storage:
    """[level][tl] -> one pool; data[level][tl][gf][comp] -> Data views"""

    def __init__(self, h: Hierarchy, ngf: int, ntl: int, device="cuda",
                 share: Optional["Storage"] = None, shared_levels=()):
        """``share`` / ``shared_levels``: levels whose pools are taken from
        another storage of a hierarchy with the same components there (the
        unchanged coarse levels of a regrid) instead of allocated"""
        self.h, self.ngf, self.ntl = h, ngf, ntl
        self.pools: List[List[torch.Tensor]] = []
        self.data: List[List[List[List[Data]]]] = []
        for l, lev in enumerate(h.levels):
            if share is not None and l in shared_levels:
                self.pools.append(share.pools[l])
                self.data.append(share.data[l])
                continue
            shapes = [_padded(c.exterior) for c in lev.comps]
            # 256-byte aligned offsets for every component array
            offs, n = [], 0
            for _ in range(ngf):
                row = []
                for (px, py, pz) in shapes:
                    row.append(n)
                    n += ((px * py * pz + 31) // 32) * 32
                offs.append(row)
            lp, ld = [], []
            for tl in range(ntl):
                pool = torch.empty(n, dtype=torch.float64, device=device)
                lp.append(pool)
                gfs = []
                for g in range(ngf):
                    comps = []
                    for c, (px, py, pz) in enumerate(shapes):
                        o = offs[g][c]
                        t = pool[o:o + px * py * pz].view(pz, py, px)
                        comps.append(Data(lev.comps[c].exterior, t))
                    gfs.append(comps)
                ld.append(gfs)
            self.pools.append(lp)
            self.data.append(ld)

    def nbytes(self) -> int:
        return sum(p.numel() * 8 for lp in self.pools for p in lp)

    def fill(self, fn, seed=0):
        """fn(x, y, z, gf, tl, rng) -> values, evaluated on every array"""
        rng = np.random.default_rng(seed)
        for l, lev in enumerate(self.h.levels):
            for tl in range(self.ntl):
                for g in range(self.ngf):
                    for c, comp in enumerate(lev.comps):
                        b = comp.exterior
                        nx, ny, nz = size(b)
                        x = b[0] + np.arange(nx) * b[6]
                        y = b[1] + np.arange(ny) * b[7]
                        z = b[2] + np.arange(nz) * b[8]
                        Z, Y, X = np.meshgrid(z, y, x, indexing="ij")
                        v = fn(X, Y, Z, g, tl, rng)
                        t = self.data[l][tl][g][c].tensor
                        full = np.zeros(tuple(t.shape))
                        full[:, :, :nx] = v
                        t.copy_(torch.from_numpy(full))


@dataclass
class Phase:
    kind: str          # "prolong", "sync", "restrict"
    level: int         # destination level
    rot: Tuple[int, ...]  # rotation of the levels involved
    ntl: int           # timelevels read (prolongation: 1 or 3)


class BergerOliger:
    """Transfer phases of one coarse step of a nested hierarchy."""

    def __init__(self, h: Hierarchy, st: Storage, order_space=5, order_time=2,
                 op=OP_LAGRANGE, cent=VERTEX, groups: int = 1, stagger: int = 0,
                 chain: bool = False, max_ctas=(0, 0)):
        """``chain``: run a step's phases as one chain (one persistent
        launch, carpet_b200.transfer.Chain) instead of one launch per phase;
        needs groups == 1 (the chain overlaps the grid functions itself)"""
        if not 1 <= groups <= st.ngf:
            raise ValueError("groups must lie in 1..ngf")
        if chain and groups != 1:
            raise ValueError("a chained step runs its grid functions in one launch: groups must be 1")
        self.use_chain = chain
        # CTAs per SM of every batch's TMA / streaming kernels (0: all that fit)
        self.max_ctas = tuple(max_ctas)
        self.chains: Dict[tuple, Chain] = {}
        if stagger < 0:
            raise ValueError("stagger must not be negative")
        self.h, self.st = h, st
        self.groups, self.stagger = groups, stagger
        self._side: List[torch.cuda.Stream] = []
        self.order_space, self.order_time = order_space, order_time
        self.op, self.cent = op, cent
        self.L = len(h.levels)
        self.batches: Dict[tuple, Batch] = {}
        self.rot = [0] * self.L  # cycles of each level modulo ntl

    # which pool holds timelevel tl of level l under rotation r
    def pool_index(self, r: int, tl: int) -> int:
        return bo.pool_index(r, tl, self.st.ntl)

    def _tl(self, l, r, tl):
        return self.st.data[l][self.pool_index(r, tl)]

    def gfs(self, grp: int) -> range:
        """grid functions of group grp (contiguous, sizes differing by one
        at most)"""
        n, G = self.st.ngf, self.groups
        return range(grp * n // G, (grp + 1) * n // G)

    def _build(self, key, grp: int) -> Batch:
        kind, l, rots, ntl = key
        b = Batch()
        h, st = self.h, self.st
        gfs = self.gfs(grp)
        # one dependency group per grid function (a chain keeps each grid
        # function's phases in order and lets the others overlap)
        for g in gfs:
            b.set_group(g)
            if kind == "sync":
                r, = rots
                arrs = self._tl(l, r, 0)
                b.add_many([(arrs[g][p.dst_comp], [arrs[g][p.src_comp]], p.dstbox, p.srcbox)
                            for p in h.sync[l]],
                           [0.0], 0.0, 1, 0, op=self.op, cent=self.cent)
            elif kind == "prolong":
                rf, rc = rots
                dst = self._tl(l, rf, 0)
                srcs = [self._tl(l - 1, rc, t) for t in range(st.ntl)]
                times, time = bo.prolong_times(ntl)
                b.add_many([(dst[g][p.dst_comp], [s[g][p.src_comp] for s in srcs], p.dstbox, p.srcbox)
                            for p in h.prolong[l]],
                           times, time, self.order_space, self.order_time, op=self.op, cent=self.cent)
            elif kind == "restrict":
                rc, rf = rots
                dst = self._tl(l, rc, 0)
                src = self._tl(l + 1, rf, 0)
                b.add_many([(dst[g][p.dst_comp], [src[g][p.src_comp]], p.dstbox, p.srcbox)
                            for p in h.restrict[l + 1]],
                           [0.0], 0.0, self.order_space, 0, op=self.op, cent=self.cent)
        b.set_max_ctas(*self.max_ctas)
        b.upload()
        return b

    def batch(self, key, grp: int = 0) -> Batch:
        """the batch of phase key for grid-function group grp"""
        k = key if grp == 0 else key + (grp,)
        if k not in self.batches:
            self.batches[k] = self._build(key, grp)
        return self.batches[k]

    def group_batches(self, key) -> List[Batch]:
        return [self.batch(key, g) for g in range(self.groups)]

    def step_phases(self) -> List[tuple]:
        """the phases of one coarse step, advancing the rotation state
        (carpet_b200.bo.step_phases)"""
        return bo.step_phases(self.L, self.st.ntl, self.rot)

    def autotune(self, keys, reps=2, stream=None):
        """tile configurations of every phase's prolongation kernels, chosen
        by timing group 0's batch (runs the phases; the groups have the same
        box-pairs); returns {phase: {variant: config}}"""
        out = {}
        for k in dict.fromkeys(keys):
            out[k] = cfg = self.batch(k).autotune(reps, stream)
            for b in self.group_batches(k)[1:]:
                for v, c in cfg.items():
                    b.set_config(c, v)
                b.upload(stream)
        return out

    def set_config(self, keys, config: int, stream=None):
        """pin every prolongation variant of the phases' batches to one tile
        configuration"""
        for k in dict.fromkeys(keys):
            for b in self.group_batches(k):
                b.set_config(config)
                b.upload(stream)

    def chain(self, keys, stream=None) -> Chain:
        """the phases as one chain, built and uploaded on first use"""
        k = tuple(keys)
        if k not in self.chains:
            c = Chain([self.batch(x) for x in keys])
            c.upload(stream)
            self.chains[k] = c
        return self.chains[k]

    def run(self, keys, stream=None, per_box=False, stagger=None):
        """launch the phases in order; with several groups, group g's chain
        runs on its own stream, forked from and joined back into stream
        (which may be capturing a graph).  With stagger > 0 group g starts
        once group 0 has completed g * stagger phases, so that the groups'
        concurrent kernels are of different kinds."""
        if stagger is None:
            stagger = self.stagger

        def launch(b, s):
            if per_box:
                b.launch_per_box(s)
            else:
                b.launch(s)
        if self.use_chain and not per_box:
            self.chain(keys, stream).launch(stream)
            return
        if self.groups == 1:
            for k in keys:
                launch(self.batch(k), stream)
            return
        main = stream if stream is not None else torch.cuda.current_stream()
        while len(self._side) < self.groups - 1:
            self._side.append(torch.cuda.Stream(device=main.device))
        side = self._side[:self.groups - 1]
        fork_at = {min(g * stagger, len(keys)): [] for g in range(1, self.groups)}
        for g in range(1, self.groups):
            fork_at[min(g * stagger, len(keys))].append(g)

        def fork(gs):
            for g in gs:
                s = side[g - 1]
                s.wait_stream(main)
                for k in keys:
                    launch(self.batch(k, g), s)
        for j, k in enumerate(keys):
            fork(fork_at.get(j, []))
            launch(self.batch(k, 0), main)
        fork(fork_at.get(len(keys), []))
        for s in side:
            main.wait_stream(s)

    def stats(self, keys):
        """totals over the phases: box-pairs, tiles, points, algorithmic
        bytes, batches (phases) and kernel launches"""
        tot = dict(pairs=0, tiles=0, points=0, bytes=0, launches=0, kernels=0)
        for k in keys:
            for b in self.group_batches(k):
                s = b.stats()
                for n in ("pairs", "tiles", "points", "bytes"):
                    tot[n] += s[n]
                tot["launches"] += 1
                tot["kernels"] += b.kernels()
        return tot
