"""Uneven mixed batches: many independent box-pairs of different sizes and
operators in one persistent-kernel launch.

``uneven_batch`` builds the workload of the batched benchmark configuration:
``npairs`` box-pairs, each with its own source and destination arrays, the
fine extent of every pair drawn per axis from U{lo..hi}, the operators mixed
40% vertex-centred Lagrange order 5, 20% vertex-centred ENO order 3, 20%
cell-centred Lagrange order 3 (prolongate_3d_cc_rf2) and 20% cell-centred
averaging restriction (restrict_3d_cc_rf2).  Index-space conventions follow
CarpetLib's: vertex-centred levels have strides 2 (coarse) and 1 (fine) with
coincident points; cell-centred levels have strides 4 and 2 with coarse
points at 4n+2 and fine points at 2m+1 (the cell centres).

Field values are the cubic of the two-level test, sum_{i+j+k<=3} c_ijk x^i
y^j z^k with seeded c_ijk ~ U(-1,1), evaluated on each source array.
"""
from __future__ import annotations

import itertools
from dataclasses import dataclass
from typing import List, Sequence

import numpy as np
import torch

from .transfer import OP_ENO, OP_LAGRANGE, VERTEX, CELL, Batch, Data

KINDS = ("vc_lagrange5", "vc_eno3", "cc_lagrange3", "cc_average")
MIX = (0.4, 0.2, 0.2, 0.2)


@dataclass
class PairSpec:
    """one box-pair: operator, source and destination extents, region"""
    kind: str
    op: int
    cent: int
    order: int
    srcbbox: tuple
    dstbbox: tuple
    reg: tuple


@dataclass
class UnevenPair:
    spec: PairSpec
    dst: Data
    src: Data


def _box(lo, up, st):
    return tuple(int(v) for v in (*lo, *up, *st))


def cubic_coeffs(seed):
    rng = np.random.default_rng(seed)
    terms = [t for t in itertools.product(range(4), repeat=3) if sum(t) <= 3]
    return terms, rng.uniform(-1, 1, len(terms))


def cubic_values(b, terms, coef, scale: float = 256.0, lib=np):
    """the cubic on the points of bbox b, shape (nz, ny, nx)"""
    n = [(b[3 + k] - b[k]) // b[6 + k] + 1 for k in range(3)]
    kw = dict(dtype=lib.float64)
    if lib is torch:
        kw["device"] = "cuda"
    x = (b[0] + lib.arange(n[0], **kw) * b[6]) / scale
    y = (b[1] + lib.arange(n[1], **kw) * b[7]) / scale
    z = (b[2] + lib.arange(n[2], **kw) * b[8]) / scale
    Z, Y, X = lib.meshgrid(z, y, x, indexing="ij")
    v = lib.zeros_like(X)
    for c, (i, j, k) in zip(coef, terms):
        v = v + float(c) * X ** i * Y ** j * Z ** k
    return v


def uneven_specs(seed: int = 3, npairs: int = 256, ext=(16, 96),
                 mix: Sequence[float] = MIX) -> List[PairSpec]:
    rng = np.random.default_rng(seed)
    counts = [int(round(m * npairs)) for m in mix]
    counts[0] += npairs - sum(counts)
    kinds = [k for k, c in zip(KINDS, counts) for _ in range(c)]
    rng.shuffle(kinds)
    specs = []
    for kind in kinds:
        e = rng.integers(ext[0], ext[1] + 1, 3)
        if kind in ("vc_lagrange5", "vc_eno3"):
            order, op = (5, OP_LAGRANGE) if kind == "vc_lagrange5" else (3, OP_ENO)
            lo, hi = (-2, 3) if order == 5 else (-1, 2)  # stencil window around c = s >> 1
            flo = rng.integers(-64, 64, 3)
            fup = flo + e - 1
            reg = _box(flo, fup, (1, 1, 1))
            clo = np.floor_divide(flo, 2) + lo - 1
            cup = np.floor_divide(fup, 2) + hi + 1
            srcb = _box(2 * clo, 2 * cup, (2, 2, 2))
            dstb = _box(flo - 2, fup + 2, (1, 1, 1))
            cent = VERTEX
        elif kind == "cc_lagrange3":
            order, op, cent = 3, OP_LAGRANGE, CELL
            flo = 2 * rng.integers(-32, 32, 3) + 1
            fup = flo + 2 * (e - 1)
            reg = _box(flo, fup, (2, 2, 2))
            c_lo = np.floor_divide(flo - 2, 4) - 3
            c_up = np.floor_divide(fup - 2, 4) + 4
            srcb = _box(4 * c_lo + 2, 4 * c_up + 2, (4, 4, 4))
            dstb = _box(flo - 4, fup + 4, (2, 2, 2))
        else:  # averaging restriction onto a coarse box of half the extent
            order, op, cent = 0, OP_LAGRANGE, CELL
            ce = np.maximum(e // 2, 1)
            clo = 4 * rng.integers(-16, 16, 3) + 2
            cup = clo + 4 * (ce - 1)
            reg = _box(clo, cup, (4, 4, 4))
            srcb = _box(clo - 3, cup + 3, (2, 2, 2))
            dstb = _box(clo - 4, cup + 4, (4, 4, 4))
        specs.append(PairSpec(kind, op, cent, order, srcb, dstb, reg))
    return specs


def uneven_pairs(specs: List[PairSpec], seed: int = 4, device="cuda") -> List[UnevenPair]:
    """device arrays for the specs: sources hold the cubic, destinations NaN"""
    terms, coef = cubic_coeffs(seed)
    pairs = []
    for sp in specs:
        src = Data(sp.srcbbox, device=device)
        dst = Data(sp.dstbbox, device=device)
        v = cubic_values(sp.srcbbox, terms, coef, lib=torch)
        src.tensor.zero_()
        src.tensor[:, :, :v.shape[2]] = v
        dst.tensor.fill_(float("nan"))
        pairs.append(UnevenPair(sp, dst, src))
    return pairs


def uneven_batch(pairs: List[UnevenPair]) -> Batch:
    """one batch holding every pair (one timelevel, time 0)"""
    b = Batch()
    for p in pairs:
        sp = p.spec
        b.add(p.dst, [p.src], [0.0], sp.reg, sp.srcbbox, 0.0, sp.order, 0, op=sp.op, cent=sp.cent)
    return b


def main(argv=None):
    """``python -m carpet_b200.uneven``: the 256-pair uneven batch alone
    (autotuned or pinned tiles, one graph replay per step), printed as one
    JSON line -- the workload the profiles of the mixed batch are taken on"""
    import argparse
    import json

    from . import transfer
    from .transfer import Graph

    p = argparse.ArgumentParser(prog="python -m carpet_b200.uneven")
    p.add_argument("--pairs", type=int, default=256)
    p.add_argument("--steps", type=int, default=20)
    p.add_argument("--warmup", type=int, default=3)
    p.add_argument("--tile-config", type=int, default=None,
                   help="pin every prolongation variant to this configuration instead of tuning")
    p.add_argument("--fp", default="exact", choices=["exact", "fma"])
    a = p.parse_args(argv)
    transfer.set_fp_mode(a.fp == "fma")
    pairs = uneven_pairs(uneven_specs(seed=3, npairs=a.pairs, ext=(16, 96)), seed=4)
    b = uneven_batch(pairs)
    st = b.stats()
    if a.tile_config is None:
        configs = sorted(set(b.autotune(reps=3).values()))
    else:
        b.set_config(a.tile_config)
        b.upload()
        configs = [a.tile_config]
    s = torch.cuda.Stream()
    g = Graph()
    with g.capture(s):
        b.launch(s)
    for _ in range(a.warmup):
        g.launch(s)
    s.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(s)
    for _ in range(a.steps):
        g.launch(s)
    e1.record(s)
    s.synchronize()
    b.check(s)
    ms = e0.elapsed_time(e1) / a.steps
    print(json.dumps({"pairs": st["pairs"], "fine_points": st["points"], "bytes": st["bytes"],
                      "ms": round(ms, 4), "gbs": round(st["bytes"] / (ms * 1e-3) / 1e9, 1),
                      "tile_configs": configs, "fp_mode": a.fp}))
    del g


if __name__ == "__main__":
    main()
