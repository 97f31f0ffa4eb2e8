"""Seeded synthetic box-pair cases for the parity tests (TEST INFRASTRUCTURE).

Each generator returns a dict describing one call of a CarpetLib operator:
source/destination arrays (numpy, stored (nz, ny, nx_pad), x fastest), their
bboxes and the region.  Geometry follows the reference's conventions:

* vertex-centred: a level with stride s has points at multiples of s; the
  coarse level has stride 2s (prolongate_3d_rf2.cc:377-387);
* cell-centred: fine stride fs = 2h (even, prolongate_3d_cc_rf2.cc:264),
  fine points at fs*m + h, coarse points (stride 2fs) at 2fs*n + fs, so a
  coarse cell centre sits halfway between two fine cell centres.

Source boxes are always large enough for the operator's full stencil, with a
random margin, so that no operator reads outside its source array.
"""
from __future__ import annotations

import numpy as np

from .binding import alloc, box_sizes


def _fill(rng, a, kind="normal"):
    if kind == "normal":
        a[...] = rng.standard_normal(a.shape)
    elif kind == "mixed":
        # magnitudes spread over many decades, signed zeros, exact integers
        v = rng.standard_normal(a.shape) * 10.0 ** rng.integers(-8, 8, a.shape)
        m = rng.random(a.shape)
        v[m < 0.05] = -0.0
        v[(m >= 0.05) & (m < 0.1)] = 0.0
        sel = (m >= 0.1) & (m < 0.2)
        v[sel] = rng.integers(-50, 50, int(sel.sum())).astype(np.float64)
        a[...] = v
    elif kind == "steps":
        # piecewise-constant with jumps: exercises the ENO limiters
        a[...] = np.sign(rng.standard_normal(a.shape)) * rng.integers(
            0, 3, a.shape).astype(np.float64)
    elif kind == "smooth":
        # smooth fields whose undivided differences keep their sign over
        # stretches and change it elsewhere: every ENO stencil choice occurs
        z, y, x = np.meshgrid(*[np.arange(n, dtype=np.float64) for n in a.shape], indexing="ij")
        g = rng.uniform(-0.5, 0.5, 3)
        f = rng.uniform(0.1, 0.9, 3)
        a[...] = np.exp(g[0] * x + g[1] * y + g[2] * z) + 0.3 * np.sin(
            f[0] * x + f[1] * y + f[2] * z + rng.uniform(0, 6.3))
    else:
        raise ValueError(kind)
    return a


def _box(lo, up, st):
    return [int(x) for x in (*lo, *up, *st)]


def vc_prolong_case(rng, order, fine_stride=1, max_ext=9, kind="normal",
                    reach=None, margin=2):
    """A vertex-centred rf2 prolongation (Lagrange of ``order`` or ENO with
    ``reach`` = (below, above) coarse points of stencil)."""
    fs, cs = fine_stride, 2 * fine_stride
    if reach is None:
        reach = (order // 2, order // 2 + 1)  # coeffs1d::imin..imax-1
    ext = rng.integers(1, max_ext + 1, 3)
    lo = rng.integers(-20, 20, 3) * fs
    up = lo + (ext - 1) * fs
    reg = _box(lo, up, (fs,) * 3)
    # coarse coverage of the stencil, then a random margin
    clo = np.floor_divide(lo, cs) - reach[0] - rng.integers(0, margin + 1, 3)
    cup = np.floor_divide(up, cs) + reach[1] + 1 + rng.integers(0, margin + 1, 3)
    srcbbox = _box(clo * cs, cup * cs, (cs,) * 3)
    dlo = lo - rng.integers(0, 3, 3) * fs
    dup = up + rng.integers(0, 3, 3) * fs
    dstbbox = _box(dlo, dup, (fs,) * 3)
    src = _fill(rng, alloc(srcbbox), kind)
    dst = alloc(dstbbox, fill=np.nan)
    return dict(src=src, srcbbox=srcbbox, dst=dst, dstbbox=dstbbox, reg=reg)


def cc_prolong_case(rng, order, half=1, max_ext=9, kind="normal", margin=2):
    """A cell-centred rf2 prolongation of ``order``."""
    h = half
    fs, cs = 2 * h, 4 * h
    ext = rng.integers(1, max_ext + 1, 3)
    m0 = rng.integers(-20, 20, 3)
    lo = m0 * fs + h
    up = lo + (ext - 1) * fs
    reg = _box(lo, up, (fs,) * 3)
    n = order + 1
    # coarse index of the fine point p: (p - fs)/cs rounded toward the cell
    # that holds it; the stencil reaches n/2+1 cells either way
    c_lo = np.floor_divide(lo - fs, cs) - (n // 2 + 1) - rng.integers(0, margin + 1, 3)
    c_up = np.floor_divide(up - fs, cs) + (n // 2 + 2) + rng.integers(0, margin + 1, 3)
    srcbbox = _box(c_lo * cs + fs, c_up * cs + fs, (cs,) * 3)
    dlo = lo - rng.integers(0, 3, 3) * fs
    dup = up + rng.integers(0, 3, 3) * fs
    dstbbox = _box(dlo, dup, (fs,) * 3)
    src = _fill(rng, alloc(srcbbox), kind)
    dst = alloc(dstbbox, fill=np.nan)
    return dict(src=src, srcbbox=srcbbox, dst=dst, dstbbox=dstbbox, reg=reg)


def vc_restrict_case(rng, fine_stride=1, max_ext=9, kind="normal"):
    """Vertex-centred injection: coarse region inside fine source."""
    fs, cs = fine_stride, 2 * fine_stride
    ext = rng.integers(1, max_ext + 1, 3)
    lo = rng.integers(-10, 10, 3) * cs
    up = lo + (ext - 1) * cs
    reg = _box(lo, up, (cs,) * 3)
    slo = lo - rng.integers(0, 3, 3) * fs
    sup = up + rng.integers(0, 3, 3) * fs
    srcbbox = _box(slo, sup, (fs,) * 3)
    dlo = lo - rng.integers(0, 3, 3) * cs
    dup = up + rng.integers(0, 3, 3) * cs
    dstbbox = _box(dlo, dup, (cs,) * 3)
    src = _fill(rng, alloc(srcbbox), kind)
    dst = alloc(dstbbox, fill=np.nan)
    return dict(src=src, srcbbox=srcbbox, dst=dst, dstbbox=dstbbox, reg=reg)


def cc_restrict_case(rng, half=1, max_ext=9, kind="normal", reach=(0, 0)):
    """Cell-centred averaging: coarse cells (stride 4h at 4h*n + 2h) over
    fine cells (stride 2h at 2h*m + h); ``reach`` = fine cells the stencil
    needs below / above a coarse cell's two children (the higher-order
    restrictions: (1, 1) for order 3, (2, 2) for order 5)."""
    h = half
    fs, cs = 2 * h, 4 * h
    ext = rng.integers(1, max_ext + 1, 3)
    n0 = rng.integers(-10, 10, 3)
    lo = n0 * cs + fs
    up = lo + (ext - 1) * cs
    reg = _box(lo, up, (cs,) * 3)
    # fine children of coarse cell c are c - h and c + h
    slo = lo - h - (reach[0] + rng.integers(0, 3, 3)) * fs
    sup = up + h + (reach[1] + rng.integers(0, 3, 3)) * fs
    srcbbox = _box(slo, sup, (fs,) * 3)
    dlo = lo - rng.integers(0, 3, 3) * cs
    dup = up + rng.integers(0, 3, 3) * cs
    dstbbox = _box(dlo, dup, (cs,) * 3)
    src = _fill(rng, alloc(srcbbox), kind)
    dst = alloc(dstbbox, fill=np.nan)
    return dict(src=src, srcbbox=srcbbox, dst=dst, dstbbox=dstbbox, reg=reg)


def copy_case(rng, stride=1, max_ext=9, slab=False, kind="normal"):
    """Same-stride copy; with ``slab`` the source region is the destination
    region shifted by a random offset (copy_3d.cc:57-58)."""
    s = stride
    ext = rng.integers(1, max_ext + 1, 3)
    lo = rng.integers(-10, 10, 3) * s
    up = lo + (ext - 1) * s
    dstreg = _box(lo, up, (s,) * 3)
    off = rng.integers(-4, 5, 3) if slab else np.zeros(3, int)
    slo, sup = lo + off * s, up + off * s
    srcbbox = _box(slo - rng.integers(0, 3, 3) * s, sup + rng.integers(0, 3, 3) * s,
                   (s,) * 3)
    dstbbox = _box(lo - rng.integers(0, 3, 3) * s, up + rng.integers(0, 3, 3) * s,
                   (s,) * 3)
    srcreg = _box(slo, sup, (s,) * 3)
    src = _fill(rng, alloc(srcbbox), kind)
    dst = alloc(dstbbox, fill=np.nan)
    return dict(src=src, srcbbox=srcbbox, dst=dst, dstbbox=dstbbox,
                srcreg=srcreg if slab else dstreg, dstreg=dstreg, reg=dstreg,
                slab=[int(x) for x in off] if slab else None)


def time_case(rng, ntl, stride=1, max_ext=9, kind="normal"):
    """Time interpolation between ``ntl`` same-shaped timelevels.  Times are
    t, t-dt, t-2dt as the timelevels are ordered in CarpetLib; the target time
    lies inside their span."""
    s = stride
    ext = rng.integers(1, max_ext + 1, 3)
    lo = rng.integers(-10, 10, 3) * s
    up = lo + (ext - 1) * s
    reg = _box(lo, up, (s,) * 3)
    srcbbox = _box(lo - rng.integers(0, 3, 3) * s, up + rng.integers(0, 3, 3) * s,
                   (s,) * 3)
    dstbbox = _box(lo - rng.integers(0, 3, 3) * s, up + rng.integers(0, 3, 3) * s,
                   (s,) * 3)
    t0 = float(rng.uniform(-2.0, 2.0))
    dt = float(rng.uniform(0.01, 0.5))
    times = [t0 - i * dt for i in range(ntl)]
    t = float(rng.uniform(times[-1], times[0]))
    srcs = [_fill(rng, alloc(srcbbox), kind) for _ in range(ntl)]
    dst = alloc(dstbbox, fill=np.nan)
    return dict(srcs=srcs, times=times, t=t, srcbbox=srcbbox, dst=dst,
                dstbbox=dstbbox, reg=reg)


def region_view(a, bbox, reg):
    """The part of array ``a`` (with bbox) covered by region ``reg``."""
    sz = box_sizes(reg)
    off = [(reg[d] - bbox[d]) // bbox[6 + d] for d in range(3)]
    return a[off[2]:off[2] + sz[2], off[1]:off[1] + sz[1], off[0]:off[0] + sz[0]]
