"""The CPU-runnable two-level case (CarpetProlongateTest-style).

A coarse 33^3 vertex-centred level and a fine level covering its central
half (33^3 fine points, split into two components along x), ghost width 3,
buffer width 3.  One grid function: the cubic sum_{i+j+k<=3} c_ijk x^i y^j z^k
with seeded c_ijk ~ U(-1,1).  The transfers are those of one coarse step of
this hierarchy: order-3 Lagrange prolongation into the fine ghost + buffer
shell, injection back onto the coarse points under the fine active region,
and the copy_3d ghost sync between the two fine components.

Order-3 Lagrange prolongation reproduces a cubic to roundoff, injection and
copy move exact values, so every destination point must hold the polynomial
(to a few ulp of its magnitude).  The GPU test runs the same schedule
through the library, batched and per box, and requires it bit-identical to
the oracle.
"""
import itertools

import numpy as np
import pytest

from carpet_b200.hierarchy import nested, size
from oracle.binding import OP_LAGRANGE, VERTEX

N = 33


def hierarchy():
    return nested(2, N, parts=[(1, 1, 1), (2, 1, 1)], ghost=3, buffer=3, order=3)


def cubic(seed=7):
    rng = np.random.default_rng(seed)
    terms = [(i, j, k) for i, j, k in itertools.product(range(4), repeat=3) if i + j + k <= 3]
    c = rng.uniform(-1, 1, len(terms))
    scale = float((N - 1) * 2)  # the coarse level spans [0, 1] in x, y, z

    def f(b):
        nx, ny, nz = size(b)
        x = (b[0] + np.arange(nx) * b[6]) / scale
        y = (b[1] + np.arange(ny) * b[7]) / scale
        z = (b[2] + np.arange(nz) * b[8]) / scale
        Z, Y, X = np.meshgrid(z, y, x, indexing="ij")
        return sum(ci * X ** i * Y ** j * Z ** k for ci, (i, j, k) in zip(c, terms))
    return f


def padded(v):
    """an (nz, ny, nx) array with x padded to an even length"""
    nz, ny, nx = v.shape
    out = np.full((nz, ny, nx + (nx & 1)), np.nan)
    out[:, :, :nx] = v
    return out


def setup(h, f):
    """coarse: the polynomial everywhere; fine: the polynomial on each
    component's interior minus the outer ghost + buffer shell, NaN elsewhere
    (what prolongation and sync must fill)"""
    coarse = [padded(f(c.exterior)) for c in h.levels[0].comps]
    fine = []
    w = h.ghost + h.buffer
    fb = h.levels[1].box
    for c in h.levels[1].comps:
        v = np.full(padded(f(c.exterior)).shape, np.nan)
        exact = f(c.exterior)
        e = c.exterior
        nx, ny, nz = size(e)
        for kk in range(nz):
            for jj in range(ny):
                for ii in range(nx):
                    p = (e[0] + ii * e[6], e[1] + jj * e[7], e[2] + kk * e[8])
                    inside = all(c.interior[d] <= p[d] <= c.interior[3 + d] for d in range(3))
                    active = all(fb[d] + w * fb[6 + d] <= p[d] <= fb[3 + d] - w * fb[6 + d]
                                 for d in range(3))
                    if inside and active:
                        v[kk, jj, ii] = exact[kk, jj, ii]
        fine.append(v)
    return coarse, fine


def run_oracle(port, h, coarse, fine):
    l0, l1 = h.levels
    for p in h.prolong[1]:
        port.transfer(OP_LAGRANGE, VERTEX, fine[p.dst_comp], l1.comps[p.dst_comp].exterior,
                      [coarse[p.src_comp]], l0.comps[p.src_comp].exterior, [0.0], p.dstbox,
                      p.srcbox, 0.0, 3, 0)
    for p in h.sync[1]:
        port.transfer(OP_LAGRANGE, VERTEX, fine[p.dst_comp], l1.comps[p.dst_comp].exterior,
                      [fine[p.src_comp]], l1.comps[p.src_comp].exterior, [0.0], p.dstbox,
                      p.srcbox, 0.0, 1, 0)
    for p in h.restrict[1]:
        port.transfer(OP_LAGRANGE, VERTEX, coarse[p.dst_comp], l0.comps[p.dst_comp].exterior,
                      [fine[p.src_comp]], l1.comps[p.src_comp].exterior, [0.0], p.dstbox,
                      p.srcbox, 0.0, 3, 0)


def check_polynomial(h, f, coarse, fine):
    for lev, arrs in ((h.levels[0], coarse), (h.levels[1], fine)):
        for c, v in zip(lev.comps, arrs):
            want = f(c.exterior)
            got = v[:, :, :want.shape[2]]
            assert not np.isnan(got).any(), "a destination point was not written"
            tol = 64 * np.finfo(float).eps * max(1.0, np.abs(want).max())
            assert np.abs(got - want).max() <= tol


def test_config1_oracle_reproduces_cubic(port):
    h = hierarchy()
    assert len(h.levels[1].comps) == 2 and size(h.levels[1].box) == (N, N, N)
    f = cubic()
    coarse, fine = setup(h, f)
    run_oracle(port, h, coarse, fine)
    check_polynomial(h, f, coarse, fine)


@pytest.mark.gpu
@pytest.mark.parametrize("form", ["batch", "per_box"])
def test_config1_gpu_matches_oracle(port, form):
    torch = pytest.importorskip("torch")
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    import carpet_b200 as cb
    cb.set_fp_mode(False)
    h = hierarchy()
    f = cubic()
    coarse, fine = setup(h, f)
    dc = [cb.Data(c.exterior, torch.from_numpy(a.copy()).cuda()) for c, a in zip(h.levels[0].comps, coarse)]
    df = [cb.Data(c.exterior, torch.from_numpy(a.copy()).cuda()) for c, a in zip(h.levels[1].comps, fine)]
    run_oracle(port, h, coarse, fine)
    phases = [
        [(df[p.dst_comp], dc[p.src_comp], p, 3) for p in h.prolong[1]],
        [(df[p.dst_comp], df[p.src_comp], p, 1) for p in h.sync[1]],
        [(dc[p.dst_comp], df[p.src_comp], p, 3) for p in h.restrict[1]],
    ]
    for ph in phases:
        b = cb.Batch()
        for dst, src, p, order in ph:
            b.add(dst, [src], [0.0], p.dstbox, p.srcbox, 0.0, order, 0)
        b.upload()
        if form == "batch":
            b.launch()
        else:
            b.launch_per_box()
        b.check()
    torch.cuda.synchronize()
    got_c = [d.tensor.cpu().numpy() for d in dc]
    got_f = [d.tensor.cpu().numpy() for d in df]
    for g, w in zip(got_c + got_f, coarse + fine):
        assert np.array_equal(np.nan_to_num(g, nan=7.0).view(np.uint64),
                              np.nan_to_num(w, nan=7.0).view(np.uint64))
    check_polynomial(h, f, got_c, got_f)
