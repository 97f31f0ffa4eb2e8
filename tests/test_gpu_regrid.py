"""Regridding a moving-box hierarchy: the old-to-new fill of every refined
level and timelevel (copies from the old level, order-5 prolongation from the
refilled coarser level), run as batches and as one CUDA graph on the GPU,
bit-identical to the oracle applying the same schedule, and covering every
point of the new components."""
import numpy as np
import pytest

from carpet_b200.moving import MovingSpec, build, old2new

SPEC = MovingSpec(nlevels=3, n0=65, nbox=33, parts0=(2, 1, 1), parts=(1, 2, 1), ghost=3, buffer=3,
                  order=5)


def test_moving_schedules_cover_every_point():
    """host side only: both hierarchies are consistent and the fill covers
    each new component's exterior exactly once with copies and prolongations"""
    h0, h1 = build(SPEC, 0), build(SPEC, SPEC.regrid_every)
    kinds = set()
    for l in range(1, SPEC.nlevels):
        assert h0.boxes[l] != h1.boxes[l]  # the regions moved
        copies, prols = old2new(h0, h1, l)  # asserts exact coverage
        kinds |= {"copy"} if copies else set()
        kinds |= {"prolong"} if prols else set()
    assert kinds == {"copy", "prolong"}


@pytest.mark.gpu
def test_regrid_fill_matches_oracle(port):
    torch = pytest.importorskip("torch")
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    import carpet_b200 as cb
    from carpet_b200.amr import Storage
    from carpet_b200.moving import Regrid
    from oracle.binding import OP_LAGRANGE, VERTEX
    cb.set_fp_mode(False)
    ngf, ntl = 2, 3
    h0, h1 = build(SPEC, 0), build(SPEC, SPEC.regrid_every)
    old = Storage(h0, ngf, ntl)
    rng = np.random.default_rng(21)
    for lp in old.pools:
        for p in lp:
            p.copy_(torch.from_numpy(rng.standard_normal(p.numel())))
    new = Storage(h1, ngf, ntl, share=old, shared_levels=(0,))
    for l in range(1, SPEC.nlevels):
        for p in new.pools[l]:
            p.fill_(float("nan"))
    # oracle state: numpy copies of every array
    onp = [[[[d.tensor.cpu().numpy().copy() for d in comps] for comps in gfs] for gfs in lev]
           for lev in old.data]
    nnp = [[[[d.tensor.cpu().numpy().copy() for d in comps] for comps in gfs] for gfs in lev]
           for lev in new.data]
    for l in range(1, SPEC.nlevels):
        copies, prols = old2new(h0, h1, l)
        for tl in range(ntl):
            for g in range(ngf):
                for p in copies:
                    port.transfer(OP_LAGRANGE, VERTEX, nnp[l][tl][g][p.dst_comp],
                                  h1.levels[l].comps[p.dst_comp].exterior,
                                  [onp[l][tl][g][p.src_comp]], h0.levels[l].comps[p.src_comp].exterior,
                                  [0.0], p.dstbox, p.srcbox, 0.0, 1, 0)
                for p in prols:
                    port.transfer(OP_LAGRANGE, VERTEX, nnp[l][tl][g][p.dst_comp],
                                  h1.levels[l].comps[p.dst_comp].exterior,
                                  [nnp[l - 1][tl][g][p.src_comp]],
                                  h1.levels[l - 1].comps[p.src_comp].exterior,
                                  [0.0], p.dstbox, p.srcbox, 0.0, 5, 0)
    rg = Regrid(h0, h1, ngf, ntl, lambda l, tl: old.data[l][tl], lambda l, tl: new.data[l][tl])
    for autotune in (False, True):
        for l in range(1, SPEC.nlevels):
            for p in new.pools[l]:
                p.fill_(float("nan"))
        rg.upload(autotune=autotune)
        for l in range(1, SPEC.nlevels):  # autotuning ran the fill: start over
            for p in new.pools[l]:
                p.fill_(float("nan"))
        s = torch.cuda.Stream()
        torch.cuda.synchronize()
        g = rg.graph(s)
        g.launch(s)
        s.synchronize()
        for b in rg.batches:
            b.check(s)
        for l in range(1, SPEC.nlevels):
            for tl in range(ntl):
                for gf in range(ngf):
                    for c, comp in enumerate(h1.levels[l].comps):
                        got = new.data[l][tl][gf][c].tensor.cpu().numpy()
                        want = nnp[l][tl][gf][c]
                        assert np.array_equal(got.view(np.uint64), want.view(np.uint64)), (l, tl, c)
                        nx = (comp.exterior[3] - comp.exterior[0]) // comp.exterior[6] + 1
                        assert not np.isnan(got[:, :, :nx]).any(), (l, tl, c)
