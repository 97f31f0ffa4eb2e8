"""Full-size checks on the benchmark workload: 5 vertex-centred levels of
129^3 points, each split into 2x2x2 components, 3 timelevels, ghost 3,
buffer 9, order-5 Lagrange prolongation with quadratic time interpolation,
injection and ghost sync -- one coarse Berger-Oliger step, FMA mode.

* the whole step on the device for every grid function, and the oracle's
  replay of the same phases for a sample of grid functions (grid functions
  never mix, so each is a full-size parity case): bit-exact;
* a separable cubic field is reproduced exactly by every operator on the
  path (Lagrange of order 5 holds cubics, the time weights of equal
  timelevels sum to one, and every intermediate value is an exactly
  representable integer multiple of a power of two), so two whole steps
  leave every point of every array bit-identical;
* the batched kernels (TMA-staged prolongation, persistent streaming
  kernels) and the per-box kernels (cp.async-staged prolongation, per-box
  streaming) give the same bits on the whole step;
* the grid functions split into groups whose phase chains run on separate
  streams (eagerly and captured as one graph, the groups started together
  or staggered by whole phases) give the same bits as one chain over all
  of them;
* with CarpetLib's own region lists (carpet_b200.dh: the outer ghost
  layer's internal ghost points prolongated instead of synced, restriction
  into the coarse ghost zones too) the step matches the oracle's replay of
  those lists, and gives the same bits as the box hierarchy's lists: a
  prolongated point and a synced copy of a prolongated point are the same
  value, and so are a restricted ghost point and the sync that overwrites
  it.
"""
import numpy as np
import pytest

from oracle.binding import OP_LAGRANGE, VERTEX

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")

LEVELS, NPOINTS = 5, 129


@pytest.fixture(scope="module")
def cgx():
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    import carpet_b200 as cb
    return cb


def workload(cb, ngf, fill, groups=1, schedule="regular", fma=True):
    from carpet_b200.amr import BergerOliger, Storage
    from carpet_b200.hierarchy import nested
    cb.set_fp_mode(fma)
    h = nested(LEVELS, NPOINTS, ghost=3, buffer=9, order=5, schedule=schedule)
    st = Storage(h, ngf, 3)
    fill(st, h)
    bo = BergerOliger(h, st, order_space=5, order_time=2, groups=groups)
    return h, st, bo


def random_fill(st, h):
    gen = torch.Generator(device="cuda")
    gen.manual_seed(7)
    for lp in st.pools:
        for p in lp:
            p.normal_(generator=gen)


def consistent_fill(st, h):
    """random values that are a function of the global point: every ghost
    zone holds its neighbours' values, as in any state a run reaches (the
    schedules may then take a point from either component)"""
    gen = torch.Generator(device="cuda")
    gen.manual_seed(11)
    for lp in st.pools:  # padding and the gaps between arrays: zero in every storage
        for p in lp:
            p.zero_()
    for l, lev in enumerate(h.levels):
        box = lev.box
        n = [(box[3 + d] - box[d]) // box[6 + d] + 1 for d in range(3)]
        for tl in range(st.ntl):
            for g in range(st.ngf):
                G = torch.randn((n[2], n[1], n[0]), generator=gen, device="cuda", dtype=torch.float64)
                for c, comp in enumerate(lev.comps):
                    e = comp.exterior
                    o = [(e[d] - box[d]) // box[6 + d] for d in range(3)]
                    m = [(e[3 + d] - e[d]) // e[6 + d] + 1 for d in range(3)]
                    st.data[l][tl][g][c].tensor[:, :, :m[0]] = \
                        G[o[2]:o[2] + m[2], o[1]:o[1] + m[1], o[0]:o[0] + m[0]]


def cubic_fill(st, h):
    """p(x) + q(y) + r(z), cubics with small integer coefficients in the
    global integer coordinates (at most 2048): values below 2^36; the same
    on every timelevel, different on every grid function"""
    for l, lev in enumerate(h.levels):
        for tl in range(st.ntl):
            for g in range(st.ngf):
                for c, comp in enumerate(lev.comps):
                    b = comp.exterior
                    t = st.data[l][tl][g][c].tensor
                    nz, ny = t.shape[0], t.shape[1]
                    nx = (b[3] - b[0]) // b[6] + 1
                    x = (b[0] + torch.arange(nx, device="cuda", dtype=torch.float64) * b[6])
                    y = (b[1] + torch.arange(ny, device="cuda", dtype=torch.float64) * b[7])
                    z = (b[2] + torch.arange(nz, device="cuda", dtype=torch.float64) * b[8])
                    px = 2 * x ** 3 - 3 * x ** 2 + x + g
                    qy = y ** 3 + 5 * y ** 2 - 7 * y
                    rz = -z ** 3 + 2 * z ** 2 + 3 * z
                    t[:, :, :nx] = rz[:, None, None] + qy[None, :, None] + px[None, None, :]


def host_copy(st, gfs):
    return {g: [[[st.data[l][p][g][c].tensor.cpu().numpy().copy()
                  for c in range(len(st.data[l][p][g]))] for p in range(st.ntl)]
                for l in range(len(st.data))] for g in gfs}


def oracle_phase(port, h, arr, key, fma=True):
    """one phase of BergerOliger on one grid function's host arrays
    arr[level][pool][comp], in the batches' own terms (carpet_b200.amr)"""
    kind, l, rots, ntl = key
    pool = lambda r, tl: (tl - r) % 3
    ext = lambda lv, c: list(h.levels[lv].comps[c].exterior)
    if kind == "sync":
        r, = rots
        a = arr[l][pool(r, 0)]
        for p in h.sync[l]:
            port.transfer(OP_LAGRANGE, VERTEX, a[p.dst_comp], ext(l, p.dst_comp), [a[p.src_comp]],
                          ext(l, p.src_comp), [0.0], list(p.dstbox), list(p.srcbox), 0.0, 1, 0,
                          fma=fma)
    elif kind == "prolong":
        rf, rc = rots
        dst = arr[l][pool(rf, 0)]
        srcs = [arr[l - 1][pool(rc, t)] for t in range(3)]
        dtc = 1.0 / 64
        times, time = [0.0, -dtc, -2 * dtc], (-dtc / 2 if ntl > 1 else 0.0)
        for p in h.prolong[l]:
            port.transfer(OP_LAGRANGE, VERTEX, dst[p.dst_comp], ext(l, p.dst_comp),
                          [s[p.src_comp] for s in srcs], ext(l - 1, p.src_comp), times,
                          list(p.dstbox), list(p.srcbox), time, 5, 2, fma=fma)
    else:
        rc, rf = rots
        dst, src = arr[l][pool(rc, 0)], arr[l + 1][pool(rf, 0)]
        for p in h.restrict[l + 1]:
            port.transfer(OP_LAGRANGE, VERTEX, dst[p.dst_comp], ext(l, p.dst_comp),
                          [src[p.src_comp]], ext(l + 1, p.src_comp), [0.0], list(p.dstbox),
                          list(p.srcbox), 0.0, 5, 0, fma=fma)


@pytest.mark.parametrize("schedule,fma", [("regular", True), ("dh", False)])
def test_bench_step_matches_oracle_on_sampled_grid_functions(cgx, port, schedule, fma):
    ngf = 25 if schedule == "regular" else 4
    h, st, bo = workload(cgx, ngf, random_fill, schedule=schedule, fma=fma)
    gfs = (0, ngf - 1)
    want = host_copy(st, gfs)
    keys = bo.step_phases()
    bo.run(keys)
    for b in bo.batches.values():
        b.check()
    torch.cuda.synchronize()
    got = host_copy(st, gfs)
    for g in gfs:
        for k in keys:
            oracle_phase(port, h, want[g], k, fma=fma)
        for l in range(LEVELS):
            for p in range(3):
                for c, a in enumerate(want[g][l][p]):
                    assert np.array_equal(a.view(np.uint64), got[g][l][p][c].view(np.uint64)), \
                        ("grid function", g, "level", l, "pool", p, "component", c)


def test_cubic_field_survives_two_steps_bit_exact(cgx):
    h, st, bo = workload(cgx, 4, cubic_fill)
    before = [[p.clone() for p in lp] for lp in st.pools]
    for _ in range(2):
        keys = bo.step_phases()
        bo.run(keys)
    for b in bo.batches.values():
        b.check()
    torch.cuda.synchronize()
    for l, (lp, bp) in enumerate(zip(st.pools, before)):
        for p, q in zip(lp, bp):
            assert torch.equal(p.view(torch.int64), q.view(torch.int64)), ("level", l)


def test_batched_and_per_box_kernels_agree_on_the_step(cgx):
    h, st, bo = workload(cgx, 4, random_fill)
    init = [[p.clone() for p in lp] for lp in st.pools]
    keys = bo.step_phases()
    bo.run(keys)
    torch.cuda.synchronize()
    batched = [[p.clone() for p in lp] for lp in st.pools]
    for lp, ip in zip(st.pools, init):
        for p, q in zip(lp, ip):
            p.copy_(q)
    bo.run(keys, per_box=True)
    for b in bo.batches.values():
        b.check()
    torch.cuda.synchronize()
    for l, (lp, bp) in enumerate(zip(st.pools, batched)):
        for p, q in zip(lp, bp):
            assert torch.equal(p.view(torch.int64), q.view(torch.int64)), ("level", l)


@pytest.mark.parametrize("groups,stagger", [(2, 0), (3, 0), (2, 1), (3, 2)])
def test_grid_function_groups_on_streams_match_one_chain(cgx, groups, stagger):
    ngf = 5
    _, st1, bo1 = workload(cgx, ngf, random_fill)
    _, st2, bo2 = workload(cgx, ngf, random_fill, groups=groups)
    bo2.stagger = stagger
    parts = [list(bo2.gfs(g)) for g in range(groups)]
    assert sum(parts, []) == list(range(ngf)) and all(parts)
    stream = torch.cuda.Stream()
    # step 1 eagerly, step 2 from a captured graph (the fork and join of the
    # groups' streams inside the capture)
    keys1 = bo1.step_phases()
    keys2 = bo2.step_phases()
    assert keys1 == keys2
    bo1.run(keys1, stream)
    bo2.run(keys2, stream)
    keys1 = bo1.step_phases()
    keys2 = bo2.step_phases()
    for k in keys2:  # build and upload outside the capture
        bo2.group_batches(k)
    stream.synchronize()
    g = cgx.Graph()
    with g.capture(stream):
        bo2.run(keys2, stream)
    bo1.run(keys1, stream)
    g.launch(stream)
    for b in list(bo1.batches.values()) + list(bo2.batches.values()):
        b.check(stream)
    stream.synchronize()
    for l, (p1, p2) in enumerate(zip(st1.pools, st2.pools)):
        for a, b in zip(p1, p2):
            assert torch.equal(a.view(torch.int64), b.view(torch.int64)), ("level", l)
    del g


def test_dh_lists_and_box_lists_give_the_same_step(cgx):
    _, s1, b1 = workload(cgx, 3, consistent_fill, fma=False)
    _, s2, b2 = workload(cgx, 3, consistent_fill, schedule="dh", fma=False)
    for _ in range(2):
        b1.run(b1.step_phases())
        b2.run(b2.step_phases())
    for b in list(b1.batches.values()) + list(b2.batches.values()):
        b.check()
    torch.cuda.synchronize()
    for l, (p1, p2) in enumerate(zip(s1.pools, s2.pools)):
        for a, b in zip(p1, p2):
            assert torch.equal(a.view(torch.int64), b.view(torch.int64)), ("level", l)
