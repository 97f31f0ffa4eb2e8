"""The dh schedule producer (cgx_dh_* / carpet_b200.dh) on the CPU.

* The C++ producer and its Python restatement give identical pair lists.
* A point-wise restatement of dh::regrid's region algebra
  (CarpetLib/src/dh.cc:300-1088) on boolean masks -- ghost zones, owned and
  buffer regions, active regions, and the order in which components are
  asked -- predicts, for every receiving point, which component sends it;
  on random irregular hierarchies (components of random sizes, refined
  regions made of one or two boxes) every point of every list is received
  exactly once, from the predicted component, and every expected point is
  received: the consistency checks of dh.cc:825-831, 971-973 and 1080-1082.
* On the nested benchmark hierarchies the derived arrays are the nested
  builder's, sync plus boundary prolongation write the same points, and
  restriction into interiors only writes the same points as the nested
  builder's restriction (into exteriors it also fills the ghost zones).
"""
import numpy as np
import pytest

from carpet_b200 import dh
from carpet_b200.hierarchy import mkbox, nested, npoints

GHOST, BUFFER, ORDER = 3, 3, 5


def as_list(pairs):
    return [(p.dst_comp, p.src_comp, tuple(p.dstbox), tuple(p.srcbox)) for p in pairs]


def same(a, b):
    L = len(a.levels)
    for l in range(L):
        assert [c.exterior for c in a.levels[l].comps] == [c.exterior for c in b.levels[l].comps]
        assert as_list(a.sync[l]) == as_list(b.sync[l]), ("sync", l)
        if l:
            assert as_list(a.prolong[l]) == as_list(b.prolong[l]), ("prolong", l)
            assert as_list(a.restrict[l]) == as_list(b.restrict[l]), ("restrict", l)


# ---------------------------------------------------------------- layouts
def split(rng, box, parts, minw):
    """random bisections of box into about `parts` components, each at least
    minw points wide"""
    out = [box]
    for _ in range(parts - 1):
        i = int(rng.integers(0, len(out)))
        b = out[i]
        d = int(rng.integers(0, 3))
        n = (b[3 + d] - b[d]) // b[6 + d] + 1
        if n < 2 * minw:
            continue
        k = int(rng.integers(minw, n - minw + 1))
        lo = list(b[:3]); up = list(b[3:6])
        up[d] = b[d] + (k - 1) * b[6 + d]
        lo2 = list(b[:3]); lo2[d] = b[d] + k * b[6 + d]
        out[i] = mkbox(lo, up, b[6:])
        out.append(mkbox(lo2, b[3:6], b[6:]))
    return out


def random_hierarchy(rng, nlevels=3, n0=(41, 53)):
    """domains and interiors of a random properly nested hierarchy"""
    s0 = 2 ** (nlevels - 1)
    n = [int(rng.integers(n0[0], n0[1] + 1)) for _ in range(3)]
    D0 = mkbox((0, 0, 0), [(m - 1) * s0 for m in n], (s0,) * 3)
    domains, interiors = [D0], [split(rng, D0, int(rng.integers(1, 6)), GHOST + 1)]
    active = D0  # a box inside the current level's active region
    for l in range(1, nlevels):
        s = s0 >> l
        cs = 2 * s
        D = mkbox(D0[:3], D0[3:6], (s,) * 3)
        # room inside the coarse active box: stencil and ghost margins
        m = (GHOST + ORDER // 2 + 2) * cs
        lo = [active[d] + m for d in range(3)]
        up = [active[3 + d] - m for d in range(3)]
        span = [(up[d] - lo[d]) // s for d in range(3)]
        if min(span) < 2 * (GHOST + BUFFER) + 4:
            break
        # work on the coarse lattice so the regions are coarse-aligned
        lo = [lo[d] + (-(lo[d] - D0[d])) % cs for d in range(3)]
        up = [up[d] - (up[d] - D0[d]) % cs for d in range(3)]
        cspan = [(up[d] - lo[d]) // cs for d in range(3)]
        wmin = (GHOST + BUFFER) // 2 + 3  # coarse points of a refined box
        if min(cspan) < wmin:
            break
        boxes = []
        if rng.random() < 0.4 and max(cspan) >= 2 * wmin + 2:
            d = int(np.argmax(cspan))
            k1 = int(rng.integers(wmin, cspan[d] - wmin))  # first box: lo .. lo + k1 coarse points
            gap = int(rng.integers(1, 4))
            for a, b in ((lo[d], lo[d] + k1 * cs), (lo[d] + (k1 + gap) * cs, up[d])):
                if b - a < wmin * cs:
                    continue
                blo, bup = list(lo), list(up)
                blo[d], bup[d] = a, b
                boxes.append(mkbox(blo, bup, (s,) * 3))
        if not boxes:
            blo, bup = [], []
            for d in range(3):
                w = int(rng.integers(wmin, cspan[d] + 1))
                o = int(rng.integers(0, cspan[d] - w + 1))
                blo.append(lo[d] + o * cs)
                bup.append(lo[d] + (o + w) * cs)
            boxes.append(mkbox(blo, bup, (s,) * 3))
        intr = []
        for b in boxes:
            intr += split(rng, b, int(rng.integers(1, 5)), GHOST + 1)
        domains.append(D)
        interiors.append(intr)
        # the next level nests inside this level's first box, shrunk by its
        # buffer width (the active part)
        src = boxes[0]
        active = mkbox([src[d] + (BUFFER + 1) * s for d in range(3)],
                       [src[3 + d] - (BUFFER + 1) * s for d in range(3)], (s,) * 3)
    return domains, interiors


# ---------------------------------------------------------------- oracle
def dilate(m, r):
    out = m.copy()
    for ax in range(3):
        acc = out.copy()
        for k in range(1, r + 1):
            acc[tuple(slice(k, None) if a == ax else slice(None) for a in range(3))] |= \
                out[tuple(slice(None, -k) if a == ax else slice(None) for a in range(3))]
            acc[tuple(slice(None, -k) if a == ax else slice(None) for a in range(3))] |= \
                out[tuple(slice(k, None) if a == ax else slice(None) for a in range(3))]
        out = acc
    return out


class Grid:
    """boolean masks over a level's domain (index = (x - lo) / stride)"""

    def __init__(self, D):
        self.D = D
        self.s = D[6]
        self.shape = tuple((D[3 + d] - D[d]) // self.s + 1 for d in range(3))

    def mask(self, b):
        m = np.zeros(self.shape, bool)
        lo = [max(0, (b[d] - self.D[d]) // self.s) for d in range(3)]
        up = [min(self.shape[d] - 1, (b[3 + d] - self.D[d]) // self.s) for d in range(3)]
        if all(lo[d] <= up[d] for d in range(3)):
            m[lo[0]:up[0] + 1, lo[1]:up[1] + 1, lo[2]:up[2] + 1] = True
        return m

    def points(self, b):
        s = b[6:]
        return [(x, y, z) for x in range(b[0], b[3] + 1, s[0]) for y in range(b[1], b[4] + 1, s[1])
                for z in range(b[2], b[5] + 1, s[2])]

    def idx(self, p):
        return tuple((p[d] - self.D[d]) // self.s for d in range(3))


def oracle(domains, interiors, into_ghosts=True):
    """per level: sync / bndprol / restrict maps {(dst comp, point): src comp}"""
    L = len(domains)
    lv = []
    for l in range(L):
        g = Grid(domains[l])
        D = domains[l]
        comps = []
        allowned = np.zeros(g.shape, bool)
        for b in interiors[l]:
            gl = [0 if b[d] == D[d] else GHOST for d in range(3)]
            gu = [0 if b[3 + d] == D[3 + d] else GHOST for d in range(3)]
            e = mkbox([b[d] - gl[d] * D[6] for d in range(3)], [b[3 + d] + gu[d] * D[6] for d in range(3)],
                      b[6:])
            comps.append(dict(intr=g.mask(b), extr=g.mask(e), ebox=e))
            allowned |= comps[-1]["intr"]
        notactive = dilate(~allowned, BUFFER)
        allactive = allowned & ~notactive
        for k in comps:
            k["buffers"] = k["intr"] & notactive
            k["active"] = k["intr"] & allactive
            k["ghosts"] = k["extr"] & ~k["intr"]
        lv.append(dict(g=g, comps=comps, allactive=allactive))
    out = []
    for l in range(L):
        F, g = lv[l], lv[l]["g"]
        sync, bnd, rest = {}, {}, {}
        for c, k in enumerate(F["comps"]):
            synced = np.zeros(g.shape, bool)
            for idx in zip(*np.nonzero(k["ghosts"])):
                for cc, o in enumerate(F["comps"]):
                    if o["intr"][idx]:
                        sync[(c, idx)] = cc
                        synced[idx] = True
                        break
            if l == 0:
                continue
            Cl, gc = lv[l - 1], lv[l - 1]["g"]
            need = (k["ghosts"] & ~synced) | k["buffers"]
            eoas = []
            for o in Cl["comps"]:
                m = np.zeros(g.shape, bool)
                ci = np.nonzero(o["active"])
                fx = [(ci[d] * gc.s + gc.D[d] - g.D[d]) // g.s for d in range(3)]
                m[tuple(fx)] = True
                eoas.append(dilate(m, 2))
            for idx in zip(*np.nonzero(need)):
                for cc, m in enumerate(eoas):
                    if m[idx]:
                        bnd[(c, idx)] = cc
                        break
                else:
                    raise AssertionError("oracle: a point nobody prolongates")
        out.append(dict(sync=sync, bndprol=bnd, restrict=rest))
    for l in range(1, L):
        F, Cl = lv[l], lv[l - 1]
        g, gc = F["g"], Cl["g"]
        # coarse points that are fine active points
        ar = np.zeros(gc.shape, bool)
        ci = np.nonzero(np.ones(gc.shape, bool))
        fx = [(ci[d] * gc.s + gc.D[d] - g.D[d]) for d in range(3)]
        ok = np.all([(fx[d] >= 0) & (fx[d] % g.s == 0) & (fx[d] // g.s < g.shape[d]) for d in range(3)], axis=0)
        sel = tuple(np.array(ci[d])[ok] for d in range(3))
        fsel = tuple((fx[d][ok] // g.s) for d in range(3))
        ar[sel] = F["allactive"][fsel]
        for oc, o in enumerate(Cl["comps"]):
            need = ar & (o["extr"] if into_ghosts else o["intr"])
            for idx in zip(*np.nonzero(need)):
                p = tuple(idx[d] * gc.s + gc.D[d] for d in range(3))
                for c, k in enumerate(F["comps"]):
                    if k["extr"][g.idx(p)]:
                        out[l - 1]["restrict"][(oc, idx)] = c
                        break
    return out, lv


def check_against_oracle(h, domains, interiors, into_ghosts=True):
    want, lv = oracle(domains, interiors, into_ghosts)
    L = len(domains)
    for l in range(L):
        g = lv[l]["g"]
        for kind, pairs in (("sync", h.sync[l]), ("bndprol", h.prolong.get(l, [])),
                            ("restrict", h.restrict.get(l + 1, []))):
            got = {}
            for p in pairs:
                for pt in g.points(p.dstbox):
                    key = (p.dst_comp, g.idx(pt))
                    assert key not in got, (kind, l, "received twice", key)
                    got[key] = p.src_comp
            assert got == want[l][kind], (kind, l)


# ---------------------------------------------------------------- tests
@pytest.mark.parametrize("seed,n0", [(s, (41, 53)) for s in range(6)] + [(s, (45, 61)) for s in (2, 6, 8)])
def test_random_hierarchies_cpp_python_and_pointwise_oracle(seed, n0):
    rng = np.random.default_rng(seed)
    domains, interiors = random_hierarchy(rng, n0=n0)
    a = dh.schedule(domains, interiors, GHOST, BUFFER, ORDER)
    b = dh.schedule_py(domains, interiors, GHOST, BUFFER, ORDER)
    same(a, b)
    check_against_oracle(a, domains, interiors)
    c = dh.schedule(domains, interiors, GHOST, BUFFER, ORDER, restrict_into_ghosts=False)
    check_against_oracle(c, domains, interiors, into_ghosts=False)


def test_nested_benchmark_hierarchy():
    h = nested(5, 129, ghost=3, buffer=9, order=5)
    doms, ints = dh.from_nested(h)
    a = dh.schedule(doms, ints, 3, 9, 5)
    same(a, dh.schedule_py(doms, ints, 3, 9, 5))
    for l in range(5):
        assert [c.exterior for c in a.levels[l].comps] == [c.exterior for c in h.levels[l].comps]
        if l == 0:
            assert sum(npoints(p.dstbox) for p in a.sync[l]) == sum(npoints(p.dstbox) for p in h.sync[l])
            continue
        # the same points written by sync and prolongation together
        assert sum(npoints(p.dstbox) for p in a.sync[l] + a.prolong[l]) == \
            sum(npoints(p.dstbox) for p in h.sync[l] + h.prolong[l])
    inner = dh.schedule(doms, ints, 3, 9, 5, restrict_into_ghosts=False)
    for l in range(1, 5):
        assert sum(npoints(p.dstbox) for p in inner.restrict[l]) == \
            sum(npoints(p.dstbox) for p in h.restrict[l])
        assert sum(npoints(p.dstbox) for p in a.restrict[l]) > sum(npoints(p.dstbox) for p in h.restrict[l])


def test_improper_nesting_is_refused():
    """a refined level whose boundary stencils leave the coarse level's
    active region: the reference's check fails, here as CGX_EINVAL"""
    h = nested(3, 33, ghost=3, buffer=9, order=5)
    doms, ints = dh.from_nested(h)
    from carpet_b200._lib import CgxError
    with pytest.raises(CgxError):
        dh.schedule(doms, ints, 3, 9, 5)
    with pytest.raises(ValueError):
        dh.schedule_py(doms, ints, 3, 9, 5)
