"""GPU parity: the sm_100a kernels through the C-ABI against the oracle.

Every case runs the same seeded inputs through ``cgx_transfer`` (and the
batched persistent kernel) and through the oracle's restatement of
``gdata::transfer_data`` (oracle/cgx_oracle.c), in the same floating-point
mode.  The bar is bit-exact: whole destination arrays are compared as bit
patterns, so values outside the region (NaN-filled) must stay untouched.
In the exact mode the oracle is itself bit-exact with CarpetLib's own
operators (tests/test_oracle.py), and so, transitively, is the GPU.
"""
import numpy as np
import pytest

from oracle import cases
from oracle.binding import (OP_COPY, OP_ENO, OP_LAGRANGE, OP_LAGRANGE_MONOTONE, OP_WENO, CELL,
                            VERTEX, OracleError, alloc)

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")


@pytest.fixture(scope="module")
def cgx():
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    import carpet_b200 as cb
    return cb


def bits_equal(a, b):
    return np.array_equal(np.ascontiguousarray(a).view(np.uint64),
                          np.ascontiguousarray(b).view(np.uint64))


def to_dev(cb, a, bbox, pad=False):
    """a device copy of a; pad=True gives the array an even, NaN-filled row
    pitch (the layout the TMA-staged prolongation kernels accept)"""
    if not pad or a.shape[2] % 2 == 0:
        return cb.Data(bbox, torch.from_numpy(a.copy()).cuda())
    full = np.full(a.shape[:2] + (a.shape[2] + 1,), np.nan)
    full[:, :, :a.shape[2]] = a
    return cb.Data(bbox, torch.from_numpy(full).cuda())


# per_box: cgx_transfer; batch: a one-pair batch on arrays of exact shape
# (TMA-staged when the row pitch is even, cp.async-staged otherwise);
# batch_pad: a batch on arrays padded to an even pitch (TMA-staged)
FORMS = ["per_box", "batch", "batch_pad"]


def timeset(rng, ntl):
    """(times, time, order_time) that select ntl timelevels"""
    t0, dt = float(rng.uniform(-1, 1)), float(rng.uniform(0.05, 0.5))
    times = [t0, t0 - dt, t0 - 2 * dt]
    if ntl == 1:
        return times, times[int(rng.integers(0, 3))], 2
    lo = times[ntl - 1]  # 2 timelevels interpolate between TL0 and TL1
    return times, float(rng.uniform(lo + 1e-3, times[0] - 1e-3)), ntl - 1


def run_pair(cb, port, c, op, cent, order, ntl, fma, rng, form="per_box"):
    times, time, ot = timeset(rng, ntl)
    srcs_np = [c["src"], c["src"] * 0.5 + 0.25, c["src"] * -1.5 + 1.0]
    want = c["dst"].copy()
    port.transfer(op, cent, want, c["dstbbox"], srcs_np, c["srcbbox"], times, c["reg"],
                  c["srcbbox"], time, order, ot, fma=fma)
    pad = form == "batch_pad"
    dst = to_dev(cb, c["dst"], c["dstbbox"], pad)
    srcs = [to_dev(cb, s, c["srcbbox"], pad) for s in srcs_np]
    cb.set_fp_mode(fma)
    if form != "per_box":
        b = cb.Batch()
        b.add(dst, srcs, times, c["reg"], c["srcbbox"], time, order, ot, op=op, cent=cent)
        b.upload()
        b.launch()
        b.check()
    else:
        cb.transfer_data(dst, srcs, times, c["reg"], c["srcbbox"], time, order, ot, op=op,
                         cent=cent)
    torch.cuda.synchronize()
    got = dst.tensor.cpu().numpy()[:, :, :want.shape[2]]
    return got, want


@pytest.mark.parametrize("form", FORMS)
@pytest.mark.parametrize("fma", [False, True], ids=["exact", "fma"])
@pytest.mark.parametrize("ntl", [1, 2, 3])
@pytest.mark.parametrize("order", [1, 3, 5, 7, 9, 11])
def test_vc_lagrange(cgx, port, order, ntl, fma, form):
    rng = np.random.default_rng(1000 + 10 * order + ntl)
    for it in range(6):
        big = it >= 4
        c = cases.vc_prolong_case(rng, order, fine_stride=int(rng.choice([1, 2])),
                                  max_ext=40 if big else 9,
                                  kind=("normal", "mixed")[it % 2])
        got, want = run_pair(cgx, port, c, OP_LAGRANGE, VERTEX, order, ntl, fma, rng, form)
        assert bits_equal(got, want), np.nanmax(np.abs(got - want))


@pytest.mark.parametrize("form", FORMS)
@pytest.mark.parametrize("fma", [False, True], ids=["exact", "fma"])
@pytest.mark.parametrize("ntl", [1, 2, 3])
@pytest.mark.parametrize("order", [0, 1, 2, 3, 4, 5])
def test_cc_lagrange(cgx, port, order, ntl, fma, form):
    rng = np.random.default_rng(2000 + 10 * order + ntl)
    for it in range(5):
        c = cases.cc_prolong_case(rng, order, half=int(rng.choice([1, 2])),
                                  max_ext=36 if it == 4 else 9,
                                  kind=("normal", "mixed")[it % 2])
        got, want = run_pair(cgx, port, c, OP_LAGRANGE, CELL, order, ntl, fma, rng, form)
        assert bits_equal(got, want)


@pytest.mark.parametrize("form", FORMS)
@pytest.mark.parametrize("fma", [False, True], ids=["exact", "fma"])
@pytest.mark.parametrize("ntl", [1, 2, 3])
def test_vc_eno(cgx, port, ntl, fma, form):
    rng = np.random.default_rng(3000 + ntl)
    for it in range(8):
        c = cases.vc_prolong_case(rng, 3, reach=(1, 2), max_ext=40 if it == 7 else 9,
                                  kind=("normal", "steps", "mixed")[it % 3])
        got, want = run_pair(cgx, port, c, OP_ENO, VERTEX, 3, ntl, fma, rng, form)
        assert bits_equal(got, want)


@pytest.mark.parametrize("form", FORMS)
@pytest.mark.parametrize("fma", [False, True], ids=["exact", "fma"])
@pytest.mark.parametrize("ntl", [1, 2, 3])
def test_o5_monotone(cgx, port, ntl, fma, form):
    """op Lagrange_monotone: prolongate_3d_o5_monotone_rf2, with ENO time
    interpolation through temporaries for 2 and 3 timelevels"""
    rng = np.random.default_rng(3200 + ntl)
    for it in range(6):
        c = cases.vc_prolong_case(rng, 5, fine_stride=int(rng.choice([1, 2])),
                                  max_ext=30 if it == 5 else 9,
                                  kind=("normal", "mixed", "steps", "smooth")[it % 4])
        got, want = run_pair(cgx, port, c, OP_LAGRANGE_MONOTONE, VERTEX, 5, ntl, fma, rng, form)
        assert bits_equal(got, want)


@pytest.mark.parametrize("form", FORMS)
@pytest.mark.parametrize("ntl", [1, 2, 3])
def test_vc_weno(cgx, port, ntl, form):
    """op WENO, vertex-centred order 5: the ENO operator (data.cc:722-752)"""
    rng = np.random.default_rng(3050 + ntl)
    for it in range(4):
        c = cases.vc_prolong_case(rng, 3, reach=(1, 2), max_ext=9, kind=("steps", "mixed")[it % 2])
        got, want = run_pair(cgx, port, c, OP_WENO, VERTEX, 5, ntl, False, rng, form)
        assert bits_equal(got, want)


@pytest.mark.parametrize("form", FORMS)
@pytest.mark.parametrize("fma", [False, True], ids=["exact", "fma"])
@pytest.mark.parametrize("ntl", [1, 2, 3])
@pytest.mark.parametrize("order_space", [2, 3, 4, 5])
def test_cc_eno(cgx, port, order_space, ntl, fma, form):
    """prolongate_3d_cc_eno_rf2 (order_space 2-4: ORDER 2, 5: ORDER 3) with
    ENO time interpolation, on data that drive every stencil choice"""
    rng = np.random.default_rng(3100 + 10 * order_space + ntl)
    lagr = 5 if order_space == 5 else 3  # the Lagrange order of the same window
    for it in range(8):
        c = cases.cc_prolong_case(rng, lagr, half=int(rng.choice([1, 2])),
                                  max_ext=36 if it == 7 else 9,
                                  kind=("normal", "mixed", "steps", "smooth")[it % 4])
        got, want = run_pair(cgx, port, c, OP_ENO, CELL, order_space, ntl, fma, rng, form)
        assert bits_equal(got, want)


@pytest.mark.parametrize("form", FORMS)
@pytest.mark.parametrize("fma", [False, True], ids=["exact", "fma"])
def test_restrict_and_copy(cgx, port, fma, form):
    rng = np.random.default_rng(4000)
    for it in range(10):
        big = it == 9
        for maker, cent in ((cases.vc_restrict_case, VERTEX), (cases.cc_restrict_case, CELL)):
            c = maker(rng, max_ext=40 if big else 9, kind="mixed")
            got, want = run_pair(cgx, port, c, OP_LAGRANGE, cent, 1, 1, fma, rng, form)
            assert bits_equal(got, want)
        c = cases.copy_case(rng, max_ext=40 if big else 9, kind="mixed")
        for ntl in (1, 2, 3):
            got, want = run_pair(cgx, port, c, OP_LAGRANGE, VERTEX, 1, ntl, fma, rng, form)
            assert bits_equal(got, want)


@pytest.mark.parametrize("form", FORMS)
@pytest.mark.parametrize("fma", [False, True], ids=["exact", "fma"])
@pytest.mark.parametrize("order", [3, 5])
def test_cc_higher_order_restriction(cgx, port, order, fma, form):
    """restrict_3d_cc_o3_rf2 / _o5_rf2, selected as CarpetLib selects them
    (use_higher_order_restriction with restriction_order_space)."""
    rng = np.random.default_rng(4200 + order)
    reach = (1, 1) if order == 3 else (2, 2)
    cgx.set_restriction(True, order)
    port.set_restriction(True, order)
    try:
        for it in range(8):
            c = cases.cc_restrict_case(rng, half=int(rng.choice([1, 2])), reach=reach,
                                       max_ext=40 if it == 7 else 9,
                                       kind=("normal", "mixed")[it % 2])
            got, want = run_pair(cgx, port, c, OP_LAGRANGE, CELL, 1, 1, fma, rng, form)
            assert bits_equal(got, want)
        # the ENO transport operator keeps the 8-cell average
        c = cases.cc_restrict_case(rng, reach=reach, kind="mixed")
        got, want = run_pair(cgx, port, c, OP_ENO, CELL, 1, 1, fma, rng, form)
        assert bits_equal(got, want)
        # a source without the stencil's reach is refused, as by the oracle
        c = cases.cc_restrict_case(rng, kind="mixed")
        reg, fs = c["reg"], c["srcbbox"][6]
        srcbbox = [reg[d] - fs // 2 for d in range(3)] + [reg[3 + d] + fs // 2 for d in range(3)] + [fs] * 3
        src = alloc(srcbbox)
        with pytest.raises(OracleError, match="stencil reaches outside"):
            port.transfer(OP_LAGRANGE, CELL, c["dst"].copy(), c["dstbbox"], [src], srcbbox, [0.0], reg,
                          srcbbox, 0.0, 1, 0, fma=fma)
        cgx.set_fp_mode(fma)
        with pytest.raises(cgx.CgxError, match="stencil reaches outside"):
            cgx.transfer_data(to_dev(cgx, c["dst"], c["dstbbox"]), [to_dev(cgx, src, srcbbox)], [0.0],
                              reg, srcbbox, 0.0, 1, 0, op=OP_LAGRANGE, cent=CELL)
    finally:
        cgx.set_restriction(False, 1)
        port.set_restriction(False, 1)


def test_copy_with_slab_offset(cgx, port):
    rng = np.random.default_rng(4100)
    for it in range(10):
        c = cases.copy_case(rng, slab=True, kind="mixed")
        want = c["dst"].copy()
        port.copy_3d(c["src"], c["srcbbox"], want, c["dstbbox"], c["srcreg"], c["dstreg"], c["slab"])
        dst = to_dev(cgx, c["dst"], c["dstbbox"])
        src = to_dev(cgx, c["src"], c["srcbbox"])
        cgx.copy_data(dst, src, c["dstreg"], c["srcreg"], slab_offset=c["slab"])
        torch.cuda.synchronize()
        assert bits_equal(dst.tensor.cpu().numpy(), want)


@pytest.mark.parametrize("fma", [False, True], ids=["exact", "fma"])
def test_batched_mixed_pairs_match_per_box_and_oracle(cgx, port, fma):
    """A batch of uneven, mixed box-pairs (each with its own destination)
    in one persistent kernel, then the same descriptors per box, then a
    CUDA-graph replay: all three bit-identical with the oracle."""
    rng = np.random.default_rng(5000)
    cgx.set_fp_mode(fma)
    b = cgx.Batch()
    items = []
    for it in range(60):
        kind = it % 6
        ntl = int(rng.integers(1, 4))
        if kind == 0:
            order = int(rng.choice([1, 3, 5]))
            c = cases.vc_prolong_case(rng, order, max_ext=int(rng.integers(3, 40)))
            op, cent = OP_LAGRANGE, VERTEX
        elif kind == 1:
            order = int(rng.integers(0, 6))
            c = cases.cc_prolong_case(rng, order, max_ext=int(rng.integers(3, 30)))
            op, cent = OP_LAGRANGE, CELL
        elif kind == 2:
            order = 3
            c = cases.vc_prolong_case(rng, 3, reach=(1, 2), max_ext=int(rng.integers(3, 30)))
            op, cent = OP_ENO, VERTEX
        elif kind == 3:
            order, op, cent = 1, OP_LAGRANGE, VERTEX
            c = cases.vc_restrict_case(rng, max_ext=int(rng.integers(3, 30)))
            ntl = 1
        elif kind == 4:
            order, op, cent = 0, OP_LAGRANGE, CELL
            c = cases.cc_restrict_case(rng, max_ext=int(rng.integers(3, 30)))
            ntl = 1
        else:
            order, op, cent = 1, OP_LAGRANGE, VERTEX
            c = cases.copy_case(rng, max_ext=int(rng.integers(3, 40)))
        times, time, ot = timeset(rng, ntl)
        srcs_np = [c["src"], c["src"] * 0.5 + 0.25, c["src"] * -1.5 + 1.0]
        want = c["dst"].copy()
        port.transfer(op, cent, want, c["dstbbox"], srcs_np, c["srcbbox"], times, c["reg"]
                      if "reg" in c else c["dstreg"], c["srcbbox"], time, order, ot, fma=fma)
        dst = to_dev(cgx, c["dst"], c["dstbbox"])
        srcs = [to_dev(cgx, s, c["srcbbox"]) for s in srcs_np]
        b.add(dst, srcs, times, c["reg"] if "reg" in c else c["dstreg"], c["srcbbox"], time,
              order, ot, op=op, cent=cent)
        items.append((dst, srcs, want, c["dst"]))
    st = b.stats()
    assert st["pairs"] == 60 and st["tiles"] > 60
    b.upload()
    modes = ["batch", "per_box", "graph"] + [f"config{c}" for c in range(5)] + ["autotuned"]
    for mode in modes:
        for dst, _, _, init in items:
            dst.tensor.copy_(torch.from_numpy(init))
        if mode.startswith("config"):
            # every prolongation variant pinned to one tile configuration
            b.set_config(int(mode[6:]))
            b.upload()
            b.launch()
        elif mode == "autotuned":
            chosen = b.autotune(reps=2)
            assert chosen and all(0 <= c < 5 for c in chosen.values())
            for dst, _, _, init in items:  # autotuning ran the batch: start over
                dst.tensor.copy_(torch.from_numpy(init))
            b.launch()
        elif mode == "batch":
            b.launch()
        elif mode == "per_box":
            b.launch_per_box()
        else:
            s = torch.cuda.Stream()
            g = cgx.Graph()
            torch.cuda.synchronize()
            with g.capture(s):
                b.launch(s)
            g.launch(s)
            g.launch(s)
            s.synchronize()
        b.check()
        torch.cuda.synchronize()
        for dst, _, want, _ in items:
            assert bits_equal(dst.tensor.cpu().numpy(), want), mode


def test_exact_mode_matches_compiled_reference(cgx):
    """Directly against CarpetLib's operators compiled from source, where
    that build travelled with the tree."""
    from oracle.binding import Ref
    if not Ref.available():
        pytest.skip("reference build absent")
    ref = Ref(False)
    rng = np.random.default_rng(6000)
    cgx.set_fp_mode(False)
    for order in (1, 3, 5):
        for it in range(4):
            c = cases.vc_prolong_case(rng, order, max_ext=30, kind="mixed")
            want = c["dst"].copy()
            ref.prolongate_3d_rf2(order, c["src"], c["srcbbox"], want, c["dstbbox"], c["reg"])
            dst = to_dev(cgx, c["dst"], c["dstbbox"])
            src = to_dev(cgx, c["src"], c["srcbbox"])
            cgx.transfer_data(dst, [src], [0.0], c["reg"], c["srcbbox"], 0.0, order, 0)
            torch.cuda.synchronize()
            assert bits_equal(dst.tensor.cpu().numpy(), want)


# ---------------------------------------------------------------- two stages
def timeset5(rng, ntl):
    """five timelevels t0, t0-dt, ...; a time that selects the first ntl
    (order_time = ntl - 1)"""
    t0, dt = float(rng.uniform(-1, 1)), float(rng.uniform(0.05, 0.5))
    times = [t0 - i * dt for i in range(5)]
    if ntl == 1:  # an exact match selects one timelevel
        return times, times[int(rng.integers(0, 5))], 2
    return times, float(rng.uniform(times[ntl - 1] + 1e-3, times[0] - 1e-3)), ntl - 1


def staged_cases(rng, big=False):
    """(case, op, cent, order_space, ntl): transfers that run through
    per-timelevel temporaries"""
    m = 30 if big else 8
    out = []
    for ntl in (4, 5):
        out.append((cases.vc_prolong_case(rng, 5, max_ext=m, kind="mixed"), OP_LAGRANGE, VERTEX, 5, ntl))
        out.append((cases.cc_prolong_case(rng, 3, max_ext=m, kind="mixed"), OP_LAGRANGE, CELL, 3, ntl))
        out.append((cases.copy_case(rng, max_ext=m, kind="mixed"), OP_LAGRANGE, VERTEX, 1, ntl))
        out.append((cases.vc_prolong_case(rng, 7, max_ext=m, kind="mixed"), OP_LAGRANGE, VERTEX, 7, ntl))
    for ntl in (2, 3):
        out.append((cases.vc_restrict_case(rng, max_ext=m, kind="mixed"), OP_LAGRANGE, VERTEX, 1, ntl))
        out.append((cases.cc_restrict_case(rng, max_ext=m, kind="mixed"), OP_LAGRANGE, CELL, 1, ntl))
        out.append((cases.cc_restrict_case(rng, max_ext=m, kind="mixed"), OP_ENO, CELL, 1, ntl))
        out.append((cases.vc_prolong_case(rng, 5, max_ext=m, kind="steps"), OP_LAGRANGE_MONOTONE,
                    VERTEX, 5, ntl))
    return out


def staged_io(cb, port, c, op, cent, order, ntl, fma, rng):
    times, time, ot = timeset5(rng, ntl)
    srcs_np = [c["src"] * (1.0 + 0.25 * i) - 0.5 * i for i in range(5)]
    reg = c.get("reg", c.get("dstreg"))
    want = c["dst"].copy()
    port.transfer(op, cent, want, c["dstbbox"], srcs_np, c["srcbbox"], times, reg, c["srcbbox"],
                  time, order, ot, fma=fma)
    dst = to_dev(cb, c["dst"], c["dstbbox"])
    srcs = [to_dev(cb, s, c["srcbbox"]) for s in srcs_np]
    return dict(dst=dst, srcs=srcs, times=times, time=time, ot=ot, reg=reg, want=want, init=c["dst"])


@pytest.mark.parametrize("fma", [False, True], ids=["exact", "fma"])
def test_staged_transfers_per_box(cgx, port, fma):
    """order_time 3 and 4 (interpolate_3d_4tl / 5tl) and restriction between
    timelevels: the spatial operator per timelevel into temporaries, then
    the time combination, as transfer_time does"""
    rng = np.random.default_rng(6000 + fma)
    cgx.set_fp_mode(fma)
    for big in (False, True):
        for c, op, cent, order, ntl in staged_cases(rng, big):
            x = staged_io(cgx, port, c, op, cent, order, ntl, fma, rng)
            cgx.transfer_data(x["dst"], x["srcs"], x["times"], x["reg"], c["srcbbox"], x["time"],
                              order, x["ot"], op=op, cent=cent)
            torch.cuda.synchronize()
            got = x["dst"].tensor.cpu().numpy()[:, :, :x["want"].shape[2]]
            assert bits_equal(got, x["want"]), (op, cent, order, ntl)


@pytest.mark.parametrize("fma", [False, True], ids=["exact", "fma"])
def test_staged_transfers_batched(cgx, port, fma):
    """staged pairs mixed with fused ones in one batch: the batch's
    persistent kernels, the per-box launches and a CUDA-graph replay"""
    rng = np.random.default_rng(6100 + fma)
    cgx.set_fp_mode(fma)
    b = cgx.Batch()
    items = []
    for c, op, cent, order, ntl in staged_cases(rng):
        x = staged_io(cgx, port, c, op, cent, order, ntl, fma, rng)
        b.add(x["dst"], x["srcs"], x["times"], x["reg"], c["srcbbox"], x["time"], order, x["ot"],
              op=op, cent=cent)
        items.append(x)
    for it in range(6):  # fused pairs alongside
        c = cases.vc_prolong_case(rng, 5, max_ext=12, kind="mixed")
        x = staged_io(cgx, port, c, OP_LAGRANGE, VERTEX, 5, 1 + it % 3, fma, rng)
        b.add(x["dst"], x["srcs"], x["times"], x["reg"], c["srcbbox"], x["time"], 5, x["ot"],
              op=OP_LAGRANGE, cent=VERTEX)
        items.append(x)
    assert b.stats()["pairs"] == len(items)
    b.upload()
    for mode in ("batch", "per_box", "graph"):
        for x in items:
            x["dst"].tensor.copy_(torch.from_numpy(x["init"]))
        if mode == "batch":
            b.launch()
        elif mode == "per_box":
            b.launch_per_box()
        else:
            s = torch.cuda.Stream()
            g = cgx.Graph()
            torch.cuda.synchronize()
            with g.capture(s):
                b.launch(s)
            g.launch(s)
            s.synchronize()
        b.check()
        torch.cuda.synchronize()
        for x in items:
            got = x["dst"].tensor.cpu().numpy()[:, :, :x["want"].shape[2]]
            assert bits_equal(got, x["want"]), mode


def test_staged_eno_family_beyond_order_time_2_is_refused(cgx, port):
    rng = np.random.default_rng(6200)
    c = cases.vc_prolong_case(rng, 3, reach=(1, 2), kind="mixed")
    times, time, ot = timeset5(rng, 4)
    srcs = [c["src"]] * 5
    with pytest.raises(OracleError, match="order_time"):
        port.transfer(OP_ENO, VERTEX, c["dst"].copy(), c["dstbbox"], srcs, c["srcbbox"], times,
                      c["reg"], c["srcbbox"], time, 3, ot)
    with pytest.raises(cgx.CgxError, match="order_time"):
        cgx.transfer_data(to_dev(cgx, c["dst"], c["dstbbox"]), [to_dev(cgx, s, c["srcbbox"]) for s in srcs],
                          times, c["reg"], c["srcbbox"], time, 3, ot, op=OP_ENO, cent=VERTEX)
