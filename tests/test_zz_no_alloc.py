"""The no-allocation entry point, cgx_transfer_pairs_noalloc.

Some callers of this library must not allocate device memory: a host code
that hands all device memory to its own pool, work issued while a CUDA graph
is being captured elsewhere in the process, or a time-step loop that cannot
take the device-wide synchronisation cudaMalloc/cudaFree bring.  For them the
persistent kernel can run with its scratch (descriptor queue, tile offsets,
work counter) in a fixed array inside the library's device image instead of
in allocated memory.

This test calls that entry point through the C-ABI twice in a row and checks
each result bit for bit against the ordinary per-box entry point
(cgx_transfer) and against the oracle on the same inputs -- the same bar as
every other parity test -- reads the kernel's status back through
cgx_noalloc_check, and checks that an over-long pair list and a call inside a
stream capture are refused.  It sits in the last collected test file and
passes both alone and after the other tests.
"""
import ctypes as C

import numpy as np
import pytest

from oracle import cases
from oracle.binding import CELL, OP_ENO, OP_LAGRANGE, OP_LAGRANGE_MONOTONE, VERTEX, Port

pytestmark = pytest.mark.gpu
torch = pytest.importorskip("torch")


def _structs():
    from carpet_b200._lib import cgx_array

    class cgx_pair(C.Structure):
        _fields_ = [("op", C.c_int), ("cent", C.c_int), ("dst", cgx_array),
                    ("srcs", cgx_array * 3), ("times", C.c_double * 3), ("nsrc", C.c_int),
                    ("dstbox", C.c_int * 9), ("srcbox", C.c_int * 9), ("has_slab", C.c_int),
                    ("slab_offset", C.c_int * 3), ("time", C.c_double),
                    ("order_space", C.c_int), ("order_time", C.c_int)]
    return cgx_array, cgx_pair


def _make_pairs(seed, n):
    """seeded mixed box-pairs: (op, cent, case, ntl, order)"""
    rng = np.random.default_rng(seed)
    out = []
    for i in range(n):
        k = i % 8
        if k == 0:
            order = int(rng.choice([1, 3, 5]))
            out.append((OP_LAGRANGE, VERTEX, cases.vc_prolong_case(rng, order, max_ext=30), order))
        elif k == 1:
            order = int(rng.integers(0, 6))
            out.append((OP_LAGRANGE, CELL, cases.cc_prolong_case(rng, order, max_ext=24), order))
        elif k == 2:
            out.append((OP_ENO, VERTEX, cases.vc_prolong_case(rng, 3, reach=(1, 2), max_ext=24), 3))
        elif k == 3:
            out.append((OP_LAGRANGE, VERTEX, cases.vc_restrict_case(rng, max_ext=24), 1))
        elif k == 4:
            out.append((OP_LAGRANGE, CELL, cases.cc_restrict_case(rng, max_ext=24), 0))
        elif k == 5:
            out.append((OP_LAGRANGE, VERTEX, cases.copy_case(rng, max_ext=30), 1))
        elif k == 6:
            out.append((OP_LAGRANGE_MONOTONE, VERTEX, cases.vc_prolong_case(rng, 5, max_ext=20), 5))
        else:
            out.append((OP_ENO, CELL, cases.cc_prolong_case(rng, 5, max_ext=20, kind="smooth"), 5))
    return out


@pytest.fixture(scope="module")
def lib():
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    from carpet_b200._lib import lib as L
    return L


def _run(lib, seed, n):
    from carpet_b200._lib import box9
    cgx_array, cgx_pair = _structs()
    lib.cgx_set_fp_mode(0)  # the reference's operation order, two roundings per multiply-add
    port = Port()
    pairs = (cgx_pair * n)()
    keep, ref_dsts, na_dsts, oracle_dsts = [], [], [], []
    t0, dt = 0.5, 0.125
    for i, (op, cent, c, order) in enumerate(_make_pairs(seed, n)):
        ntl = 1 + i % 3
        # restriction, and the monotone operator (between timelevels it runs
        # through temporaries, which this entry point does not allocate)
        if c["srcbbox"][6] < c["dstbbox"][6] or op == OP_LAGRANGE_MONOTONE:
            ntl = 1
        times = [t0, t0 - dt, t0 - 2 * dt]
        time = t0 if ntl == 1 else t0 - dt / (3 if ntl == 2 else 2)
        ot = 2 if ntl != 2 else 1
        srcs_np = [c["src"], c["src"] * 0.5 + 0.25, c["src"] * -1.5 + 1.0]
        srcs = [torch.from_numpy(s.copy()).cuda() for s in srcs_np]
        d_ref = torch.from_numpy(c["dst"].copy()).cuda()
        d_na = torch.from_numpy(c["dst"].copy()).cuda()
        keep += srcs
        ref_dsts.append(d_ref)
        na_dsts.append((d_na, torch.from_numpy(c["dst"].copy()).cuda()))

        def arr(t, bbox):
            a = cgx_array()
            a.data = t.data_ptr()
            a.padext[:] = (t.shape[2], t.shape[1], t.shape[0])
            a.bbox[:] = bbox
            return a

        p = pairs[i]
        p.op, p.cent = op, cent
        p.dst = arr(d_na, c["dstbbox"])
        for t in range(3):
            p.srcs[t] = arr(srcs[t], c["srcbbox"])
        p.times[:] = times
        p.nsrc = 3
        p.dstbox[:] = c["reg"]
        p.srcbox[:] = c["srcbbox"]
        p.has_slab = 0
        p.time = time
        p.order_space, p.order_time = order, ot
        # the existing per-box entry point on the same arguments
        dref = arr(d_ref, c["dstbbox"])
        sarr = (cgx_array * 3)(*[arr(s, c["srcbbox"]) for s in srcs])
        ts = (C.c_double * 3)(*times)
        rc = lib.cgx_transfer(op, cent, C.byref(dref), sarr, ts, 3, box9(c["reg"]),
                              box9(c["srcbbox"]), None, time, order, ot, None)
        assert rc == 0, lib.cgx_last_error()
        # and the oracle on the same arguments
        want = c["dst"].copy()
        port.transfer(op, cent, want, c["dstbbox"], srcs_np, c["srcbbox"], times, c["reg"],
                      c["srcbbox"], time, order, ot)
        oracle_dsts.append(want)
    torch.cuda.synchronize()
    return pairs, keep, ref_dsts, na_dsts, oracle_dsts


def test_noalloc_matches_per_box_and_oracle_twice(lib):
    pairs, keep, ref_dsts, na_dsts, oracle_dsts = _run(lib, 777, 48)
    n = len(ref_dsts)
    for call in range(2):
        for d, init in na_dsts:
            d.copy_(init)
        rc = lib.cgx_transfer_pairs_noalloc(pairs, n, None)
        assert rc == 0, lib.cgx_last_error()
        assert lib.cgx_noalloc_check(None) == 0, lib.cgx_last_error()
        for i, ((d, _), r, o) in enumerate(zip(na_dsts, ref_dsts, oracle_dsts)):
            a = d.cpu().numpy().view(np.uint64)
            assert np.array_equal(a, r.cpu().numpy().view(np.uint64)), (call, i, "per box")
            assert np.array_equal(a, o.view(np.uint64)), (call, i, "oracle")


def test_noalloc_second_list_reuses_scratch(lib):
    """a different, shorter list right after: the shared scratch keeps the
    previous call's contents, and the counter must start from zero again"""
    pairs, keep, ref_dsts, na_dsts, oracle_dsts = _run(lib, 778, 17)
    rc = lib.cgx_transfer_pairs_noalloc(pairs, len(ref_dsts), None)
    assert rc == 0, lib.cgx_last_error()
    assert lib.cgx_noalloc_check(None) == 0, lib.cgx_last_error()
    for (d, _), r, o in zip(na_dsts, ref_dsts, oracle_dsts):
        assert np.array_equal(d.cpu().numpy().view(np.uint64), r.cpu().numpy().view(np.uint64))
        assert np.array_equal(d.cpu().numpy().view(np.uint64), o.view(np.uint64))


def test_noalloc_refuses_stream_capture(lib):
    """the descriptors come from host memory that the call does not keep, so
    a call on a stream under capture is refused and the capture ends cleanly"""
    pairs, keep, ref_dsts, na_dsts, _ = _run(lib, 780, 4)
    s = torch.cuda.Stream()
    sp = C.c_void_p(s.cuda_stream)
    lib.cgx_graph_begin.argtypes = [C.c_void_p]
    lib.cgx_graph_end.argtypes = [C.c_void_p, C.POINTER(C.c_void_p)]
    lib.cgx_graph_destroy.argtypes = [C.c_void_p]
    assert lib.cgx_graph_begin(sp) == 0, lib.cgx_last_error()
    rc = lib.cgx_transfer_pairs_noalloc(pairs, len(ref_dsts), sp)
    g = C.c_void_p()
    assert lib.cgx_graph_end(sp, C.byref(g)) == 0, lib.cgx_last_error()
    lib.cgx_graph_destroy(g)
    assert rc == 2
    assert b"capture" in lib.cgx_last_error()


def test_noalloc_rejects_too_many_pairs(lib):
    _, cgx_pair = _structs()
    n = 2049
    pairs = (cgx_pair * n)()
    rc = lib.cgx_transfer_pairs_noalloc(pairs, n, None)
    assert rc == 1
    assert b"2048" in lib.cgx_last_error()


def test_noalloc_refuses_pairs_that_need_temporaries(lib):
    """a restriction between timelevels runs through per-timelevel
    temporaries, which this entry point does not allocate"""
    from carpet_b200._lib import box9  # noqa: F401  (loads the library)
    cgx_array, cgx_pair = _structs()
    rng = np.random.default_rng(779)
    c = cases.vc_restrict_case(rng, max_ext=8)
    src = torch.from_numpy(c["src"].copy()).cuda()
    dst = torch.from_numpy(c["dst"].copy()).cuda()

    def arr(t, bbox):
        a = cgx_array()
        a.data = t.data_ptr()
        a.padext[:] = (t.shape[2], t.shape[1], t.shape[0])
        a.bbox[:] = bbox
        return a

    pairs = (cgx_pair * 1)()
    p = pairs[0]
    p.op, p.cent = OP_LAGRANGE, VERTEX
    p.dst = arr(dst, c["dstbbox"])
    for t in range(3):
        p.srcs[t] = arr(src, c["srcbbox"])
    p.times[:] = [0.5, 0.375, 0.25]
    p.nsrc = 3
    p.dstbox[:] = c["reg"]
    p.srcbox[:] = c["srcbbox"]
    p.has_slab = 0
    p.time = 0.45
    p.order_space, p.order_time = 1, 2
    rc = lib.cgx_transfer_pairs_noalloc(pairs, 1, None)
    assert rc == 2, lib.cgx_last_error()
    assert b"temporaries" in lib.cgx_last_error()
