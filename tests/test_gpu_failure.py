"""Failure detection without a GPU fault: the bounded device waits.

Every wait of the kernels on a device event -- a TMA copy landing on its
mbarrier, a chain tile's dependency counter -- gives up after about a second,
records CGX_EDEVICE in the launch's status word and lets the launch drain,
so that the context stays usable.  These tests make such waits run out with
the library's failure-injection hooks (a plane that is never staged; a
dependency count that is never reached), check that the host reads
CGX_EDEVICE, and then check that the next normal launch on the same context
is bit-exact with the oracle.  No test faults, traps or hangs the GPU.
"""
import numpy as np
import pytest

from oracle import cases
from oracle.binding import OP_LAGRANGE, VERTEX, Port

pytestmark = pytest.mark.gpu
torch = pytest.importorskip("torch")

EDEVICE = 5


@pytest.fixture(scope="module")
def cb():
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    import carpet_b200
    return carpet_b200


def _prolong_batch(cb, seed):
    """one order-5 prolongation with 3-timelevel time interpolation on arrays
    the TMA kernels stage; returns (batch, destination, expected, keep)"""
    rng = np.random.default_rng(seed)
    c = cases.vc_prolong_case(rng, 5, max_ext=40)
    times, time = [1.0, 0.75, 0.5], 0.875
    srcs_np = [c["src"], c["src"] * 0.5, c["src"] - 1.0]
    want = c["dst"].copy()
    Port().transfer(OP_LAGRANGE, VERTEX, want, c["dstbbox"], srcs_np, c["srcbbox"], times, c["reg"],
                    c["srcbbox"], time, 5, 2)
    dst = cb.Data(c["dstbbox"], torch.from_numpy(c["dst"].copy()).cuda())
    srcs = [cb.Data(c["srcbbox"], torch.from_numpy(s.copy()).cuda()) for s in srcs_np]
    b = cb.Batch()
    b.add(dst, srcs, times, c["reg"], c["srcbbox"], time, 5, 2)
    b.upload()
    return b, dst, want, (srcs, c)


def test_tma_wait_runs_out_and_context_recovers(cb):
    from carpet_b200._lib import lib
    cb.set_fp_mode(False)
    b, dst, want, keep = _prolong_batch(cb, 71)
    init = dst.tensor.clone()
    assert b.kernels() >= 1
    assert lib.cgx_debug_skip_tma_plane(1) == 0
    try:
        b.launch()
        with pytest.raises(cb.CgxError) as e:
            b.check()
        assert e.value.code == EDEVICE
    finally:
        lib.cgx_debug_skip_tma_plane(0)
    # the same batch, normal again, on the same context
    dst.tensor.copy_(init)
    b.launch()
    b.check()
    torch.cuda.synchronize()
    got = dst.tensor.cpu().numpy()
    assert np.array_equal(got.view(np.uint64), want.view(np.uint64))


def test_chain_dependency_wait_runs_out_and_context_recovers(cb):
    """two dependent batches in one chain: the second waits for the first
    (same group); with the hold, the count it waits for is never reached"""
    from carpet_b200._lib import lib
    cb.set_fp_mode(False)
    b0, d0, want0, k0 = _prolong_batch(cb, 72)
    rng = np.random.default_rng(73)
    c = cases.copy_case(rng, max_ext=30)
    want1 = c["dst"].copy()
    Port().copy_3d(c["src"], c["srcbbox"], want1, c["dstbbox"], c["srcreg"], c["dstreg"], None)
    d1 = cb.Data(c["dstbbox"], torch.from_numpy(c["dst"].copy()).cuda())
    s1 = cb.Data(c["srcbbox"], torch.from_numpy(c["src"].copy()).cuda())
    b1 = cb.Batch()
    b1.add(d1, [s1], [0.0], c["dstreg"], c["srcreg"], 0.0, 1, 0)
    b1.upload()
    ch = cb.Chain([b0, b1])
    assert lib.cgx_chain_debug_hold(ch.h, 1) == 0
    ch.upload()
    i0, i1 = d0.tensor.clone(), d1.tensor.clone()
    ch.launch()
    with pytest.raises(cb.CgxError) as e:
        ch.check()
    assert e.value.code == EDEVICE
    # without the hold: both batches complete, bit-exact
    assert lib.cgx_chain_debug_hold(ch.h, 0) == 0
    ch.upload()
    d0.tensor.copy_(i0)
    d1.tensor.copy_(i1)
    ch.launch()
    ch.check()
    torch.cuda.synchronize()
    assert np.array_equal(d0.tensor.cpu().numpy().view(np.uint64), want0.view(np.uint64))
    assert np.array_equal(d1.tensor.cpu().numpy().view(np.uint64), want1.view(np.uint64))


def test_served_wait_runs_out_is_reported(cb):
    """a served launch whose prolongation kernel gives up a bounded wait:
    the server reads the launch's status back when it retires the slot, and
    drain() reports CGX_EDEVICE with the worker's message; a new server on
    the same context then gives what the requests give served alone"""
    from carpet_b200._lib import lib
    from carpet_b200.serve import (SERVE_BATCHED, SERVE_PLAIN, Ensemble, Server, ops_for,
                                   request_key)
    cb.set_fp_mode(False)
    sv = Server(mode=SERVE_BATCHED)
    ens = Ensemble(sv, nhier=2, size_range=(24, 24), seed=5)
    rng = np.random.default_rng(1)
    keys = [request_key(ens, m, 1, rng) for m in range(2)]  # boundary prolongations
    init = ens.snapshot()
    lib.cgx_debug_skip_tma_plane(1)
    try:
        sv.replay(ops_for(ens.ops, keys), [0.0] * len(keys))
        with pytest.raises(cb.CgxError) as err:
            sv.drain()
    finally:
        lib.cgx_debug_skip_tma_plane(0)
    assert err.value.code == EDEVICE and "device wait ran out" in str(err.value)
    sv.close()
    again, plain = Server(mode=SERVE_BATCHED), Server(mode=SERVE_PLAIN)
    ops_again, ops_plain = ens.define(again), ens.define(plain)
    ens.restore(init)
    again.replay(ops_for(ops_again, keys), [0.0] * len(keys))
    again.drain()
    got = [[p.clone() for p in ens.state(m)] for m in range(2)]
    ens.restore(init)
    for k in keys:
        plain.submit(ops_plain[k])
        plain.drain()
    for m in range(2):
        assert all(torch.equal(a.view(torch.int64), b.view(torch.int64))
                   for a, b in zip(got[m], ens.state(m)))
    again.close()
    plain.close()
