"""The served form on the GPU: many small hierarchies behind the request
server (cgx_server_* in include/cgx.h).

* Continuous batching keeps each hierarchy's requests in arrival order, so
  the final grid data after a Poisson stream served batched is bit-for-bit
  the data after serving the same stream one request at a time through the
  per-box drop-in (every request alone, in order).
* Admission refuses hierarchies beyond the HBM budget and admits again once
  memory is released.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu
torch = pytest.importorskip("torch")


@pytest.fixture(scope="module")
def cgx():
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    import carpet_b200 as cb
    return cb


def _state(ens):
    return [p.clone() for m in ens.members for lp in m.storage.pools for p in lp]


def test_batched_stream_equals_requests_alone(cgx):
    from carpet_b200.serve import (SERVE_BATCHED, SERVE_PLAIN, Ensemble, Server, ops_for,
                                   poisson_trace)
    cgx.set_fp_mode(True)
    batched = Server(mode=SERVE_BATCHED)
    plain = Server(mode=SERVE_PLAIN)
    ens = Ensemble(batched, nhier=8, size_range=(24, 40), seed=11)
    plain_ops = ens.define(plain)
    keys, arr = poisson_trace(ens, rate=1e5, n=300, seed=3)
    init = ens.snapshot()
    batched.replay(ops_for(ens.ops, keys), arr)
    batched.drain()
    rb = batched.report()
    got = _state(ens)
    ens.restore(init)
    plain.replay(ops_for(plain_ops, keys), arr)
    plain.drain()
    rp = plain.report()
    want = _state(ens)
    assert rb["requests"] == rp["requests"] == 300
    assert rb["launches"] < rp["launches"]          # batched: fewer, larger launches
    assert rb["mean_batch"] > 1.0                   # requests really overlapped
    assert 0 < rb["p50_ms"] <= rb["p99_ms"]
    for a, b in zip(got, want):
        assert torch.equal(a.view(torch.int64), b.view(torch.int64))
    batched.close()
    plain.close()


def test_admission_against_budget(cgx):
    from carpet_b200.amr import storage_bytes
    from carpet_b200.hierarchy import nested
    from carpet_b200.serve import SERVE_BATCHED, Ensemble, Server
    h = nested(3, (25, 25, 25), parts=(2, 1, 1), ghost=3, buffer=3, order=5)
    one = storage_bytes(h, 4, 3)
    sv = Server(mode=SERVE_BATCHED, hbm_budget=int(2.5 * one))
    ens = Ensemble(sv, nhier=5, size_range=(24, 24), seed=0)
    assert len(ens.members) == 2 and ens.deferred == 3
    assert not sv.admit(one)
    ens.close()                      # releases the admitted hierarchies
    assert sv.admit(one) and sv.admit(one)
    sv.close()
