"""The served form on the GPU: many small hierarchies behind the request
server (cgx_server_* in include/cgx.h).

* Continuous batching keeps each hierarchy's requests in arrival order, so
  the final grid data after a Poisson stream served batched is bit-for-bit
  the data after serving the same stream one request at a time through the
  per-box drop-in (every request alone, in order).
* Per request: in rounds where every hierarchy receives exactly one request
  (sync, prolongation, restriction or regrid fill), all of a round's
  requests are served together in the mix and, separately, each alone; every
  hierarchy's arrays -- that request's result -- agree bit for bit.
* Admission refuses hierarchies beyond the HBM budget; once a hierarchy is
  retired, a waiting one is admitted while the server runs, its operations
  are defined mid-stream, and its requests are served as they would be alone.
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
    return [p.clone() for m in range(len(ens.members)) if not ens.members[m].retired
            for p in ens.state(m)]


def _equal(xs, ys):
    return len(xs) == len(ys) and all(torch.equal(a.view(torch.int64), b.view(torch.int64))
                                      for a, b in zip(xs, ys))


@pytest.mark.parametrize("config,burst,pool", [(0, False, 65536), (2, False, 65536), (0, True, 65536),
                                               (2, True, 65536), (1, True, 16)])
def test_batched_stream_equals_requests_alone(cgx, config, burst, pool):
    """a Poisson stream, or the same requests submitted at once (every
    launch then takes the next request of hierarchies still in flight on
    another slot, ordered on the device by the slots' completion events), in
    several tile configurations; with a descriptor pool of 16 entries at
    first, which the operations' definitions grow many times over"""
    from carpet_b200.serve import (SERVE_BATCHED, SERVE_PLAIN, Ensemble, Server, ops_for,
                                   poisson_trace)
    cgx.set_fp_mode(False)
    batched = Server(mode=SERVE_BATCHED, max_pairs=pool)
    batched.set_config(config)
    plain = Server(mode=SERVE_PLAIN)
    ens = Ensemble(batched, nhier=8, size_range=(24, 40), seed=11, regrid=True)
    plain_ops = ens.define(plain)
    keys, arr = poisson_trace(ens, rate=1e5, n=300, seed=3, mix=(0.55, 0.25, 0.15, 0.05))
    if burst:
        arr = [0.0] * len(keys)
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
    assert rb["bytes"] == rp["bytes"] > 0
    assert _equal(got, want)
    batched.close()
    plain.close()


def test_each_request_alone_equals_in_mix(cgx):
    """rounds of one request per hierarchy: the round served as one burst
    (continuously batched, requests of different hierarchies overlapping on
    the GPU) against each request served alone"""
    from carpet_b200.serve import SERVE_BATCHED, SERVE_PLAIN, Ensemble, Server, ops_for, request_key
    cgx.set_fp_mode(False)
    batched = Server(mode=SERVE_BATCHED)
    plain = Server(mode=SERVE_PLAIN)
    ens = Ensemble(batched, nhier=12, size_range=(24, 48), seed=21, regrid=True)
    plain_ops = ens.define(plain)
    rng = np.random.default_rng(5)
    kinds = set()
    for rnd in range(4):
        keys = []
        for m in range(len(ens.members)):
            k = int(rng.integers(0, 4))
            keys.append(request_key(ens, m, k, rng))
            kinds.add(k)
        before = ens.snapshot()
        batched.replay(ops_for(ens.ops, keys), [0.0] * len(keys))  # one burst
        batched.drain()
        mix = [[p.clone() for p in ens.state(m)] for m in range(len(ens.members))]
        ens.restore(before)
        for key in keys:                                # each request alone
            plain.submit(plain_ops[key])
            plain.drain()
        for m in range(len(ens.members)):
            assert _equal(mix[m], ens.state(m)), (rnd, keys[m])
    assert kinds == {0, 1, 2, 3}
    assert batched.report()["mean_batch"] > 1.0
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


def test_admission_while_serving(cgx):
    """a waiting hierarchy is admitted mid-stream after another retires; its
    operations are defined on the running server and its requests give what
    they give served alone"""
    from carpet_b200.amr import storage_bytes
    from carpet_b200.hierarchy import nested
    from carpet_b200.serve import (SERVE_BATCHED, SERVE_PLAIN, Ensemble, Server, ops_for,
                                   poisson_trace, request_key)
    cgx.set_fp_mode(False)
    h = nested(3, (25, 25, 25), parts=(2, 1, 1), ghost=3, buffer=3, order=5)
    one = storage_bytes(h, 4, 3)
    # a small descriptor pool: the operations defined mid-stream grow it while
    # the worker launches from it
    sv = Server(mode=SERVE_BATCHED, hbm_budget=int(3.5 * one), max_pairs=64)
    plain = Server(mode=SERVE_PLAIN)
    ens = Ensemble(sv, nhier=5, size_range=(24, 24), seed=7)
    assert len(ens.members) == 3 and ens.deferred == 2
    keys, arr = poisson_trace(ens, rate=2e4, n=120, seed=9)
    sv.replay(ops_for(ens.ops, keys), arr)          # starts the worker
    sv.drain()
    ens.retire(0)                                   # its memory returns to the budget
    new, (plain_ops,) = ens.admit_pending([plain])  # defined while sv runs
    assert len(new) == 1 and ens.deferred == 1
    m = new[0]
    init = [p.clone() for p in ens.state(m)]
    rng = np.random.default_rng(3)
    # work queued on the other hierarchies, then more definitions: the pool
    # grows (copied into a larger allocation) while those launches read it
    busy = [request_key(ens, 1 + i % 2, int(rng.integers(0, 3)), rng) for i in range(200)]
    sv.replay(ops_for(ens.ops, busy), [0.0] * len(busy))
    for _ in range(3):
        ops_now = ens.define(sv)
    sv.drain()
    mine = [request_key(ens, m, int(rng.integers(0, 3)), rng) for _ in range(20)]
    others = [request_key(ens, 1 + i % 2, int(rng.integers(0, 3)), rng) for i in range(20)]
    stream = [k for pair in zip(mine, others) for k in pair]
    sv.replay(ops_for(ops_now, stream), [1e-5 * i for i in range(len(stream))])
    sv.drain()
    got = [p.clone() for p in ens.state(m)]
    for p, q in zip(ens.state(m), init):
        p.copy_(q)
    for k in mine:                                  # alone, one at a time
        plain.submit(plain_ops[k])
        plain.drain()
    assert _equal(got, ens.state(m))
    sv.close()
    plain.close()


def test_each_request_type_matches_the_oracle(cgx):
    """every operation of a hierarchy -- the sync of each level, the
    boundary prolongation of each refined level (order 5, 3-timelevel time
    interpolation), the restriction into each coarser level and the regrid
    fill of the moved finest level -- served through the batched server
    gives, bit for bit, what the oracle gives for the same box-pairs on
    host copies of the same arrays"""
    from carpet_b200.moving import old2new
    from carpet_b200.serve import SERVE_BATCHED, Ensemble, Server
    from oracle.binding import OP_LAGRANGE, VERTEX, Port
    cgx.set_fp_mode(False)
    port = Port()
    sv = Server(mode=SERVE_BATCHED)
    ens = Ensemble(sv, nhier=2, size_range=(24, 32), seed=17, regrid=True)
    m = 1
    mem = ens.members[m]
    h, st, L = mem.hier, mem.storage, len(mem.hier.levels)
    dtc = 1.0 / 64
    times3 = [0.0, -dtc, -2 * dtc]
    kinds = set()
    for key in sorted(k for k in ens.ops if k[0] == m):
        _, kind, l = key
        calls = []  # (dst, srcs, dstbox, srcbox, times, time, order_space, order_time)
        for g in range(st.ngf):
            if kind == "sync":
                a = st.data[l][0][g]
                calls += [(a[p.dst_comp], [a[p.src_comp]], p.dstbox, p.srcbox, [0.0], 0.0, 1, 0)
                          for p in h.sync[l]]
            elif kind == "prolong":
                calls += [(st.data[l][0][g][p.dst_comp], [st.data[l - 1][t][g][p.src_comp] for t in range(3)],
                           p.dstbox, p.srcbox, times3, -dtc / 2, 5, 2) for p in h.prolong[l]]
            elif kind == "restrict":
                calls += [(st.data[l][0][g][p.dst_comp], [st.data[l + 1][0][g][p.src_comp]], p.dstbox,
                           p.srcbox, [0.0], 0.0, 5, 0) for p in h.restrict[l + 1]]
        if kind == "regrid":
            copies, prols = old2new(h, mem.moved, l)
            for tl in range(st.ntl):
                dst = mem.moved_storage.data[l][tl]
                for g in range(st.ngf):
                    calls += [(dst[g][p.dst_comp], [st.data[l][tl][g][p.src_comp]], p.dstbox, p.srcbox,
                               [0.0], 0.0, 1, 0) for p in copies]
                    calls += [(dst[g][p.dst_comp], [st.data[l - 1][tl][g][p.src_comp]], p.dstbox,
                               p.srcbox, [0.0], 0.0, 5, 0) for p in prols]
        assert calls, key
        kinds.add(kind)
        datas = {}
        for dst, srcs, *_ in calls:
            for d in [dst] + srcs:
                datas[id(d)] = d
        host = {i: d.tensor.cpu().numpy().copy() for i, d in datas.items()}
        for dst, srcs, dbox, sbox, tms, t, osp, ot in calls:
            port.transfer(OP_LAGRANGE, VERTEX, host[id(dst)], list(dst.extent), [host[id(s)] for s in srcs],
                          list(srcs[0].extent), tms, list(dbox), list(sbox), t, osp, ot)
        sv.submit(ens.ops[key])
        sv.drain()
        for i, d in datas.items():
            assert np.array_equal(d.tensor.cpu().numpy().view(np.uint64), host[i].view(np.uint64)), key
    assert kinds == {"sync", "prolong", "restrict", "regrid"}
    sv.close()
