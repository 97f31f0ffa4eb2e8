"""The chain form (cgx_chain_*): a whole coarse Berger-Oliger step as one
persistent launch with per-grid-function dependency counters.

The same seeded hierarchy is stepped twice from identical states: once with
one launch per phase (the batched form, each phase a batch in the call
order of Carpet/src/Evolve.cc:44-121) and once as a chain; every array of
every level and timelevel must agree bit for bit, after one step and after
three (the timelevel rotation), eagerly and replayed from a CUDA graph, in
both floating-point modes.  Also: the chain refuses what its kernel does
not run, and its status reads clean.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu
torch = pytest.importorskip("torch")


@pytest.fixture(scope="module")
def cb():
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    import carpet_b200
    return carpet_b200


def _pair(cb, levels, npts, ngf, seed):
    from carpet_b200.amr import BergerOliger, Storage
    from carpet_b200.hierarchy import nested
    h = nested(levels, npts, ghost=3, buffer=9, order=5)
    a = Storage(h, ngf, 3)
    b = Storage(h, ngf, 3)
    g = torch.Generator(device="cuda").manual_seed(seed)
    for la, lb in zip(a.pools, b.pools):
        for p, q in zip(la, lb):
            p.copy_(torch.randn(p.shape, generator=g, device="cuda", dtype=torch.float64))
            q.copy_(p)
    return h, a, b, BergerOliger(h, a, order_space=5, order_time=2), \
        BergerOliger(h, b, order_space=5, order_time=2, chain=True)


def _same(a, b):
    for la, lb in zip(a.pools, b.pools):
        for p, q in zip(la, lb):
            if not torch.equal(p.view(torch.int64), q.view(torch.int64)):
                return False
    return True


@pytest.mark.parametrize("fma", [False, True], ids=["exact", "fma"])
def test_chain_step_matches_phase_launches(cb, fma):
    cb.set_fp_mode(fma)
    h, sa, sb, ref, ch = _pair(cb, 4, 33, 5, 11)
    s = torch.cuda.Stream()
    for step in range(3):
        ka, kb = ref.step_phases(), ch.step_phases()
        assert ka == kb
        ref.run(ka, s)
        ch.run(kb, s)
        s.synchronize()
        for c in ch.chains.values():
            c.check(s)
        assert _same(sa, sb), f"step {step}"
    cb.set_fp_mode(False)


def test_chain_graph_replay(cb):
    cb.set_fp_mode(False)
    h, sa, sb, ref, ch = _pair(cb, 5, 33, 4, 12)
    s = torch.cuda.Stream()
    keys = [ch.step_phases() for _ in range(3)]
    ref.rot = [0] * ref.L
    rkeys = [ref.step_phases() for _ in range(3)]
    assert keys == rkeys
    graphs = []
    for k in keys:
        ch.chain(k, s)  # upload outside the capture
        g = cb.Graph()
        with g.capture(s):
            ch.run(k, s)
        graphs.append(g)
    for step in range(6):
        ref.run(rkeys[step % 3], s)
        graphs[step % 3].launch(s)
    s.synchronize()
    for c in ch.chains.values():
        c.check(s)
    assert _same(sa, sb)


def test_chain_matches_at_bench_scale(cb):
    """the benchmark hierarchy (5 levels of 129^3, 2x2x2 components) with
    6 grid functions: the chain's dependency counters under a full load"""
    cb.set_fp_mode(False)
    h, sa, sb, ref, ch = _pair(cb, 5, 129, 6, 13)
    s = torch.cuda.Stream()
    for step in range(2):
        ref.run(ref.step_phases(), s)
        ch.run(ch.step_phases(), s)
    s.synchronize()
    for c in ch.chains.values():
        c.check(s)
    assert _same(sa, sb)


def test_chain_refuses_other_operators(cb):
    from oracle import cases
    rng = np.random.default_rng(5)
    c = cases.cc_prolong_case(rng, 3, max_ext=12)
    dst = cb.Data(c["dstbbox"], torch.from_numpy(c["dst"].copy()).cuda())
    src = cb.Data(c["srcbbox"], torch.from_numpy(c["src"].copy()).cuda())
    b = cb.Batch()
    b.add(dst, [src], [0.0], c["reg"], c["srcbbox"], 0.0, 3, 0, cent=cb.CELL)
    ch = cb.Chain([b])
    with pytest.raises(cb.CgxError) as e:
        ch.upload()
    assert e.value.code == 2  # CGX_EUNSUPPORTED
