"""The batched uneven configuration on the GPU: box-pairs of uneven sizes and
mixed operators (vertex-centred Lagrange order 5, ENO order 3, cell-centred
Lagrange order 3, cell-centred averaging) in one batch, autotuned, launched
directly and replayed from a CUDA graph, and the same descriptors launched
per box -- all bit-identical to the oracle on the same source values."""
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


@pytest.mark.parametrize("fma", [False, True], ids=["exact", "fma"])
def test_uneven_batch_matches_oracle(cb, port, fma):
    from carpet_b200.uneven import uneven_batch, uneven_pairs, uneven_specs
    cb.set_fp_mode(fma)
    specs = uneven_specs(seed=11, npairs=40, ext=(16, 40))
    assert {s.kind for s in specs} == {"vc_lagrange5", "vc_eno3", "cc_lagrange3", "cc_average"}
    pairs = uneven_pairs(specs, seed=12)
    want = []
    for p in pairs:
        sp = p.spec
        w = p.dst.tensor.cpu().numpy().copy()
        port.transfer(sp.op, sp.cent, w, sp.dstbbox, [p.src.tensor.cpu().numpy()], sp.srcbbox, [0.0],
                      sp.reg, sp.srcbbox, 0.0, sp.order, 0, fma=fma)
        want.append(w)
    init = [p.dst.tensor.clone() for p in pairs]
    b = uneven_batch(pairs)
    chosen = b.autotune(reps=2)
    assert chosen  # the prolongation variants present were tuned
    s = torch.cuda.Stream()
    for mode in ("batch", "graph", "per_box"):
        for p, i in zip(pairs, init):
            p.dst.tensor.copy_(i)
        torch.cuda.synchronize()
        if mode == "batch":
            b.launch(s)
        elif mode == "graph":
            g = cb.Graph()
            with g.capture(s):
                b.launch(s)
            g.launch(s)
        else:
            b.launch_per_box(s)
        s.synchronize()
        b.check(s)
        for p, w in zip(pairs, want):
            got = p.dst.tensor.cpu().numpy()
            assert np.array_equal(got.view(np.uint64), w.view(np.uint64)), (mode, p.spec.kind)
