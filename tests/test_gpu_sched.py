"""GPU tests of the repair variants and the learned scheduler.

- every BFS variant (incremental, top-down traversal, direction-optimizing traversal) and
  every CC variant (incremental, recompute) gives the exact solution of the current graph
  after every batch, and the commit copies back only changed entries;
- the probe's variants agree vertex for vertex and its features equal the oracle's;
- the cost model's device gradients equal the float64 oracle's (relative 1e-4), its fp32
  and bf16 forward passes match, and training reduces the loss;
- trained on probed batches, the model picks variants whose total repair time on held-out
  streams is below the plain engine's (always incremental), and the engine's on-device
  decisions equal the argmin of the same model's bf16 forward pass on the same features.
"""
import numpy as np
import pytest

import scout_b200 as sb
from gpu_util import stream
from oracle import oracle as orc
from oracle import sched_oracle as so

pytestmark = pytest.mark.gpu


class Mirror:
    def __init__(self, off, adj):
        self.g = orc.Graph(off, adj)

    def apply(self, b):
        pairs = [p for p in b.tolist() if p[0] != p[1]]
        flags = [not self.g.is_adjacent(u, v) for u, v in pairs]
        for (u, v), f in zip(pairs, flags):
            (self.g.insert if f else self.g.remove)(u, v)
        return self.g.csr()


def _batches(off, adj):
    return (list(stream(off, adj, sb.STREAM_PREFERENTIAL, 20000, 2, seed=61))
            + list(stream(off, adj, sb.STREAM_LOWDEG, 20000, 2, seed=62, insert_ratio=0.1, lowdeg_frac=0.6))
            + list(stream(off, adj, sb.STREAM_MIXED, 500, 2, seed=63)))


@pytest.mark.parametrize("sched", [{"mode": 1}, {"mode": 2, "frontier": 1}, {"mode": 2, "frontier": 2}])
def test_bfs_variants_exact(rmat16, sched):
    off, adj = rmat16[1]
    m = Mirror(off, adj)
    init = orc.gt_bfs(off, adj, 0)
    mirror = init.copy()
    want_variant = 0 if sched["mode"] == 1 else sched["frontier"]
    with sb.Context(0) as ctx:
        ctx.load_csr(off, adj)
        ctx.upload("bfs", init)
        for b in _batches(off, adj):
            before = mirror.copy()
            st = ctx.repair("bfs", b, sched=sched)
            assert st["variant"] == want_variant
            o, a = m.apply(b)
            got = ctx.download("bfs")
            assert np.array_equal(got, orc.gt_bfs(o, a, 0))
            assert ctx.commit("bfs", mirror) == int((before != got).sum())
            if want_variant:   # a traversal lists exactly the changed levels (the diff pass)
                assert st["changed"] == int((before != got).sum()), "the commit list holds unchanged entries"
            assert np.array_equal(mirror, got)


@pytest.mark.parametrize("sched", [{"mode": 1}, {"mode": 2}])
def test_cc_variants_exact(rmat16, sched):
    off, adj = rmat16[1]
    m = Mirror(off, adj)
    init = orc.gt_cc(off, adj)
    mirror = init.copy()
    with sb.Context(0) as ctx:
        ctx.load_csr(off, adj)
        ctx.upload("cc", init)
        for b in _batches(off, adj):
            before = mirror.copy()
            st = ctx.repair("cc", b, sched=sched)
            assert st["variant"] == (1 if sched["mode"] == 2 else 0)
            o, a = m.apply(b)
            got = ctx.download("cc")
            assert np.array_equal(got, orc.gt_cc(o, a))
            assert ctx.commit("cc", mirror) == int((before != got).sum())
            assert np.array_equal(mirror, got)


@pytest.mark.parametrize("problem", ["bfs", "cc"])
def test_probe_agrees_and_features_match_oracle(rmat16, problem):
    off, adj = rmat16[1]
    m = Mirror(off, adj)
    init = orc.gt_bfs(off, adj, 0) if problem == "bfs" else orc.gt_cc(off, adj)
    mirror = init.copy()
    r = np.random.default_rng(5)
    with sb.Context(0) as ctx:
        ctx.load_csr(off, adj)
        ctx.upload(problem, init)
        prev = 0.0
        for b in _batches(off, adj)[:5]:
            # distinct pairs so that every toggle is applied (the oracle's feature rule)
            key = np.minimum(b[:, 0], b[:, 1]).astype(np.int64) << 32 | np.maximum(b[:, 0], b[:, 1])
            _, first = np.unique(key, return_index=True)
            b = b[np.sort(first)]
            b = b[b[:, 0] != b[:, 1]]
            b = b[r.permutation(len(b))]
            o0, a0 = m.g.csr()
            lv = ctx.download("bfs") if problem == "bfs" else None
            st, ms, f = ctx.repair_probe(problem, b)
            nv = 3
            assert (ms[:nv] > 0).all()
            want = so.features(o0, a0, b, problem, level=lv, prev_ms=prev)
            np.testing.assert_allclose(f, want, atol=1e-5)
            prev = float(ms[:nv].min())
            o, a = m.apply(b)
            got = ctx.download(problem)
            truth = orc.gt_bfs(o, a, 0) if problem == "bfs" else orc.gt_cc(o, a)
            assert np.array_equal(got, truth)
            ctx.commit(problem, mirror)
            assert np.array_equal(mirror, got)


def _bf16_round(w):
    """fp32 -> bf16 (round to nearest, ties to even) -> fp32."""
    u = np.ascontiguousarray(w, dtype=np.float32).view(np.uint32).astype(np.uint64)
    u = ((u + 0x7FFF + ((u >> 16) & 1)) >> 16) << 16
    return u.astype(np.uint32).view(np.float32)


def test_mlp_gradients_match_oracle():
    r = np.random.default_rng(11)
    n = 300
    x = r.uniform(0, 1, (n, 24)).astype(np.float32)
    t = r.normal(0, 1, (n, 4)).astype(np.float32)
    mk = (r.uniform(0, 1, (n, 4)) < 0.75).astype(np.float32)
    with sb.MLP(0, seed=3) as net:
        w = net.params
        loss, g = net.loss_grad(x, t, mk)
        L, g_ref = so.loss_grad(w.astype(np.float64), x, t, mk)
        assert abs(loss - L) <= 1e-4 * abs(L)
        # relative to the gradient's scale (fp32 tiles summed atomically)
        err = np.abs(g - g_ref).max() / np.abs(g_ref).max()
        assert err < 1e-4, err
        y = net.forward(x)
        np.testing.assert_allclose(y, so.forward(w, x), rtol=1e-4, atol=1e-4)
        yb = net.forward(x, bf16=True)
        np.testing.assert_allclose(yb, so.forward(_bf16_round(w), x), rtol=1e-3, atol=1e-3)


def test_mlp_training_reduces_loss():
    r = np.random.default_rng(12)
    n = 4096
    x = r.uniform(0, 1, (n, 24)).astype(np.float32)
    t = np.stack([x[:, 0] * 2 - x[:, 1], np.sin(3 * x[:, 2]), x[:, 3] * x[:, 4], x[:, 5:10].sum(1) / 5], 1)
    mk = np.ones((n, 4), dtype=np.float32)
    with sb.MLP(0, seed=4) as net:
        l0, _ = net.loss_grad(x, t, mk)
        losses = net.train(x, t, mk, epochs=60, batch=128, lr=3e-3, seed=1)
        l1, _ = net.loss_grad(x, t, mk)
    assert np.isfinite(losses).all()
    assert l1 < 0.1 * l0, (l0, l1)
    assert losses[-1] < losses[0]


def test_learned_scheduler_beats_plain_on_held_out_streams():
    from scout_b200 import learn
    specs_tr = learn.default_specs("bfs", range(3), scales=(14, 16), sizes=(100, 2000, 30000, 120000))
    specs_ev = learn.default_specs("bfs", range(50, 52), scales=(14, 16), sizes=(100, 2000, 30000, 120000))
    graphs = {}
    tr = learn.collect("bfs", specs_tr, graphs=graphs)
    ev = learn.collect("bfs", specs_ev, graphs=graphs)
    params, losses = learn.train(tr, epochs=300)
    assert losses[-1] < losses[0]
    res = learn.evaluate(params, ev, "bfs")
    print(res)
    # the learned choice costs less repair time than always-incremental, and its regret
    # against the per-batch best variant is smaller
    assert res["learned_ms"] < res["plain_ms"], res
    assert res["learned_regret"] < res["plain_regret"], res

    # the engine's own on-device decision equals the bf16 model's argmin on the features
    g = graphs[(16, 16, 150)]
    off, adj = g.arrays()
    m = Mirror(off, adj)
    init = orc.gt_bfs(off, adj, 0)
    batches = stream(off, adj, sb.STREAM_LOWDEG, 60000, 2, seed=71, insert_ratio=0.3, lowdeg_frac=0.3)
    small = stream(off, adj, sb.STREAM_MIXED, 200, 2, seed=72)
    with sb.Context(0) as ctx:
        ctx.load_csr(off, adj)
        ctx.upload("bfs", init)
        ctx.sched_install("bfs", params)
        for b in list(batches) + list(small):
            st = ctx.repair("bfs", b, sched={"policy": 1})
            f, y, d = ctx.sched_last()
            assert d == st["variant"]
            pick = learn.choose(params, f[None, :], 3)[0]
            assert d == pick
            o, a = m.apply(b)
            assert np.array_equal(ctx.download("bfs"), orc.gt_bfs(o, a, 0))
        ctx.sched_install("bfs", None)
        st = ctx.repair("bfs", small[0], sched={"policy": 1})
        assert st["variant"] == 0, "without a model the plain policy runs"
