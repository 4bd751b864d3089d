"""GPU: BFS levels are bit-exact against a from-scratch BFS of the current graph after every
batch, and against the reference rule's levels wherever that rule is exact."""
import numpy as np
import pytest

import scout_b200 as sb
from oracle import oracle as orc
from gpu_util import stream

pytestmark = pytest.mark.gpu


def _run(off, adj, batches, source=0, check_ref=True):
    init = orc.gt_bfs(off, adj, source)
    ref = orc.Engine("bfs", off, adj, init)
    g = orc.Graph(off, adj)
    mirror = init.copy()
    with sb.Context(0) as ctx:
        ctx.load_csr(off, adj)
        ctx.set_source(source)
        ctx.upload("bfs", init)
        for b in batches:
            st = ctx.repair("bfs", b)
            flags = [not g.is_adjacent(u, v) for u, v in b.tolist() if u != v]
            for (u, v), f in zip([p for p in b.tolist() if p[0] != p[1]], flags):
                (g.insert if f else g.remove)(u, v)
            o, a = g.csr()
            truth = orc.gt_bfs(o, a, source)
            got = ctx.download("bfs")
            assert np.array_equal(got, truth), f"levels differ at {np.flatnonzero(got != truth)[:10]}"
            before = mirror.copy()
            changed = ctx.commit("bfs", mirror)
            assert np.array_equal(mirror, truth)
            assert changed == int((before != truth).sum())
            ref.batch(b)
            s = ref.stats()
            if check_ref and s["deferred"] == 0 and s["truncated"] == 0 and np.array_equal(ref.solution(), truth):
                assert np.array_equal(got, ref.solution())
        st = ctx.recompute_bfs(source)
        assert np.array_equal(ctx.download("bfs"), orc.gt_bfs(*g.csr(), source))
    return st


def test_sample(sample_graph, sample_batches):
    off, adj = sample_graph
    _run(off, adj, sample_batches)


@pytest.mark.parametrize("kind,m,k,ratio", [(sb.STREAM_MIXED, 1000, 10, 0.5),
                                            (sb.STREAM_PREFERENTIAL, 10000, 3, 0.5),
                                            (sb.STREAM_LOWDEG, 4000, 3, 0.0),
                                            (sb.STREAM_MIXED, 3000, 3, 1.0)])
def test_rmat16_streams(rmat16, kind, m, k, ratio):
    off, adj = rmat16[1]
    _run(off, adj, stream(off, adj, kind, m, k, seed=31, insert_ratio=ratio, lowdeg_frac=0.5))


def test_disconnecting_deletions_and_other_source():
    # two paths joined by a bridge, plus an isolated vertex: deleting the bridge strands half
    n = 41
    edges = [(i, i + 1) for i in range(19)] + [(20 + i, 21 + i) for i in range(19)] + [(19, 20), (5, 30)]
    rows = [[] for _ in range(n)]
    for u, v in edges:
        rows[u].append(v)
        rows[v].append(u)
    off = np.concatenate([[0], np.cumsum([len(r) for r in rows])]).astype(np.int64)
    adj = np.concatenate([sorted(r) for r in rows if r]).astype(np.int32)
    batches = [np.array([[19, 20]], np.int32), np.array([[5, 30]], np.int32), np.array([[19, 20], [40, 0]], np.int32),
               np.array([[40, 0], [3, 4], [10, 11]], np.int32)]
    _run(off, adj, batches, source=0)
    _run(off, adj, batches, source=25)
