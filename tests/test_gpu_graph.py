"""GPU: the HBM graph store (load, classification, batch merge, staging, compaction) against
the oracle's restatement of the reference scratchpad (FlashGraph.h:200-388)."""
import numpy as np
import pytest

import scout_b200 as sb
from oracle import oracle as orc
from gpu_util import assert_same_graph, sorted_rows, stream

pytestmark = pytest.mark.gpu


def _ctx_with(off, adj, problem="bfs"):
    ctx = sb.Context(0)
    ctx.load_csr(off, adj)
    ctx.upload(problem, orc.gt_bfs(off, adj, 0))
    return ctx


def test_load_and_download(sample_graph):
    off, adj = sample_graph
    with sb.Context(0) as ctx:
        ctx.load_csr(off, adj)
        o, a = ctx.graph()
        assert np.array_equal(o, off) and np.array_equal(a, adj)
        assert ctx.info()["nnz"] == len(adj)


def test_classify_matches_reference_adjacency(rmat16):
    off, adj = rmat16[1]
    rng = np.random.default_rng(0)
    pairs = rng.integers(0, 65536, size=(20000, 2)).astype(np.int32)
    src = np.repeat(np.arange(65536), np.diff(off))
    pick = rng.integers(0, len(adj), 20000)
    pairs = np.concatenate([pairs, np.stack([src[pick], adj[pick]], 1).astype(np.int32)])
    g = orc.Graph(off, adj)
    with sb.Context(0) as ctx:
        ctx.load_csr(off, adj)
        got = ctx.classify(pairs)
    want = np.array([255 if u == v else (0 if g.is_adjacent(u, v) else 1) for u, v in pairs.tolist()], dtype=np.uint8)
    assert np.array_equal(got, want)


def test_batches_merge_like_the_scratchpad(sample_graph, sample_batches):
    off, adj = sample_graph
    e = orc.Engine("bfs", off, adj, orc.gt_bfs(off, adj, 0))
    with _ctx_with(off, adj) as ctx:
        for b in sample_batches:
            st = ctx.repair("bfs", b)
            e.batch(b)
            assert_same_graph(ctx, e.graph())
            s = e.stats()
        assert ctx.info()["nnz"] == len(e.graph().csr()[1])


@pytest.mark.parametrize("kind,m,k", [(sb.STREAM_MIXED, 1000, 10), (sb.STREAM_PREFERENTIAL, 20000, 3),
                                      (sb.STREAM_LOWDEG, 5000, 3)])
def test_rmat_streams_merge(rmat16, kind, m, k):
    off, adj = rmat16[1]
    batches = stream(off, adj, kind, m, k, seed=21, insert_ratio=0.5 if kind != sb.STREAM_LOWDEG else 0.3,
                     lowdeg_frac=0.3)
    g = orc.Graph(off, adj)
    with _ctx_with(off, adj) as ctx:
        for b in batches:
            st = ctx.repair("bfs", b)
            ins = 0
            for u, v in b.tolist():   # classify against the pre-batch graph, then apply
                pass
            flags = [not g.is_adjacent(u, v) for u, v in b.tolist()]
            assert st["insertions"] == sum(flags) and st["deletions"] == len(flags) - sum(flags)
            for (u, v), f in zip(b.tolist(), flags):
                (g.insert if f else g.remove)(u, v)
            assert_same_graph(ctx, g)


def test_duplicates_and_invalid_edits(sample_graph):
    off, adj = sample_graph
    u0, v0 = 0, int(adj[off[0]])   # an existing edge
    batch = np.array([[3, 1500], [3, 1500], [u0, v0], [v0, u0], [5, 5], [-1, 3], [2000, 1], [7, 9]], dtype=np.int32)
    e = orc.Engine("bfs", off, adj, orc.gt_bfs(off, adj, 0))
    with _ctx_with(off, adj) as ctx:
        st = ctx.repair("bfs", batch)
        e.batch(batch)
        assert st["edits"] == 5   # self-loop and out-of-range ids are dropped, as parse_batch_file does
        assert_same_graph(ctx, e.graph())
        # a later batch deletes one copy of the pair inserted twice (the scratchpad forgets one)
        st = ctx.repair("bfs", np.array([[1500, 3]], dtype=np.int32))
        e.batch(np.array([[1500, 3]], dtype=np.int32))
        assert st["deletions"] == 1
        assert_same_graph(ctx, e.graph())
        st = ctx.repair("bfs", np.zeros((0, 2), dtype=np.int32))
        assert st["edits"] == 0
        assert_same_graph(ctx, e.graph())


def test_explicit_ops_are_conditional(sample_graph):
    off, adj = sample_graph
    u0, v0 = 0, int(adj[off[0]])
    u1, v1 = 1, int(adj[off[1]])
    batch = np.array([[u0, v0], [3, 1500], [4, 1501], [u1, v1]], dtype=np.int32)
    ops = np.array([sb.OP_INSERT, sb.OP_DELETE, sb.OP_INSERT, sb.OP_DELETE], dtype=np.uint8)
    g = orc.Graph(off, adj)
    with _ctx_with(off, adj) as ctx:
        st = ctx.repair("bfs", batch, ops=ops)
        assert st["insertions"] == 2 and st["deletions"] == 2
        # inserting a present edge and deleting an absent one change nothing
        # (scout_mis.cu:743-749); the other two are applied
        g.insert(4, 1501)
        g.remove(u1, v1)
        assert_same_graph(ctx, g)


def test_stage_rows_sorts_and_validates():
    rng = np.random.default_rng(5)
    n = 300
    rows = [np.unique(rng.integers(0, n, rng.integers(0, 40))) for _ in range(n)]
    off = np.concatenate([[0], np.cumsum([len(r) for r in rows])]).astype(np.int64)
    elems = np.concatenate([rng.permutation(r) for r in rows]).astype(np.int32)
    with sb.Context(0) as ctx:
        ctx.reserve(n, len(elems))
        ctx.stage_rows(0, np.arange(n // 2), off[: n // 2 + 1], elems[: off[n // 2]])
        ctx.stage_rows(1, np.arange(n // 2, n), off[n // 2:] - off[n // 2], elems[off[n // 2]:])
        ctx.seal()
        o, a = ctx.graph()
        assert np.array_equal(o, off)
        assert np.array_equal(a, np.concatenate(rows).astype(np.int32))
    with sb.Context(0) as ctx:
        ctx.reserve(4, 2)
        ctx.stage_rows(0, [0], [0, 2], [1, 9])
        with pytest.raises(sb.ScoutError):
            ctx.seal()


def test_compaction_preserves_rows(rmat16):
    off, adj = rmat16[1]
    batches = stream(off, adj, sb.STREAM_PREFERENTIAL, 20000, 4, seed=9)
    with _ctx_with(off, adj) as ctx:
        for b in batches:
            ctx.repair("bfs", b)
        before = ctx.graph()
        used = ctx.info()["pool_used"]
        ctx.compact()
        after = ctx.graph()
        assert ctx.info()["pool_used"] < used
        assert np.array_equal(before[0], after[0]) and np.array_equal(before[1], after[1])


def test_budget_is_enforced(rmat16):
    off, adj = rmat16[1]
    with sb.Context(0, budget_bytes=1 << 20) as ctx:
        with pytest.raises(sb.ScoutError) as e:
            ctx.load_csr(off, adj)
        assert e.value.code == -3
