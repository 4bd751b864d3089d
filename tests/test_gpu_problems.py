"""GPU parity of the coloring, CC and MIS engines against the oracle after every batch.

- coloring: bit-exact with the reference rule (scout_coloring.cu:46-100, 243-277) wherever the
  reference did not truncate a round; always a proper colouring;
- CC: the exact partition of the current graph (min-vertex-id labels) after every batch, and
  equal to the reference rule's partition whenever it had no deferred deletion pending;
- MIS: bit-exact with the oracle's vertex-id-priority restatement; independent and maximal.
"""
import os

import numpy as np
import pytest

import scout_b200 as sb
from conftest import SAMPLE
from oracle import oracle as orc
from gpu_util import stream

pytestmark = pytest.mark.gpu


class Mirror:
    """Oracle graph kept in step with the device through the toggle rule."""

    def __init__(self, off, adj):
        self.g = orc.Graph(off, adj)

    def apply(self, b):
        pairs = [p for p in b.tolist() if p[0] != p[1]]
        flags = [not self.g.is_adjacent(u, v) for u, v in pairs]
        for (u, v), f in zip(pairs, flags):
            (self.g.insert if f else self.g.remove)(u, v)
        return self.g.csr()


def _streams(off, adj):
    return {
        "mixed": stream(off, adj, sb.STREAM_MIXED, 1000, 8, seed=41),
        "preferential": stream(off, adj, sb.STREAM_PREFERENTIAL, 20000, 3, seed=42),
        "lowdeg_deletions": stream(off, adj, sb.STREAM_LOWDEG, 5000, 3, seed=43, insert_ratio=0.1, lowdeg_frac=0.6),
    }


# ---- coloring --------------------------------------------------------------------------
def _coloring(off, adj, init, batches):
    ref = orc.Engine("coloring", off, adj, init)
    m = Mirror(off, adj)
    mirror = init.copy()
    exact = 0
    with sb.Context(0) as ctx:
        ctx.load_csr(off, adj)
        ctx.upload("coloring", init)
        for b in batches:
            st = ctx.repair("coloring", b)
            o, a = m.apply(b)
            got = ctx.download("coloring")
            assert orc.check_coloring(o, a, got) == 0, "not a proper colouring"
            ref.batch(b)
            s = ref.stats()
            if s["truncated"] == 0:
                assert np.array_equal(got, ref.solution()), "differs from the reference rule"
                exact += 1
            ctx.commit("coloring", mirror)
            assert np.array_equal(mirror, got)
            assert st["conflicts"] >= 0
    return exact


def test_coloring_sample(sample_graph, sample_batches):
    off, adj = sample_graph
    init, _ = sb.load_state(os.path.join(SAMPLE, "sample_colors.txt"), "coloring", 2000)
    assert _coloring(off, adj, init, sample_batches) == 5


@pytest.mark.parametrize("kind", ["mixed", "preferential", "lowdeg_deletions"])
def test_coloring_rmat16(rmat16, kind):
    off, adj = rmat16[1]
    batches = _streams(off, adj)[kind]
    assert _coloring(off, adj, orc.gt_greedy_color(off, adj), batches) == len(batches)


def test_coloring_stats_match_reference(rmat16):
    off, adj = rmat16[1]
    init = orc.gt_greedy_color(off, adj)
    b = stream(off, adj, sb.STREAM_PREFERENTIAL, 30000, 1, seed=44)[0]
    ref = orc.Engine("coloring", off, adj, init)
    ref.batch(b)
    with sb.Context(0) as ctx:
        ctx.load_csr(off, adj)
        ctx.upload("coloring", init)
        st = ctx.repair("coloring", b)
    s = ref.stats()
    assert st["conflicts"] == s["conflict"] and st["rounds"] == s["rounds"]
    assert st["insertions"] == s["ins"] and st["deletions"] == s["del"]


# ---- CC --------------------------------------------------------------------------------
def _cc(off, adj, batches, sched=None, check_ref=True):
    init = orc.gt_cc(off, adj)
    ref = orc.Engine("cc", off, adj, init)
    m = Mirror(off, adj)
    mirror = init.copy()
    with sb.Context(0) as ctx:
        ctx.load_csr(off, adj)
        ctx.upload("cc", init)
        for b in batches:
            st = ctx.repair("cc", b, sched=sched)
            o, a = m.apply(b)
            got = ctx.download("cc")
            truth = orc.gt_cc(o, a)
            assert np.array_equal(got, truth), f"partition differs at {np.flatnonzero(got != truth)[:10]}"
            ctx.commit("cc", mirror)
            assert np.array_equal(mirror, truth)
            ref.batch(b)
            if check_ref and ref.stats()["deferred"] == 0:
                assert np.array_equal(got, ref.solution())
        st = ctx.recompute_cc()
        assert np.array_equal(ctx.download("cc"), orc.gt_cc(*m.g.csr()))


def test_cc_sample(sample_graph, sample_batches):
    off, adj = sample_graph
    _cc(off, adj, sample_batches)


@pytest.mark.parametrize("kind", ["mixed", "preferential", "lowdeg_deletions"])
def test_cc_rmat16(rmat16, kind):
    off, adj = rmat16[1]
    _cc(off, adj, _streams(off, adj)[kind])


def test_cc_forced_recompute_paths(rmat16):
    off, adj = rmat16[1]
    batches = _streams(off, adj)["lowdeg_deletions"]
    _cc(off, adj, batches, sched={"search_bound": 3}, check_ref=False)   # most searches give up
    _cc(off, adj, batches[:1], sched={"mode": 2}, check_ref=False)       # full recompute per batch


def test_cc_bridges_and_small_components():
    # a chain of triangles joined by bridges, plus isolated vertices; deleting bridges splits
    n = 60
    edges = []
    for t in range(15):
        a, b, c = 3 * t, 3 * t + 1, 3 * t + 2
        edges += [(a, b), (b, c), (a, c)]
        if t:
            edges.append((3 * t - 1, a))
    rows = [[] for _ in range(n)]
    for u, v in edges:
        rows[u].append(v)
        rows[v].append(u)
    off = np.concatenate([[0], np.cumsum([len(r) for r in rows])]).astype(np.int64)
    adj = np.concatenate([sorted(r) for r in rows if r]).astype(np.int32)
    batches = [np.array([[5, 6]], np.int32), np.array([[2, 3], [11, 12], [20, 21]], np.int32),
               np.array([[0, 1], [0, 2], [50, 51], [2, 3]], np.int32), np.array([[5, 6], [44, 45], [30, 59]], np.int32)]
    _cc(off, adj, batches)


# ---- MIS -------------------------------------------------------------------------------
def _mis(off, adj, batches):
    init = orc.gt_greedy_mis(off, adj)
    idp = orc.Engine("mis_id", off, adj, init)
    ref = orc.Engine("mis", off, adj, init, against_base=True)
    m = Mirror(off, adj)
    mirror = init.copy()
    with sb.Context(0) as ctx:
        ctx.load_csr(off, adj)
        ctx.upload("mis", init)
        for b in batches:
            ctx.repair("mis", b)
            o, a = m.apply(b)
            got = ctx.download("mis")
            assert orc.check_mis(o, a, got) == (0, 0), "not independent and maximal"
            idp.batch(b)
            assert np.array_equal(got, idp.solution()), "differs from the id-priority rule"
            ref.batch(b)
            ctx.commit("mis", mirror)
            assert np.array_equal(mirror, got)
    return int(got.sum()), int(ref.solution().sum())


def test_mis_sample(sample_graph, sample_batches):
    off, adj = sample_graph
    ours, theirs = _mis(off, adj, sample_batches)
    # The reference rule re-admits at most one vertex per dropped one and is not maximal in
    # general; the id-priority set is maximal. The size difference is the logged divergence.
    print(f"MIS size after 5 sample batches: engine {ours}, reference rule {theirs}")
    assert ours > 0 and theirs > 0


@pytest.mark.parametrize("kind", ["mixed", "preferential", "lowdeg_deletions"])
def test_mis_rmat16(rmat16, kind):
    off, adj = rmat16[1]
    _mis(off, adj, _streams(off, adj)[kind])
