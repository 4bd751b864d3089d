"""GPU parity of the batched multi-stream engine.

Several independent streams of one problem, over different graphs and with uneven batch
sizes, run as a disjoint union in one device store, a round at a time. After every round each
stream's solution must equal, bit for bit, the solution the single-stream engine computes for
that stream alone, and for BFS and CC also the ground truth of the stream's current graph;
the per-stream commit mirrors must track the device state.
"""
import numpy as np
import pytest

import scout_b200 as sb
from gpu_util import stream
from oracle import oracle as orc

pytestmark = pytest.mark.gpu


class Mirror:
    def __init__(self, off, adj):
        self.g = orc.Graph(off, adj)

    def apply(self, b):
        pairs = [p for p in b.tolist() if p[0] != p[1] and 0 <= min(p) and max(p) < self.n]
        flags = [not self.g.is_adjacent(u, v) for u, v in pairs]
        for (u, v), f in zip(pairs, flags):
            (self.g.insert if f else self.g.remove)(u, v)
        return self.g.csr()


def _init(problem, off, adj):
    return {"bfs": lambda: orc.gt_bfs(off, adj, 0), "cc": lambda: orc.gt_cc(off, adj),
            "coloring": lambda: orc.gt_greedy_color(off, adj), "mis": lambda: orc.gt_greedy_mis(off, adj)}[problem]()


def _streams():
    gs = [sb.gen_rmat(10, 8, seed=5).arrays(), sb.gen_rmat(12, 16, seed=6).arrays(), sb.gen_rmat(14, 16, seed=7).arrays()]
    specs = [(0, sb.STREAM_MIXED, [50, 300, 20, 700]), (1, sb.STREAM_PREFERENTIAL, [2000, 100, 5000, 40]),
             (2, sb.STREAM_LOWDEG, [10, 8000, 300, 3000]), (1, sb.STREAM_MIXED, [400, 400, 400, 400]),
             (2, sb.STREAM_PREFERENTIAL, [30000, 5, 600, 9000])]
    out = []
    for i, (gi, kind, sizes) in enumerate(specs):
        off, adj = gs[gi]
        h = sb.HostCsr.from_arrays(off, adj)
        s = h.stream(kind, sum(sizes), 1, insert_ratio=0.4, lowdeg_frac=0.5, seed=90 + i)
        b = np.cumsum([0] + sizes)
        batches = [np.ascontiguousarray(s[b[j]:b[j + 1]]) for j in range(len(sizes))]
        if i == 3:   # out-of-range and self-loop edits are skipped per stream
            batches[1] = np.concatenate([batches[1], [[0, len(off) + 5], [3, 3], [-1, 2]]]).astype(np.int32)
        out.append((off, adj, batches))
    return out


@pytest.mark.parametrize("problem", ["bfs", "cc", "coloring", "mis"])
@pytest.mark.parametrize("learned", [False, True])
def test_union_equals_streams_alone(problem, learned):
    if learned and problem not in ("bfs", "cc"):
        pytest.skip("the learned scheduler applies to BFS and CC")
    streams = _streams()
    arrivals = []
    for j in range(4):
        for sid in (3, 0, 4, 1, 2):
            arrivals.append((sid, streams[sid][2][j]))
    rounds = sb.form_rounds(arrivals, 12000)
    assert len(rounds) < len(arrivals)
    sched = {"policy": 1} if learned else None
    with sb.MultiEngine(problem) as me:
        singles, mirrors, truths = [], [], []
        for off, adj, _ in streams:
            init = _init(problem, off, adj)
            me.add_stream(off, adj, init, 0)
            ctx = sb.Context(0)
            ctx.load_csr(off, adj)
            ctx.upload(problem, init)
            singles.append(ctx)
            mirrors.append(init.copy())
            mm = Mirror(off, adj)
            mm.n = len(off) - 1
            truths.append(mm)
        if learned:
            # a model that always prefers the traversal (variant 1 for CC, 2 for BFS): bias-only output
            w = np.zeros(6020, dtype=np.float32)
            w[6016:6020] = [1.0, 0.5 if problem == "cc" else 0.9, 0.5, 0.0]
            me.context.sched_install(problem, w)
        for rd in rounds:
            st = me.round(rd, sched=sched)
            if learned:
                assert st["variant"] != 0
            me.commit(mirrors)
            for sid, b in rd:
                singles[sid].repair(problem, b)
                want = singles[sid].download(problem)
                got = me.download(sid)
                assert np.array_equal(got, want), f"stream {sid} differs from its single-stream run"
                assert np.array_equal(mirrors[sid], got)
                o, a = truths[sid].apply(b)
                if problem == "bfs":
                    assert np.array_equal(got, orc.gt_bfs(o, a, 0))
                elif problem == "cc":
                    assert np.array_equal(got, orc.gt_cc(o, a))
                elif problem == "coloring":
                    assert orc.check_coloring(o, a, got) == 0
                else:
                    assert orc.check_mis(o, a, got) == (0, 0)
        for c in singles:
            c.close()


@pytest.mark.parametrize("problem", ["bfs", "cc", "coloring", "mis"])
def test_union_with_a_large_stream(problem):
    """A stream on an R-MAT scale-19 graph (about 16 M directed entries) with a 10^6-edit batch
    shares rounds with two small streams; every stream equals its single-stream run and, for
    BFS and CC, the ground truth of its current graph."""
    specs = [(19, 16, sb.STREAM_PREFERENTIAL, [1_000_000, 2000]), (14, 16, sb.STREAM_MIXED, [500, 20000]),
             (12, 8, sb.STREAM_PREFERENTIAL, [100, 100])]
    streams = []
    for i, (sc, ef, kind, sizes) in enumerate(specs):
        h = sb.gen_rmat(sc, ef, seed=70 + i)
        off, adj = h.arrays()
        s = h.stream(kind, sum(sizes), 1, insert_ratio=0.5, seed=170 + i)
        b = np.cumsum([0] + sizes)
        streams.append((off, adj, [np.ascontiguousarray(s[b[j]:b[j + 1]]) for j in range(len(sizes))]))
    arrivals = [(sid, streams[sid][2][j]) for j in range(2) for sid in (0, 1, 2)]
    rounds = sb.form_rounds(arrivals, 1 << 21)
    with sb.MultiEngine(problem) as me:
        singles, truths = [], []
        for off, adj, _ in streams:
            init = _init(problem, off, adj)
            me.add_stream(off, adj, init, 0)
            ctx = sb.Context(0)
            ctx.load_csr(off, adj)
            ctx.upload(problem, init)
            singles.append(ctx)
            truths.append(orc.Graph(off, adj))
        me.reserve_batches(1 << 21)
        for rd in rounds:
            me.round(rd)
            for sid, b in rd:
                singles[sid].repair(problem, b)
                got = me.download(sid)
                assert np.array_equal(got, singles[sid].download(problem)), f"stream {sid} differs"
                truths[sid].toggle_batch(b)
                o, a = truths[sid].csr()
                if problem == "bfs":
                    assert np.array_equal(got, orc.gt_bfs(o, a, 0))
                elif problem == "cc":
                    assert np.array_equal(got, orc.gt_cc(o, a))
                elif problem == "coloring":
                    assert orc.check_coloring(o, a, got) == 0
                else:
                    assert orc.check_mis(o, a, got) == (0, 0)
        for c in singles:
            c.close()
