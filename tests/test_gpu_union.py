"""GPU parity of the fused round: four union stores, one per problem, whose repairs run in ONE
persistent kernel per round (scout_multi_stage + scout_multi_run_all). The streams span
several graphs and uneven batch sizes; after every round each stream's solution equals, bit
for bit, what the single-stream engine computes for that stream alone, and for BFS and CC
the ground truth of the stream's current graph. A round may leave out problems, and an
engine without a staged round is refused."""
import numpy as np
import pytest

import scout_b200 as sb
from oracle import oracle as orc

pytestmark = pytest.mark.gpu

PROBLEMS = ["bfs", "cc", "coloring", "mis"]


def _init(problem, off, adj):
    return {"bfs": lambda: orc.gt_bfs(off, adj, 0), "cc": lambda: orc.gt_cc(off, adj),
            "coloring": lambda: orc.gt_greedy_color(off, adj), "mis": lambda: orc.gt_greedy_mis(off, adj)}[problem]()


def _streams(pi):
    """Three streams per problem over R-MAT graphs of scales 10-14, four batches each."""
    specs = [(10, 8, sb.STREAM_MIXED, [60, 400, 30, 900]), (12, 16, sb.STREAM_PREFERENTIAL, [3000, 150, 6000, 50]),
             (14, 16, sb.STREAM_LOWDEG, [20, 9000, 400, 2500])]
    out = []
    for i, (sc, ef, kind, sizes) in enumerate(specs):
        h = sb.gen_rmat(sc, ef, seed=300 + 10 * pi + i)
        off, adj = h.arrays()
        s = h.stream(kind, sum(sizes), 1, insert_ratio=0.4, lowdeg_frac=0.5, seed=600 + 10 * pi + i)
        b = np.cumsum([0] + sizes)
        out.append((off, adj, [np.ascontiguousarray(s[b[j]:b[j + 1]]) for j in range(len(sizes))]))
    return out


def _check(problem, got, o, a):
    if problem == "bfs":
        assert np.array_equal(got, orc.gt_bfs(o, a, 0))
    elif problem == "cc":
        assert np.array_equal(got, orc.gt_cc(o, a))
    elif problem == "coloring":
        assert orc.check_coloring(o, a, got) == 0
    else:
        assert orc.check_mis(o, a, got) == (0, 0)


def test_fused_round_equals_streams_alone():
    engines, singles, truths, data = [], [], [], []
    try:
        for pi, problem in enumerate(PROBLEMS):
            me = sb.MultiEngine(problem)
            engines.append(me)
            streams = _streams(pi)
            data.append(streams)
            sg, tr = [], []
            for off, adj, _ in streams:
                init = _init(problem, off, adj)
                me.add_stream(off, adj, init, 0)
                ctx = sb.Context(0)
                ctx.load_csr(off, adj)
                ctx.upload(problem, init)
                sg.append(ctx)
                tr.append(orc.Graph(off, adj))
            singles.append(sg)
            truths.append(tr)
            me.seal()
        for j in range(4):
            # the third round leaves colouring out: a fused round takes any subset of the problems
            members = [pi for pi in range(4) if not (j == 2 and PROBLEMS[pi] == "coloring")]
            for pi in members:
                engines[pi].stage([(sid, data[pi][sid][2][j]) for sid in range(3)])
            stats = sb.run_fused_round([engines[pi] for pi in members])
            assert len(stats) == len(members)
            assert len({s["ms_repair"] for s in stats}) == 1   # one shared launch
            for pi in members:
                problem = PROBLEMS[pi]
                for sid in range(3):
                    b = data[pi][sid][2][j]
                    singles[pi][sid].repair(problem, b)
                    want = singles[pi][sid].download(problem)
                    got = engines[pi].download(sid)
                    assert np.array_equal(got, want), f"{problem} stream {sid} round {j}"
                    truths[pi][sid].toggle_batch(b)
                    o, a = truths[pi][sid].csr()
                    _check(problem, got, o, a)
        # an engine without a staged round is refused, and nothing runs
        engines[0].stage([(0, data[0][0][2][0][:10])])
        with pytest.raises(sb.ScoutError):
            sb.run_fused_round([engines[0], engines[1]])
        with pytest.raises(sb.ScoutError):   # two engines of one problem
            engines[0].stage([(0, data[0][0][2][0][:10])])
            sb.run_fused_round([engines[0], engines[0]])
    finally:
        for sg in singles:
            for c in sg:
                c.close()
        for me in engines:
            me.close()
