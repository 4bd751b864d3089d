"""Initial solutions computed on the device (scout_seed) equal the reference seeding tools'
rules, restated by the oracle and pinned to the tools' own output: greedy MIS and greedy
smallest-free colouring in vertex-id order, BFS levels, min-id component labels; on the
loaded graph and again after batches have changed it."""
import numpy as np
import pytest

import scout_b200 as sb
from gpu_util import stream
from oracle import oracle as orc

pytestmark = pytest.mark.gpu

TRUTH = {"mis": lambda o, a: orc.gt_greedy_mis(o, a), "coloring": lambda o, a: orc.gt_greedy_color(o, a),
         "bfs": lambda o, a: orc.gt_bfs(o, a, 0), "cc": lambda o, a: orc.gt_cc(o, a)}


@pytest.mark.parametrize("problem", ["mis", "coloring", "bfs", "cc"])
def test_seed_matches_tools(sample_graph, rmat16, problem):
    for off, adj in (sample_graph, rmat16[1]):
        with sb.Context(0) as ctx:
            ctx.load_csr(off, adj)
            ctx.seed(problem, 0)
            assert np.array_equal(ctx.download(problem), TRUTH[problem](off, adj))


@pytest.mark.parametrize("problem", ["mis", "coloring"])
def test_seed_after_batches(rmat16, problem):
    off, adj = rmat16[1]
    g = orc.Graph(off, adj)
    with sb.Context(0) as ctx:
        ctx.load_csr(off, adj)
        ctx.upload("bfs", orc.gt_bfs(off, adj, 0))
        for b in stream(off, adj, sb.STREAM_MIXED, 3000, 3, seed=17):
            ctx.repair("bfs", b)
            pairs = [p for p in b.tolist() if p[0] != p[1]]
            flags = [not g.is_adjacent(u, v) for u, v in pairs]
            for (u, v), f in zip(pairs, flags):
                (g.insert if f else g.remove)(u, v)
        ctx.seed(problem, 0)
        o, a = g.csr()
        assert np.array_equal(ctx.download(problem), TRUTH[problem](o, a))
