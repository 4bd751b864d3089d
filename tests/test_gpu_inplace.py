"""Rows that only lose entries are compacted where they lie: rows of 200 to 5000 entries lose
scattered entries and long runs of consecutive ones (rows of one 4096-entry slice go through one
warp of the slice merge, the short background rows through the short-row merge). A row longer
than a slice is compacted in place by one block in the tiered store, and rewritten at the pool
tail by the slice merge in the all-HBM store. After every batch the adjacency equals the oracle
scratchpad's, and the pool tail moves by exactly the rows rewritten elsewhere: none in the
tiered store, the rows longer than a slice in the all-HBM store."""
import numpy as np
import pytest

import scout_b200 as sb
from gpu_util import sorted_rows
from oracle import oracle as orc

pytestmark = pytest.mark.gpu

HUBS = {0: 5000, 1: 3000, 2: 2048, 3: 1500, 4: 200}   # vertex: row length
SLICE = 4096   # entries of one slice of the slice merge


def _graph(n=6000):
    rows = [set() for _ in range(n)]
    rng = np.random.default_rng(7)
    for h, d in HUBS.items():
        for v in rng.choice(np.arange(10, n), size=d, replace=False):
            rows[h].add(int(v))
            rows[int(v)].add(h)
    for _ in range(4000):   # a sparse background so the other rows are not empty
        u, v = (int(x) for x in rng.integers(10, n, 2))
        if u != v:
            rows[u].add(v)
            rows[v].add(u)
    off = np.concatenate([[0], np.cumsum([len(r) for r in rows])]).astype(np.int64)
    adj = np.concatenate([sorted(r) for r in rows]).astype(np.int32)
    return off, adj


def _deletions(off, adj, rng):
    """Scattered deletions and a run of consecutive entries from every hub row."""
    out = []
    for h in HUBS:
        row = adj[off[h]:off[h + 1]]
        run0 = int(rng.integers(0, max(1, len(row) - 600)))
        pick = set(range(run0, min(len(row), run0 + 500)))                        # consecutive run
        pick |= set(int(i) for i in rng.choice(len(row), size=len(row) // 8, replace=False))   # scattered
        out += [(h, int(row[i])) for i in sorted(pick)]
    return np.array(out, dtype=np.int32)


@pytest.mark.parametrize("tiered", [False, True])
def test_deletion_only_rows_compact_in_place(tiered):
    off, adj = _graph()
    rng = np.random.default_rng(11)
    og = orc.Graph(off, adj)
    with sb.Context(0) as ctx:
        if tiered:
            ctx.load_tiered(off, adj, hbm_entries=len(adj) // 2)
        else:
            ctx.load_csr(off, adj)
        ctx.upload("bfs", orc.gt_bfs(off, adj, 0))
        used0 = ctx.info()["pool_used"]
        tiers0 = ctx.tier_info()
        cur_off, cur_adj = off, adj
        grown = 0
        for k in range(3):
            b = _deletions(cur_off, cur_adj, rng)
            if not tiered:   # rows past one slice are rewritten at the tail (their old length)
                grown += sum(int(cur_off[h + 1] - cur_off[h]) for h in HUBS if cur_off[h + 1] - cur_off[h] > SLICE)
            st = ctx.repair("bfs", b)
            assert st["deletions"] == len(b) and st["insertions"] == 0
            og.toggle_batch(b)
            cur_off, cur_adj = sorted_rows(*og.csr())
            o, a = ctx.graph()
            assert np.array_equal(o, cur_off) and np.array_equal(a, cur_adj), f"batch {k + 1}"
            assert np.array_equal(ctx.download("bfs"), orc.gt_bfs(cur_off, cur_adj, 0))
            assert ctx.info()["pool_used"] == used0 + grown, "a deletion-only row was rewritten elsewhere"
            if tiered:
                assert ctx.tier_info()["host_used"] == tiers0["host_used"]
