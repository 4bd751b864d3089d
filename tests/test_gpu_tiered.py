"""Out-of-core (tiered) graph store: hot rows in a small HBM pool, the rest in mapped
page-locked host memory read in place, rewritten rows moved to HBM, short rows evicted back
to the host pool when the HBM pool fills. After every batch the adjacency and the solution must equal an
ordinary single-tier context's, bit for bit."""
import numpy as np
import pytest

import scout_b200 as sb
from gpu_util import stream

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("problem", ["bfs", "cc", "coloring", "mis"])
def test_tiered_equals_single_tier(rmat16, problem):
    g, (off, adj) = rmat16
    init = g.init_state(problem, 0)
    batches = (list(stream(off, adj, sb.STREAM_PREFERENTIAL, 30000, 2, seed=91))
               + list(stream(off, adj, sb.STREAM_PREFERENTIAL, 200, 8, seed=94))
               + list(stream(off, adj, sb.STREAM_LOWDEG, 20000, 2, seed=92, insert_ratio=0.3, lowdeg_frac=0.3))
               + list(stream(off, adj, sb.STREAM_MIXED, 400, 3, seed=93)))
    nnz = len(adj)
    with sb.Context(0) as t, sb.Context(0) as ref:
        t.load_tiered(off, adj, hbm_entries=nnz // 3)
        ref.load_csr(off, adj)
        info = t.tier_info()
        assert info["host_used"] > 0 and info["hbm_used"] <= nnz // 6 + 1
        for c in (t, ref):
            c.upload(problem, init)
        mt, mr = init.copy(), init.copy()
        for b in batches:
            t.repair(problem, b)
            ref.repair(problem, b)
            t.commit(problem, mt)
            ref.commit(problem, mr)
            assert np.array_equal(t.download(problem), ref.download(problem))
            assert np.array_equal(mt, mr)
        o1, a1 = t.graph()
        o2, a2 = ref.graph()
        assert np.array_equal(o1, o2) and np.array_equal(a1, a2)
        info = t.tier_info()
        assert info["evicted"] > 0, "the medium batches should have made the HBM pool evict rows"


@pytest.mark.parametrize("problem", ["bfs", "cc"])
def test_tiny_hbm_pool_stays_exact(rmat16, problem):
    """An HBM pool of 5% of the graph under large batches: rows move back and forth between
    the tiers on every batch (evictions, host-pool writes and compactions), results exact."""
    g, (off, adj) = rmat16
    init = g.init_state(problem, 0)
    batches = list(stream(off, adj, sb.STREAM_PREFERENTIAL, 30000, 3, seed=95))
    with sb.Context(0) as t, sb.Context(0) as ref:
        t.load_tiered(off, adj, hbm_entries=len(adj) // 20)
        ref.load_csr(off, adj)
        for c in (t, ref):
            c.upload(problem, init)
        for b in batches:
            t.repair(problem, b)
            ref.repair(problem, b)
            assert np.array_equal(t.download(problem), ref.download(problem))
        o1, a1 = t.graph()
        o2, a2 = ref.graph()
        assert np.array_equal(o1, o2) and np.array_equal(a1, a2)
        assert t.tier_info()["evicted"] > 0


@pytest.mark.parametrize("problem", ["bfs", "cc", "coloring", "mis"])
@pytest.mark.parametrize("hbm_frac", [3, 20])
def test_prefetched_gather_stays_exact(rmat16, problem, hbm_frac):
    """scout_prefetch hints every next batch: during each repair the next batch's cold
    endpoint rows are gathered into HBM on a copy stream, descriptors switched while the repair
    reads them. Adjacency and solution still equal a single-tier context's after every batch,
    and the gathers really ran (rows moved, bytes read over the host link). A pool of 1/20 of
    the graph leaves the gather little room and forces evictions between the gathers."""
    g, (off, adj) = rmat16
    init = g.init_state(problem, 0)
    batches = (list(stream(off, adj, sb.STREAM_LOWDEG, 20000, 3, seed=96, insert_ratio=0.3, lowdeg_frac=0.3))
               + list(stream(off, adj, sb.STREAM_PREFERENTIAL, 5000, 3, seed=97)))
    with sb.Context(0) as t, sb.Context(0) as ref:
        t.load_tiered(off, adj, hbm_entries=len(adj) // hbm_frac)
        ref.load_csr(off, adj)
        for c in (t, ref):
            c.upload(problem, init)
        t.reserve_batches(max(len(b) for b in batches))
        gathered = 0
        for k, b in enumerate(batches):
            if k + 1 < len(batches):
                t.prefetch(batches[k + 1])
            st = t.repair(problem, b)
            ref.repair(problem, b)
            gathered += st["gather_rows"]
            if st["gather_rows"]:
                assert st["gather_bytes"] > 0 and st["ms_gather"] > 0
            assert np.array_equal(t.download(problem), ref.download(problem)), f"batch {k + 1}"
        o1, a1 = t.graph()
        o2, a2 = ref.graph()
        assert np.array_equal(o1, o2) and np.array_equal(a1, a2)
        assert gathered > 0
