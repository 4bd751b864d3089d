"""The fetch of batch K+1 during the repair of batch K on an all-HBM store: scout_prefetch hints
the next batch, the repair copies its edits to the device on the copy stream, and the next
repair reads that copy (scout_sched.prefetched) instead of uploading. Every batch's solution
and adjacency equal those of a context that uploads every batch itself, for page-locked and
pageable hints, for hints that are never used, and for a declared hint whose count does not
match (the edits are then uploaded)."""
import numpy as np
import pytest

import scout_b200 as sb
from gpu_util import stream
from oracle import oracle as orc

pytestmark = pytest.mark.gpu


def _batches(off, adj):
    sizes = [3000, 20000, 500, 20000, 3000]
    return [stream(off, adj, sb.STREAM_PREFERENTIAL, m, 1, seed=400 + i)[0] for i, m in enumerate(sizes)]


@pytest.mark.parametrize("problem", ["bfs", "coloring"])
@pytest.mark.parametrize("pinned", [True, False])
def test_prefetched_edits_match_uploaded_ones(rmat16, problem, pinned):
    g, (off, adj) = rmat16
    init = g.init_state(problem, 0)
    batches = _batches(off, adj)
    if pinned:
        batches = [sb.pinned_copy(b) for b in batches]
    og = orc.Graph(off, adj)
    with sb.Context(0) as t, sb.Context(0) as ref:
        for c in (t, ref):
            c.load_csr(off, adj)
            c.upload(problem, init)
        t.reserve_batches(max(len(b) for b in batches))
        for k, b in enumerate(batches):
            if k + 1 < len(batches):
                t.prefetch(batches[k + 1])
            st = t.repair(problem, b)
            sr = ref.repair(problem, np.array(b))
            assert st["edits"] == sr["edits"] and st["h2d_bytes"] == sr["h2d_bytes"]
            assert np.array_equal(t.download(problem), ref.download(problem)), f"batch {k + 1}"
            og.toggle_batch(np.asarray(b))
        o1, a1 = t.graph()
        o2, a2 = ref.graph()
        assert np.array_equal(o1, o2) and np.array_equal(a1, a2)
        if problem == "bfs":
            o, a = og.csr()
            assert np.array_equal(t.download("bfs"), orc.gt_bfs(o, a, 0))


def test_unused_and_mismatched_hints(rmat16):
    g, (off, adj) = rmat16
    init = g.init_state("bfs", 0)
    b = _batches(off, adj)
    with sb.Context(0) as t, sb.Context(0) as ref:
        for c in (t, ref):
            c.load_csr(off, adj)
            c.upload("bfs", init)
        # a hint, then a different batch: it is uploaded; the hinted one later too
        t.prefetch(b[1])
        t.repair("bfs", b[0])
        ref.repair("bfs", b[0])
        t.repair("bfs", b[1])
        ref.repair("bfs", b[1])
        assert np.array_equal(t.download("bfs"), ref.download("bfs"))
        # a hint of 20000 edits whose copy is made, then a declared batch of another count
        t.prefetch(b[3])
        t.repair("bfs", b[2])
        ref.repair("bfs", b[2])
        t.repair("bfs", b[4], sched={"prefetched": 1})
        ref.repair("bfs", b[4])
        assert np.array_equal(t.download("bfs"), ref.download("bfs"))
        o1, a1 = t.graph()
        o2, a2 = ref.graph()
        assert np.array_equal(o1, o2) and np.array_equal(a1, a2)
