"""scout_reserve: after it, batches up to the reserved size allocate no device memory (the
context's held bytes stay constant through repairs and a compaction) and give the same
results as an unreserved context."""
import numpy as np
import pytest

import scout_b200 as sb
from gpu_util import stream

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("problem", ["bfs", "cc", "coloring", "mis"])
def test_reserved_context_allocates_nothing(rmat16, problem):
    g, (off, adj) = rmat16
    init = g.init_state(problem, 0)
    batches = (list(stream(off, adj, sb.STREAM_PREFERENTIAL, 40000, 4, seed=81))
               + list(stream(off, adj, sb.STREAM_MIXED, 300, 4, seed=82)))
    with sb.Context(0) as a, sb.Context(0) as b:
        for c in (a, b):
            c.load_csr(off, adj)
            c.upload(problem, init)
        a.reserve_batches(40000)
        held = a.held_bytes()
        for k, e in enumerate(batches):
            if k == 4:
                a.compact()   # the reserved spare pool is the compaction target
            a.repair(problem, e)
            b.repair(problem, e)
            assert a.held_bytes() == held, "a repair allocated device memory after scout_reserve"
            assert np.array_equal(a.download(problem), b.download(problem))
