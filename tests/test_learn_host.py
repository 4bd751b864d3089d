"""Host-side helpers of the learned scheduler's data collection (no GPU): stream sizes that fit
the generators, and multi-stream arrivals that keep every stream's batches in order."""
import numpy as np

import scout_b200 as sb
from scout_b200 import learn


def test_fit_sizes_respects_the_deletion_budget():
    for nnz, ins in ((1000, 0.5), (100000, 0.3), (64, 0.0)):
        sizes = learn.fit_sizes([10 ** 6, 500, 3000], nnz, ins)
        assert all(z >= 1 for z in sizes)
        assert sum(sizes) * (1 - ins) <= nnz / 2 + len(sizes)
    assert learn.fit_sizes([10, 20], 10 ** 6, 0.5) == [10, 20]


def test_multi_arrivals_keep_stream_order_and_generate():
    spec = learn.MultiSpec([(8, 8), (9, 16)], streams_per_graph=2, nbatches=3, seed=4)
    graphs = [sb.gen_rmat(sc, ef, seed=spec.seed * 100 + i) for i, (sc, ef) in enumerate(spec.graphs)]
    per_stream, arrivals = learn.multi_arrivals(spec, graphs)
    assert len(per_stream) == 4 and len(arrivals) == 12
    seen = {}
    for sid, b in arrivals:
        k = seen.get(sid, 0)
        assert np.array_equal(b, per_stream[sid][1][k])
        seen[sid] = k + 1
        gi = per_stream[sid][0]
        assert b.max() < graphs[gi].n
    rounds = sb.form_rounds(arrivals, 1 << 20)
    assert sum(len(r) for r in rounds) == 12


def test_targets_mask_absent_variants():
    t, m = learn.targets([1.0, -1.0, 0.5], 7)
    assert list(m) == [1, 0, 1, 1]
    assert abs(t[0] - np.log2(1001.0) / 4) < 1e-6 and abs(t[3] - 3 / 24) < 1e-6
