"""Pins the oracle's engine restatements to what the reference's own engines printed.

golden/ref_engines.json was recorded on a B200 by running the reference binaries (compiled
from its sources by oracle/build_ref.sh) on every prefix of two streams: the bundled sample
(5 batches) and an R-MAT scale-16 mixed stream (10 x 1000 toggles, regenerated here
bit-identically). For BFS, colouring and CC the reference is deterministic on these inputs, so
every printed counter and final value must match the oracle exactly; the MIS engine is racy,
so its sets are validated and their sizes compared.
"""
import json
import os

import numpy as np
import pytest

import scout_b200 as sb
from conftest import GOLDEN, SAMPLE
from oracle import oracle as orc

GOLD = json.load(open(os.path.join(GOLDEN, "ref_engines.json")))
INIT = {"mis": "sample_mis.txt", "coloring": "sample_colors.txt", "bfs": "sample_bfs.txt",
        "cc": "sample_components.txt"}


def _case(name, rmat16):
    if name == "sample":
        off, adj, _ = sb.read_egr(os.path.join(SAMPLE, "sample.egr"))
        init = {p: sb.load_state(os.path.join(SAMPLE, f), p, 2000)[0] for p, f in INIT.items()}
        batches = [sb.parse_batch_file(os.path.join(SAMPLE, "batches", f"{k}.mtx"), 2000) for k in range(1, 6)]
    else:
        rc = GOLD["_rmat16_case"]
        g, (off, adj) = rmat16
        assert (rc["scale"], rc["edge_factor"], rc["seed"]) == (16, 16, 1)
        st = g.stream(sb.STREAM_MIXED, rc["batch_size"], rc["batches"], seed=rc["stream_seed"])
        batches = list(st.reshape(rc["batches"], rc["batch_size"], 2))
        init = {p: g.init_state(p, 0) for p in INIT}
    return off, adj, init, batches


def _stream(problem, off, adj, init, batches):
    """One pass: yields (k, engine, stats before batch k, stats after batch k, final value
    after the prefix's end-of-stream catch-up). The catch-up of the reference (a full BFS /
    recompute when a deletion was deferred) equals the ground truth of the current graph, so
    it is computed without disturbing the engine."""
    e = orc.Engine(problem, off, adj, init, against_base=(problem == "mis"))
    for k, b in enumerate(batches, start=1):
        s0 = e.stats()
        e.batch(b)
        s1 = e.stats()
        sol = e.solution()
        if problem in ("bfs", "cc") and s1["deferred"] > 0:
            o, a = e.graph().csr()
            sol = orc.gt_bfs(o, a, 0) if problem == "bfs" else orc.gt_cc(o, a)
        yield k, e, s0, s1, sol


@pytest.mark.parametrize("case", ["sample", "rmat16"])
def test_bfs_counters_and_levels(case, rmat16):
    off, adj, init, batches = _case(case, rmat16)
    gold = GOLD[case]["bfs"]
    last = gold[str(len(batches))]["batches"]
    for k, e, s0, s, sol in _stream("bfs", off, adj, init["bfs"], batches):
        line = last[k - 1]
        assert (s["ins"] - s0["ins"], s["del"] - s0["del"], s["fallback"] - s0["fallback"]) == (
            line["insertions"], line["deletions"], line["fallback"])
        st = gold[str(k)]["stats"]
        assert (s["ins"], s["ins_noop"], s["ins_repaired"]) == (st["insertions"]["total"], st["insertions"]["noop"],
                                                                 st["insertions"]["repaired"])
        assert (s["del"], s["del_noop"], s["del_local"], s["fallback"], s["deferred"]) == (
            st["deletions"]["total"], st["deletions"]["noop"], st["deletions"]["local"], st["deletions"]["fallback"],
            st["deletions"]["deferred"])
        assert int((sol >= 0).sum()) == gold[str(k)]["final"]


@pytest.mark.parametrize("case", ["sample", "rmat16"])
def test_coloring_counters_and_colours(case, rmat16):
    off, adj, init, batches = _case(case, rmat16)
    gold = GOLD[case]["coloring"]
    last = gold[str(len(batches))]["batches"]
    for k, e, s0, s, sol in _stream("coloring", off, adj, init["coloring"], batches):
        line = last[k - 1]
        assert (s["ins"] - s0["ins"], s["conflict"] - s0["conflict"], s["rounds"] - s0["rounds"]) == (
            line["insertions"], line["conflicts"], line["rounds"])
        st = gold[str(k)]["stats"]
        assert (s["ins"], s["ins_noop"], s["conflict"]) == (st["insertions"]["total"], st["insertions"]["noop"],
                                                            st["insertions"]["conflict"])
        assert (s["rounds"], s["max_rounds"]) == (st["rounds"]["total"], st["rounds"]["max"])
        assert int(sol.max()) + 1 == gold[str(k)]["final"]


@pytest.mark.parametrize("case", ["sample", "rmat16"])
def test_cc_counters_and_components(case, rmat16):
    off, adj, init, batches = _case(case, rmat16)
    gold = GOLD[case]["cc"]
    last = gold[str(len(batches))]["batches"]
    for k, e, s0, s, sol in _stream("cc", off, adj, init["cc"], batches):
        line = last[k - 1]
        assert (s["ins"] - s0["ins"], s["del"] - s0["del"]) == (line["insertions"], line["deletions"])
        st = gold[str(k)]["stats"]
        assert (s["ins"], s["merged"], s["ins_noop"]) == (st["insertions"]["total"], st["insertions"]["merged"],
                                                          st["insertions"]["noop"])
        assert (s["del"], s["del_noop"], s["still_connected"], s["split"], s["deferred"]) == (
            st["deletions"]["total"], st["deletions"]["noop"], st["deletions"]["still_connected"],
            st["deletions"]["definitive_split"], st["deletions"]["deferred"])
        assert len(np.unique(sol)) == gold[str(k)]["final"]


@pytest.mark.parametrize("case", ["sample", "rmat16"])
def test_mis_reference_sets_are_independent_and_sized_alike(case, rmat16):
    off, adj, init, batches = _case(case, rmat16)
    ours = orc.Engine("mis_id", off, adj, init["mis"], against_base=True)
    for k, e, _, _, sol in _stream("mis", off, adj, init["mis"], batches):
        rec = GOLD[case]["mis"][str(k)]
        ours.batch(batches[k - 1])
        o, a = ours.graph().csr()
        assert orc.check_mis(o, a, ours.solution()) == (0, 0)
        ref_size = rec["final"]
        if "mis_ids" in rec:   # the reference's own set on the final graph: always independent
            flags = np.zeros(len(off) - 1, dtype=np.int32)
            flags[np.array(rec["mis_ids"], dtype=np.int64) - 1] = 1
            assert orc.check_mis(o, a, flags)[0] == 0
            assert int(flags.sum()) == ref_size
        # the restatement's set and the reference's racy set stay within 2% of each other
        assert abs(int(sol.sum()) - ref_size) <= max(5, 0.02 * ref_size)
