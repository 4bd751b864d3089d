"""Pins the oracle (and the package's seeding tools) to the reference's own outputs.

- the sample's shipped initial states (datasets/sample) are exact CPU recomputations:
  BFS from 0, min-id components, greedy MIS in id order;
- tools/compute_initial_mis.py and tools/greedy_color.cpp were run on the sample and on the
  R-MAT scale-16 graph (golden.json holds the hashes of what they wrote).
"""
import hashlib
import json
import os

import numpy as np

from conftest import GOLDEN, SAMPLE

import scout_b200 as sb
from oracle import oracle as orc

GOLD = json.load(open(os.path.join(GOLDEN, "golden.json")))


def _mis_file_sha(flags):
    txt = "".join(f"{v + 1}\n" for v in np.flatnonzero(flags))
    return hashlib.sha256(txt.encode()).hexdigest()


def _colors_file_sha(colors):
    txt = "".join(f"{c}\n" for c in colors)
    return hashlib.sha256(txt.encode()).hexdigest()


def test_sample_initial_states_are_exact(sample_graph):
    off, adj = sample_graph
    lev, _ = sb.load_state(os.path.join(SAMPLE, "sample_bfs.txt"), "bfs", 2000)
    assert np.array_equal(orc.gt_bfs(off, adj, 0), lev)
    lab, _ = sb.load_state(os.path.join(SAMPLE, "sample_components.txt"), "cc", 2000)
    assert np.array_equal(orc.gt_cc(off, adj), lab)
    mis, _ = sb.load_state(os.path.join(SAMPLE, "sample_mis.txt"), "mis", 2000)
    assert np.array_equal(orc.gt_greedy_mis(off, adj), mis)
    col, _ = sb.load_state(os.path.join(SAMPLE, "sample_colors.txt"), "coloring", 2000)
    assert orc.check_coloring(off, adj, col) == 0   # ECL-GC colouring: proper, not greedy


def test_reference_tools_on_sample(sample_graph):
    off, adj = sample_graph
    g = GOLD["tools"]["sample"]
    gm = orc.gt_greedy_mis(off, adj)
    assert gm.sum() == g["mis_count"] and _mis_file_sha(gm) == g["mis_sha256"]
    gc = orc.gt_greedy_color(off, adj)
    assert gc.max() + 1 == g["colors_used"] and _colors_file_sha(gc) == g["colors_sha256"]
    ref_cols = np.loadtxt(os.path.join(GOLDEN, "sample_greedy_colors.txt"), dtype=np.int32)
    assert np.array_equal(gc, ref_cols)


def test_reference_tools_on_rmat16(rmat16, tmp_path):
    g, (off, adj) = rmat16
    gold = GOLD["tools"]["rmat16_ef16_seed1"]
    p = tmp_path / "r.egr"
    sb.write_egr(str(p), off, adj, wide=False)
    assert hashlib.sha256(p.read_bytes()).hexdigest() == gold["egr_sha256"]   # generator is deterministic
    gm = orc.gt_greedy_mis(off, adj)
    assert _mis_file_sha(gm) == gold["mis_sha256"]
    gc = orc.gt_greedy_color(off, adj)
    assert _colors_file_sha(gc) == gold["colors_sha256"] and gc.max() + 1 == gold["colors_used"]
    # the package's seeding tools agree with the oracle (and so with the reference tools)
    assert np.array_equal(g.init_state("mis"), gm)
    assert np.array_equal(g.init_state("coloring"), gc)
    assert np.array_equal(g.init_state("bfs"), orc.gt_bfs(off, adj, 0))
    assert np.array_equal(g.init_state("cc"), orc.gt_cc(off, adj))
