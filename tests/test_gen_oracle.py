"""The oracle's numpy generator (oracle/gen_oracle.py) reproduces the package generator byte for
byte, and its file writers produce what the package's readers parse back. The benchmark's
reference arm builds its inputs with it, so the process that runs the reference's programs
maps no library of this package."""
import os

import numpy as np
import pytest

import scout_b200 as sb
from oracle import gen_oracle as go
from oracle import oracle as orc


@pytest.mark.parametrize("scale,ef,seed", [(8, 4, 5), (11, 16, 2), (13, 32, 29)])
def test_rmat_is_byte_identical(scale, ef, seed):
    off, adj = go.gen_rmat(scale, ef, seed=seed, chunk=1 << 14)
    g = sb.gen_rmat(scale, ef, seed=seed)
    o2, a2 = g.arrays()
    assert np.array_equal(off, o2) and np.array_equal(adj, a2)


@pytest.mark.parametrize("kind", [go.STREAM_MIXED, go.STREAM_PREFERENTIAL])
@pytest.mark.parametrize("ratio", [0.5, 0.3, 1.0])
def test_stream_is_byte_identical(kind, ratio):
    g = sb.gen_rmat(13, 16, seed=3)
    off, adj = g.arrays()
    total = 6000
    # small blocks force several sampling blocks per phase
    got = go.gen_stream(off, adj, kind, total, ratio, seed=91, block=1 << 10)
    want = g.stream(kind, total, 1, insert_ratio=ratio, seed=91)
    assert np.array_equal(got, want)


def test_initial_states_match_the_package_seeders():
    g = sb.gen_rmat(12, 16, seed=2)
    off, adj = g.arrays()
    assert np.array_equal(orc.gt_bfs(off, adj, 0), g.init_state("bfs", 0))
    assert np.array_equal(orc.gt_greedy_color(off, adj), g.init_state("coloring"))
    assert np.array_equal(orc.gt_cc(off, adj), g.init_state("cc"))
    assert np.array_equal(orc.gt_greedy_mis(off, adj), g.init_state("mis"))


def test_writers_round_trip(tmp_path):
    g = sb.gen_rmat(10, 8, seed=4)
    off, adj = g.arrays()
    egr = os.path.join(tmp_path, "g.egr")
    go.write_egr_narrow(egr, off, adj)
    o2, a2, wide = sb.read_egr(egr)
    assert not wide and np.array_equal(o2, off) and np.array_equal(a2, adj)
    s = go.gen_stream(off, adj, go.STREAM_PREFERENTIAL, 300, 0.5, seed=5)
    go.write_batch_folder(os.path.join(tmp_path, "b"), [s[:100], s[100:]])
    assert np.array_equal(sb.parse_batch_file(os.path.join(tmp_path, "b", "1.mtx"), len(off) - 1), s[:100])
    assert np.array_equal(sb.parse_batch_file(os.path.join(tmp_path, "b", "2.mtx"), len(off) - 1), s[100:])
    for p, sol in [("bfs", g.init_state("bfs", 0)), ("coloring", g.init_state("coloring")),
                   ("cc", g.init_state("cc")), ("mis", g.init_state("mis"))]:
        path = os.path.join(tmp_path, f"{p}.txt")
        go.write_state(path, p, sol)
        back, _ = sb.load_state(path, p, len(off) - 1)
        assert np.array_equal(back, sol), p
