"""Host-side helpers of bench.py (no GPU): the launch knobs a tuned set passes to the batched
arms, per-size rates, the cycled batch sizes, the config both arms print, and the DRAM
traffic read from the committed ncu summary."""
import argparse

import bench


def test_launch_knobs_drop_the_plain_variant():
    tuned = {"blocks_per_sm": 4, "chunk_log2": 8, "lanes_per_vertex": 64, "mode": 2, "frontier": 1}
    assert bench.launch_knobs(tuned) == {"blocks_per_sm": 4, "chunk_log2": 8, "lanes_per_vertex": 64}
    assert bench.launch_knobs({}) == {}
    assert bench.launch_knobs(None) == {}


def test_per_size_rates():
    edits = [10_000, 100_000, 10_000, 1_000_000]
    ms = [1.0, 2.0, 1.0, 4.0]
    sizes = [10_000, 100_000, 10_000, 1_000_000]
    r = bench.per_size_rates(edits, ms, sizes)
    assert r == {"10000": 20_000 / 2e-3, "100000": 100_000 / 2e-3, "1000000": 1_000_000 / 4e-3}


def test_batch_sizes_cycle_and_config():
    sizes = bench.batch_sizes(20, 5)
    assert len(sizes) == 25 and sizes[:3] == list(bench.SIZES) and sizes[24] == bench.SIZES[24 % 3]
    a = argparse.Namespace(scale=22, seed=2, warmup=5)
    c1 = bench.workload_config(a, 4194304, 128308376, sizes, ["bfs", "coloring"], 1)
    c2 = bench.workload_config(a, 4194304, 128308376, sizes, ["bfs", "coloring"], 1)
    assert c1 == c2 and c1["batch_sizes"] == sizes[5:]
    assert "R-MAT scale 22" in c1["workload"] and c1["graph_bytes"] == 4 * 128308376 + 8 * 4194304


def test_profiled_traffic_reads_the_committed_summary():
    assert bench.profiled_traffic("k_bfs", 22) == 60080000.0
    assert bench.profiled_traffic("k_bfs", 20) == 48444544.0
    assert bench.profiled_traffic("k_bfs", 19) is None
    assert bench.profiled_traffic("k_cc", 22) is None
