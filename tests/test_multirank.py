"""Replica sharding across ranks (the multi-GPU form of the engine): every rank repairs its own
seeded update stream with no collective on the data path; the job's throughput is the sum of
the ranks' updates over the slowest rank's time. Two gloo ranks on the CPU, the oracle standing
in for each rank's engine."""
import os
import socket

import numpy as np
import pytest
import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_stream(rank: int):
    import scout_b200 as sb
    g = sb.gen_rmat(10, 8, seed=3)
    off, adj = g.arrays()
    stream = g.stream(sb.STREAM_PREFERENTIAL, 300, 1, insert_ratio=0.5, seed=1000 + rank)
    return g, off, adj, stream


def _worker(rank, world, port, q):
    import sys
    sys.path.insert(0, ROOT)
    os.environ.update(RANK=str(rank), WORLD_SIZE=str(world), LOCAL_RANK=str(rank),
                      MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    import bench
    from oracle import oracle as orc
    d = bench.Dist(backend="gloo")
    try:
        g, off, adj, stream = _rank_stream(rank)
        eng = orc.Engine("bfs", off, adj, g.init_state("bfs", 0))
        d.barrier()
        eng.batch(stream)
        eng.finish()   # the reference engine's end-of-stream catch-up traversal
        elapsed = 0.5 + rank   # stands in for the rank's measured device time
        d.barrier()
        total = d.reduce(float(len(stream)), "sum")
        slowest = d.reduce(elapsed, "max")
        q.put((rank, total, slowest, eng.solution().tobytes()))
    finally:
        d.close()


def test_two_replicas_gloo():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    res = [q.get(timeout=240) for _ in procs]
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    res.sort()
    # every rank sees the whole-job aggregates: sum of updates, max of times
    for _, total, slowest, _ in res:
        assert total == 600.0 and slowest == 1.5
    # the replicas ran different streams and each rank's state is its own stream's
    from oracle import oracle as orc
    sols = []
    for rank, _, _, sol in res:
        g, off, adj, stream = _rank_stream(rank)
        ref = orc.Engine("bfs", off, adj, g.init_state("bfs", 0))
        ref.batch(stream)
        ref.finish()
        got = np.frombuffer(sol, dtype=np.int32)
        assert np.array_equal(got, ref.solution())
        assert np.array_equal(got, orc.gt_bfs(*ref.graph().csr(), 0))
        sols.append(got)
    s0, s1 = _rank_stream(0)[3], _rank_stream(1)[3]
    assert not np.array_equal(s0, s1)


def test_single_rank_has_no_process_group():
    import sys
    sys.path.insert(0, ROOT)
    import bench
    os.environ.pop("WORLD_SIZE", None)
    d = bench.Dist()
    assert d.world == 1 and d.pg is None
    assert d.reduce(3.0, "sum") == 3.0 and d.reduce(2.0, "max") == 2.0
    d.barrier()
    d.close()
