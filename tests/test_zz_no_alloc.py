"""The allocation-free BFS entry point (scout_bfs_levels_noalloc) gives the same levels as the
context-based full recompute (scout_recompute_bfs) and as the oracle's from-scratch BFS, call
after call.

Callers of this entry point cannot allocate device memory themselves (a foreign allocator or
fixed arena owns the device memory, real-time code); the library keeps its working buffers in
a static device array instead, so repeated calls reuse it. This file is
collected last so a failure here leaves every other test already run; it passes alone in a
fresh process too.
"""
import ctypes

import numpy as np
import pytest

import scout_b200 as sb
from oracle import oracle as orc
from scout_b200._lib import LIB

pytestmark = pytest.mark.gpu

MAX_VERTICES = 1 << 20


def _levels_via_context(off, adj, source):
    with sb.Context(0) as ctx:
        ctx.load_csr(off, adj)
        ctx.upload("bfs", np.full(len(off) - 1, -1, dtype=np.int32))
        ctx.recompute_bfs(source)
        return ctx.download("bfs")


def _levels_noalloc(torch, d_off, d_adj, n, source, d_level):
    rc = LIB.scout_bfs_levels_noalloc(ctypes.c_void_p(d_off.data_ptr()), ctypes.c_void_p(d_adj.data_ptr()), n,
                                      source, ctypes.c_void_p(d_level.data_ptr()),
                                      ctypes.c_void_p(torch.cuda.current_stream().cuda_stream))
    assert rc == 0, LIB.scout_last_error(None)
    return d_level.cpu().numpy()


def _graphs(sample_graph, rmat16):
    yield "sample", sample_graph[0], sample_graph[1], 0
    yield "sample_src1663", sample_graph[0], sample_graph[1], 1663   # isolated source
    yield "rmat16", rmat16[1][0], rmat16[1][1], 0
    yield "rmat16_src777", rmat16[1][0], rmat16[1][1], 777


def test_noalloc_bfs_matches_recompute_twice(sample_graph, rmat16):
    torch = pytest.importorskip("torch")
    for name, off, adj, src in _graphs(sample_graph, rmat16):
        n = len(off) - 1
        want = _levels_via_context(off, adj, src)
        assert np.array_equal(want, orc.gt_bfs(off, adj, src)), f"{name}: the context recompute differs"
        d_off = torch.from_numpy(np.ascontiguousarray(off, dtype=np.int64)).cuda()
        d_adj = torch.from_numpy(np.ascontiguousarray(adj, dtype=np.int32)).cuda()
        d_lev = torch.full((n,), 12345, dtype=torch.int32, device="cuda")
        for call in range(2):   # the static array keeps the previous call's contents
            got = _levels_noalloc(torch, d_off, d_adj, n, src, d_lev)
            assert np.array_equal(got, want), f"{name}: call {call + 1} differs"
        # the first call of the process loaded the kernel's module, which places the static
        # array on the device; calls after it take no device memory
        torch.cuda.synchronize()
        free0 = torch.cuda.mem_get_info()[0]
        for call in range(2):
            got = _levels_noalloc(torch, d_off, d_adj, n, src, d_lev)
            assert np.array_equal(got, want), f"{name}: call {call + 3} differs"
        assert torch.cuda.mem_get_info()[0] == free0, f"{name}: device memory was allocated"


def test_noalloc_refuses_oversized_graphs():
    torch = pytest.importorskip("torch")
    d = torch.zeros(4, dtype=torch.int64, device="cuda")
    rc = LIB.scout_bfs_levels_noalloc(ctypes.c_void_p(d.data_ptr()), ctypes.c_void_p(d.data_ptr()), MAX_VERTICES + 1,
                                      0, ctypes.c_void_p(d.data_ptr()), None)
    assert rc == -3   # SCOUT_E_CAPACITY
    assert b"at most 1048576" in LIB.scout_last_error(None)
