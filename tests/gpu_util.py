"""Helpers shared by the GPU parity tests."""
import numpy as np

from oracle import oracle as orc


def sorted_rows(off, adj):
    """Canonical form of a CSR: every row sorted (the device keeps rows ascending)."""
    out = adj.copy()
    for v in range(len(off) - 1):
        out[off[v]:off[v + 1]].sort()
    return off, out


def assert_same_graph(ctx, oracle_graph):
    o1, a1 = ctx.graph()
    o2, a2 = sorted_rows(*oracle_graph.csr())
    assert np.array_equal(o1, o2), "row lengths differ"
    assert np.array_equal(a1, a2), "row contents differ"


def stream(off, adj, kind, m, k, seed, insert_ratio=0.5, lowdeg_frac=0.0):
    import scout_b200 as sb
    g = sb.HostCsr.from_arrays(off, adj)
    return g.stream(kind, m, k, insert_ratio=insert_ratio, lowdeg_frac=lowdeg_frac, seed=seed).reshape(k, m, 2)
