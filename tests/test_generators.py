"""Synthetic workloads: R-MAT graphs and update streams (no GPU)."""
import numpy as np
import pytest

import scout_b200 as sb


def test_rmat_is_simple_symmetric_sorted(rmat16):
    g, (off, adj) = rmat16
    n = g.n
    assert n == 65536 and off[0] == 0 and off[-1] == len(adj)
    src = np.repeat(np.arange(n), np.diff(off))
    assert not np.any(src == adj), "self-loop"
    keys = src.astype(np.int64) * n + adj
    assert np.all(np.diff(keys) > 0), "rows sorted, no duplicates"
    rev = np.sort(adj.astype(np.int64) * n + src)
    assert np.array_equal(rev, keys), "symmetric"
    # R-MAT(.57,.19,.19,.05) skew: vertex 0 is the hub
    assert np.argmax(np.diff(off)) == 0 and 1.5e6 < len(adj) < 2.1e6


def test_rmat_deterministic():
    a = sb.gen_rmat(12, 8, seed=5).arrays()
    b = sb.gen_rmat(12, 8, seed=5).arrays()
    c = sb.gen_rmat(12, 8, seed=6).arrays()
    assert np.array_equal(a[1], b[1]) and not np.array_equal(a[1], c[1])


@pytest.mark.parametrize("kind", [sb.STREAM_MIXED, sb.STREAM_PREFERENTIAL, sb.STREAM_LOWDEG])
def test_streams(kind, rmat16):
    g, (off, adj) = rmat16
    n = g.n
    s = g.stream(kind, 1000, 10, insert_ratio=0.5 if kind != sb.STREAM_LOWDEG else 0.3, lowdeg_frac=0.3, seed=3)
    assert s.shape == (10000, 2)
    assert np.all(s[:, 0] < s[:, 1]) and np.all(s >= 0) and np.all(s < n)
    keys = s[:, 0].astype(np.int64) * n + s[:, 1]
    assert len(np.unique(keys)) == len(keys), "each pair once per stream"
    src = np.repeat(np.arange(n), np.diff(off))
    edge_keys = set((src.astype(np.int64) * n + adj).tolist())
    existing = np.array([k in edge_keys for k in keys.tolist()])
    frac_del = existing.mean()
    want = 0.5 if kind != sb.STREAM_LOWDEG else 0.7
    assert abs(frac_del - want) < 1e-9
    deg = np.diff(off)
    if kind == sb.STREAM_PREFERENTIAL:
        ins = s[~existing]
        assert deg[ins].mean() > 5 * deg.mean(), "insert endpoints proportional to degree"
    if kind == sb.STREAM_LOWDEG:
        # deletions whose first endpoint is drawn with probability 1/degree touch far
        # lower-degree vertices than deletions drawn uniformly over the edges
        low = g.stream(kind, 1000, 2, insert_ratio=0.0, lowdeg_frac=1.0, seed=4)
        uni = g.stream(kind, 1000, 2, insert_ratio=0.0, lowdeg_frac=0.0, seed=4)
        mlow = np.median(np.minimum(deg[low[:, 0]], deg[low[:, 1]]))
        muni = np.median(np.minimum(deg[uni[:, 0]], deg[uni[:, 1]]))
        assert mlow * 4 < muni
    # deterministic
    assert np.array_equal(s, g.stream(kind, 1000, 10, insert_ratio=0.5 if kind != sb.STREAM_LOWDEG else 0.3,
                                      lowdeg_frac=0.3, seed=3))


def test_stream_rejects_impossible_requests():
    g = sb.HostCsr.from_arrays([0, 1, 2], [1, 0])
    with pytest.raises(sb.ScoutError):
        g.stream(sb.STREAM_MIXED, 10, 1, insert_ratio=0.0)
