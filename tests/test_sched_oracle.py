"""CPU pins of the scheduler oracle: the hand-written backpropagation of the cost model
against central finite differences, and the targets rule shared with the package."""
import numpy as np

from oracle import sched_oracle as so


def _case(seed, n=40):
    r = np.random.default_rng(seed)
    w = r.normal(0, 0.3, so.NPARAM)
    x = r.uniform(0, 1, (n, so.IN))
    t = r.normal(0, 1, (n, so.OUT))
    m = (r.uniform(0, 1, (n, so.OUT)) < 0.8).astype(np.float64)
    m[0, :] = 1.0
    return w, x, t, m


def test_layout():
    assert so.NPARAM == 6020
    assert (so.OFF_B1, so.OFF_W2, so.OFF_B2, so.OFF_W3, so.OFF_B3) == (1536, 1600, 5696, 5760, 6016)


def test_backprop_matches_finite_differences():
    w, x, t, m = _case(3)
    L, g = so.loss_grad(w, x, t, m)
    assert abs(L - so.loss(w, x, t, m)) < 1e-12
    r = np.random.default_rng(7)
    # every bias and a sample of every weight matrix
    idx = list(range(so.OFF_B1, so.OFF_W2)) + list(range(so.OFF_B2, so.OFF_W3)) + list(range(so.OFF_B3, so.NPARAM))
    for lo, hi in ((so.OFF_W1, so.OFF_B1), (so.OFF_W2, so.OFF_B2), (so.OFF_W3, so.OFF_B3)):
        idx += r.choice(np.arange(lo, hi), 40, replace=False).tolist()
    fd = so.finite_diff_grad(w, x, t, m, idx)
    np.testing.assert_allclose(g[idx], fd, rtol=1e-5, atol=1e-8)


def test_masked_targets_do_not_contribute():
    w, x, t, m = _case(5)
    m[:, 2] = 0.0
    t2 = t.copy()
    t2[:, 2] += 100.0
    assert abs(so.loss(w, x, t, m) - so.loss(w, x, t2, m)) < 1e-12


def test_targets_rule_matches_package():
    from scout_b200 import learn
    for ms, ch in (([0.5, 2.0, 1.0], 10), ([0.01, 3.0, -1.0], 0), ([10.0, 0.2, -1.0], 123456)):
        t1, m1 = so.targets(ms, ch)
        t2, m2 = learn.targets(ms, ch)
        np.testing.assert_array_equal(m1, m2)
        np.testing.assert_allclose(t1, t2, rtol=1e-7)


def test_features_of_a_tiny_graph():
    # path 0-1-2-3 plus edge 1-3; BFS levels from 0: 0 1 2 2
    off = np.array([0, 1, 4, 6, 8], dtype=np.int64)
    adj = np.array([1, 0, 2, 3, 1, 3, 1, 2], dtype=np.int32)
    level = np.array([0, 1, 2, 2])
    f = so.features(off, adj, np.array([[1, 2], [0, 3]]), "bfs", level=level, prev_ms=1.0)
    assert f[1] == 0.5 and f[2] == 0.5                 # one deletion (1-2), one insertion (0-3)
    assert abs(f[22] - 0.5) < 1e-12                    # of 1->2 and 2->1, only 1->2 is a tree edge
    assert abs(f[3:19].sum() - 1.0) < 1e-12
    assert abs(f[23] - np.log2(1001.0) / 16) < 1e-12
