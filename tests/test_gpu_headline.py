"""GPU parity at the headline workload, for all four problems.

R-MAT scale 22, edge factor 16 (4,194,304 vertices, 128 M directed entries), seed 2, and the
benchmark's own preferential 50/50 toggle stream (seed 1002), cut into batches of 10^5, 10^6,
10^5 and 10^6 edits. After every batch:

- BFS: levels bit-exact with a from-scratch BFS of the current graph;
- CC: labels bit-exact with the min-vertex-id partition of the current graph;
- colouring: proper, and bit-exact with the oracle's restatement of the reference rounds
  (scout_coloring.cu:46-100, 243-277) wherever that rule did not truncate a round (a
  truncated batch is logged with the colour counts of both);
- MIS: independent and maximal, and bit-exact with the oracle's vertex-id-priority rule.

The graph after each batch is computed here from sorted (u << 32 | v) keys with the toggle
rule of cli_setup.h:87-103 (every toggle classified against the graph before its batch).
"""
import numpy as np
import pytest

import scout_b200 as sb
from oracle import oracle as orc

pytestmark = pytest.mark.gpu

SIZES = (100_000, 1_000_000, 100_000, 1_000_000)
U64 = np.uint64


def _member(sorted_keys, q):
    at = np.searchsorted(sorted_keys, q)
    return (at < len(sorted_keys)) & (sorted_keys[np.minimum(at, len(sorted_keys) - 1)] == q)


def _apply(keys, b):
    u = b[:, 0].astype(U64)
    v = b[:, 1].astype(U64)
    fwd = (u << U64(32)) | v
    bwd = (v << U64(32)) | u
    present = _member(keys, fwd)
    gone = np.sort(np.concatenate((fwd[present], bwd[present])))
    kept = keys[~_member(gone, keys)] if len(gone) else keys
    new = np.sort(np.concatenate((fwd[~present], bwd[~present])))
    return np.sort(np.concatenate((kept, new)), kind="stable")


def _csr(keys, n):
    rows = (keys >> U64(32)).astype(np.int64)
    off = np.zeros(n + 1, dtype=np.int64)
    np.cumsum(np.bincount(rows, minlength=n), out=off[1:])
    return off, (keys & U64(0xFFFFFFFF)).astype(np.int32)


@pytest.fixture(scope="module")
def headline():
    g = sb.gen_rmat(22, 16, seed=2)
    off, adj = g.arrays()
    n = len(off) - 1
    s = g.stream(sb.STREAM_PREFERENTIAL, sum(SIZES), 1, insert_ratio=0.5, seed=1002)
    bounds = np.cumsum([0] + list(SIZES))
    batches = [np.ascontiguousarray(s[bounds[i]:bounds[i + 1]]) for i in range(len(SIZES))]
    keys = (np.repeat(np.arange(n, dtype=U64), np.diff(off)) << U64(32)) | adj.astype(U64)
    states = []
    for b in batches:
        keys = _apply(keys, b)
        states.append(_csr(keys, n))
    return off, adj, batches, states


def _run(problem, off, adj, init, batches, check):
    mirror = init.copy()
    with sb.Context(0) as ctx:
        ctx.load_csr(off, adj)
        ctx.upload(problem, init)
        ctx.reserve_batches(max(len(b) for b in batches))
        for k, b in enumerate(batches):
            ctx.repair(problem, b)
            got = ctx.download(problem)
            ctx.commit(problem, mirror)
            assert np.array_equal(mirror, got), f"{problem}: host mirror differs after batch {k + 1}"
            check(k, got)


def test_headline_bfs(headline):
    off, adj, batches, states = headline

    def check(k, got):
        truth = orc.gt_bfs(*states[k], 0)
        bad = np.flatnonzero(got != truth)
        assert len(bad) == 0, f"batch {k + 1}: {len(bad)} levels differ, first at {bad[:8]}"

    _run("bfs", off, adj, orc.gt_bfs(off, adj, 0), batches, check)


def test_headline_cc(headline):
    off, adj, batches, states = headline

    def check(k, got):
        truth = orc.gt_cc(*states[k])
        bad = np.flatnonzero(got != truth)
        assert len(bad) == 0, f"batch {k + 1}: {len(bad)} labels differ, first at {bad[:8]}"

    _run("cc", off, adj, orc.gt_cc(off, adj), batches, check)


def test_headline_coloring(headline):
    off, adj, batches, states = headline
    init = orc.gt_greedy_color(off, adj)
    ref = orc.Engine("coloring", off, adj, init)
    exact = []

    def check(k, got):
        assert orc.check_coloring(*states[k], got) == 0, f"batch {k + 1}: not a proper colouring"
        ref.batch(batches[k])
        st = ref.stats()
        want = ref.solution()
        if st["truncated"] == 0:
            assert np.array_equal(got, want), f"batch {k + 1}: differs from the reference rule"
            exact.append(k)
        else:
            print(f"coloring batch {k + 1}: reference truncated {st['truncated']} rounds; colours "
                  f"{int(got.max()) + 1} here vs {int(want.max()) + 1} in the reference rule")

    _run("coloring", off, adj, init, batches, check)
    assert exact, "no batch was comparable with the reference rule"


def test_headline_mis(headline):
    off, adj, batches, states = headline
    init = orc.gt_greedy_mis(off, adj)
    ref = orc.Engine("mis_id", off, adj, init)

    def check(k, got):
        bad, undominated = orc.check_mis(*states[k], got)
        assert bad == 0, f"batch {k + 1}: {bad} adjacent members"
        assert undominated == 0, f"batch {k + 1}: {undominated} undominated non-members"
        ref.batch(batches[k])
        assert np.array_equal(got, ref.solution()), f"batch {k + 1}: differs from the id-priority rule"

    _run("mis", off, adj, init, batches, check)
