"""Host-side parity with the reference's own code (no GPU).

The commands in golden/ref_core_cmds.txt were run through the reference's FlashGraph.h,
cli_setup.h, chunking.h and flash_compactor.h (oracle/ref_core_driver, compiled from the
reference tree); golden/ref_core_out.txt is what they printed. Both the package's host
scratchpad (scout_b200.HybridGraph) and the oracle replay the commands and must print the
same lines.
"""
import hashlib
import json
import os
import shutil

import numpy as np
import pytest

from conftest import GOLDEN, SAMPLE

import scout_b200 as sb
from oracle import oracle as orc


def _cmds():
    with open(os.path.join(GOLDEN, "ref_core_cmds.txt")) as f:
        return [l.replace("@GOLDEN@", GOLDEN) for l in f.read().splitlines() if l.strip()]


def _expected():
    with open(os.path.join(GOLDEN, "ref_core_out.txt")) as f:
        return f.read().splitlines()


def _bound_by_cumulative_degree(deg, cand, cap):   # chunking.h:20-32
    n = probe = 0
    for v in cand:
        if n >= cap:
            break
        d = deg(v)
        if probe + d > cap:
            break
        probe += d
        n += 1
    return n


def _replay(is_adj, insert, remove, row, degree, n=2000):
    out = []
    for line in _cmds():
        t = line.split()
        if t[0] in ("ins", "del", "adj"):
            u, v = int(t[1]), int(t[2])
            if t[0] == "ins":
                insert(u, v)
            elif t[0] == "del":
                remove(u, v)
            else:
                out.append(f"adj {u} {v} {1 if is_adj(u, v) else 0}")
        elif t[0] == "row":
            v = int(t[1])
            r = row(v)
            out.append(f"row {v} {degree(v)}:" + "".join(f" {x}" for x in r))
        elif t[0] == "parse":
            pairs = sb.parse_batch_file(t[1], int(t[2]))
            out.append(f"parse {len(pairs)}")
            # classification against the graph as it stands before the batch
            for u, v in pairs.tolist():
                out.append(f"{u} {v} {0 if is_adj(u, v) else 1}")
        elif t[0] == "ints":
            vals = sb.read_ints(t[1])
            out.append(f"ints {len(vals)}:" + "".join(f" {x}" for x in vals.tolist()))
        elif t[0] == "chunk":
            cap = int(t[1])
            out.append(f"chunk {_bound_by_cumulative_degree(degree, [int(x) for x in t[2:]], cap)}")
    return out


def test_package_scratchpad_matches_reference(tmp_path):
    egr = tmp_path / "g.egr"
    shutil.copyfile(os.path.join(SAMPLE, "sample.egr"), egr)
    h = sb.HybridGraph(str(egr))
    got = _replay(h.is_adjacent, h.insert, h.remove, h.neighbors, h.degree)
    exp = _expected()
    assert got == exp[: len(got)]
    # compaction: byte-identical wide .egr, then the rows read back from the new mapping
    out = tmp_path / "compacted.egr"
    h.compact(str(out))
    gold = json.load(open(os.path.join(GOLDEN, "golden.json")))
    assert hashlib.sha256(out.read_bytes()).hexdigest() == gold["compacted_sample_sha256"]
    tail = exp[len(got):]
    assert tail[0] == f"compacted 2000 {sb.read_egr(str(out))[0][-1]}"
    for line in tail[1:]:
        v = int(line.split()[1])
        assert line == f"row {v} {h.degree(v)}:" + "".join(f" {x}" for x in h.neighbors(v))


def test_oracle_scratchpad_matches_reference(sample_graph):
    off, adj = sample_graph
    g = orc.Graph(off, adj)

    def degree(v):
        return len(g.row(v))

    got = _replay(g.is_adjacent, g.insert, g.remove, g.row, degree)
    assert got == _expected()[: len(got)]


def test_egr_roundtrip_narrow_and_wide(tmp_path, sample_graph):
    off, adj = sample_graph
    for wide in (False, True):
        p = tmp_path / f"g{int(wide)}.egr"
        sb.write_egr(str(p), off, adj, wide=wide)
        o2, a2, w2 = sb.read_egr(str(p))
        assert w2 == wide
        assert np.array_equal(o2, off) and np.array_equal(a2, adj)
    # the sample itself is wide; rewriting it wide reproduces its bytes
    p = tmp_path / "w.egr"
    sb.write_egr(str(p), off, adj, wide=True)
    assert p.read_bytes() == open(os.path.join(SAMPLE, "sample.egr"), "rb").read()


def test_egr_rejects_truncated_and_bad_headers(tmp_path):
    raw = open(os.path.join(SAMPLE, "sample.egr"), "rb").read()
    for cut in (0, 4, 12, 100, len(raw) - 4):
        p = tmp_path / f"t{cut}.egr"
        p.write_bytes(raw[:cut])
        with pytest.raises(sb.ScoutError) as e:
            sb.read_egr(str(p))
        assert e.value.code == -7
    p = tmp_path / "neg.egr"
    p.write_bytes(np.array([5, -3], dtype=np.int32).tobytes())
    with pytest.raises(sb.ScoutError):
        sb.read_egr(str(p))
    with pytest.raises(sb.ScoutError) as e:
        sb.read_egr(str(tmp_path / "missing.egr"))
    assert e.value.code == -6


def test_initial_state_decoding(tmp_path):
    n = 2000
    mis, cnt = sb.load_state(os.path.join(SAMPLE, "sample_mis.txt"), "mis", n)
    assert cnt == 533 and mis.sum() == 533
    col, used = sb.load_state(os.path.join(SAMPLE, "sample_colors.txt"), "coloring", n)
    assert used == col.max() + 1 == 6
    lev, reached = sb.load_state(os.path.join(SAMPLE, "sample_bfs.txt"), "bfs", n)
    assert reached == (lev >= 0).sum() and lev[0] == 0
    lab, comps = sb.load_state(os.path.join(SAMPLE, "sample_components.txt"), "cc", n)
    assert comps == 2 and set(np.unique(lab).tolist()) == {0, 1663}
    # reference corner cases: repeated MIS ids count twice, short colour files pad with 0,
    # out-of-range ids are skipped, an odd trailing BFS value is ignored
    p = tmp_path / "s.txt"
    p.write_text("3\n3\n0\n9\n")
    f, c = sb.load_state(str(p), "mis", 5)
    assert c == 2 and f.tolist() == [0, 0, 1, 0, 0]
    f, c = sb.load_state(str(p), "coloring", 6)
    assert f.tolist() == [3, 3, 0, 9, 0, 0] and c == 10
    p.write_text("1 0\n2 1\n7 3\n4")
    f, c = sb.load_state(str(p), "bfs", 5)
    assert f.tolist() == [0, 1, -1, -1, -1] and c == 2
    p.write_text("0\n0\n1\n2\n")
    f, c = sb.load_state(str(p), "cc", 5)
    assert f.tolist() == [0, 0, 0, 0, 4] and c == 2
    p.write_text("1\n0\n")   # parent cycle: the reference would loop forever
    with pytest.raises(sb.ScoutError):
        sb.load_state(str(p), "cc", 2)


def test_state_and_batch_writers_roundtrip(tmp_path):
    rng = np.random.default_rng(3)
    n = 50
    for prob, sol in (("mis", (rng.random(n) < 0.3).astype(np.int32)), ("coloring", rng.integers(0, 9, n)),
                      ("bfs", rng.integers(-1, 7, n)), ("cc", np.sort(rng.integers(0, n, n)))):
        p = tmp_path / f"{prob}.txt"
        sb.write_state(str(p), prob, sol)
        back, _ = sb.load_state(str(p), prob, n)
        if prob == "cc":
            assert np.array_equal(orc.canonical_labels(back), orc.canonical_labels(np.minimum(sol, np.arange(n)) * 0 + back))
        else:
            assert np.array_equal(back, np.asarray(sol, dtype=np.int32))
    e = rng.integers(0, n, size=(30, 2)).astype(np.int32)
    e = e[e[:, 0] != e[:, 1]][:20]
    sb.write_batch_folder(str(tmp_path / "b"), e, 10, 2)
    got = np.concatenate([sb.parse_batch_file(str(tmp_path / "b" / f"{k}.mtx"), n) for k in (1, 2)])
    assert np.array_equal(got, e)


def test_parallel_batch_parse_equals_serial(tmp_path):
    """A batch file large enough to be parsed in parallel chunks gives the same edits, in file
    order, as the line-by-line rule (malformed lines, out-of-range ids and self-loops dropped)."""
    import numpy as np

    import scout_b200 as sb
    r = np.random.default_rng(4)
    n = 5000
    lines, want = [], []
    for i in range(300000):
        u, v = int(r.integers(0, n + 3)), int(r.integers(0, n + 3))
        k = i % 97
        if k == 0:
            lines.append("garbage line")
            continue
        if k == 1:
            lines.append(f"  {u + 1}\t{v + 1}  extra")
        else:
            lines.append(f"{u + 1} {v + 1}")
        if 0 <= u < n and 0 <= v < n and u != v:
            want.append((u, v))
    p = tmp_path / "big.mtx"
    p.write_text("\n".join(lines) + "\n")
    got = sb.parse_batch_file(str(p), n)
    assert np.array_equal(got, np.array(want, dtype=np.int32).reshape(-1, 2))


def test_compaction_spanning_rewrite_windows(tmp_path):
    """The rewrite gathers rows over the host threads in windows of 2^25 entries: a graph of
    more than one window, with toggles spread over the id range, compacts to the rows the
    scratchpad held (unedited rows byte for byte the base's, edited rows in the reference's
    order: base minus tombstones, then additions)."""
    g = sb.gen_rmat(20, 18, seed=11)
    off, adj = g.arrays()
    assert off[-1] > (1 << 25)
    src = tmp_path / "g.egr"
    sb.write_egr(str(src), off, adj)
    h = sb.HybridGraph(str(src))
    n = len(off) - 1
    rng = np.random.default_rng(5)
    edited = set()
    for u, v in rng.integers(0, n, size=(3000, 2)).tolist():
        if u == v:
            continue
        if h.is_adjacent(u, v):
            h.remove(u, v)
            h.remove(v, u)
        else:
            h.insert(u, v)
            h.insert(v, u)
        edited.update((u, v))
    want = {v: h.neighbors(v).copy() for v in edited}
    out = tmp_path / "c.egr"
    h.compact(str(out))
    off2, adj2, _ = sb.read_egr(str(out))
    deg, deg2 = np.diff(off), np.diff(off2)
    mask = np.ones(n, dtype=bool)
    mask[list(edited)] = False
    assert np.array_equal(deg[mask], deg2[mask])
    keep = np.repeat(mask, deg)
    keep2 = np.repeat(mask, deg2)
    assert np.array_equal(adj[keep], adj2[keep2])
    for v, row in want.items():
        assert np.array_equal(adj2[off2[v]:off2[v + 1]], row), f"row {v}"
