"""GPU: the drop-in binaries on the bundled sample, checked against the oracle."""
import os
import re
import shutil
import subprocess

import numpy as np
import pytest

import scout_b200 as sb
from conftest import ROOT, SAMPLE
from oracle import oracle as orc

pytestmark = pytest.mark.gpu

INIT = {"mis": "sample_mis.txt", "coloring": "sample_colors.txt", "bfs": "sample_bfs.txt",
        "cc": "sample_components.txt"}


def _run(p, tmp_path, nb=5, env=None, via_run_sh=False):
    egr = tmp_path / "sample.egr"
    shutil.copyfile(os.path.join(SAMPLE, "sample.egr"), egr)
    if via_run_sh:
        cmd = ["bash", os.path.join(ROOT, "run.sh"), f"--problem={p}", f"--graph={egr}",
               f"--init={os.path.join(SAMPLE, INIT[p])}", f"--batch={os.path.join(SAMPLE, 'batches')}",
               f"--num-batches={nb}"]
    else:
        cmd = [os.path.join(ROOT, "bin", f"scout_{p}"), str(egr), os.path.join(SAMPLE, INIT[p]),
               os.path.join(SAMPLE, "batches"), str(nb), "0"]
    r = subprocess.run(cmd, capture_output=True, text=True, cwd=tmp_path, env=dict(os.environ, **(env or {})),
                       timeout=300)
    assert r.returncode == 0, r.stderr
    return r.stdout, egr


def _final(out):
    m = re.findall(r"^Final [a-zA-Z ]+:\s+(\d+)$", out, re.M)
    return int(m[-1])


def _oracle_after(problem, nb, against_base=False):
    off, adj, _ = sb.read_egr(os.path.join(SAMPLE, "sample.egr"))
    state = "mis" if problem == "mis_id" else problem
    init, _ = sb.load_state(os.path.join(SAMPLE, INIT[state]), state, 2000)
    eng = orc.Engine(problem, off, adj, init, against_base=against_base)
    for k in range(1, nb + 1):
        eng.batch(sb.parse_batch_file(os.path.join(SAMPLE, "batches", f"{k}.mtx"), 2000))
    return eng


def test_bfs_cli(tmp_path):
    out, _ = _run("bfs", tmp_path)
    lines = re.findall(r"^Batch (\d+)/5 \| edges=(\d+) \| time=[0-9.]+ms \| insertions=(\d+) \| deletions=(\d+)", out, re.M)
    assert len(lines) == 5 and all(int(e) == 50 for _, e, _, _ in lines)
    assert out.count("[STAGE] batch=") == 5 and "=== FINAL SUMMARY ===" in out
    eng = _oracle_after("bfs", 5)
    o, a = eng.graph().csr()
    assert _final(out) == int((orc.gt_bfs(o, a, 0) >= 0).sum())
    # end-of-run breakdown (scout_bfs.cu:607-613): the parts add up to the totals
    ins = re.search(r"^Insertions: (\d+) \(noop=(\d+), repaired=(\d+)\)$", out, re.M)
    dels = re.search(r"^Deletions:  (\d+) \(noop=(\d+), local=(\d+), fallback=(\d+), deferred=0\)$", out, re.M)
    assert ins and dels, out[-600:]
    assert int(ins.group(1)) == int(ins.group(2)) + int(ins.group(3)) == sum(int(x[2]) for x in lines)
    assert int(dels.group(1)) == sum(int(dels.group(k)) for k in (2, 3, 4)) == sum(int(x[3]) for x in lines)
    assert "GPU kernel:" in out


def test_coloring_cli(tmp_path):
    out, _ = _run("coloring", tmp_path)
    eng = _oracle_after("coloring", 5)
    assert _final(out) == int(eng.solution().max()) + 1
    conf = [int(x) for x in re.findall(r"\| conflicts=(\d+)", out)]
    assert sum(conf) == eng.stats()["conflict"]
    ins = re.search(r"^Insertions: (\d+) \(noop=(\d+), conflict=(\d+)\)$", out, re.M)
    assert ins and int(ins.group(3)) == sum(conf) and int(ins.group(1)) == int(ins.group(2)) + int(ins.group(3))
    assert re.search(r"^Speculative rounds: total=\d+ max_in_single_batch=\d+$", out, re.M)


def test_cc_cli(tmp_path):
    out, _ = _run("cc", tmp_path)
    eng = _oracle_after("cc", 5)
    o, a = eng.graph().csr()
    assert _final(out) == len(np.unique(orc.gt_cc(o, a)))
    # scout_cc.cu:531-539 (the sample's batches only delete edges, none a bridge)
    ins = re.search(r"^Insertions: (\d+) \(noop=(\d+), merged=(\d+)\)$", out, re.M)
    dels = re.search(r"^Deletions:  (\d+) \(noop=0, still_connected=(\d+), definitive_split=(\d+), "
                     r"fallback=(\d+), deferred=0\)$", out, re.M)
    assert ins and dels, out[-600:]
    assert int(ins.group(1)) == int(ins.group(2)) + int(ins.group(3))
    assert int(ins.group(3)) == eng.stats()["merged"]
    assert int(dels.group(1)) == sum(int(dels.group(k)) for k in (2, 3, 4))
    assert int(dels.group(2)) == eng.stats()["still_connected"]


def test_mis_cli_writes_set_and_compacts(tmp_path):
    out, egr = _run("mis", tmp_path)
    fn = tmp_path / "datasets" / "Final_MISs" / "sample_flash_final_mis.txt"
    ids = np.array([int(x) for x in fn.read_text().split()], dtype=np.int64) - 1
    flags = np.zeros(2000, dtype=np.int32)
    flags[ids] = 1
    eng = _oracle_after("mis_id", 5, against_base=True)
    assert np.array_equal(flags, eng.solution())
    assert _final(out) == int(flags.sum())
    # the input .egr was rewritten in place: the reference compactor's bytes for the same edits
    off, adj, wide = sb.read_egr(str(egr))
    assert wide
    o2, a2 = eng.graph().csr()
    assert np.array_equal(off, o2) and np.array_equal(adj, a2)
    assert orc.check_mis(off, adj, flags) == (0, 0)


def test_mis_cli_skip_compaction_and_run_sh(tmp_path):
    out, egr = _run("mis", tmp_path, env={"SCOUT_SKIP_COMPACTION": "1"}, via_run_sh=True)
    assert "[SCOUT_SKIP_COMPACTION=1]" in out
    assert egr.read_bytes() == open(os.path.join(SAMPLE, "sample.egr"), "rb").read()
