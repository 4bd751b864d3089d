"""Records what the reference's own engines print on the bundled sample and on an R-MAT
scale-16 stream, for every prefix of the batch stream. Needs a GPU and oracle/_ref/ (built by
oracle/build_ref.sh from the reference sources); run on a machine with a B200:

    python tests/golden/make_ref_engine_golden.py ref_engines.json

and commit the JSON as tests/golden/ref_engines.json. Each entry holds the per-batch lines
(edges, counters) and the final summary (solution measure, insertion/deletion breakdowns).
The R-MAT case is regenerated bit-identically by the package's seeded generators, so the
tests replay it without shipping its files.
"""
from __future__ import annotations

import json
import os
import re
import subprocess
import sys
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

import scout_b200 as sb  # noqa: E402

REF = os.path.join(ROOT, "oracle", "_ref")
BATCH_RE = re.compile(r"^Batch (\d+)/(\d+) \| edges=(\d+) \| time=[0-9.]+ms(.*)$")
KV_RE = re.compile(r" \| (\w+)=(-?\d+)")
FINAL_RE = re.compile(r"^Final (.+?):\s+(-?\d+)$")
STATS_RE = re.compile(r"^(Insertions|Deletions):\s+(\d+) \((.*)\)$")
ROUNDS_RE = re.compile(r"^Speculative rounds: total=(\d+) max_in_single_batch=(\d+)$")
STATE_FILE = {"mis": "mis", "coloring": "coloring", "bfs": "bfs", "cc": "cc"}

RMAT = {"scale": 16, "edge_factor": 16, "seed": 1, "stream": "mixed", "batch_size": 1000, "batches": 10,
        "stream_seed": 1}


def parse(out: str) -> dict:
    rec = {"batches": [], "final": None, "stats": {}}
    for line in out.splitlines():
        m = BATCH_RE.match(line)
        if m:
            kv = {k: int(v) for k, v in KV_RE.findall(m.group(4))}
            rec["batches"].append({"i": int(m.group(1)), "edges": int(m.group(3)), **kv})
            continue
        m = FINAL_RE.match(line.strip())
        if m:
            rec["final"] = int(m.group(2))
            continue
        m = STATS_RE.match(line.strip())
        if m:
            d = {"total": int(m.group(2))}
            for part in m.group(3).split(","):
                if "=" in part:
                    k, v = part.strip().split("=")
                    d[k] = int(v)
            rec["stats"][m.group(1).lower()] = d
            continue
        m = ROUNDS_RE.match(line.strip())
        if m:
            rec["stats"]["rounds"] = {"total": int(m.group(1)), "max": int(m.group(2))}
    return rec


def run_case(name, egr, states, bdir, nb, out):
    for p in ("bfs", "coloring", "cc", "mis"):
        for k in range(1, nb + 1):
            with tempfile.TemporaryDirectory() as td:
                env = dict(os.environ, SCOUT_SKIP_COMPACTION="1")
                r = subprocess.run([os.path.join(REF, f"scout_{p}"), egr, states[p], bdir, str(k), "0"],
                                   capture_output=True, text=True, env=env, cwd=td, timeout=600)
                rec = parse(r.stdout)
                rec["rc"] = r.returncode
                if p == "mis":
                    fn = os.path.join(td, "datasets", "Final_MISs", os.path.splitext(os.path.basename(egr))[0]
                                      + "_flash_final_mis.txt")
                    if os.path.exists(fn):
                        rec["mis_ids"] = [int(x) for x in open(fn).read().split()]
            out.setdefault(name, {}).setdefault(p, {})[str(k)] = rec
            print(name, p, k, rec["final"], flush=True)


def main():
    dst = sys.argv[1] if len(sys.argv) > 1 else os.path.join(HERE, "ref_engines.json")
    out = {}
    s = os.path.join(HERE, "sample")
    states = {"mis": f"{s}/sample_mis.txt", "coloring": f"{s}/sample_colors.txt", "bfs": f"{s}/sample_bfs.txt",
              "cc": f"{s}/sample_components.txt"}
    run_case("sample", f"{s}/sample.egr", states, f"{s}/batches", 5, out)
    with tempfile.TemporaryDirectory() as td:
        g = sb.gen_rmat(RMAT["scale"], RMAT["edge_factor"], seed=RMAT["seed"])
        off, adj = g.arrays()
        egr = os.path.join(td, "rmat16.egr")
        sb.write_egr(egr, off, adj, wide=False)
        st = g.stream(sb.STREAM_MIXED, RMAT["batch_size"], RMAT["batches"], seed=RMAT["stream_seed"])
        sb.write_batch_folder(os.path.join(td, "b"), st, RMAT["batch_size"], RMAT["batches"])
        states = {}
        for p in ("mis", "coloring", "bfs", "cc"):
            states[p] = os.path.join(td, f"{p}.txt")
            sb.write_state(states[p], p, g.init_state(p, 0))
        run_case("rmat16", egr, states, os.path.join(td, "b"), RMAT["batches"], out)
    out["_rmat16_case"] = RMAT
    with open(dst, "w") as f:
        json.dump(out, f, sort_keys=True)
    print("wrote", dst)


if __name__ == "__main__":
    main()
