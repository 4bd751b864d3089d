"""Generates the committed golden fixtures from the reference itself.

Run where the reference tree is available ($SCOUT_REFERENCE_DIR, else `reference` beside the
repository root) after
`bash oracle/build_ref.sh`:

    python tests/golden/make_golden.py

Writes into tests/golden/:
  sample/                     the reference's bundled sample dataset (its only fixture)
  ref_core_cmds.txt / ref_core_out.txt
                              commands replayed through the reference's own FlashGraph.h /
                              cli_setup.h / chunking.h / flash_compactor.h (oracle/_ref/
                              ref_core_driver) and the output they printed
  malformed_batch.mtx, malformed_ints.txt
                              hand-made inputs exercising the parser's skip rules
  golden.json                 hashes and counts from the reference's seeding tools
                              (tools/compute_initial_mis.py, tools/greedy_color.cpp) on the
                              sample and on the R-MAT scale-16 graph of the MIS workload
"""
from __future__ import annotations

import hashlib
import json
import os
import shutil
import subprocess
import sys
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)
REF = os.environ.get("SCOUT_REFERENCE_DIR") or os.path.join(os.path.dirname(ROOT), "reference")
REF_BIN = os.path.join(ROOT, "oracle", "_ref")


def sha(path: str) -> str:
    with open(path, "rb") as f:
        return hashlib.sha256(f.read()).hexdigest()


def copy_sample() -> None:
    src = os.path.join(REF, "datasets", "sample")
    dst = os.path.join(HERE, "sample")
    os.makedirs(os.path.join(dst, "batches"), exist_ok=True)
    for f in ("sample.egr", "sample_mis.txt", "sample_colors.txt", "sample_bfs.txt", "sample_components.txt"):
        shutil.copyfile(os.path.join(src, f), os.path.join(dst, f))
    for k in range(1, 6):
        shutil.copyfile(os.path.join(src, "batches", f"{k}.mtx"), os.path.join(dst, "batches", f"{k}.mtx"))


def malformed_inputs() -> None:
    with open(os.path.join(HERE, "malformed_batch.mtx"), "w") as f:
        f.write("%%MatrixMarket matrix coordinate pattern symmetric\n"
                "% comment line\n"
                "217 1391\n"          # a real sample edge (deletion)
                "1 1\n"               # self-loop: skipped
                "0 5\n"               # id 0 -> -1: out of range
                "2001 4\n"            # beyond n
                "  5\t 9 trailing tokens\n"
                "12abc 5\n"           # second token fails to parse
                "7 8x\n"              # accepted: 8 then garbage
                "+3 -4\n"             # -4 out of range
                "99999999999 3\n"     # overflow: skipped
                "1391 217\n"          # the same edge reversed (classified against the same state)
                "\n"
                "10 11")              # no trailing newline
    with open(os.path.join(HERE, "malformed_ints.txt"), "w") as f:
        f.write("1 2\n-3 x4 5-6\n+7\n\n  8 9999999999999 -\n10")


def core_commands(n: int) -> str:
    rng = np.random.default_rng(7)
    egr = os.path.join(HERE, "sample", "sample.egr")
    import scout_b200 as sb
    off, adj, _ = sb.read_egr(egr)
    cmds = []
    # deletions of base edges, re-insertions (un-tombstone), insertions of new edges,
    # deletion of added edges, duplicate insertions, adjacency probes and row dumps
    base_edges = [(v, int(adj[i])) for v in range(0, n, 97) for i in range(off[v], min(off[v + 1], off[v] + 2))]
    for u, v in base_edges[:12]:
        cmds += [f"del {u} {v}", f"adj {u} {v}", f"adj {v} {u}", f"row {u}", f"row {v}"]
    for u, v in base_edges[:4]:
        cmds += [f"ins {u} {v}", f"row {u}", f"adj {u} {v}"]
    for _ in range(10):
        u, v = (int(x) for x in rng.integers(0, n, 2))
        if u == v:
            continue
        cmds += [f"adj {u} {v}", f"ins {u} {v}", f"row {u}", f"row {v}", f"adj {v} {u}"]
    cmds += ["ins 3 1500", "ins 3 1500", "row 3", "row 1500", "del 3 1500", "row 3", "adj 3 1500",
             "del 3 1500", "row 3", "adj 1500 3", "ins 1663 5", "row 1663", "row 5"]
    for k in range(1, 6):
        cmds.append(f"parse {os.path.join(HERE, 'sample', 'batches', f'{k}.mtx')} {n}")
    cmds.append(f"parse {os.path.join(HERE, 'malformed_batch.mtx')} {n}")
    cmds.append(f"ints {os.path.join(HERE, 'malformed_ints.txt')}")
    cmds += ["chunk 40 0 1 2 3 4 5 6 7 8 9", "chunk 3 0 1 2", "chunk 100000 5 6 7", "chunk 5 1663 1663 0"]
    return "\n".join(cmds) + "\n"


def run_core_driver(n: int) -> None:
    cmds = core_commands(n)
    with open(os.path.join(HERE, "ref_core_cmds.txt"), "w") as f:
        f.write(cmds.replace(HERE, "@GOLDEN@"))
    with tempfile.TemporaryDirectory() as td:
        work_egr = os.path.join(td, "g.egr")
        shutil.copyfile(os.path.join(HERE, "sample", "sample.egr"), work_egr)
        out_egr = os.path.join(td, "compacted.egr")
        r = subprocess.run([os.path.join(REF_BIN, "ref_core_driver"), work_egr],
                           input=cmds + f"compact {out_egr}\n" + "row 3\nrow 1663\n", capture_output=True,
                           text=True, check=True)
        with open(os.path.join(HERE, "ref_core_out.txt"), "w") as f:
            f.write(r.stdout.replace(out_egr, "@OUT@"))
        return sha(out_egr), os.path.getsize(out_egr)


def tool_outputs() -> dict:
    import scout_b200 as sb
    res = {}
    with tempfile.TemporaryDirectory() as td:
        graphs = {"sample": os.path.join(HERE, "sample", "sample.egr")}
        g = sb.gen_rmat(16, 16, seed=1)
        off, adj = g.arrays()
        p = os.path.join(td, "rmat16.egr")
        sb.write_egr(p, off, adj, wide=False)
        graphs["rmat16_ef16_seed1"] = p
        for name, egr in graphs.items():
            mis_out = os.path.join(td, name + "_mis.txt")
            subprocess.run([sys.executable, os.path.join(REF, "tools", "compute_initial_mis.py"), "--egr", egr,
                            "--out", mis_out], check=True, capture_output=True)
            egr_copy = os.path.join(td, name + "_copy.egr")
            shutil.copyfile(egr, egr_copy)
            subprocess.run([os.path.join(REF_BIN, "greedy_color"), egr_copy], check=True, capture_output=True)
            col = egr_copy + ".colors.txt"
            colors = np.loadtxt(col, dtype=np.int64)
            with open(mis_out) as f:
                mis_count = sum(1 for line in f if line.strip())
            res[name] = {"egr_sha256": sha(egr), "mis_sha256": sha(mis_out), "mis_count": mis_count,
                         "colors_sha256": sha(col), "colors_used": int(colors.max()) + 1}
            if name == "sample":
                shutil.copyfile(col, os.path.join(HERE, "sample_greedy_colors.txt"))
    return res


def main() -> None:
    if not os.path.isdir(REF):
        raise SystemExit(f"reference tree not found at {REF}")
    copy_sample()
    malformed_inputs()
    n = 2000
    compact_sha, compact_size = run_core_driver(n)
    gold = {"reference_dir_layout": "datasets/sample, tools/, core/",
            "compacted_sample_sha256": compact_sha, "compacted_sample_bytes": compact_size,
            "tools": tool_outputs()}
    with open(os.path.join(HERE, "golden.json"), "w") as f:
        json.dump(gold, f, indent=1, sort_keys=True)
    print(json.dumps(gold, indent=1))


if __name__ == "__main__":
    main()
