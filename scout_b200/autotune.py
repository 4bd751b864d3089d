"""Autotuner of the engine's launch knobs.

Knobs (all exact: they change speed, never results; every configuration's final solution is
checksummed and the sweep fails if two differ):
  blocks_per_sm     resident blocks per SM of the persistent repair kernels (1, 2, 4): more
                    blocks hide latency, fewer make each grid barrier cheaper
  chunk_log2        BFS queue item = 2^chunk_log2 row entries (8 .. 13): smaller items spread a
                    hub's row over more warps, larger ones cost fewer queue entries
  lanes_per_vertex  BFS: most lanes sharing one queue item when a round has fewer items than
                    warps (32, 64, 128, 256, 1024, i.e. 1-32 warps; 0 = as many as useful)
  mode / frontier   the plain engine's repair variant: incremental, or a full traversal with a
                    queue frontier (top-down) or a bitmap frontier (direction-optimizing); CC:
                    incremental or a recompute of every class. The learned scheduler picks the
                    variant per batch instead
  round_cap         multi-stream engine: most edits per round (2^16 .. 2^22): larger rounds
                    amortise the per-round fixed cost over more streams, smaller ones bound the
                    latency a small batch waits behind large ones

Each configuration replays the same sample batches from the same starting state on a fresh
context and is scored by the library's device time (CUDA events on its stream) over the
sample, after one warm-up batch. The defaults (blocks 4, chunk 10, lanes 0, incremental) are
always among the configurations, so the choice is never slower than them on the sample.

    python -m scout_b200.autotune --out scout_b200/tuned.json
"""
from __future__ import annotations

import argparse
import itertools
import json
import time

import numpy as np

from . import engine as E
from ._lib import STREAM_PREFERENTIAL

BLOCKS = (1, 2, 4)
CHUNKS = (8, 10, 12)
LANES = (0, 32, 64, 128, 256, 1024)
CAPS = (1 << 16, 1 << 18, 1 << 20, 1 << 22)
DEFAULT = {"blocks_per_sm": 4, "chunk_log2": 10, "lanes_per_vertex": 0, "mode": 0, "frontier": 0}
# plain repair variants: (mode, frontier); SCOUT_MODE_RECOMPUTE = 2, QUEUE = 1, BITMAP = 2
VARIANTS = {"bfs": ((0, 0), (2, 1), (2, 2)), "cc": ((0, 0), (2, 0))}


def _device_ms(st: dict) -> float:
    return st["ms_compact"] + st["ms_update"] + st["ms_repair"]


def run_config(problem, off, adj, init, batches, sched: dict, device: int = 0, model=None):
    """(device ms over batches[1:], crc32 of the final solution) of one configuration."""
    import zlib
    sd = dict(sched)
    if model is not None:
        sd["policy"] = 1
    with E.Context(device) as ctx:
        ctx.load_csr(off, adj)
        ctx.upload(problem, init)
        if model is not None:
            ctx.sched_install(problem, model)
        ctx.reserve_batches(max(len(b) for b in batches))
        ctx.repair(problem, batches[0], sched=sd)
        ms = sum(_device_ms(ctx.repair(problem, b, sched=sd)) for b in batches[1:])
        crc = zlib.crc32(np.ascontiguousarray(ctx.download(problem)).tobytes())
    return ms, crc


def tune_single(problem, off, adj, init, batches, device: int = 0, blocks=BLOCKS, chunks=CHUNKS, lanes=LANES,
                model=None, variants: bool = True) -> dict:
    """Sweeps blocks_per_sm x chunk_log2 (chunk only matters for BFS), then at the best of
    those lanes_per_vertex (BFS) and the plain repair variant (BFS, CC) on one stream."""
    chunks = chunks if problem == "bfs" else (10,)
    table = []

    def run(cfg):
        ms, crc = run_config(problem, off, adj, init, batches, cfg, device, model)
        row = dict(cfg, device_ms=ms, solution_crc=crc)
        table.append(row)
        return row

    run(dict(DEFAULT))
    for bps, ch in itertools.product(blocks, chunks):
        cfg = dict(DEFAULT, blocks_per_sm=bps, chunk_log2=ch)
        if cfg != DEFAULT:
            run(cfg)
    best = dict(min(table, key=lambda r: r["device_ms"]))
    if problem == "bfs":
        base = {k: best[k] for k in DEFAULT}
        for lv in lanes:
            cfg = dict(base, lanes_per_vertex=lv)
            if cfg != base:
                run(cfg)
        best = dict(min(table, key=lambda r: r["device_ms"]))
    if variants and problem in VARIANTS and model is None:
        base = {k: best[k] for k in DEFAULT}
        for mode, fr in VARIANTS[problem]:
            cfg = dict(base, mode=mode, frontier=fr)
            if cfg != base:
                run(cfg)
        best = dict(min(table, key=lambda r: r["device_ms"]))
    crcs = {r["solution_crc"] for r in table}
    if len(crcs) != 1:
        raise RuntimeError(f"{problem}: launch knobs changed the solution ({len(crcs)} different results)")
    return {"problem": problem, "best": {k: best[k] for k in DEFAULT}, "table": table}


def tune_rounds(problem, streams, arrivals, device: int = 0, caps=CAPS, sched=None, p99_ms: float = 8.0) -> dict:
    """Sweeps the multi-stream round cap. streams: [(off, adj, init)], arrivals:
    [(stream index, edges)] in arrival order. Every batch waits for its whole round, so its
    latency is the host wall time of its round's synchronous calls. The choice is the cap with
    the least total wall time among those whose p99 batch latency stays within p99_ms (the
    smallest cap when none does): larger rounds amortise the per-round cost, smaller ones bound
    how long a small batch waits behind large ones."""
    table = []
    for cap in caps:
        with E.MultiEngine(problem, device) as me:
            for off, adj, init in streams:
                me.add_stream(off, adj, init, 0)
            me.seal()
            me.reserve_batches(max(cap, max(len(b) for _, b in arrivals)))
            rounds = E.form_rounds(arrivals, cap)
            lat = []
            t0 = time.perf_counter()
            dev = 0.0
            for rd in rounds:
                t1 = time.perf_counter()
                dev += _device_ms(me.round(rd, sched=sched))
                lat += [1e3 * (time.perf_counter() - t1)] * len(rd)
            wall = 1e3 * (time.perf_counter() - t0)
        table.append({"round_cap": cap, "rounds": len(rounds), "device_ms": dev, "wall_ms": wall,
                      "p99_batch_ms": float(np.percentile(lat, 99))})
    return {"problem": problem, "p99_bound_ms": p99_ms, "best": {"round_cap": choose_round_cap(table, p99_ms)},
            "table": table}


def choose_round_cap(table, p99_ms: float, slack: float = 0.05) -> int:
    """Among the caps whose p99 batch latency stays within p99_ms, the smallest one whose total
    wall time is within `slack` of the fastest (bigger rounds that barely raise throughput only
    add latency); the smallest cap when none meets the bound."""
    ok = [r for r in table if r["p99_batch_ms"] <= p99_ms]
    if not ok:
        return min(r["round_cap"] for r in table)
    fastest = min(r["wall_ms"] for r in ok)
    return min(r["round_cap"] for r in ok if r["wall_ms"] <= (1 + slack) * fastest)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--out", default="")
    ap.add_argument("--scale", type=int, default=22)
    ap.add_argument("--device", type=int, default=0)
    ap.add_argument("--p99-ms", type=float, default=8.0, help="latency bound of the multi-stream round cap")
    a = ap.parse_args()
    g = E.gen_rmat(a.scale, 16, seed=2)
    off, adj = g.arrays()
    sizes = [10_000, 100_000, 1_000_000, 10_000, 100_000, 1_000_000, 10_000]
    s = g.stream(STREAM_PREFERENTIAL, sum(sizes), 1, insert_ratio=0.5, seed=77)
    b = np.cumsum([0] + sizes)
    batches = [np.ascontiguousarray(s[b[i]:b[i + 1]]) for i in range(len(sizes))]
    report = {"workload": f"R-MAT scale {a.scale} EF16 seed 2, preferential 50/50 batches {sizes}"}
    for p in ("bfs", "coloring", "cc", "mis"):
        r = tune_single(p, off, adj, g.init_state(p, 0), batches, a.device)
        report[p] = r
        print(json.dumps(r), flush=True)
    small = [E.gen_rmat(sc, 16, seed=60 + sc) for sc in (12, 14, 16, 18)]
    streams = [(h.arrays()[0], h.arrays()[1], h.init_state("bfs", 0)) for h in small for _ in range(4)]
    rng = np.random.default_rng(5)
    arrivals = []
    for j in range(6):
        for i in rng.permutation(len(streams)):
            h = small[i // 4]
            m = int(min(h.nnz // 4, round(10 ** rng.uniform(2, 5))))
            arrivals.append((int(i), h.stream(STREAM_PREFERENTIAL, m, 1, insert_ratio=0.5, seed=1000 * j + int(i))))
    report["rounds"] = tune_rounds("bfs", streams, arrivals, a.device, p99_ms=a.p99_ms)
    print(json.dumps(report["rounds"]), flush=True)
    tuned = {p: report[p]["best"] for p in ("bfs", "coloring", "cc", "mis")}
    tuned["round_cap"] = report["rounds"]["best"]["round_cap"]
    tuned["report"] = report
    if a.out:
        with open(a.out, "w") as f:
            json.dump(tuned, f, indent=1)


if __name__ == "__main__":
    main()
