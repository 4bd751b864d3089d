#!/usr/bin/env python3
"""Edge-updates/s of the B200 dynamic-graph repair engine.

Workload (one step = one batch of toggled edges through the hot path): an R-MAT graph of
scale 22 (4,194,304 vertices, edge factor 16, a/b/c/d = .57/.19/.19/.05, symmetrised, no
self-loops or duplicates, ~128M directed entries, 0.5 GB of adjacency: larger than the 126 MB
L2), initial BFS levels from vertex 0 and a greedy smallest-free colouring; batches of
10^4, 10^5 and 10^6 toggles whose endpoints are drawn proportional to degree, half
deletions of existing edges and half insertions of non-edges. Seeded synthetic data.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl scout|reference]

value  edge-updates/s with the edits already in HBM: classification + merge into the rows +
       repair, from the library's CUDA events on its own stream.
e2e    the same through the public C ABI with host buffers: each step copies the edits from
       page-locked host memory, repairs and copies the changed solution entries back into a
       host mirror (scout_repair + scout_commit), timed with CUDA events around the step loop.
Multi-GPU (torchrun): every rank runs an independent replica stream (no collective on the
data path), value = all ranks' updates / max over ranks of the elapsed time.
"""
from __future__ import annotations

import argparse
import json
import os
import re
import shutil
import statistics
import subprocess
import sys
import tempfile
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

SIZES = (10_000, 100_000, 1_000_000)
METRIC = "edge-updates/sec per problem"


def parse_args():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=12)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="scout", choices=["scout", "reference"])
    ap.add_argument("--scale", type=int, default=22)
    ap.add_argument("--problems", default="bfs,coloring")
    ap.add_argument("--seed", type=int, default=2)
    ap.add_argument("--cpu-seconds", type=float, default=15.0)
    ap.add_argument("--ref-timeout", type=float, default=1500.0,
                    help="seconds the reference programs may run in total (reference arm)")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--verbose", action="store_true", help="per-batch statistics on stderr")
    ap.add_argument("--model", default=os.path.join(ROOT, "scout_b200", "sched_model.npz"),
                    help="trained scheduler model (BFS/CC); the plain policy runs without it")
    ap.add_argument("--tuned", default=os.path.join(ROOT, "scout_b200", "tuned.json"),
                    help="autotuned launch knobs (python -m scout_b200.autotune); defaults without it")
    ap.add_argument("--no-multi", action="store_true", help="skip the multi-stream section")
    ap.add_argument("--multi-batches", type=int, default=6, help="batches per stream in the multi-stream section")
    ap.add_argument("--no-ooc", action="store_true", help="skip the out-of-core section")
    ap.add_argument("--ooc-scale", type=int, default=23)
    ap.add_argument("--ooc-batches", type=int, default=5)
    ap.add_argument("--ooc-edits", type=int, default=100_000)
    return ap.parse_args()


# ---------------------------------------------------------------------------------------
# distributed plumbing (replicas only)
# ---------------------------------------------------------------------------------------
class Dist:
    """Replica plumbing: one process per GPU, no collective on the data path. The process
    group only carries the start/stop barriers and the two scalar reductions of the result
    (NCCL with CUDA, gloo without, as in the CPU tests)."""

    def __init__(self, backend: str | None = None):
        self.rank = int(os.environ.get("RANK", 0))
        self.world = int(os.environ.get("WORLD_SIZE", 1))
        self.local = int(os.environ.get("LOCAL_RANK", 0))
        self.pg = None
        self.backend = backend
        if self.world > 1:
            import datetime

            import torch
            import torch.distributed as dist
            if self.backend is None:
                self.backend = "nccl" if torch.cuda.is_available() else "gloo"
            dist.init_process_group(self.backend, timeout=datetime.timedelta(seconds=120))
            self.pg = dist

    def _dev(self):
        return f"cuda:{self.local}" if self.backend == "nccl" else "cpu"

    def barrier(self):
        if self.pg:
            import torch
            t = torch.zeros(1, device=self._dev())
            self.pg.all_reduce(t)
            if self.backend == "nccl":
                torch.cuda.synchronize(self.local)

    def reduce(self, x: float, op: str) -> float:
        if not self.pg:
            return x
        import torch
        t = torch.tensor([x], dtype=torch.float64, device=self._dev())
        self.pg.all_reduce(t, op=self.pg.ReduceOp.MAX if op == "max" else self.pg.ReduceOp.SUM)
        return float(t.item())

    def close(self):
        if self.pg:
            self.pg.destroy_process_group()
            self.pg = None


# ---------------------------------------------------------------------------------------
# workload
# ---------------------------------------------------------------------------------------
def batch_sizes(steps: int, warmup: int):
    return [SIZES[i % len(SIZES)] for i in range(warmup + steps)]


def workload_config(a, n: int, nnz: int, sizes, problems, world: int) -> dict:
    """The `config` object of both arms' lines (identical for the same arguments)."""
    return {"workload": f"R-MAT scale {a.scale} EF16 (.57/.19/.19/.05) seed {a.seed}; "
                        f"preferential 50/50 toggles; batch sizes {list(SIZES)} cycled; problems {problems}",
            "vertices": n, "directed_entries": nnz, "graph_bytes": 4 * nnz + 8 * n,
            "l2": "inputs larger than L2 (0.5 GB adjacency vs 126 MB L2); no flush",
            "parallelism": f"replicas x{world}", "batch_sizes": list(sizes[a.warmup:])}


def per_size_rates(edits, ms, sizes) -> dict:
    """edge-updates/s per batch size, from per-batch (edits, ms) of the timed batches."""
    out = {}
    for z in sorted(set(sizes)):
        e = sum(x for x, s_ in zip(edits, sizes) if s_ == z)
        t = sum(x for x, s_ in zip(ms, sizes) if s_ == z)
        if t > 0:
            out[str(z)] = e / (t / 1e3)
    return out


def make_workload(scale: int, seed: int, stream_seed: int, sizes):
    import scout_b200 as sb
    g = sb.gen_rmat(scale, 16, seed=seed)
    off, adj = g.arrays()
    total = sum(sizes)
    s = g.stream(sb.STREAM_PREFERENTIAL, total, 1, insert_ratio=0.5, seed=stream_seed)
    bounds = np.cumsum([0] + list(sizes))
    batches = [np.ascontiguousarray(s[bounds[i]:bounds[i + 1]]) for i in range(len(sizes))]
    init = {"bfs": g.init_state("bfs", 0), "coloring": g.init_state("coloring"), "cc": g.init_state("cc"),
            "mis": g.init_state("mis")}
    return g, off, adj, batches, init


class Clocks:
    """SM clock and throttle-reason sampling during the timed loops only.

    The timed region lasts tens of milliseconds, shorter than nvidia-smi's 200 ms loop, so the
    clocks are polled through NVML every 5 ms from a thread while a timed loop runs (the same
    counters nvidia-smi reports: clocks.sm, clocks.max.sm, clocks_event_reasons.*)."""

    REASONS = {"hw_slowdown": 0x8, "sw_thermal_slowdown": 0x20, "hw_thermal_slowdown": 0x40,
               "sw_power_cap": 0x4}

    def __init__(self, gpu: int):
        self.gpu = gpu
        self.samples = []
        self.reasons = 0
        self._stop = threading.Event()
        self._t = None
        self.h = None
        self.max_mhz = None
        try:
            import pynvml
            pynvml.nvmlInit()
            self.nv = pynvml
            self.h = pynvml.nvmlDeviceGetHandleByIndex(gpu)
            self.max_mhz = float(pynvml.nvmlDeviceGetMaxClockInfo(self.h, pynvml.NVML_CLOCK_SM))
        except Exception:
            self.h = None

    def _run(self):
        while not self._stop.is_set():
            try:
                self.samples.append(float(self.nv.nvmlDeviceGetClockInfo(self.h, self.nv.NVML_CLOCK_SM)))
                self.reasons |= int(self.nv.nvmlDeviceGetCurrentClocksEventReasons(self.h))
            except Exception:
                pass
            self._stop.wait(0.005)

    def start(self):
        if self.h is not None:
            self._stop.clear()
            self._t = threading.Thread(target=self._run, daemon=True)
            self._t.start()

    def stop(self):
        if self._t:
            self._stop.set()
            self._t.join()
            self._t = None

    def summary(self) -> dict:
        if not self.samples:
            return {"sm_mhz": None, "sm_max_mhz": self.max_mhz, "reasons": ["unsampled"], "samples": 0}
        return {"sm_mhz": statistics.median(self.samples), "sm_max_mhz": self.max_mhz,
                "sm_mhz_min": min(self.samples), "sm_mhz_max": max(self.samples),
                "reasons": sorted(k for k, bit in self.REASONS.items() if self.reasons & bit),
                "samples": len(self.samples), "source": "NVML, 5 ms polling inside the timed loops"}


def profiled_traffic(kernel: str, scale: int):
    """DRAM bytes per launch (dram__bytes_read.sum + dram__bytes_write.sum) of `kernel` on this
    workload, from the committed ncu summary profiles/roofline_traffic.txt (lines:
    kernel scale bytes_per_launch), or None when it holds no capture of that kernel and scale."""
    p = os.path.join(ROOT, "profiles", "roofline_traffic.txt")
    if not os.path.exists(p):
        return None
    for line in open(p):
        f = line.split()
        if len(f) >= 3 and not line.startswith("#") and f[0] == kernel and f[1] == str(scale):
            return float(f[2])
    return None


def measured_peak():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        d = json.load(open(p))
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


# ---------------------------------------------------------------------------------------
# scout arm
# ---------------------------------------------------------------------------------------
def load_model(path):
    """Trained scheduler parameters per problem ({"bfs": 6020 floats, "cc": ...}), or {}."""
    if not path or not os.path.exists(path):
        return {}
    d = np.load(path, allow_pickle=False)
    return {k: np.asarray(d[k], dtype=np.float32) for k in ("bfs", "cc") if k in d.files}


LAUNCH_KNOBS = ("blocks_per_sm", "chunk_log2", "lanes_per_vertex")


def launch_knobs(knobs: dict) -> dict:
    """The launch knobs of a tuned set, without its plain repair variant (mode, frontier): that
    choice was tuned on one stream of the headline workload; union rounds and tiered batches
    leave the variant to the plain default or the learned scheduler."""
    return {k: v for k, v in (knobs or {}).items() if k in LAUNCH_KNOBS}


def load_tuned(path):
    """Autotuned knobs: {problem: {"blocks_per_sm", "chunk_log2"}, "round_cap": int}, or {}."""
    if not path or not os.path.exists(path):
        return {}
    with open(path) as f:
        d = json.load(f)
    d.pop("report", None)
    return d


def run_problem(problem, off, adj, init, batches, warmup, steps, device, dist, clocks, verbose=False, model=None,
                tune=None):
    import torch

    import scout_b200 as sb
    ctx = sb.Context(device)
    ctx.load_csr(off, adj)
    ctx.upload(problem, init)
    sched = dict(tune or {})
    if model is not None:
        ctx.sched_install(problem, model)
        sched["policy"] = 1
    ctx.reserve_batches(max(len(b) for b in batches))   # no allocation inside the timed loop
    mirror = init.copy()
    # each step's edits are read from page-locked host memory (copied there before timing); the
    # next step's edits are hinted (prefetch) so that their host-to-device copy overlaps this
    # step's repair, as a stream consumer that knows its next batch does
    batches = [sb.pinned_copy(b) for b in batches[:warmup + steps]]
    nb = len(batches)
    for i, b in enumerate(batches[:warmup]):
        if i + 1 < nb:
            ctx.prefetch(batches[i + 1])
        ctx.repair(problem, b, sched=sched)
        ctx.commit(problem, mirror)
    timed = batches[warmup:warmup + steps]
    per = []
    torch.cuda.set_device(device)
    dist.barrier()
    torch.cuda.synchronize(device)
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    clocks.start()
    ev0.record()
    for i, b in enumerate(timed):
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record()
        if i + 1 < len(timed):
            ctx.prefetch(timed[i + 1])
        st = ctx.repair(problem, b, sched=sched)
        changed = ctx.commit(problem, mirror)
        e1.record()
        st["commit_changed"] = changed
        st["_ev"] = (e0, e1)
        per.append(st)
    ev1.record()
    torch.cuda.synchronize(device)
    clocks.stop()
    dist.barrier()
    e2e_ms = ev0.elapsed_time(ev1)
    for st in per:
        e0, e1 = st.pop("_ev")
        st["ms_step"] = e0.elapsed_time(e1)
        if verbose:
            keep = ("edits", "ms_step", "ms_h2d", "ms_update", "ms_repair", "rounds", "changed", "launches", "variant",
                    "hbm_bytes", "update_bytes")
            d = {k: (round(st[k], 3) if isinstance(st[k], float) else st[k]) for k in keep}
            d["phase_ms"] = [round(x, 3) for x in st["phase_ms"]]
            print(problem, json.dumps(d), file=sys.stderr, flush=True)
    ctx.close()
    return per, e2e_ms


def cpu_baseline(problems, off, adj, init, batches, seconds):
    """The oracle (single-thread CPU restatement of the reference engine) on a bounded sample:
    the same stream's batches in order, about seconds / len(problems) per problem."""
    from oracle import oracle as orc
    edits = 0
    t_used = 0.0
    parts = []
    for p in problems:
        eng = orc.Engine(p, off, adj, init[p])
        t_p = 0.0
        k = e_p = 0
        for b in batches:
            if t_p >= seconds / len(problems):
                break
            t0 = time.perf_counter()
            eng.batch(b)
            t_p += time.perf_counter() - t0
            e_p += len(b)
            k += 1
        parts.append(f"{p}: first {k} batches ({e_p} toggles) in {t_p:.1f} s")
        edits += e_p
        t_used += t_p
    return {"value": edits / t_used if t_used else None, "unit": "edge-updates/s", "cores": 1, "kind": "port",
            "sample": "oracle restatement of the reference engine, single-threaded, on the same stream; "
                      + "; ".join(parts)}


def cpu_recompute_baseline(problems, off, adj, batches, warmup, seconds):
    """All-core from-scratch recompute on the host (oracle/cpu_recompute.cpp, OpenMP): the
    oracle's graph follows the stream with the toggle rule, and after each timed batch of the
    sample every problem's solution is recomputed from scratch (parallel BFS, CAS union-find;
    greedy colouring and MIS are sequential by definition). edge-updates/s = the sample's edits
    per problem / the recompute seconds (the graph updates themselves are not charged)."""
    from oracle import oracle as orc
    g = orc.Graph(off, adj)
    for b in batches[:warmup]:
        g.toggle_batch(b)
    per = {p: [0, 0.0] for p in problems}
    t0 = time.perf_counter()
    k = 0
    for b in batches[warmup:]:
        if time.perf_counter() - t0 > seconds and k >= 1:
            break
        g.toggle_batch(b)
        o, a_ = g.csr()
        for p in problems:
            _, t = orc.cpu_recompute(p, o, a_, 0)
            per[p][0] += len(b)
            per[p][1] += t
        k += 1
    edits = sum(v[0] for v in per.values())
    secs = sum(v[1] for v in per.values())
    return {"value": edits / secs if secs else None, "unit": "edge-updates/s", "cores": orc.cpu_threads(),
            "kind": "from-scratch recompute",
            "per_problem": {p: (v[0] / v[1] if v[1] else None) for p, v in per.items()},
            "sample": f"the first {k} timed batches of the same stream ({per[problems[0]][0]} toggles), each "
                      f"followed by a from-scratch recompute of {problems} on {orc.cpu_threads()} threads"}


def scout_arm(a, dist):
    import scout_b200 as sb
    sizes = batch_sizes(a.steps, a.warmup)
    g, off, adj, batches, init = make_workload(a.scale, a.seed, 1000 + a.seed + dist.rank, sizes)
    problems = [p.strip() for p in a.problems.split(",") if p.strip()]
    device = dist.local
    results = {}
    plain = {}
    model = load_model(a.model)
    tuned = load_tuned(a.tuned)
    clocks = Clocks(device)
    for p in problems:
        # the engine as deployed: the learned scheduler where a model exists (BFS, CC) and the
        # autotuned knobs, and the plain engine (no scheduler, default knobs) beside it
        results[p] = run_problem(p, off, adj, init[p], batches, a.warmup, a.steps, device, dist, clocks, a.verbose,
                                 model=model.get(p), tune=tuned.get(p))
        if p in model or p in tuned:
            plain[p] = run_problem(p, off, adj, init[p], batches, a.warmup, a.steps, device, dist, clocks, a.verbose)
    clk = clocks.summary()
    peak, peak_kind = measured_peak()
    per_problem = {}
    tot_edits = tot_e2e = tot_dev = 0.0
    all_ms = []
    bytes_rep = bytes_upd = ms_rep = ms_upd = 0.0
    launches = h2d = d2h = 0
    for p, (per, e2e_ms) in results.items():
        edits = sum(s["edits"] for s in per)
        dev_ms = sum(s["ms_compact"] + s["ms_update"] + s["ms_repair"] for s in per)
        per_problem[p] = {"edge_updates_per_s": edits / (dev_ms / 1e3), "e2e_edge_updates_per_s": edits / (e2e_ms / 1e3),
                          "p50_batch_ms": float(np.percentile([s["ms_step"] for s in per], 50)),
                          "p99_batch_ms": float(np.percentile([s["ms_step"] for s in per], 99)),
                          "batches": len(per), "edits": edits,
                          "repair_ms": sum(s["ms_repair"] for s in per), "update_ms": sum(s["ms_update"] for s in per),
                          "compact_ms": sum(s["ms_compact"] for s in per),
                          "h2d_ms": sum(s["ms_h2d"] for s in per), "rounds": sum(s["rounds"] for s in per),
                          "changed": sum(s["commit_changed"] for s in per),
                          "scheduler": "learned" if p in model else "plain", "knobs": tuned.get(p, {}),
                          "variants": [int(s["variant"]) for s in per],
                          "per_size": per_size_rates([s["edits"] for s in per], [s["ms_step"] for s in per],
                                                     sizes[a.warmup:a.warmup + len(per)])}
        if p in plain:
            pp, pe = plain[p]
            pdev = sum(s["ms_compact"] + s["ms_update"] + s["ms_repair"] for s in pp)
            per_problem[p]["plain"] = {"edge_updates_per_s": edits / (pdev / 1e3),
                                       "e2e_edge_updates_per_s": edits / (pe / 1e3),
                                       "repair_ms": sum(s["ms_repair"] for s in pp),
                                       "p99_batch_ms": float(np.percentile([s["ms_step"] for s in pp], 99))}
        tot_edits += edits
        tot_e2e += e2e_ms
        tot_dev += dev_ms
        all_ms += [s["ms_step"] for s in per]
        bytes_rep += sum(s["hbm_bytes"] for s in per)
        bytes_upd += sum(s["update_bytes"] for s in per)
        ms_rep += sum(s["ms_repair"] for s in per)
        ms_upd += sum(s["ms_update"] for s in per)
        launches += sum(s["launches"] for s in per)
        h2d += sum(s["h2d_bytes"] for s in per)
        d2h += sum(s["d2h_bytes"] + 8 * s["commit_changed"] for s in per)
    n_steps = sum(len(r[0]) for r in results.values())
    # whole job over ranks
    edits_all = dist.reduce(tot_edits, "sum")
    dev_s = dist.reduce(tot_dev / 1e3, "max")
    e2e_s = dist.reduce(tot_e2e / 1e3, "max")
    # Roofline of the dominant kernel: the repair kernel (one cooperative launch per batch,
    # k_<problem>) with the largest event-timed total; the launch list of the same workload
    # ranks it first. Achieved = its algorithmic bytes / its event time. The batch-merge
    # pipeline (about fifteen short kernels per batch) is reported beside it.
    rep = {p: (sum(s["hbm_bytes"] for s in per), sum(s["ms_repair"] for s in per), len(per))
           for p, (per, _) in results.items()}
    kp = max(rep, key=lambda p: rep[p][1])
    b, ms, nl = rep[kp]
    achieved = b / (ms / 1e3) / 1e9 if ms else 0.0
    line = {
        "metric": METRIC, "value": edits_all / dev_s if dev_s else None, "unit": "edge-updates/s",
        "n_gpus": dist.world, "steps": a.steps, "warmup": a.warmup,
        "ms_per_step": 1e3 * e2e_s / max(n_steps, 1), "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "int32", "data": "synthetic (seeded R-MAT + preferential toggle stream)",
        "config": workload_config(a, int(g.n), int(g.nnz), sizes, problems, dist.world),
        "p50_batch_ms": float(np.percentile(all_ms, 50)), "p99_batch_ms": float(np.percentile(all_ms, 99)),
        "per_problem": per_problem,
        "e2e": {"value": edits_all / e2e_s if e2e_s else None, "unit": "edge-updates/s",
                "h2d_bytes_per_step": int(h2d / max(n_steps, 1)), "d2h_bytes_per_step": int(d2h / max(n_steps, 1))},
        "roofline": {"bound": "hbm", "kernel": f"k_{kp}", "achieved": achieved, "peak": peak, "unit": "GB/s",
                     "frac": achieved / peak, "peak_kind": peak_kind, "traffic": profiled_traffic(f"k_{kp}", a.scale),
                     "algorithmic_bytes_per_launch": b / max(nl, 1), "ms_per_launch": ms / max(nl, 1),
                     "launches": nl},
        "roofline_merge": {"kernels": "k_classify .. k_merge_slices (batch merge pipeline)",
                           "achieved": bytes_upd / (ms_upd / 1e3) / 1e9 if ms_upd else 0.0,
                           "frac": (bytes_upd / (ms_upd / 1e3) / 1e9) / peak if ms_upd else 0.0,
                           "ms": ms_upd, "bytes": bytes_upd},
        "gpu_launches": int(launches), "clocks": clk,
    }
    if dist.rank == 0 and dist.world == 1 and not a.no_cpu_baseline:
        line["cpu_baseline"] = cpu_baseline(problems, off, adj, init, batches, a.cpu_seconds)
        line["cpu_recompute"] = cpu_recompute_baseline(problems, off, adj, batches, a.warmup, a.cpu_seconds)
    if dist.world == 1 and not a.no_multi:
        del g, off, adj, batches, init
        line["multi_stream"] = multi_stream(a, device, model, tuned)
    if dist.world == 1 and not a.no_ooc:
        line["out_of_core"] = out_of_core(a, device, model, tuned, a.ooc_batches, a.ooc_edits)
    return line


# ---------------------------------------------------------------------------------------
# out-of-core section: a graph 4.3x larger than its HBM pool (the 16 GB / 69 GB ratio)
# ---------------------------------------------------------------------------------------
def h2d_peak_gbs(device: int, mib: int = 1024, reps: int = 5) -> float:
    """Host-to-device copy bandwidth from page-locked memory (the host link's measured peak):
    the best of `reps` copies of `mib` MiB, timed with CUDA events."""
    import torch
    src = torch.empty(mib << 20, dtype=torch.uint8).pin_memory()
    dst = torch.empty(mib << 20, dtype=torch.uint8, device=f"cuda:{device}")
    best = 0.0
    for _ in range(reps + 1):
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        dst.copy_(src, non_blocking=True)
        e1.record()
        torch.cuda.synchronize(device)
        best = max(best, (mib << 20) / (e0.elapsed_time(e1) / 1e3) / 1e9)
    del src, dst
    return best


def out_of_core(a, device, model, tuned, nbatches: int = 6, m: int = 1_000_000):
    """BFS and CC streams of deletion-heavy batches (70% deletions of existing edges, 30% of
    them with a low-degree first endpoint; 30% uniform insertions) on an R-MAT graph of scale
    a.ooc_scale, edge factor 32, whose HBM element pool holds 23% of the adjacency: hot rows
    in HBM, the rest in mapped page-locked host memory. Arms on the tiered store: plain (cold
    rows read in place, plain scheduling), learned (the cost model picks the variant),
    batched (each batch's cold endpoint rows gathered into HBM on a copy stream during the
    previous batch's repair, scout_prefetch) and learned + batched; the all-in-HBM engine on the
    same stream for scale. The gather's bytes over its time, against the measured host-link
    peak, is the host-link roofline."""
    import scout_b200 as sb
    g = sb.gen_rmat(a.ooc_scale, 32, seed=29)
    off, adj = g.arrays()
    nnz = int(g.nnz)
    hbm = int(0.23 * nnz)
    s = g.stream(sb.STREAM_LOWDEG, m, nbatches, insert_ratio=0.3, lowdeg_frac=0.3, seed=2929)
    batches = [sb.pinned_copy(x) for x in s.reshape(nbatches, m, 2)]
    peak = h2d_peak_gbs(device)
    out = {"workload": f"R-MAT scale {a.ooc_scale} EF32 seed 29 ({g.n} vertices, {nnz} directed entries, "
                       f"{4 * nnz / 1e9:.2f} GB adjacency); HBM pool {hbm} entries (23%); {nbatches} batches of "
                       f"{m} toggles: 70% deletions (30% low-degree first endpoint), 30% uniform insertions",
           "vertices": int(g.n), "directed_entries": nnz, "h2d_peak_gbs": peak,
           "h2d_peak": "best of 5 copies of 1 GiB from page-locked host memory, CUDA events"}
    for p in ("bfs", "cc"):
        init = g.init_state(p, 0)
        res = {}
        arms = [("tiered_plain", True, None, False), ("tiered_batched", True, None, True)]
        if p in model:
            arms += [("tiered_learned", True, model[p], False), ("tiered_learned_batched", True, model[p], True)]
        arms.append(("in_hbm_plain", False, None, False))
        for arm, tier, mdl, batched in arms:
            with sb.Context(device) as ctx:
                if tier:
                    ctx.load_tiered(off, adj, hbm_entries=hbm)
                else:
                    ctx.load_csr(off, adj)
                ctx.upload(p, init)
                # the plain arms run the default knobs; the others the autotuned ones
                sched = {} if arm in ("tiered_plain", "in_hbm_plain") else launch_knobs(tuned.get(p, {}))
                if mdl is not None:
                    ctx.sched_install(p, mdl)
                    sched["policy"] = 1
                ctx.reserve_batches(m)
                mirror = init.copy()
                dev = wall = 0.0
                lat, variants = [], []
                g_bytes = g_ms = 0.0
                g_rows = 0
                for k, b in enumerate(batches):
                    t0 = time.perf_counter()
                    if batched and k + 1 < len(batches):
                        ctx.prefetch(batches[k + 1])
                    st = ctx.repair(p, b, sched=sched)
                    ctx.commit(p, mirror)
                    dt = 1e3 * (time.perf_counter() - t0)
                    wall += dt
                    lat.append(dt)
                    dev += st["ms_compact"] + st["ms_update"] + st["ms_repair"]
                    variants.append(int(st["variant"]))
                    g_bytes += st["gather_bytes"]
                    g_ms += st["ms_gather"]
                    g_rows += st["gather_rows"]
                    if a.verbose:
                        print(f"out_of_core {p} {arm}: wall {dt:.1f} ms, update {st['ms_update']:.1f}, repair "
                              f"{st['ms_repair']:.1f}, compact {st['ms_compact']:.1f}, gather {st['ms_gather']:.1f} ms "
                              f"({st['gather_rows']} rows), variant {st['variant']}, tiers {ctx.tier_info()}",
                              file=sys.stderr, flush=True)
                info = ctx.tier_info()
            edits = nbatches * m
            r = {"edge_updates_per_s": edits / (dev / 1e3), "e2e_edge_updates_per_s": edits / (wall / 1e3),
                 "p50_batch_ms": float(np.percentile(lat, 50)), "p99_batch_ms": float(np.percentile(lat, 99)),
                 "variants": variants, "hbm_used": info["hbm_used"], "host_used": info["host_used"],
                 "evicted": info["evicted"]}
            if batched:
                gbs = g_bytes / (g_ms / 1e3) / 1e9 if g_ms else 0.0
                r["gather"] = {"rows": g_rows, "bytes": g_bytes, "ms": g_ms, "achieved_gbs": gbs,
                               "frac_of_h2d_peak": gbs / peak if peak else None}
            res[arm] = r
        base = res["tiered_plain"]["e2e_edge_updates_per_s"]
        for r in res.values():
            r["e2e_vs_tiered_plain"] = r["e2e_edge_updates_per_s"] / base
        out[p] = res
    return out


# ---------------------------------------------------------------------------------------
# multi-stream section: 64 independent streams over the four problems and 8 graphs
# ---------------------------------------------------------------------------------------
MULTI_GRAPHS = [(14, 8), (15, 16), (16, 32), (17, 8), (18, 16), (19, 32), (20, 8), (22, 16)]
MULTI_PROBLEMS = ("bfs", "cc", "coloring", "mis")


def multi_workload(nbatches: int, seed: int = 7):
    """64 streams: stream i serves problem i % 4 on graph (i // 4) % 8 (scales 14-22, edge
    factors 8-32, seeded); each has `nbatches` preferential 50/50 toggle batches whose sizes
    are log-uniform in [100, 10^6], capped at a quarter of the graph's directed entries (and
    scaled down where a stream would delete more edges than its graph has). The
    arrival order interleaves the streams at random (seeded), each stream in its own order."""
    import scout_b200 as sb
    from scout_b200.learn import fit_sizes
    rng = np.random.default_rng(seed)
    graphs = []
    for gi, (sc, ef) in enumerate(MULTI_GRAPHS):
        g = sb.gen_rmat(sc, ef, seed=50 + gi)
        graphs.append(g)
    streams = []
    for i in range(64):
        p = MULTI_PROBLEMS[i % 4]
        gi = (i // 4) % 8
        g = graphs[gi]
        cap = max(100, g.nnz // 4)
        sizes = fit_sizes([int(min(cap, round(10 ** rng.uniform(2, 6)))) for _ in range(nbatches)], g.nnz, 0.5)
        s = g.stream(sb.STREAM_PREFERENTIAL, sum(sizes), 1, insert_ratio=0.5, seed=9000 + i)
        b = np.cumsum([0] + sizes)
        streams.append({"problem": p, "graph": gi, "batches": [np.ascontiguousarray(s[b[j]:b[j + 1]])
                                                                for j in range(nbatches)]})
    order = np.repeat(np.arange(64), nbatches)
    rng.shuffle(order)
    nxt = [0] * 64
    arrivals = []
    for i in order.tolist():
        arrivals.append((i, nxt[i]))
        nxt[i] += 1
    return graphs, streams, arrivals


def multi_stream(a, device, model, tuned):
    """Plain (one context per stream, batches one at a time in arrival order), batched (one
    union store per problem, rounds), learned+batched (the same with the scheduler model) and
    fused (the four union stores at once, one repair launch per round across problems) on the
    same 64-stream workload. Times: device CUDA events of the library per batch or round
    (edits already copied), and host wall time of the synchronous calls (copies in, commit out)."""
    import scout_b200 as sb
    graphs, streams, arrivals = multi_workload(a.multi_batches)
    arrays = [g.arrays() for g in graphs]
    inits = {}
    for st in streams:
        key = (st["problem"], st["graph"])
        if key not in inits:
            inits[key] = graphs[st["graph"]].init_state(st["problem"], 0)
    total_edits = sum(len(st["batches"][j]) for st in streams for j in range(len(st["batches"])))
    out = {"workload": "64 streams (16 per problem: bfs, cc, coloring, mis) over 8 R-MAT graphs "
                       f"{MULTI_GRAPHS} (scale, edge factor); {a.multi_batches} preferential 50/50 batches per "
                       "stream, sizes log-uniform in [100, 1e6] capped at nnz/4; seeded random interleaving",
           "batches": len(arrivals), "edits": int(total_edits)}
    arms = {"plain": None, "batched": None}
    if model:
        arms["learned_batched"] = model
    res = {k: {"dev_ms": 0.0, "wall_ms": 0.0, "lat": [], "rounds": 0} for k in arms}
    for p in MULTI_PROBLEMS:
        sids = [i for i, st in enumerate(streams) if st["problem"] == p]
        arr_p = [(i, j) for i, j in arrivals if streams[i]["problem"] == p]
        # plain: a context per stream
        ctxs, mirrors = {}, {}
        for i in sids:
            off, adj = arrays[streams[i]["graph"]]
            c = sb.Context(device)
            c.load_csr(off, adj)
            c.upload(p, inits[(p, streams[i]["graph"])])
            c.reserve_batches(max(len(b) for b in streams[i]["batches"]))
            ctxs[i] = c
            mirrors[i] = inits[(p, streams[i]["graph"])].copy()
        pinned = {(i, j): sb.pinned_copy(streams[i]["batches"][j]) for i, j in arr_p}
        t0 = time.perf_counter()
        for i, j in arr_p:
            t1 = time.perf_counter()
            st = ctxs[i].repair(p, pinned[(i, j)])
            ctxs[i].commit(p, mirrors[i])
            res["plain"]["lat"].append(1e3 * (time.perf_counter() - t1))
            res["plain"]["dev_ms"] += st["ms_compact"] + st["ms_update"] + st["ms_repair"]
        res["plain"]["wall_ms"] += 1e3 * (time.perf_counter() - t0)
        res["plain"]["rounds"] += len(arr_p)
        for c in ctxs.values():
            c.close()
        # batched (and learned + batched): one union store per problem, rounds of many streams
        for arm, mdl in arms.items():
            if arm == "plain":
                continue
            me = sb.MultiEngine(p, device)
            local = {}
            for i in sids:
                off, adj = arrays[streams[i]["graph"]]
                local[i] = me.add_stream(off, adj, inits[(p, streams[i]["graph"])], 0)
            me.seal()
            cap = int(tuned.get("round_cap", 1 << 21))
            me.reserve_batches(max(cap, max(len(pinned[(i, j)]) for i, j in arr_p)))
            sched = launch_knobs(tuned.get(p, {}))
            if mdl is not None and p in mdl:
                me.context.sched_install(p, mdl[p])
                sched["policy"] = 1
            mir = [inits[(p, streams[i]["graph"])].copy() for i in sids]
            rounds = sb.form_rounds([(local[i], pinned[(i, j)]) for i, j in arr_p], cap)
            t0 = time.perf_counter()
            for rd in rounds:
                t1 = time.perf_counter()
                st = me.round(rd, sched=sched)
                me.commit(mir)
                dt = 1e3 * (time.perf_counter() - t1)
                res[arm]["lat"] += [dt] * len(rd)
                res[arm]["dev_ms"] += st["ms_compact"] + st["ms_update"] + st["ms_repair"]
            res[arm]["wall_ms"] += 1e3 * (time.perf_counter() - t0)
            res[arm]["rounds"] += len(rounds)
            me.close()
    # fused: the four union stores at once; a round's four merges, then ONE persistent kernel
    # running the four repairs (scout_multi_run_all), the rounds of each problem as above
    res["fused"] = {"dev_ms": 0.0, "wall_ms": 0.0, "lat": [], "rounds": 0}
    engines, mirs, rounds_p, pinned_all = {}, {}, {}, {}
    cap = int(tuned.get("round_cap", 1 << 21))
    sched = launch_knobs(tuned.get("bfs", {}))
    for p in MULTI_PROBLEMS:
        sids = [i for i, st in enumerate(streams) if st["problem"] == p]
        arr_p = [(i, j) for i, j in arrivals if streams[i]["problem"] == p]
        me = sb.MultiEngine(p, device, budget_bytes=36 << 30)   # four stores side by side
        local = {}
        for i in sids:
            off, adj = arrays[streams[i]["graph"]]
            local[i] = me.add_stream(off, adj, inits[(p, streams[i]["graph"])], 0)
        me.seal()
        pinned_all[p] = {(i, j): sb.pinned_copy(streams[i]["batches"][j]) for i, j in arr_p}
        me.reserve_batches(max(cap, max(len(b) for b in pinned_all[p].values())))
        engines[p] = me
        mirs[p] = [inits[(p, streams[i]["graph"])].copy() for i in sids]
        rounds_p[p] = sb.form_rounds([(local[i], pinned_all[p][(i, j)]) for i, j in arr_p], cap)
    nr = max(len(r) for r in rounds_p.values())
    t0 = time.perf_counter()
    for r in range(nr):
        members = [p for p in MULTI_PROBLEMS if r < len(rounds_p[p])]
        t1 = time.perf_counter()
        for p in members:
            engines[p].stage(rounds_p[p][r])
        sts = sb.run_fused_round([engines[p] for p in members], sched=sched)
        for p in members:
            engines[p].commit(mirs[p])
        dt = 1e3 * (time.perf_counter() - t1)
        res["fused"]["lat"] += [dt] * sum(len(rounds_p[p][r]) for p in members)
        res["fused"]["dev_ms"] += sum(x["ms_compact"] + x["ms_update"] for x in sts) + sts[0]["ms_repair"]
    res["fused"]["wall_ms"] = 1e3 * (time.perf_counter() - t0)
    res["fused"]["rounds"] = nr
    for me in engines.values():
        me.close()
    arms["fused"] = None
    for arm, r in res.items():
        out[arm] = {"edge_updates_per_s": total_edits / (r["dev_ms"] / 1e3),
                    "e2e_edge_updates_per_s": total_edits / (r["wall_ms"] / 1e3),
                    "p50_batch_ms": float(np.percentile(r["lat"], 50)),
                    "p99_batch_ms": float(np.percentile(r["lat"], 99)),
                    ("repair_launches" if arm == "fused" else "launch_rounds"): r["rounds"]}
    base = out["plain"]["e2e_edge_updates_per_s"]
    for arm in arms:
        out[arm]["e2e_vs_plain"] = out[arm]["e2e_edge_updates_per_s"] / base
    return out


# ---------------------------------------------------------------------------------------
# reference arm: the reference's own programs (oracle/_ref, compiled from its sources)
# ---------------------------------------------------------------------------------------
BATCH_RE = re.compile(r"^Batch (\d+)/(\d+) \| edges=(\d+) \| time=([0-9.]+)ms(.*)$")
FALLBACK_RE = re.compile(r"fallback=(\d+)")
DEFERRED_RE = re.compile(r"^\[DEFERRED FALLBACK\] done in ([0-9.]+) ms")


def reference_workload(a, sizes):
    """The scout arm's workload rebuilt without this package's library: the numpy
    restatement of the generator (byte-identical, tests/test_gen_oracle.py) and the oracle's
    initial-state solvers (BFS from vertex 0, greedy smallest-free colouring in id order,
    min-id components, greedy MIS in id order)."""
    from oracle import gen_oracle as go
    from oracle import oracle as orc
    off, adj = go.gen_rmat(a.scale, 16, seed=a.seed)
    s = go.gen_stream(off, adj, go.STREAM_PREFERENTIAL, sum(sizes), 0.5, seed=1000 + a.seed)
    bounds = np.cumsum([0] + list(sizes))
    batches = [s[bounds[i]:bounds[i + 1]] for i in range(len(sizes))]
    init = {"bfs": lambda: orc.gt_bfs(off, adj, 0), "coloring": lambda: orc.gt_greedy_color(off, adj),
            "cc": lambda: orc.gt_cc(off, adj), "mis": lambda: orc.gt_greedy_mis(off, adj)}
    return off, adj, batches, init


def run_reference_program(path, egr, state, bdir, nb, gpu, timeout, cwd):
    """Runs one reference binary over the batch folder; returns (per-batch rows, deferred
    catch-up ms, complete, wall seconds). A row is (batch, edits, ms, fallback count)."""
    cmd = [path, egr, state, bdir, str(nb), str(gpu)]
    env = dict(os.environ, SCOUT_SKIP_COMPACTION="1")
    t0 = time.perf_counter()
    complete = True
    try:
        r = subprocess.run(cmd, capture_output=True, text=True, timeout=timeout, env=env, cwd=cwd)
        out = r.stdout
        complete = r.returncode == 0
    except subprocess.TimeoutExpired as e:
        out = e.stdout.decode() if isinstance(e.stdout, bytes) else (e.stdout or "")
        complete = False
    wall = time.perf_counter() - t0
    rows, deferred = [], 0.0
    for line in out.splitlines():
        m = BATCH_RE.match(line)
        if m:
            fb = FALLBACK_RE.search(m.group(5))
            rows.append((int(m.group(1)), int(m.group(3)), float(m.group(4)), int(fb.group(1)) if fb else 0))
            continue
        d = DEFERRED_RE.match(line)
        if d:
            deferred += float(d.group(1))
    complete = complete and len(rows) == nb
    return rows, deferred, complete, wall


def reference_arm(a, dist):
    """The unmodified reference programs (src/<problem>/scout_<problem>.cu built for sm_100a
    by oracle/build_ref.sh) on exactly the scout arm's workload: the same graph written as a
    narrow .egr, the same warm-up + timed batches as a batch folder, the same initial states.
    Each program runs the whole folder; the timed batches are those after the warm-up, their
    time from the program's own per-batch `time=` lines. The end-of-stream catch-up traversal
    (SCOUT_DEFER_FALLBACK, the reference default) is what makes the deferred batches exact, so
    its time is charged to the timed batches in proportion to their deferred cascades."""
    sizes = batch_sizes(a.steps, a.warmup)
    problems = [p.strip() for p in a.problems.split(",") if p.strip()]
    ref_dir = os.path.join(ROOT, "oracle", "_ref")
    cores = os.cpu_count()
    t_gen = time.perf_counter()
    off, adj, batches, init = reference_workload(a, sizes)
    n, nnz = len(off) - 1, int(off[-1])
    config = workload_config(a, n, nnz, sizes, problems, dist.world)
    base = {"impl": "reference", "metric": METRIC, "unit": "edge-updates/s", "n_gpus": dist.world,
            "steps": a.steps, "warmup": a.warmup, "higher_is_better": True, "dtype": "int32",
            "data": "synthetic (seeded R-MAT + preferential toggle stream)", "config": config}
    missing = [p for p in problems if not os.path.exists(os.path.join(ref_dir, f"scout_{p}"))]
    if missing:
        return dict(base, unavailable=f"reference programs not built for {missing} (oracle/build_ref.sh needs the "
                                      f"reference sources)")
    from oracle import gen_oracle as go
    per_problem = {}
    edits_t = ms_t = 0.0
    complete = True
    with tempfile.TemporaryDirectory() as td:
        egr = os.path.join(td, "g.egr")
        go.write_egr_narrow(egr, off, adj)
        bdir = os.path.join(td, "batches")
        go.write_batch_folder(bdir, batches)
        gen_s = time.perf_counter() - t_gen
        budget = a.ref_timeout
        for p in problems:
            st = os.path.join(td, f"{p}.txt")
            go.write_state(st, p, init[p]())
            rows, deferred, ok, wall = run_reference_program(os.path.join(ref_dir, f"scout_{p}"), egr, st, bdir,
                                                             len(batches), dist.local, max(60.0, budget), td)
            budget -= wall
            complete = complete and ok
            timed = [r for r in rows if r[0] > a.warmup]
            fb_all = sum(r[3] for r in rows)
            fb_timed = sum(r[3] for r in timed)
            share = deferred * (fb_timed / fb_all) if fb_all else 0.0
            e = sum(r[1] for r in timed)
            ms = sum(r[2] for r in timed) + share
            per_problem[p] = {"edge_updates_per_s": e / (ms / 1e3) if ms else None, "batches_timed": len(timed),
                              "edits": e, "ms": ms, "deferred_catch_up_ms": deferred,
                              "deferred_charged_ms": share, "complete": ok, "program_wall_s": wall,
                              "per_size": per_size_rates([r[1] for r in timed], [r[2] for r in timed],
                                                         [sizes[r[0] - 1] for r in timed])}
            edits_t += e
            ms_t += ms
    val = edits_t / (ms_t / 1e3) if ms_t else None
    sample = (f"reference programs (src/*/scout_*.cu built for sm_100a, OpenMP host fetch on {cores} threads) on "
              f"the full workload: {len(batches)} batches, the last {a.steps} timed from their own per-batch "
              f"time= lines plus the charged share of the deferred catch-up; inputs generated in {gen_s:.0f} s "
              f"by the oracle's numpy generator")
    return dict(base, value=val, ms_per_step=ms_t / max(1, a.steps * len(problems)), complete=complete,
                per_problem=per_problem,
                cpu_baseline={"value": val, "unit": "edge-updates/s", "cores": cores, "kind": "reference",
                              "sample": sample},
                e2e={"value": val, "unit": "edge-updates/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0})


def main():
    a = parse_args()
    dist = Dist()
    try:
        if a.impl == "reference":
            if dist.rank != 0:
                return
            line = reference_arm(a, dist)
        else:
            line = scout_arm(a, dist)
        if dist.rank == 0:
            print(json.dumps(line), flush=True)
    finally:
        dist.close()


if __name__ == "__main__":
    main()
