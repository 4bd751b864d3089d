"""The learned scheduler's data, training and evaluation.

The plain engine runs every BFS/CC batch with the incremental repair. The learned engine
lets a cost model, evaluated on the device after the batch merge, pick among the exact
repair variants of the problem (BFS: 0 incremental, 1 top-down traversal, 2
direction-optimizing traversal; CC: 0 incremental, 1 recompute of every class). All
variants give identical solutions, so the choice only moves time.

    python -m scout_b200.learn --out scout_b200/sched_model.npz   # collect, train, evaluate

Data: every batch of a set of seeded R-MAT graphs and update streams is run through
``Context.repair_probe``, which merges the batch once and times every variant from the same
pre-repair state. A sample is (24 features, targets = log2 of each variant's repair time
and of the changed-vertex count, mask). Training uses the library's own device kernels
(``MLP.train``); evaluation uses the bf16 inference the engine runs and reports, on held-out
seeds, the total repair time of the plain choice (always incremental), of the learned choice
and of the best variant per batch (oracle-best), and the regrets against oracle-best.
"""
from __future__ import annotations

import argparse
import json
import math
import time
from dataclasses import dataclass, field

import numpy as np

from . import engine as E
from ._lib import STREAM_LOWDEG, STREAM_MIXED, STREAM_PREFERENTIAL

VARIANTS = {"bfs": 3, "cc": 2}
VARIANT_NAMES = {"bfs": ["incremental", "top-down traversal", "direction-optimizing traversal"],
                 "cc": ["incremental", "recompute"]}


def targets(variant_ms, changed):
    """log2(1 + repair microseconds) / 4 per variant (mask 0 where absent) and
    log2(1 + changed vertices) / 24."""
    t = np.zeros(4, dtype=np.float32)
    m = np.zeros(4, dtype=np.float32)
    for v in range(3):
        if variant_ms[v] >= 0:
            t[v] = math.log2(1.0 + 1000.0 * variant_ms[v]) / 4.0
            m[v] = 1.0
    t[3] = math.log2(1.0 + changed) / 24.0
    m[3] = 1.0
    return t, m


@dataclass
class StreamSpec:
    """One seeded update stream over one seeded R-MAT graph."""
    scale: int
    edge_factor: int
    kind: int                  # STREAM_MIXED / STREAM_PREFERENTIAL / STREAM_LOWDEG
    sizes: list
    insert_ratio: float = 0.5
    graph_seed: int = 1
    stream_seed: int = 1
    lowdeg_p: float = 0.3


@dataclass
class Dataset:
    x: list = field(default_factory=list)
    t: list = field(default_factory=list)
    m: list = field(default_factory=list)
    ms: list = field(default_factory=list)
    tag: list = field(default_factory=list)

    def add(self, f, ms, changed, tag):
        t, m = targets(ms, changed)
        self.x.append(np.asarray(f, dtype=np.float32))
        self.t.append(t)
        self.m.append(m)
        self.ms.append(np.asarray(ms, dtype=np.float64))
        self.tag.append(tag)

    def arrays(self):
        return (np.stack(self.x), np.stack(self.t), np.stack(self.m), np.stack(self.ms))

    def __len__(self):
        return len(self.x)


def _stream(g, spec: StreamSpec):
    total = int(sum(spec.sizes))
    s = g.stream(spec.kind, total, 1, insert_ratio=spec.insert_ratio,
                 lowdeg_frac=spec.lowdeg_p if spec.kind == STREAM_LOWDEG else 0.0, seed=spec.stream_seed)
    bounds = np.cumsum([0] + list(spec.sizes))
    return [np.ascontiguousarray(s[bounds[i]:bounds[i + 1]]) for i in range(len(spec.sizes))]


def collect(problem: str, specs, device: int = 0, data: Dataset | None = None, graphs: dict | None = None,
            log=None) -> Dataset:
    """Probes every batch of every stream; returns the samples (features, targets, mask)."""
    data = data or Dataset()
    graphs = graphs if graphs is not None else {}
    for spec in specs:
        key = (spec.scale, spec.edge_factor, spec.graph_seed)
        if key not in graphs:
            graphs[key] = E.gen_rmat(spec.scale, spec.edge_factor, seed=spec.graph_seed)
        g = graphs[key]
        off, adj = g.arrays()
        init = g.init_state(problem, 0)
        batches = _stream(g, spec)
        t0 = time.time()
        with E.Context(device) as ctx:
            ctx.load_csr(off, adj)
            ctx.upload(problem, init)
            for b in batches:
                st, ms, f = ctx.repair_probe(problem, b)
                data.add(f, ms, st["changed"], (spec.scale, spec.kind, len(b)))
        if log:
            log(f"{problem}: scale {spec.scale} kind {spec.kind} seed {spec.stream_seed}: "
                f"{len(batches)} batches in {time.time() - t0:.1f} s")
    return data


def train(data: Dataset, device: int = 0, epochs: int = 300, batch: int = 128, lr: float = 2e-3, seed: int = 0):
    """Trains the cost model on the device; returns (fp32 parameters, per-epoch loss)."""
    x, t, m, _ = data.arrays()
    with E.MLP(device, seed=seed) as net:
        losses = net.train(x, t, m, epochs=epochs, batch=batch, lr=lr, seed=seed)
        return net.params, losses


def choose(params, x, nvariants: int, device: int = 0, bf16: bool = True) -> np.ndarray:
    """The variant the engine's device scheduler would pick for each feature row."""
    with E.MLP(device) as net:
        net.params = params
        y = net.forward(x, bf16=bf16)
    return np.argmin(y[:, :nvariants], axis=1)


def evaluate(params, data: Dataset, problem: str, device: int = 0) -> dict:
    """Total repair time (ms) of plain (always incremental), learned and oracle-best choices
    over the probed batches of `data`, and the regrets against oracle-best."""
    x, _, _, ms = data.arrays()
    nv = VARIANTS[problem]
    ms = ms[:, :nv]
    pick = choose(params, x, nv, device)
    best = ms.min(1)
    t_plain = float(ms[:, 0].sum())
    t_learned = float(ms[np.arange(len(ms)), pick].sum())
    t_best = float(best.sum())
    return {"problem": problem, "batches": int(len(ms)), "plain_ms": t_plain, "learned_ms": t_learned,
            "oracle_best_ms": t_best, "plain_regret": t_plain / t_best - 1.0,
            "learned_regret": t_learned / t_best - 1.0, "speedup_vs_plain": t_plain / t_learned,
            "picked": {VARIANT_NAMES[problem][v]: int((pick == v).sum()) for v in range(nv)},
            "best": {VARIANT_NAMES[problem][v]: int((ms.argmin(1) == v).sum()) for v in range(nv)}}


def default_specs(problem: str, seeds, scales=(16, 18, 20), sizes=(100, 1_000, 10_000, 100_000, 300_000),
                  graph_seeds=None):
    """Streams spanning the regimes where each variant wins: small batches (incremental),
    large preferential batches and deletion-heavy low-degree batches (traversals). Stream s
    runs on graph seed graph_seeds[s % len(graph_seeds)] (default: its own graph, 100 + s)."""
    specs = []
    for s in seeds:
        gseed = 100 + s if not graph_seeds else graph_seeds[s % len(graph_seeds)]
        for sc in scales:
            cap = 1 << (sc + 2)
            sz = [z for z in sizes if z <= cap]
            seq = [sz[(i * 7 + s) % len(sz)] for i in range(12)]
            specs.append(StreamSpec(sc, 16, STREAM_PREFERENTIAL, seq, 0.5, graph_seed=gseed, stream_seed=1000 + s))
            specs.append(StreamSpec(sc, 16, STREAM_LOWDEG, seq, 0.3, graph_seed=gseed, stream_seed=2000 + s))
            specs.append(StreamSpec(sc, 16, STREAM_MIXED, seq, 0.5, graph_seed=gseed, stream_seed=3000 + s))
    return specs


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--out", default="")
    ap.add_argument("--problems", default="bfs,cc")
    ap.add_argument("--train-seeds", type=int, default=6)
    ap.add_argument("--eval-seeds", type=int, default=2)
    ap.add_argument("--scales", default="16,18,20")
    ap.add_argument("--sizes", default="100,1000,10000,100000,300000,1000000")
    ap.add_argument("--epochs", type=int, default=400)
    ap.add_argument("--device", type=int, default=0)
    a = ap.parse_args()
    scales = tuple(int(x) for x in a.scales.split(","))
    out = {}
    report = {}
    for p in [x.strip() for x in a.problems.split(",") if x.strip()]:
        log = lambda s: print(s, flush=True)  # noqa: E731
        graphs: dict = {}
        sizes = tuple(int(x) for x in a.sizes.split(","))
        tr = collect(p, default_specs(p, range(a.train_seeds), scales, sizes, graph_seeds=(100, 101)), a.device,
                     graphs=graphs, log=log)
        ev = collect(p, default_specs(p, range(100, 100 + a.eval_seeds), scales, sizes, graph_seeds=(200,)),
                     a.device, graphs=graphs, log=log)
        params, losses = train(tr, a.device, epochs=a.epochs)
        report[p] = {"train_samples": len(tr), "eval_samples": len(ev), "final_loss": float(losses[-1]),
                     "first_loss": float(losses[0]), "eval": evaluate(params, ev, p, a.device),
                     "train_fit": evaluate(params, tr, p, a.device)}
        out[p] = params
        print(json.dumps(report[p]), flush=True)
    if a.out:
        np.savez(a.out, **out, report=np.array(json.dumps(report)))


if __name__ == "__main__":
    main()
