"""The learned scheduler's data, training and evaluation.

The plain engine runs every BFS/CC batch with the incremental repair. The learned engine
lets a cost model, evaluated on the device after the batch merge, pick among the exact
repair variants of the problem (BFS: 0 incremental, 1 top-down traversal, 2
direction-optimizing traversal; CC: 0 incremental, 1 recompute of every class, 2 recompute of
the classes an unsettled deletion touches). All variants give identical solutions, so the
choice only moves time.

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

VARIANTS = {"bfs": 3, "cc": 3}
VARIANT_NAMES = {"bfs": ["incremental", "top-down traversal", "direction-optimizing traversal"],
                 "cc": ["incremental", "recompute", "recompute touched classes"]}
# the device scheduler leaves the incremental repair only for a predicted gain above this
# (target units: log2(1 + microseconds) / 4, so 0.05 is about 15%)
MARGIN = 0.05


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


@dataclass
class MultiSpec:
    """A multi-stream workload: streams_per_graph streams on each seeded graph (scale, edge
    factor), nbatches batches per stream with log-uniform sizes in [100, 10^6] (capped at a
    quarter of the graph's entries), kinds drawn per stream, seeded random interleaving, and
    rounds formed with round_cap."""
    graphs: list
    streams_per_graph: int
    nbatches: int
    seed: int
    round_cap: int = 1 << 20


def fit_sizes(sizes, nnz: int, insert_ratio: float):
    """Scales a stream's batch sizes down so its deletions fit the graph: the generators draw
    distinct existing edges, at most nnz / 2 (undirected) per stream."""
    limit = int(0.95 * nnz / (2.0 * max(1e-9, 1.0 - insert_ratio)))
    tot = sum(sizes)
    if tot <= limit:
        return list(sizes)
    return [max(1, int(z * limit / tot)) for z in sizes]


def multi_arrivals(spec: MultiSpec, graphs):
    """(stream graph index, batch) arrivals of a MultiSpec over its generated graphs."""
    rng = np.random.default_rng(spec.seed)
    per_stream = []
    for gi, g in enumerate(graphs):
        for r in range(spec.streams_per_graph):
            cap = max(100, g.nnz // 4)
            sizes = [int(min(cap, round(10 ** rng.uniform(2, 6)))) for _ in range(spec.nbatches)]
            kind = int(rng.integers(0, 3))
            ins = 0.5 if kind != STREAM_LOWDEG else 0.3
            sizes = fit_sizes(sizes, g.nnz, ins)
            s = g.stream(kind, sum(sizes), 1, insert_ratio=ins,
                         lowdeg_frac=0.3 if kind == STREAM_LOWDEG else 0.0, seed=spec.seed * 1000 + len(per_stream))
            b = np.cumsum([0] + sizes)
            per_stream.append((gi, [np.ascontiguousarray(s[b[j]:b[j + 1]]) for j in range(len(sizes))]))
    order = np.repeat(np.arange(len(per_stream)), spec.nbatches)
    rng.shuffle(order)
    nxt = [0] * len(per_stream)
    arrivals = []
    for i in order.tolist():
        arrivals.append((i, per_stream[i][1][nxt[i]]))
        nxt[i] += 1
    return per_stream, arrivals


def collect_multi(problem: str, specs, device: int = 0, data: Dataset | None = None, log=None) -> Dataset:
    """Probes every round of every multi-stream workload (the union batch of the round)."""
    data = data or Dataset()
    for spec in specs:
        graphs = [E.gen_rmat(sc, ef, seed=spec.seed * 100 + i) for i, (sc, ef) in enumerate(spec.graphs)]
        per_stream, arrivals = multi_arrivals(spec, graphs)
        t0 = time.time()
        with E.MultiEngine(problem, device) as me:
            inits = {}
            for gi, _ in per_stream:
                if gi not in inits:
                    inits[gi] = graphs[gi].init_state(problem, 0)
                off, adj = graphs[gi].arrays()
                me.add_stream(off, adj, inits[gi], 0)
            me.seal()
            rounds = E.form_rounds(arrivals, spec.round_cap)
            me.reserve_batches(max(spec.round_cap, max(len(b) for _, b in arrivals)))
            for rd in rounds:
                st, ms, f = me.probe(rd)
                data.add(f, ms, st["changed"], ("multi", len(rd), int(sum(len(b) for _, b in rd))))
        if log:
            log(f"{problem}: multi-stream {spec.graphs} x{spec.streams_per_graph}: {len(rounds)} rounds in "
                f"{time.time() - t0:.1f} s")
    return data


def default_multi_specs(seeds, big: bool = True):
    """Unions like the benchmark's: 8 graphs of scales 12-22 (or 12-20), two streams each."""
    out = []
    for s in seeds:
        gs = [(12, 8), (14, 16), (15, 32), (16, 8), (17, 16), (18, 32), (20, 8)] + ([(22, 16)] if big else [(19, 16)])
        out.append(MultiSpec(gs, 2, 6, seed=s))
        out.append(MultiSpec(gs[:5], 3, 6, seed=s + 500, round_cap=1 << 18))
    return out


def train(data: Dataset, device: int = 0, epochs: int = 300, batch: int = 128, lr: float = 2e-3, seed: int = 0):
    """Trains the cost model on the device; returns (fp32 parameters, per-epoch loss)."""
    x, t, m, _ = data.arrays()
    with E.MLP(device, seed=seed) as net:
        losses = net.train(x, t, m, epochs=epochs, batch=batch, lr=lr, seed=seed)
        return net.params, losses


def choose(params, x, nvariants: int, device: int = 0, bf16: bool = True) -> np.ndarray:
    """The variant the engine's device scheduler picks for each feature row: the cheapest
    predicted one among those beating the incremental repair by more than MARGIN."""
    with E.MLP(device) as net:
        net.params = params
        y = net.forward(x, bf16=bf16)
    pick = np.zeros(len(y), dtype=np.int64)
    for i in range(len(y)):
        best, by = 0, np.float32(y[i, 0]) - np.float32(MARGIN)
        for v in range(1, nvariants):
            if y[i, v] < by:
                best, by = v, y[i, v]
        pick[i] = best
    return pick


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
    ap.add_argument("--multi-seeds", type=int, default=3)
    ap.add_argument("--multi-weight", type=int, default=4, help="copies of each union-round sample in training")
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
        trm = collect_multi(p, default_multi_specs(range(1, 1 + a.multi_seeds)), a.device, log=log)
        evm = collect_multi(p, default_multi_specs([77], big=True)[:1], a.device, log=log)
        both = Dataset()
        for d, w in ((tr, 1), (trm, a.multi_weight)):
            for _ in range(w):
                both.x += d.x
                both.t += d.t
                both.m += d.m
                both.ms += d.ms
                both.tag += d.tag
        params, losses = train(both, a.device, epochs=a.epochs)
        report[p] = {"train_samples": len(tr), "train_rounds": len(trm), "eval_samples": len(ev),
                     "eval_rounds": len(evm), "final_loss": float(losses[-1]), "first_loss": float(losses[0]),
                     "eval": evaluate(params, ev, p, a.device), "eval_rounds_result": evaluate(params, evm, p, a.device),
                     "train_fit": evaluate(params, tr, p, a.device), "train_rounds_fit": evaluate(params, trm, p, a.device)}
        out[p] = params
        print(json.dumps(report[p]), flush=True)
    if a.out:
        np.savez(a.out, **out, report=np.array(json.dumps(report)))


if __name__ == "__main__":
    main()
