"""ORACLE -- test and benchmark infrastructure, not product code.

A numpy restatement of the package's seeded workload generator (R-MAT graphs and toggle
streams) plus plain writers of the reference's file formats (.egr, batch folders, initial
states). `bench.py --impl reference` builds its inputs with this module, so the process that
times the reference's own programs maps no library of this package; `tests/test_gen_oracle.py`
checks that it reproduces the package generator byte for byte.

Random draws: splitmix64 (Steele, Lea, Flood, OOPSLA 2014). The R-MAT bits of edge i come from
mix64(h ^ (64 i + l)) for even levels l (low word at l, high word at l + 1); a stream's k-th
draw is mix64(s0 + k * golden) with s0 = mix64(seed ^ 0x5C07), so every draw is a pure function
of its index and whole blocks of draws are computed at once.

File formats (README.md:118-137 of the reference): narrow .egr = int32 nodes, int32 entries,
int32 nindex[n + 1], int32 nlist[E]; batch files `1.mtx..K.mtx` of 1-indexed `u v` lines;
BFS state `v level` (1-indexed v), colouring one colour per line, CC one label per line, MIS
the 1-indexed ids of the members.
"""
from __future__ import annotations

import os

import numpy as np

U64 = np.uint64
GOLDEN = U64(0x9E3779B97F4A7C15)
_M1 = U64(0xBF58476D1CE4E5B9)
_M2 = U64(0x94D049BB133111EB)
MASK64 = (1 << 64) - 1

STREAM_MIXED, STREAM_PREFERENTIAL = 0, 1


def mix64(z: np.ndarray) -> np.ndarray:
    """splitmix64 finaliser on a uint64 array (wrapping arithmetic)."""
    z = z + GOLDEN
    z = (z ^ (z >> U64(30))) * _M1
    z = (z ^ (z >> U64(27))) * _M2
    return z ^ (z >> U64(31))


def _mix64_int(z: int) -> int:
    return int(mix64(np.array([z & MASK64], dtype=U64))[0])


def gen_rmat(scale: int, edge_factor: int = 16, a: float = 0.57, b: float = 0.19, c: float = 0.19,
             seed: int = 1, chunk: int = 1 << 22):
    """Symmetrised R-MAT graph without self-loops or duplicate entries, both directions kept,
    rows sorted ascending. Returns (off int64[n + 1], adj int32[nnz])."""
    n = 1 << scale
    m = n * edge_factor
    ta = U64(int(a * 4294967296.0))
    tab = U64(int((a + b) * 4294967296.0))
    tabc = U64(int((a + b + c) * 4294967296.0))
    h = U64(_mix64_int((seed * 0x2545F4914F6CDD1D + 0xA0761D6478BD642F) & MASK64))
    lo32 = U64(0xFFFFFFFF)
    parts = []
    with np.errstate(over="ignore"):
        for i0 in range(0, m, chunk):
            i = np.arange(i0, min(m, i0 + chunk), dtype=U64)
            u = np.zeros(len(i), dtype=U64)
            v = np.zeros(len(i), dtype=U64)
            r = None
            for lv in range(scale):
                if lv % 2 == 0:
                    r = mix64(h ^ (i * U64(64) + U64(lv)))
                x = (r >> U64(32)) if lv % 2 else (r & lo32)
                bu = (x >= tab).astype(U64)
                bv = ((x >= ta) & (x < tab)) | (x >= tabc)
                u = (u << U64(1)) | bu
                v = (v << U64(1)) | bv.astype(U64)
            keep = u != v
            u, v = u[keep], v[keep]
            parts.append((u << U64(scale)) | v)
            parts.append((v << U64(scale)) | u)
    keys = np.concatenate(parts)
    del parts
    keys.sort()
    if len(keys):
        keys = keys[np.concatenate(([True], keys[1:] != keys[:-1]))]
    rows = (keys >> U64(scale)).astype(np.int64)
    off = np.zeros(n + 1, dtype=np.int64)
    np.cumsum(np.bincount(rows, minlength=n), out=off[1:])
    adj = (keys & U64(n - 1)).astype(np.int32)
    return off, adj


class _Draws:
    """The stream sampler's sequence of 64-bit draws, read in blocks."""

    def __init__(self, seed: int):
        self.s0 = U64(_mix64_int((seed ^ 0x5C07) & MASK64))
        self.k = 0   # draws consumed

    def block(self, count: int) -> np.ndarray:
        idx = np.arange(self.k + 1, self.k + 1 + count, dtype=U64)
        with np.errstate(over="ignore"):
            return mix64(self.s0 + idx * GOLDEN)




def _first_new(keys: np.ndarray, valid: np.ndarray, used: np.ndarray) -> np.ndarray:
    """Indices (in order) of candidates that are valid, not in `used` (sorted) and the first
    occurrence of their key among the valid candidates of this block."""
    cand = np.flatnonzero(valid)
    if len(cand) == 0:
        return cand
    k = keys[cand]
    order = np.argsort(k, kind="stable")
    ks = k[order]
    head = np.concatenate(([True], ks[1:] != ks[:-1]))
    firsts = np.sort(cand[order[head]])
    kf = keys[firsts]
    if len(used):
        hit = _member(used, kf)
        firsts = firsts[~hit]
    return firsts


def _member(sorted_keys: np.ndarray, q: np.ndarray) -> np.ndarray:
    """q[i] in sorted_keys, for unsorted q (queries sorted first for locality)."""
    order = np.argsort(q, kind="stable")
    qs = q[order]
    at = np.searchsorted(sorted_keys, qs)
    hit_s = (at < len(sorted_keys)) & (sorted_keys[np.minimum(at, len(sorted_keys) - 1)] == qs)
    hit = np.empty(len(q), dtype=bool)
    hit[order] = hit_s
    return hit


def gen_stream(off, adj, kind: int, total: int, insert_ratio: float = 0.5, seed: int = 1,
               block: int = 1 << 21) -> np.ndarray:
    """`total` toggles (int32 pairs, min id first): deletions of distinct existing edges
    (first endpoint proportional to degree: a uniform directed entry), then insertions of
    distinct non-edges (both endpoints proportional to degree for the preferential kind,
    uniform for the mixed kind), shuffled with Fisher-Yates."""
    off = np.asarray(off, dtype=np.int64)
    adj = np.asarray(adj, dtype=np.int32)
    n = len(off) - 1
    nnz = int(off[-1])
    n_ins = int(np.floor(total * insert_ratio + 0.5))
    n_del = total - n_ins
    if 2 * n_del > nnz:
        raise ValueError("stream asks for more deletions than the graph has edges")
    # row of a directed entry: searchsorted(nindex, pos, side="right") - 1, tabulated
    row_of = np.repeat(np.arange(n, dtype=np.int32), np.diff(off))
    edge_keys = None
    d = _Draws(seed)
    used = np.zeros(0, dtype=U64)
    out_keys = []
    # deletions: one draw per try
    got = 0
    while got < n_del:
        r = d.block(block)
        pos = (r % U64(nnz)).astype(np.int64)
        u = row_of[pos].astype(np.int64)
        v = adj[pos].astype(np.int64)
        lo, hi = np.minimum(u, v), np.maximum(u, v)
        keys = (lo.astype(U64) << U64(32)) | hi.astype(U64)
        acc = _first_new(keys, u != v, used)
        need = n_del - got
        if len(acc) >= need:
            acc = acc[:need]
            d.k += int(acc[-1]) + 1
        else:
            d.k += block
        out_keys.append(keys[acc])
        used = np.sort(np.concatenate((used, keys[acc])))
        got += len(acc)
    # insertions: two draws per try
    if n_ins > 0:
        edge_keys = (row_of.astype(U64) << U64(32)) | adj.astype(U64)
        if np.any(edge_keys[1:] < edge_keys[:-1]):
            edge_keys = np.sort(edge_keys)
    got = 0
    while got < n_ins:
        r = d.block(2 * block)
        if kind == STREAM_PREFERENTIAL:
            u = row_of[(r[0::2] % U64(nnz)).astype(np.int64)].astype(np.int64)
            v = row_of[(r[1::2] % U64(nnz)).astype(np.int64)].astype(np.int64)
        else:
            u = (r[0::2] % U64(n)).astype(np.int64)
            v = (r[1::2] % U64(n)).astype(np.int64)
        lo, hi = np.minimum(u, v), np.maximum(u, v)
        keys = (lo.astype(U64) << U64(32)) | hi.astype(U64)
        probe = (u.astype(U64) << U64(32)) | v.astype(U64)
        adjacent = _member(edge_keys, probe)
        acc = _first_new(keys, (u != v) & ~adjacent, used)
        need = n_ins - got
        if len(acc) >= need:
            acc = acc[:need]
            d.k += 2 * (int(acc[-1]) + 1)
        else:
            d.k += 2 * block
        out_keys.append(keys[acc])
        used = np.sort(np.concatenate((used, keys[acc])))
        got += len(acc)
    pool = np.concatenate(out_keys) if out_keys else np.zeros(0, dtype=U64)
    # Fisher-Yates: for i = total-1 .. 1, j = draw % (i + 1), swap
    if total > 1:
        i = np.arange(total - 1, 0, -1, dtype=U64)
        js = (d.block(total - 1) % (i + U64(1))).tolist()
        a = pool.tolist()
        t = 0
        for ii in range(total - 1, 0, -1):
            j = js[t]
            t += 1
            a[ii], a[j] = a[j], a[ii]
        pool = np.array(a, dtype=U64)
    e = np.empty((total, 2), dtype=np.int32)
    e[:, 0] = (pool >> U64(32)).astype(np.int32)
    e[:, 1] = (pool & U64(0xFFFFFFFF)).astype(np.int32)
    return e


# ---- file writers (the reference's input formats) ----------------------------------------------
def write_egr_narrow(path: str, off, adj) -> None:
    off = np.asarray(off, dtype=np.int64)
    n = len(off) - 1
    nnz = int(off[-1])
    if nnz > 2**31 - 1:
        raise ValueError("narrow .egr needs fewer than 2^31 entries")
    with open(path, "wb") as f:
        f.write(np.array([n, nnz], dtype=np.int32).tobytes())
        f.write(off.astype(np.int32).tobytes())
        f.write(np.ascontiguousarray(adj, dtype=np.int32)[:nnz].tobytes())


def write_batch(path: str, edges) -> None:
    e = np.asarray(edges, dtype=np.int64).reshape(-1, 2) + 1
    with open(path, "w") as f:
        if len(e):
            f.write("\n".join(f"{u} {v}" for u, v in e.tolist()))
            f.write("\n")


def write_batch_folder(folder: str, batches) -> None:
    os.makedirs(folder, exist_ok=True)
    for k, b in enumerate(batches):
        write_batch(os.path.join(folder, f"{k + 1}.mtx"), b)


def write_state(path: str, problem: str, sol) -> None:
    s = np.asarray(sol, dtype=np.int64)
    with open(path, "w") as f:
        if problem == "bfs":
            lines = (f"{v + 1} {x}" for v, x in enumerate(s.tolist()))
        elif problem == "mis":
            lines = (str(v + 1) for v in np.flatnonzero(s).tolist())
        elif problem in ("coloring", "cc"):
            lines = (str(x) for x in s.tolist())
        else:
            raise ValueError(f"unknown problem {problem}")
        for ln in lines:
            f.write(ln)
            f.write("\n")
