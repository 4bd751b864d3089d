"""ORACLE -- test infrastructure, not product code.

ctypes wrapper of oracle/liboracle.so, the single-threaded CPU restatement of the reference
engines (see the header of oracle/oracle.cpp for the rule-by-rule citations). Only tests/,
__graft_entry__.smoke() and the cpu_baseline leg of bench.py use it, always as the checker.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "liboracle.so")
PROBLEM = {"mis": 0, "coloring": 1, "bfs": 2, "cc": 3, "mis_id": 4}
STAT = ["ins", "del", "ins_noop", "del_noop", "conflict", "deferred", "fallback", "truncated", "rounds",
        "still_connected", "split", "inconclusive", "touched", "ins_repaired", "del_local", "merged",
        "max_rounds", "changed"]

_i32p = C.POINTER(C.c_int32)
_i64p = C.POINTER(C.c_int64)


SOURCES = ("oracle.cpp", "cpu_recompute.cpp")


def _load() -> C.CDLL:
    srcs = [os.path.join(_HERE, f) for f in SOURCES]
    if not os.path.exists(LIB_PATH) or os.path.getmtime(LIB_PATH) < max(os.path.getmtime(s) for s in srcs):
        objs = [LIB_PATH + f".{i}.o" for i in range(len(srcs))]
        for src, obj in zip(srcs, objs):   # OpenMP at compile time, libgomp named at link time
            subprocess.check_call(["g++", "-O2", "-std=c++17", "-fPIC", "-fopenmp", "-c", src, "-o", obj])
        subprocess.check_call(["g++", "-shared"] + objs + ["-l:libgomp.so.1", "-o", LIB_PATH])
        for obj in objs:
            os.remove(obj)
    lib = C.CDLL(LIB_PATH)
    sig = {
        "orc_graph_new": (C.c_void_p, [C.c_int64, _i64p, _i32p]),
        "orc_graph_free": (None, [C.c_void_p]),
        "orc_graph_is_adjacent": (C.c_int, [C.c_void_p, C.c_int, C.c_int]),
        "orc_graph_insert": (None, [C.c_void_p, C.c_int, C.c_int]),
        "orc_graph_remove": (None, [C.c_void_p, C.c_int, C.c_int]),
        "orc_graph_degree": (C.c_int64, [C.c_void_p, C.c_int]),
        "orc_graph_row": (C.c_int64, [C.c_void_p, C.c_int, _i32p, C.c_int64]),
        "orc_graph_nnz": (C.c_int64, [C.c_void_p]),
        "orc_graph_export": (None, [C.c_void_p, _i64p, _i32p]),
        "orc_graph_toggle_batch": (None, [C.c_void_p, _i32p, C.c_int64]),
        "orc_cpu_recompute": (C.c_double, [C.c_int, C.c_int64, _i64p, _i32p, C.c_int32, C.c_int, _i32p]),
        "orc_cpu_threads": (C.c_int, []),
        "orc_engine_new": (C.c_void_p, [C.c_int, C.c_int64, _i64p, _i32p, _i32p, C.c_int64, C.c_int]),
        "orc_engine_free": (None, [C.c_void_p]),
        "orc_engine_batch": (None, [C.c_void_p, _i32p, C.c_int64]),
        "orc_engine_finish": (None, [C.c_void_p]),
        "orc_engine_solution": (None, [C.c_void_p, _i32p]),
        "orc_engine_stats": (None, [C.c_void_p, _i64p]),
        "orc_engine_graph": (C.c_void_p, [C.c_void_p]),
        "orc_gt_bfs": (None, [C.c_int64, _i64p, _i32p, C.c_int, _i32p]),
        "orc_gt_cc": (None, [C.c_int64, _i64p, _i32p, _i32p]),
        "orc_gt_greedy_color": (None, [C.c_int64, _i64p, _i32p, _i32p]),
        "orc_gt_greedy_mis": (None, [C.c_int64, _i64p, _i32p, _i32p]),
        "orc_check_mis": (C.c_int64, [C.c_int64, _i64p, _i32p, _i32p, _i64p]),
        "orc_check_coloring": (C.c_int64, [C.c_int64, _i64p, _i32p, _i32p]),
    }
    for k, (r, a) in sig.items():
        f = getattr(lib, k)
        f.restype = r
        f.argtypes = a
    return lib


LIB = _load()


def _p32(a):
    return a.ctypes.data_as(_i32p)


def _p64(a):
    return a.ctypes.data_as(_i64p)


def _csr(off, adj):
    return np.ascontiguousarray(off, dtype=np.int64), np.ascontiguousarray(adj, dtype=np.int32)


class Graph:
    """Base CSR + the reference scratchpad (FlashGraph.h:200-388)."""

    def __init__(self, off, adj, handle=None, owner=None):
        if handle is None:
            off, adj = _csr(off, adj)
            handle = LIB.orc_graph_new(len(off) - 1, _p64(off), _p32(adj))
            self._own = True
        else:
            self._own = False
        self._h = handle
        self._owner = owner
        self.n = len(off) - 1 if off is not None else None

    def is_adjacent(self, u, v):
        return bool(LIB.orc_graph_is_adjacent(self._h, u, v))

    def insert(self, u, v):
        LIB.orc_graph_insert(self._h, u, v)

    def remove(self, u, v):
        LIB.orc_graph_remove(self._h, u, v)

    def row(self, v):
        d = LIB.orc_graph_degree(self._h, v)
        out = np.zeros(max(d, 1), dtype=np.int32)
        LIB.orc_graph_row(self._h, v, _p32(out), len(out))
        return out[:d]

    def toggle_batch(self, edges):
        """Applies a batch of toggles, each classified against the pre-batch graph."""
        e = np.ascontiguousarray(edges, dtype=np.int32).reshape(-1, 2)
        LIB.orc_graph_toggle_batch(self._h, _p32(e), len(e))

    def csr(self):
        nnz = LIB.orc_graph_nnz(self._h)
        off = np.zeros(self.n + 1, dtype=np.int64)
        adj = np.zeros(max(nnz, 1), dtype=np.int32)
        LIB.orc_graph_export(self._h, _p64(off), _p32(adj))
        return off, adj[:nnz]

    def __del__(self):
        if getattr(self, "_own", False) and self._h:
            LIB.orc_graph_free(self._h)
            self._h = None


class Engine:
    """Reference rule restatement of one engine (problem in PROBLEM)."""

    def __init__(self, problem: str, off, adj, init, bound: int = -1, defer: bool = True,
                 against_base: bool = False):
        off, adj = _csr(off, adj)
        init = np.ascontiguousarray(init, dtype=np.int32)
        flags = (1 if defer else 0) | (2 if against_base else 0)
        self._h = LIB.orc_engine_new(PROBLEM[problem], len(off) - 1, _p64(off), _p32(adj), _p32(init), bound, flags)
        if not self._h:
            raise ValueError("unknown problem")
        self.n = len(off) - 1
        self.problem = problem

    def batch(self, edges) -> None:
        e = np.ascontiguousarray(edges, dtype=np.int32).reshape(-1, 2)
        LIB.orc_engine_batch(self._h, _p32(e), len(e))

    def finish(self) -> None:
        LIB.orc_engine_finish(self._h)

    def solution(self) -> np.ndarray:
        out = np.zeros(self.n, dtype=np.int32)
        LIB.orc_engine_solution(self._h, _p32(out))
        return out

    def stats(self) -> dict:
        out = np.zeros(32, dtype=np.int64)
        LIB.orc_engine_stats(self._h, _p64(out))
        return {k: int(out[i]) for i, k in enumerate(STAT)}

    def graph(self) -> Graph:
        g = Graph(None, None, handle=LIB.orc_engine_graph(self._h), owner=self)
        g.n = self.n
        return g

    def __del__(self):
        if getattr(self, "_h", None):
            LIB.orc_engine_free(self._h)
            self._h = None


# ---- ground truth ------------------------------------------------------------------------
def gt_bfs(off, adj, source=0):
    off, adj = _csr(off, adj)
    out = np.zeros(len(off) - 1, dtype=np.int32)
    LIB.orc_gt_bfs(len(off) - 1, _p64(off), _p32(adj), source, _p32(out))
    return out


def gt_cc(off, adj):
    off, adj = _csr(off, adj)
    out = np.zeros(len(off) - 1, dtype=np.int32)
    LIB.orc_gt_cc(len(off) - 1, _p64(off), _p32(adj), _p32(out))
    return out


def gt_greedy_color(off, adj):
    off, adj = _csr(off, adj)
    out = np.zeros(len(off) - 1, dtype=np.int32)
    LIB.orc_gt_greedy_color(len(off) - 1, _p64(off), _p32(adj), _p32(out))
    return out


def gt_greedy_mis(off, adj):
    off, adj = _csr(off, adj)
    out = np.zeros(len(off) - 1, dtype=np.int32)
    LIB.orc_gt_greedy_mis(len(off) - 1, _p64(off), _p32(adj), _p32(out))
    return out


def check_mis(off, adj, flags):
    """Returns (independence violations, undominated non-members)."""
    off, adj = _csr(off, adj)
    f = np.ascontiguousarray(flags, dtype=np.int32)
    und = C.c_int64()
    bad = LIB.orc_check_mis(len(off) - 1, _p64(off), _p32(adj), _p32(f), C.byref(und))
    return int(bad), int(und.value)


def check_coloring(off, adj, color):
    """Number of directed entries whose endpoints share a colour."""
    off, adj = _csr(off, adj)
    c = np.ascontiguousarray(color, dtype=np.int32)
    return int(LIB.orc_check_coloring(len(off) - 1, _p64(off), _p32(adj), _p32(c)))


def canonical_labels(labels) -> np.ndarray:
    """Relabels any partition by the minimum vertex id of each class."""
    lab = np.asarray(labels)
    _, first = np.unique(lab, return_index=True)
    mapping = dict(zip(lab[first].tolist(), first.tolist()))
    return np.array([mapping[x] for x in lab.tolist()], dtype=np.int32)


# ---- all-core from-scratch recompute (a benchmark baseline, oracle/cpu_recompute.cpp) ---------
RECOMPUTE = {"mis": 0, "coloring": 1, "bfs": 2, "cc": 3}


def cpu_recompute(problem: str, off, adj, source: int = 0, threads: int = 0):
    """(solution, seconds) of a from-scratch recompute on `threads` host threads (0: all)."""
    off, adj = _csr(off, adj)
    out = np.zeros(len(off) - 1, dtype=np.int32)
    t = LIB.orc_cpu_recompute(RECOMPUTE[problem], len(off) - 1, _p64(off), _p32(adj), source, threads, _p32(out))
    return out, float(t)


def cpu_threads() -> int:
    return int(LIB.orc_cpu_threads())
