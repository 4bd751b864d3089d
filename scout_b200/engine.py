"""Python face of libscout.so: numpy in, numpy out.

    ctx = Context(device=0)
    ctx.load_csr(off, adj)                  # graph resident in HBM
    ctx.upload("bfs", levels)               # maintained solution
    stats = ctx.repair("bfs", edges)        # one batch of toggles (N x 2 int32, 0-indexed)
    changed = ctx.commit("bfs", mirror)     # changed entries copied into a host mirror

Host-only helpers (no GPU): R-MAT generation, update streams, initial states, .egr and
text-format I/O, and the storage-resident hybrid graph.
"""
from __future__ import annotations

import ctypes as C
import weakref
from typing import Optional

import numpy as np

from . import _lib
from ._lib import LIB, PROBLEMS, ScoutBatchStats, ScoutEdge, ScoutSched


class ScoutError(RuntimeError):
    def __init__(self, code: int, msg: str):
        super().__init__(f"{_lib.ERRORS.get(code, code)}: {msg}")
        self.code = code


def _check(rc: int, ctx=None) -> None:
    if rc != _lib.SCOUT_OK:
        msg = LIB.scout_last_error(ctx)
        raise ScoutError(rc, msg.decode() if msg else "")


def _i32(a) -> np.ndarray:
    return np.ascontiguousarray(a, dtype=np.int32)


def _i64(a) -> np.ndarray:
    return np.ascontiguousarray(a, dtype=np.int64)


def _p32(a: np.ndarray):
    return a.ctypes.data_as(C.POINTER(C.c_int32))


def _p64(a: np.ndarray):
    return a.ctypes.data_as(C.POINTER(C.c_int64))


def _pf32(a: np.ndarray):
    return a.ctypes.data_as(C.POINTER(C.c_float))


def _pedge(a: np.ndarray):
    return a.ctypes.data_as(C.POINTER(ScoutEdge))


def _prob(p) -> int:
    return PROBLEMS[p] if isinstance(p, str) else int(p)


def as_edges(e) -> np.ndarray:
    a = _i32(e)
    if a.ndim != 2 or a.shape[1] != 2:
        raise ValueError("edges must have shape (m, 2)")
    return a


def pinned_empty(shape, dtype=np.int32) -> np.ndarray:
    """An uninitialised array in page-locked host memory (scout_host_alloc): edit batches in
    such memory are copied to the device without the staging copy."""
    dt = np.dtype(dtype)
    count = int(np.prod(shape)) if np.ndim(shape) else int(shape)
    nbytes = max(count * dt.itemsize, 1)
    ptr = C.c_void_p()
    _check(LIB.scout_host_alloc(nbytes, C.byref(ptr)))
    buf = (C.c_uint8 * nbytes).from_address(ptr.value)
    weakref.finalize(buf, LIB.scout_host_free, ptr.value)
    return np.frombuffer(buf, dtype=dt, count=count).reshape(shape)


def pinned_copy(a) -> np.ndarray:
    a = np.ascontiguousarray(a)
    out = pinned_empty(a.shape, a.dtype)
    out[...] = a
    return out


def device_count() -> int:
    n = C.c_int(0)
    _check(LIB.scout_device_count(C.byref(n)))
    return n.value


class Context:
    """One device context: an HBM graph store plus the maintained solutions."""

    def __init__(self, device: int = 0, budget_bytes: int = 0):
        h = C.c_void_p()
        _check(LIB.scout_ctx_create(int(device), int(budget_bytes), C.byref(h)))
        self._h = h
        self._own = True
        self.n = 0

    @classmethod
    def _borrow(cls, handle) -> "Context":
        """A view of a context owned by someone else (a MultiEngine); never destroyed here."""
        self = cls.__new__(cls)
        self._h = C.c_void_p(handle) if not isinstance(handle, C.c_void_p) else handle
        self._own = False
        self.n = 0
        return self

    def close(self) -> None:
        if self._h and self._own:
            LIB.scout_ctx_destroy(self._h)
        self._h = None

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def _c(self, rc: int) -> None:
        _check(rc, self._h)

    # ---- graph ------------------------------------------------------------------------
    def load_csr(self, off, adj) -> None:
        off = _i64(off)
        adj = _i32(adj)
        n = len(off) - 1
        self._c(LIB.scout_graph_load_csr(self._h, n, _p64(off), _p32(adj)))
        self.n = n

    def load_tiered(self, off, adj, hbm_entries: int = 0) -> None:
        """Out-of-core load: hot rows in an HBM pool of hbm_entries elements (0: from the
        budget), the rest in mapped page-locked host memory read in place."""
        off = _i64(off)
        adj = _i32(adj)
        self._c(LIB.scout_graph_load_tiered(self._h, len(off) - 1, _p64(off), _p32(adj), int(hbm_entries)))
        self.n = len(off) - 1

    def tier_info(self) -> dict:
        v = [C.c_int64() for _ in range(6)]
        self._c(LIB.scout_graph_tier_info(self._h, *[C.byref(x) for x in v]))
        return dict(zip(("hbm_cap", "hbm_used", "host_cap", "host_used", "evicted", "host_batches"),
                        (x.value for x in v)))

    def reserve(self, n: int, nnz: int) -> None:
        self._c(LIB.scout_graph_reserve(self._h, int(n), int(nnz)))
        self.n = int(n)

    def stage_rows(self, slot: int, ids, offs, elems) -> None:
        ids, offs, elems = _i32(ids), _i64(offs), _i32(elems)
        self._c(LIB.scout_stage_rows(self._h, int(slot), _p32(ids), _p64(offs), _p32(elems), len(ids),
                                     int(offs[-1] - offs[0]) if len(offs) else 0))

    def seal(self) -> None:
        self._c(LIB.scout_graph_seal(self._h))

    def info(self) -> dict:
        v = [C.c_int64() for _ in range(4)]
        self._c(LIB.scout_graph_info(self._h, *[C.byref(x) for x in v]))
        return dict(zip(("n", "nnz", "pool_used", "pool_cap"), (x.value for x in v)))

    def graph(self):
        """Current adjacency as CSR (rows ascending)."""
        n = self.info()["n"]
        off = np.zeros(n + 1, dtype=np.int64)
        rc = LIB.scout_graph_download(self._h, _p64(off), None, 0)
        if rc not in (_lib.SCOUT_OK, -3):
            self._c(rc)
        adj = np.zeros(max(int(off[n]), 1), dtype=np.int32)
        self._c(LIB.scout_graph_download(self._h, _p64(off), _p32(adj), len(adj)))
        return off, adj[: int(off[n])]

    def compact(self) -> None:
        self._c(LIB.scout_graph_compact(self._h))

    def classify(self, edges) -> np.ndarray:
        e = as_edges(edges)
        out = np.zeros(len(e), dtype=np.uint8)
        self._c(LIB.scout_classify(self._h, _pedge(e), len(e), out.ctypes.data_as(C.POINTER(C.c_uint8))))
        return out

    # ---- state ------------------------------------------------------------------------
    def upload(self, problem, sol) -> None:
        s = _i32(sol)
        self._c(LIB.scout_state_upload(self._h, _prob(problem), _p32(s), len(s)))

    def download(self, problem) -> np.ndarray:
        out = np.zeros(self.n, dtype=np.int32)
        self._c(LIB.scout_state_download(self._h, _prob(problem), _p32(out), self.n))
        return out

    def set_source(self, s: int) -> None:
        self._c(LIB.scout_set_source(self._h, int(s)))

    # ---- repair -----------------------------------------------------------------------
    def repair(self, problem, edges, ops=None, sched: Optional[dict] = None) -> dict:
        # the batch hinted by the last prefetch(): its device copy is already on the way
        pf = getattr(self, "_pf", None)
        hinted = pf is not None and edges is pf and ops is None
        self._pf = None
        e = as_edges(edges)
        st = ScoutBatchStats()
        sd = ScoutSched()
        for k, v in (sched or {}).items():
            setattr(sd, k, v)
        if hinted:
            sd.prefetched = 1
        op = None
        if ops is not None:
            ops = np.ascontiguousarray(ops, dtype=np.uint8)
            op = ops.ctypes.data_as(C.POINTER(C.c_uint8))
        self._c(LIB.scout_repair(self._h, _prob(problem), _pedge(e), op, len(e), C.byref(sd), C.byref(st)))
        return st.as_dict()

    def prefetch(self, next_edges) -> None:
        """Hint the edits of the batch after the next repair: that repair copies them to the
        device while it runs (and, tiered store, gathers their cold rows into HBM), and a later
        repair() given the same object uses the copy. A page-locked array (pinned_copy) is read
        in place and must stay unchanged until then."""
        e = as_edges(next_edges)
        self._c(LIB.scout_prefetch(self._h, _pedge(e), len(e)))
        # a converted temporary was copied by the call; only the caller's own array, passed to
        # repair() unchanged, is declared as the hinted batch
        self._pf = next_edges if e is next_edges else None

    def repair_probe(self, problem, edges, ops=None, sched: Optional[dict] = None):
        """One batch, every repair variant timed from the same pre-repair state (results must
        agree). Returns (stats, variant_ms[3] with -1 for absent variants, features[24])."""
        e = as_edges(edges)
        st = ScoutBatchStats()
        sd = ScoutSched()
        for k, v in (sched or {}).items():
            setattr(sd, k, v)
        op = None
        if ops is not None:
            ops = np.ascontiguousarray(ops, dtype=np.uint8)
            op = ops.ctypes.data_as(C.POINTER(C.c_uint8))
        ms = np.zeros(3, dtype=np.float64)
        feat = np.zeros(24, dtype=np.float32)
        self._c(LIB.scout_repair_probe(self._h, _prob(problem), _pedge(e), op, len(e), C.byref(sd),
                                       ms.ctypes.data_as(C.POINTER(C.c_double)), _pf32(feat), C.byref(st)))
        return st.as_dict(), ms, feat

    def sched_install(self, problem, params) -> None:
        """Installs a cost model (6020 fp32 parameters) for BFS or CC; None removes it."""
        if params is None:
            self._c(LIB.scout_sched_install(self._h, _prob(problem), None, 0))
            return
        w = np.ascontiguousarray(params, dtype=np.float32)
        self._c(LIB.scout_sched_install(self._h, _prob(problem), _pf32(w), w.size))

    def sched_last(self):
        """(features[24], predictions[4], decision) of the last repair that ran the scheduler."""
        f = np.zeros(24, dtype=np.float32)
        y = np.zeros(4, dtype=np.float32)
        d = C.c_int32()
        self._c(LIB.scout_sched_last(self._h, _pf32(f), _pf32(y), C.byref(d)))
        return f, y, d.value

    def commit(self, problem, mirror: np.ndarray) -> int:
        if mirror.dtype != np.int32 or not mirror.flags.c_contiguous:
            raise ValueError("mirror must be a contiguous int32 array")
        ch = C.c_int64()
        self._c(LIB.scout_commit(self._h, _prob(problem), _p32(mirror), len(mirror), C.byref(ch)))
        return ch.value

    def recompute_bfs(self, source: int = 0) -> dict:
        st = ScoutBatchStats()
        self._c(LIB.scout_recompute_bfs(self._h, int(source), C.byref(st)))
        return st.as_dict()

    def recompute_cc(self) -> dict:
        st = ScoutBatchStats()
        self._c(LIB.scout_recompute_cc(self._h, C.byref(st)))
        return st.as_dict()

    def seed(self, problem, source: int = 0) -> dict:
        """Initial solution computed on the device from the current graph (greedy MIS and
        colouring in vertex-id order, BFS levels from source, min-id components)."""
        st = ScoutBatchStats()
        self._c(LIB.scout_seed(self._h, _prob(problem), int(source), C.byref(st)))
        return st.as_dict()

    def held_bytes(self) -> int:
        """Device bytes the context holds (every allocation counts against its budget)."""
        v = C.c_uint64()
        self._c(LIB.scout_ctx_info(self._h, None, 0, C.byref(v)))
        return v.value

    def reserve_batches(self, max_edits: int) -> None:
        """Allocates now every buffer batches of up to max_edits edits would grow later."""
        self._c(LIB.scout_reserve(self._h, int(max_edits)))

    def sync(self, timeout_us: int = 0) -> None:
        self._c(LIB.scout_sync(self._h, int(timeout_us)))


def form_rounds(arrivals, max_edits: int):
    """Groups (stream_id, batch) arrivals into rounds for MultiEngine.round: each batch goes
    to the earliest round after its stream's previous batch that still has room for it
    (at most max_edits per round, a larger batch alone), so every stream keeps its order and
    small batches of many streams share a round. Returns a list of [(stream_id, batch), ...]."""
    rounds, totals, last = [], [], {}
    for sid, b in arrivals:
        r = last.get(sid, -1) + 1
        while r < len(rounds) and totals[r] > 0 and totals[r] + len(b) > max_edits:
            r += 1
        while r >= len(rounds):
            rounds.append([])
            totals.append(0)
        rounds[r].append((sid, b))
        totals[r] += len(b)
        last[sid] = r
    return rounds


class MultiEngine:
    """Batched multi-stream engine: K independent streams of one problem (each with its own
    graph and solution) kept as a disjoint union in one device store; a round runs at most
    one batch per stream as a single batch of the union. Ids stay stream-local."""

    def __init__(self, problem, device: int = 0, budget_bytes: int = 0):
        h = C.c_void_p()
        _check(LIB.scout_multi_create(int(device), _prob(problem), int(budget_bytes), C.byref(h)))
        self._h = h
        self.problem = problem
        self.sizes = []

    def close(self) -> None:
        if self._h:
            LIB.scout_multi_destroy(self._h)
            self._h = None

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def _c(self, rc: int) -> None:
        _check(rc, LIB.scout_multi_context(self._h) if self._h else None)

    @property
    def context(self) -> "Context":
        """The underlying device context (not owned): scheduler install, graph info."""
        return Context._borrow(LIB.scout_multi_context(self._h))

    def add_stream(self, off, adj, init, source: int = 0) -> int:
        off = _i64(off)
        adj = _i32(adj)
        init = _i32(init)
        sid = C.c_int32()
        self._c(LIB.scout_multi_add_stream(self._h, len(off) - 1, _p64(off), _p32(adj), _p32(init), int(source),
                                           C.byref(sid)))
        self.sizes.append(len(off) - 1)
        return sid.value

    def seal(self) -> None:
        self._c(LIB.scout_multi_seal(self._h))

    def reserve_batches(self, max_round_edits: int) -> None:
        self._c(LIB.scout_multi_reserve(self._h, int(max_round_edits)))

    def round(self, batches, sched: Optional[dict] = None) -> dict:
        """batches: [(stream_id, edges), ...] with distinct stream ids."""
        k = len(batches)
        ids = np.array([s for s, _ in batches], dtype=np.int32)
        arrs = [as_edges(b) for _, b in batches]
        ptrs = (C.POINTER(ScoutEdge) * max(k, 1))(*[_pedge(a) for a in arrs])
        counts = np.array([len(a) for a in arrs], dtype=np.int64)
        st = ScoutBatchStats()
        sd = ScoutSched()
        for key, v in (sched or {}).items():
            setattr(sd, key, v)
        self._c(LIB.scout_multi_round(self._h, k, _p32(ids), ptrs, _p64(counts), None, C.byref(sd), C.byref(st)))
        return st.as_dict()

    def stage(self, batches) -> None:
        """Assemble a round ([(stream_id, edges), ...]) for run_fused_round."""
        k = len(batches)
        ids = np.array([s for s, _ in batches], dtype=np.int32)
        arrs = [as_edges(b) for _, b in batches]
        ptrs = (C.POINTER(ScoutEdge) * max(k, 1))(*[_pedge(a) for a in arrs])
        counts = np.array([len(a) for a in arrs], dtype=np.int64)
        self._c(LIB.scout_multi_stage(self._h, k, _p32(ids), ptrs, _p64(counts), None))

    def probe(self, batches, sched: Optional[dict] = None):
        """A round through Context.repair_probe semantics: (stats, variant_ms[3], features[24])."""
        k = len(batches)
        ids = np.array([s for s, _ in batches], dtype=np.int32)
        arrs = [as_edges(b) for _, b in batches]
        ptrs = (C.POINTER(ScoutEdge) * max(k, 1))(*[_pedge(a) for a in arrs])
        counts = np.array([len(a) for a in arrs], dtype=np.int64)
        st = ScoutBatchStats()
        sd = ScoutSched()
        for key, v in (sched or {}).items():
            setattr(sd, key, v)
        ms = np.zeros(3, dtype=np.float64)
        feat = np.zeros(24, dtype=np.float32)
        self._c(LIB.scout_multi_probe(self._h, k, _p32(ids), ptrs, _p64(counts), None, C.byref(sd),
                                      ms.ctypes.data_as(C.POINTER(C.c_double)), _pf32(feat), C.byref(st)))
        return st.as_dict(), ms, feat

    def commit(self, mirrors) -> int:
        """mirrors[k]: int32 host mirror of stream k (None to skip)."""
        for m in mirrors:
            if m is not None and (m.dtype != np.int32 or not m.flags.c_contiguous):
                raise ValueError("mirrors must be contiguous int32 arrays")
        arr = (C.POINTER(C.c_int32) * len(mirrors))(*[(_p32(m) if m is not None else None) for m in mirrors])
        ch = C.c_int64()
        self._c(LIB.scout_multi_commit(self._h, arr, C.byref(ch)))
        return ch.value

    def download(self, sid: int) -> np.ndarray:
        out = np.zeros(self.sizes[sid], dtype=np.int32)
        self._c(LIB.scout_multi_download(self._h, int(sid), _p32(out), len(out)))
        return out


class MLP:
    """The scheduler's cost model (24-64-64-4 ReLU perceptron) on the device: fp32 master
    parameters trained by the library's own forward/backward/Adam kernels, bf16 copy for
    inference. Parameters are one flat vector of 6020 values (W1, b1, W2, b2, W3, b3; row j
    of a weight matrix = input weights of unit j)."""

    NPARAM = 6020

    def __init__(self, device: int = 0, seed: int = 0):
        h = C.c_void_p()
        _check(LIB.scout_mlp_create(int(device), int(seed), C.byref(h)))
        self._h = h

    def close(self) -> None:
        if self._h:
            LIB.scout_mlp_destroy(self._h)
            self._h = None

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    @property
    def params(self) -> np.ndarray:
        w = np.zeros(self.NPARAM, dtype=np.float32)
        _check(LIB.scout_mlp_get_params(self._h, _pf32(w), self.NPARAM))
        return w

    @params.setter
    def params(self, w) -> None:
        w = np.ascontiguousarray(w, dtype=np.float32)
        _check(LIB.scout_mlp_set_params(self._h, _pf32(w), w.size))

    def forward(self, x, bf16: bool = False) -> np.ndarray:
        x = np.ascontiguousarray(x, dtype=np.float32).reshape(-1, 24)
        y = np.zeros((len(x), 4), dtype=np.float32)
        _check(LIB.scout_mlp_forward(self._h, _pf32(x), len(x), int(bf16), _pf32(y)))
        return y

    def loss_grad(self, x, t, mask):
        x = np.ascontiguousarray(x, dtype=np.float32).reshape(-1, 24)
        t = np.ascontiguousarray(t, dtype=np.float32).reshape(-1, 4)
        m = np.ascontiguousarray(mask, dtype=np.float32).reshape(-1, 4)
        loss = C.c_float()
        g = np.zeros(self.NPARAM, dtype=np.float32)
        _check(LIB.scout_mlp_loss_grad(self._h, _pf32(x), _pf32(t), _pf32(m), len(x), C.byref(loss), _pf32(g)))
        return float(loss.value), g

    def train(self, x, t, mask, epochs: int = 200, batch: int = 256, lr: float = 3e-3, seed: int = 0) -> np.ndarray:
        x = np.ascontiguousarray(x, dtype=np.float32).reshape(-1, 24)
        t = np.ascontiguousarray(t, dtype=np.float32).reshape(-1, 4)
        m = np.ascontiguousarray(mask, dtype=np.float32).reshape(-1, 4)
        losses = np.zeros(max(epochs, 1), dtype=np.float32)
        _check(LIB.scout_mlp_train(self._h, _pf32(x), _pf32(t), _pf32(m), len(x), int(epochs), int(batch),
                                   float(lr), int(seed), _pf32(losses)))
        return losses[:epochs]


# ---------------------------------------------------------------------------------------
# Host-only helpers
# ---------------------------------------------------------------------------------------
class HostCsr:
    def __init__(self, handle):
        self._h = handle

    @classmethod
    def from_arrays(cls, off, adj) -> "HostCsr":
        off, adj = _i64(off), _i32(adj)
        h = C.c_void_p()
        _check(LIB.scout_csr_from_arrays(len(off) - 1, _p64(off), _p32(adj), C.byref(h)))
        return cls(h)

    @property
    def n(self) -> int:
        return LIB.scout_csr_nodes(self._h)

    @property
    def nnz(self) -> int:
        return LIB.scout_csr_nnz(self._h)

    def arrays(self):
        n, nnz = self.n, self.nnz
        off = np.ctypeslib.as_array(LIB.scout_csr_offsets(self._h), shape=(n + 1,)).copy()
        adj = np.ctypeslib.as_array(LIB.scout_csr_adj(self._h), shape=(max(nnz, 1),))[:nnz].copy()
        return off, adj

    def stream(self, kind: int, batch_size: int, nbatches: int, insert_ratio: float = 0.5,
               lowdeg_frac: float = 0.0, seed: int = 1) -> np.ndarray:
        out = np.zeros((batch_size * nbatches, 2), dtype=np.int32)
        _check(LIB.scout_gen_stream(self._h, int(kind), int(batch_size), int(nbatches), float(insert_ratio),
                                    float(lowdeg_frac), int(seed), _pedge(out)))
        return out

    def init_state(self, problem, source: int = 0) -> np.ndarray:
        out = np.zeros(self.n, dtype=np.int32)
        _check(LIB.scout_init_state(self._h, _prob(problem), int(source), _p32(out)))
        return out

    def close(self) -> None:
        if self._h:
            LIB.scout_csr_free(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def gen_rmat(scale: int, edge_factor: int = 16, a: float = 0.57, b: float = 0.19, c: float = 0.19,
             seed: int = 1) -> HostCsr:
    h = C.c_void_p()
    _check(LIB.scout_gen_rmat(int(scale), int(edge_factor), a, b, c, int(seed), C.byref(h)))
    return HostCsr(h)


def read_egr(path: str):
    h = C.c_void_p()
    _check(LIB.scout_egr_open(path.encode(), 1, C.byref(h)))
    try:
        n = LIB.scout_egr_nodes(h)
        e = LIB.scout_egr_edges(h)
        off = np.zeros(n + 1, dtype=np.int64)
        _check(LIB.scout_egr_offsets(h, _p64(off)))
        adj = np.ctypeslib.as_array(LIB.scout_egr_nlist(h), shape=(max(e, 1),))[:e].copy() if e else np.zeros(0, np.int32)
        wide = bool(LIB.scout_egr_is_wide(h))
    finally:
        LIB.scout_egr_close(h)
    return off, adj, wide


def write_egr(path: str, off, adj, wide: bool = False) -> None:
    off, adj = _i64(off), _i32(adj)
    _check(LIB.scout_egr_write(path.encode(), len(off) - 1, _p64(off), _p32(adj), int(wide)))


def parse_batch_file(path: str, n: int) -> np.ndarray:
    m = C.c_int64()
    rc = LIB.scout_parse_batch_file(path.encode(), int(n), None, 0, C.byref(m))
    if rc not in (_lib.SCOUT_OK, -3):
        _check(rc)
    out = np.zeros((max(m.value, 1), 2), dtype=np.int32)
    _check(LIB.scout_parse_batch_file(path.encode(), int(n), _pedge(out), len(out), C.byref(m)))
    return out[: m.value]


def read_ints(path: str) -> np.ndarray:
    m = C.c_int64()
    rc = LIB.scout_read_ints(path.encode(), None, 0, C.byref(m))
    if rc not in (_lib.SCOUT_OK, -3):
        _check(rc)
    out = np.zeros(max(m.value, 1), dtype=np.int64)
    _check(LIB.scout_read_ints(path.encode(), _p64(out), len(out), C.byref(m)))
    return out[: m.value]


def load_state(path: str, problem, n: int):
    sol = np.zeros(n, dtype=np.int32)
    aux = C.c_int64()
    _check(LIB.scout_load_state(path.encode(), _prob(problem), int(n), _p32(sol), C.byref(aux)))
    return sol, aux.value


def write_state(path: str, problem, sol) -> None:
    s = _i32(sol)
    _check(LIB.scout_write_state(path.encode(), _prob(problem), len(s), _p32(s)))


def write_batch_folder(path: str, edges, batch_size: int, nbatches: int) -> None:
    e = as_edges(edges)
    if len(e) < batch_size * nbatches:
        raise ValueError("not enough edges for the requested batches")
    _check(LIB.scout_write_batch_folder(path.encode(), _pedge(e), int(batch_size), int(nbatches)))


class HybridGraph:
    """Storage-resident .egr (mmap) + edge-update scratchpad (host)."""

    def __init__(self, path: str, madv_random: bool = True):
        h = C.c_void_p()
        _check(LIB.scout_hgraph_open(path.encode(), int(madv_random), C.byref(h)))
        self._h = h

    @property
    def n(self) -> int:
        return LIB.scout_hgraph_nodes(self._h)

    def is_adjacent(self, u: int, v: int) -> bool:
        r = LIB.scout_hgraph_is_adjacent(self._h, u, v)
        if r < 0:
            _check(r)
        return bool(r)

    def insert(self, u: int, v: int) -> None:
        _check(LIB.scout_hgraph_insert(self._h, u, v))

    def remove(self, u: int, v: int) -> None:
        _check(LIB.scout_hgraph_remove(self._h, u, v))

    def degree(self, v: int) -> int:
        d = LIB.scout_hgraph_degree(self._h, v)
        if d < 0:
            _check(int(d))
        return d

    def neighbors(self, v: int) -> np.ndarray:
        d = self.degree(v)
        out = np.zeros(max(d, 1), dtype=np.int32)
        LIB.scout_hgraph_neighbors(self._h, v, _p32(out), len(out))
        return out[:d]

    def compact(self, out_path: str) -> None:
        _check(LIB.scout_hgraph_compact(self._h, out_path.encode()))

    def fetch_all(self, ctx: Context, slab_elems: int = 0) -> None:
        _check(LIB.scout_fetch_all(self._h, ctx._h, int(slab_elems)), ctx._h)
        ctx.n = self.n

    def close(self) -> None:
        if self._h:
            LIB.scout_hgraph_close(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

def run_fused_round(engines, sched: Optional[dict] = None) -> list:
    """One round of several MultiEngines of distinct problems, each staged with stage(): their
    merges, then ONE persistent kernel running all their repairs (scout_multi_run_all).
    Returns each engine's stats; commit each engine as after round()."""
    ne = len(engines)
    hs = (C.c_void_p * max(ne, 1))(*[e._h for e in engines])
    sts = (ScoutBatchStats * max(ne, 1))()
    sd = ScoutSched()
    for key, v in (sched or {}).items():
        setattr(sd, key, v)
    rc = LIB.scout_multi_run_all(ne, hs, C.byref(sd), sts)
    _check(rc, LIB.scout_multi_context(engines[0]._h) if ne else None)
    return [sts[i].as_dict() for i in range(ne)]
