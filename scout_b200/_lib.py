"""ctypes bindings of include/scout_gpu.h and include/scout_host.h (libscout.so).

The library is built in-tree by ``python -m scout_b200.build``; importing this module
without it raises immediately (there is no fallback implementation).
"""
from __future__ import annotations

import ctypes as C
import os

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "lib", "libscout.so")

SCOUT_OK = 0
ERRORS = {
    -1: "SCOUT_E_INVALID", -2: "SCOUT_E_CUDA", -3: "SCOUT_E_CAPACITY", -4: "SCOUT_E_TIMEOUT",
    -5: "SCOUT_E_STATE", -6: "SCOUT_E_IO", -7: "SCOUT_E_FORMAT", -8: "SCOUT_E_NODEV",
}
PROBLEMS = {"mis": 0, "coloring": 1, "bfs": 2, "cc": 3}
OP_TOGGLE, OP_INSERT, OP_DELETE = 0, 1, 2
STREAM_MIXED, STREAM_PREFERENTIAL, STREAM_LOWDEG = 0, 1, 2


class ScoutEdge(C.Structure):
    _fields_ = [("u", C.c_int32), ("v", C.c_int32)]


class ScoutSched(C.Structure):
    _fields_ = [("policy", C.c_int32), ("mode", C.c_int32), ("frontier", C.c_int32),
                ("lanes_per_vertex", C.c_int32), ("search_bound", C.c_int64), ("search_limit", C.c_int64),
                ("blocks_per_sm", C.c_int32), ("chunk_log2", C.c_int32), ("prefetched", C.c_int32),
                ("pad0", C.c_int32), ("reserved", C.c_int64 * 1)]


class ScoutBatchStats(C.Structure):
    _fields_ = [("edits", C.c_int64), ("insertions", C.c_int64), ("deletions", C.c_int64),
                ("noop", C.c_int64), ("conflicts", C.c_int64), ("affected", C.c_int64),
                ("changed", C.c_int64), ("rounds", C.c_int64), ("recomputes", C.c_int64),
                ("splits", C.c_int64), ("searches", C.c_int64), ("hbm_bytes", C.c_int64),
                ("h2d_bytes", C.c_int64), ("d2h_bytes", C.c_int64), ("ms_update", C.c_double),
                ("ms_repair", C.c_double), ("ms_commit", C.c_double), ("ms_total", C.c_double),
                ("update_bytes", C.c_int64), ("launches", C.c_int64), ("ms_h2d", C.c_double),
                ("phase_ms", C.c_double * 4), ("variant", C.c_int64), ("ms_compact", C.c_double),
                ("compactions", C.c_int64), ("ins_effective", C.c_int64), ("del_effective", C.c_int64),
                ("ms_gather", C.c_double), ("gather_rows", C.c_int64), ("gather_bytes", C.c_int64)]

    def as_dict(self) -> dict:
        d = {f: getattr(self, f) for f, _ in self._fields_ if f not in ("reserved", "phase_ms")}
        d["phase_ms"] = list(self.phase_ms)
        return d


_vp = C.c_void_p
_i32p = C.POINTER(C.c_int32)
_i64p = C.POINTER(C.c_int64)
_u8p = C.POINTER(C.c_uint8)
_edgep = C.POINTER(ScoutEdge)
_f32p = C.POINTER(C.c_float)
_f64p = C.POINTER(C.c_double)

# (name, restype, argtypes) for every symbol the two headers declare.
SIGNATURES = [
    # scout_gpu.h
    ("scout_ctx_create", C.c_int, [C.c_int, C.c_uint64, C.POINTER(_vp)]),
    ("scout_ctx_destroy", C.c_int, [_vp]),
    ("scout_last_error", C.c_char_p, [_vp]),
    ("scout_device_count", C.c_int, [C.POINTER(C.c_int)]),
    ("scout_ctx_info", C.c_int, [_vp, C.c_char_p, C.c_int, C.POINTER(C.c_uint64)]),
    ("scout_graph_reserve", C.c_int, [_vp, C.c_int64, C.c_int64]),
    ("scout_stage_rows", C.c_int, [_vp, C.c_int, _i32p, _i64p, _i32p, C.c_int64, C.c_int64]),
    ("scout_graph_seal", C.c_int, [_vp]),
    ("scout_graph_load_csr", C.c_int, [_vp, C.c_int64, _i64p, _i32p]),
    ("scout_graph_info", C.c_int, [_vp, _i64p, _i64p, _i64p, _i64p]),
    ("scout_graph_download", C.c_int, [_vp, _i64p, _i32p, C.c_int64]),
    ("scout_graph_load_tiered", C.c_int, [_vp, C.c_int64, _i64p, _i32p, C.c_int64]),
    ("scout_graph_tier_info", C.c_int, [_vp, _i64p, _i64p, _i64p, _i64p, _i64p, _i64p]),
    ("scout_graph_compact", C.c_int, [_vp]),
    ("scout_classify", C.c_int, [_vp, _edgep, C.c_int64, _u8p]),
    ("scout_state_upload", C.c_int, [_vp, C.c_int, _i32p, C.c_int64]),
    ("scout_state_download", C.c_int, [_vp, C.c_int, _i32p, C.c_int64]),
    ("scout_set_source", C.c_int, [_vp, C.c_int32]),
    ("scout_repair", C.c_int, [_vp, C.c_int, _edgep, _u8p, C.c_int64, C.POINTER(ScoutSched),
                               C.POINTER(ScoutBatchStats)]),
    ("scout_repair_mis", C.c_int, [_vp, _edgep, _u8p, C.c_int64, C.POINTER(ScoutSched), C.POINTER(ScoutBatchStats)]),
    ("scout_repair_coloring", C.c_int, [_vp, _edgep, _u8p, C.c_int64, C.POINTER(ScoutSched),
                                        C.POINTER(ScoutBatchStats)]),
    ("scout_repair_bfs", C.c_int, [_vp, _edgep, _u8p, C.c_int64, C.POINTER(ScoutSched), C.POINTER(ScoutBatchStats)]),
    ("scout_repair_cc", C.c_int, [_vp, _edgep, _u8p, C.c_int64, C.POINTER(ScoutSched), C.POINTER(ScoutBatchStats)]),
    ("scout_prefetch", C.c_int, [_vp, _edgep, C.c_int64]),
    ("scout_commit", C.c_int, [_vp, C.c_int, _i32p, C.c_int64, _i64p]),
    ("scout_recompute_bfs", C.c_int, [_vp, C.c_int32, C.POINTER(ScoutBatchStats)]),
    ("scout_recompute_cc", C.c_int, [_vp, C.POINTER(ScoutBatchStats)]),
    ("scout_sync", C.c_int, [_vp, C.c_int64]),
    ("scout_host_alloc", C.c_int, [C.c_uint64, C.POINTER(_vp)]),
    ("scout_host_free", C.c_int, [_vp]),
    ("scout_sched_install", C.c_int, [_vp, C.c_int, _f32p, C.c_int64]),
    ("scout_sched_last", C.c_int, [_vp, _f32p, _f32p, _i32p]),
    ("scout_repair_probe", C.c_int, [_vp, C.c_int, _edgep, _u8p, C.c_int64, C.POINTER(ScoutSched), _f64p, _f32p,
                                     C.POINTER(ScoutBatchStats)]),
    ("scout_mlp_create", C.c_int, [C.c_int, C.c_uint64, C.POINTER(_vp)]),
    ("scout_mlp_destroy", C.c_int, [_vp]),
    ("scout_mlp_get_params", C.c_int, [_vp, _f32p, C.c_int64]),
    ("scout_mlp_set_params", C.c_int, [_vp, _f32p, C.c_int64]),
    ("scout_mlp_forward", C.c_int, [_vp, _f32p, C.c_int64, C.c_int, _f32p]),
    ("scout_mlp_loss_grad", C.c_int, [_vp, _f32p, _f32p, _f32p, C.c_int64, _f32p, _f32p]),
    ("scout_mlp_train", C.c_int, [_vp, _f32p, _f32p, _f32p, C.c_int64, C.c_int, C.c_int, C.c_float, C.c_uint64, _f32p]),
    ("scout_multi_create", C.c_int, [C.c_int, C.c_int, C.c_uint64, C.POINTER(_vp)]),
    ("scout_multi_destroy", C.c_int, [_vp]),
    ("scout_multi_context", _vp, [_vp]),
    ("scout_multi_add_stream", C.c_int, [_vp, C.c_int64, _i64p, _i32p, _i32p, C.c_int32, _i32p]),
    ("scout_multi_seal", C.c_int, [_vp]),
    ("scout_multi_round", C.c_int, [_vp, C.c_int32, _i32p, C.POINTER(_edgep), _i64p, C.POINTER(_u8p),
                                    C.POINTER(ScoutSched), C.POINTER(ScoutBatchStats)]),
    ("scout_multi_probe", C.c_int, [_vp, C.c_int32, _i32p, C.POINTER(_edgep), _i64p, C.POINTER(_u8p),
                                    C.POINTER(ScoutSched), _f64p, _f32p, C.POINTER(ScoutBatchStats)]),
    ("scout_multi_stage", C.c_int, [_vp, C.c_int32, _i32p, C.POINTER(_edgep), _i64p, C.POINTER(_u8p)]),
    ("scout_multi_run_all", C.c_int, [C.c_int32, C.POINTER(_vp), C.POINTER(ScoutSched), C.POINTER(ScoutBatchStats)]),
    ("scout_multi_commit", C.c_int, [_vp, C.POINTER(_i32p), _i64p]),
    ("scout_multi_download", C.c_int, [_vp, C.c_int32, _i32p, C.c_int64]),
    ("scout_multi_streams", C.c_int, [_vp, _i32p, _i64p]),
    ("scout_reserve", C.c_int, [_vp, C.c_int64]),
    ("scout_seed", C.c_int, [_vp, C.c_int, C.c_int32, C.POINTER(ScoutBatchStats)]),
    ("scout_multi_reserve", C.c_int, [_vp, C.c_int64]),
    ("scout_bfs_levels_noalloc", C.c_int, [C.c_void_p, C.c_void_p, C.c_int64, C.c_int32, C.c_void_p, C.c_void_p]),
    # scout_host.h
    ("scout_egr_open", C.c_int, [C.c_char_p, C.c_int, C.POINTER(_vp)]),
    ("scout_egr_close", C.c_int, [_vp]),
    ("scout_egr_nodes", C.c_int64, [_vp]),
    ("scout_egr_edges", C.c_int64, [_vp]),
    ("scout_egr_is_wide", C.c_int, [_vp]),
    ("scout_egr_offsets", C.c_int, [_vp, _i64p]),
    ("scout_egr_nlist", _i32p, [_vp]),
    ("scout_egr_write", C.c_int, [C.c_char_p, C.c_int64, _i64p, _i32p, C.c_int]),
    ("scout_hgraph_open", C.c_int, [C.c_char_p, C.c_int, C.POINTER(_vp)]),
    ("scout_hgraph_close", C.c_int, [_vp]),
    ("scout_hgraph_nodes", C.c_int64, [_vp]),
    ("scout_hgraph_is_adjacent", C.c_int, [_vp, C.c_int32, C.c_int32]),
    ("scout_hgraph_insert", C.c_int, [_vp, C.c_int32, C.c_int32]),
    ("scout_hgraph_remove", C.c_int, [_vp, C.c_int32, C.c_int32]),
    ("scout_hgraph_degree", C.c_int64, [_vp, C.c_int32]),
    ("scout_hgraph_neighbors", C.c_int64, [_vp, C.c_int32, _i32p, C.c_int64]),
    ("scout_hgraph_delta_edits", C.c_int64, [_vp]),
    ("scout_hgraph_compact", C.c_int, [_vp, C.c_char_p]),
    ("scout_fetch_all", C.c_int, [_vp, _vp, C.c_int64]),
    ("scout_fetch_rows", C.c_int, [_vp, _vp, _i32p, C.c_int64]),
    ("scout_parse_batch_file", C.c_int, [C.c_char_p, C.c_int64, _edgep, C.c_int64, _i64p]),
    ("scout_read_ints", C.c_int, [C.c_char_p, _i64p, C.c_int64, _i64p]),
    ("scout_load_state", C.c_int, [C.c_char_p, C.c_int, C.c_int64, _i32p, _i64p]),
    ("scout_write_state", C.c_int, [C.c_char_p, C.c_int, C.c_int64, _i32p]),
    ("scout_write_batch_folder", C.c_int, [C.c_char_p, _edgep, C.c_int64, C.c_int64]),
    ("scout_gen_rmat", C.c_int, [C.c_int, C.c_int, C.c_double, C.c_double, C.c_double, C.c_uint64, C.POINTER(_vp)]),
    ("scout_csr_from_arrays", C.c_int, [C.c_int64, _i64p, _i32p, C.POINTER(_vp)]),
    ("scout_csr_free", C.c_int, [_vp]),
    ("scout_csr_nodes", C.c_int64, [_vp]),
    ("scout_csr_nnz", C.c_int64, [_vp]),
    ("scout_csr_offsets", _i64p, [_vp]),
    ("scout_csr_adj", _i32p, [_vp]),
    ("scout_gen_stream", C.c_int, [_vp, C.c_int, C.c_int64, C.c_int64, C.c_double, C.c_double, C.c_uint64, _edgep]),
    ("scout_init_state", C.c_int, [_vp, C.c_int, C.c_int32, _i32p]),
]


def load() -> C.CDLL:
    if not os.path.exists(LIB_PATH):
        raise ImportError(f"{LIB_PATH} is missing: build the CUDA extension with `python -m scout_b200.build`")
    lib = C.CDLL(LIB_PATH)
    for name, res, args in SIGNATURES:
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    return lib


class _Lazy:
    """Loads libscout.so on first use, so the package (and its build recipe) imports before
    the library exists; any call without the built library raises ImportError."""

    _lib = None

    def __getattr__(self, name):
        if _Lazy._lib is None:
            _Lazy._lib = load()
        return getattr(_Lazy._lib, name)


LIB = _Lazy()
