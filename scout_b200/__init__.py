"""scout-b200: B200-native (sm_100a) storage-resident dynamic-graph repair engine for MIS,
colouring, BFS levels and connected components, with the reference SCOUT's drop-in surface
(bin/scout_<problem>, .egr CSR, batch folders, initial-state and solution files)."""
from .engine import (MLP, Context, MultiEngine, form_rounds, HostCsr, HybridGraph, ScoutError, as_edges, device_count, gen_rmat,
                     load_state, parse_batch_file, pinned_copy, pinned_empty, read_egr, read_ints,
                     run_fused_round, write_batch_folder, write_egr, write_state)
from ._lib import OP_DELETE, OP_INSERT, OP_TOGGLE, PROBLEMS, STREAM_LOWDEG, STREAM_MIXED, STREAM_PREFERENTIAL

__all__ = ["MLP", "Context", "MultiEngine", "form_rounds", "HostCsr", "HybridGraph", "ScoutError", "as_edges", "device_count", "gen_rmat",
           "load_state", "parse_batch_file", "pinned_copy", "pinned_empty", "read_egr", "read_ints", "run_fused_round", "write_batch_folder", "write_egr",
           "write_state", "OP_DELETE", "OP_INSERT", "OP_TOGGLE", "PROBLEMS", "STREAM_LOWDEG",
           "STREAM_MIXED", "STREAM_PREFERENTIAL"]
