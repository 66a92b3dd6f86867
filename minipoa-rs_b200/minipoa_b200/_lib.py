"""ctypes binding of libminipoa_b200.so (the C ABI of include/minipoa_b200.h).

The library is loaded from this package directory. There is no fallback:
when the shared library is missing, importing the binding raises.
"""
from __future__ import annotations

import ctypes
import os

from .params import CParams

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libminipoa_b200.so")

POA_OK, POA_ERR_ALIGN, POA_ERR_INVALID, POA_ERR_CUDA, POA_ERR_ALLOC, POA_ERR_UNSUPPORTED, POA_ERR_TIMEOUT = range(7)


class AlignedBaseC(ctypes.Structure):
    _fields_ = [("node", ctypes.c_int64), ("base", ctypes.c_int64), ("aligned", ctypes.c_int64)]


class GraphSizes(ctypes.Structure):
    _fields_ = [("n_nodes", ctypes.c_int64), ("n_edges", ctypes.c_int64), ("n_paths", ctypes.c_int64),
                ("path_items", ctypes.c_int64), ("alphabet", ctypes.c_int64),
                ("n_rank", ctypes.c_int64)]


class MinimizerC(ctypes.Structure):
    _fields_ = [("value", ctypes.c_uint64), ("end", ctypes.c_int64), ("span", ctypes.c_int64)]


class AnchorC(ctypes.Structure):
    _fields_ = [("target_end", ctypes.c_int64), ("query_end", ctypes.c_int64), ("span", ctypes.c_int64),
                ("adaptive_before", ctypes.c_int32), ("reserved", ctypes.c_int32)]


class ServerJobInfo(ctypes.Structure):
    _fields_ = [("state", ctypes.c_int32), ("reserved", ctypes.c_int32), ("cells", ctypes.c_uint64),
                ("queued_ms", ctypes.c_double), ("latency_ms", ctypes.c_double)]


class ServerStats(ctypes.Structure):
    _fields_ = [("done_jobs", ctypes.c_uint64), ("done_cells", ctypes.c_uint64), ("waves", ctypes.c_uint64),
                ("queued", ctypes.c_uint64), ("kernel_launches", ctypes.c_uint64), ("pool_bytes", ctypes.c_uint64),
                ("pool_used", ctypes.c_uint64), ("busy_s", ctypes.c_double)]


POA_SERVER_QUEUED, POA_SERVER_RUNNING, POA_SERVER_DONE, POA_SERVER_FAILED, POA_SERVER_PARKED = range(5)


class BatchStats(ctypes.Structure):
    _fields_ = [("cells", ctypes.c_uint64), ("reads", ctypes.c_uint64), ("device_ms", ctypes.c_double),
                ("launches", ctypes.c_int32), ("relaunches", ctypes.c_int32), ("slots", ctypes.c_int32),
                ("reserved", ctypes.c_int32), ("kernel_ms", ctypes.c_double), ("dp_bytes", ctypes.c_uint64),
                ("pred_cells", ctypes.c_uint64), ("far_preds", ctypes.c_uint64), ("rows_g4", ctypes.c_uint64),
                ("rows_generic", ctypes.c_uint64), ("coop_jobs", ctypes.c_int32), ("wave_reads", ctypes.c_int32),
                ("phase_cycles", ctypes.c_uint64 * 4)]


class BatchTuning(ctypes.Structure):
    _fields_ = [("warps_per_sm", ctypes.c_int32), ("giant_alone", ctypes.c_int32), ("giant_factor", ctypes.c_double),
                ("device_ms", ctypes.c_double), ("trials", ctypes.c_int32), ("reserved2", ctypes.c_int32)]


# name -> (restype, argtypes); every function declared in include/minipoa_b200.h
P = ctypes.POINTER
_vp = ctypes.c_void_p
_i64 = ctypes.c_int64
_u64 = ctypes.c_uint64
_i32 = ctypes.c_int32
_u8p = P(ctypes.c_uint8)
_cp = P(CParams)
_ccp = P(ctypes.c_char_p)
SIGNATURES = {
    "poa_dp_backend": (ctypes.c_char_p, []),
    "poa_ctx_create": (ctypes.c_int, [ctypes.c_int, _u64, P(_vp)]),
    "poa_ctx_destroy": (None, [_vp]),
    "poa_ctx_tune_windows": (ctypes.c_int, [_vp, _i32]),
    "poa_ctx_window_stats": (ctypes.c_int, [_vp, P(_u64), P(_u64), P(_u64)]),
    "poa_last_error": (ctypes.c_char_p, [_vp]),
    "poa_free": (None, [_vp]),
    "poa_params_validate": (ctypes.c_int, [_vp, _cp]),
    "poa_graph_new": (ctypes.c_int, [_vp, _cp, P(_vp)]),
    "poa_graph_free": (None, [_vp]),
    "poa_graph_read_gfa": (ctypes.c_int, [_vp, _cp, ctypes.c_char_p, _i64, P(_vp), P(_vp), P(_i64)]),
    "poa_align_sequences": (ctypes.c_int, [_vp, _cp, _i64, P(_u8p), P(_i64), P(_vp)]),
    "poa_extend_graph": (ctypes.c_int, [_vp, _cp, _vp, _i64, P(_u8p), P(_i64), _i64]),
    "poa_align": (ctypes.c_int, [_vp, _cp, _vp, _u8p, _i64, P(P(AlignedBaseC)), P(_i64)]),
    "poa_poa": (ctypes.c_int, [_vp, _cp, _vp, _i64, _i64, _u8p, _i64, _i32, _u64, _i32, _i32,
                               P(P(AlignedBaseC)), P(_i64)]),
    "poa_graph_add_path": (ctypes.c_int, [_vp, _vp, _i64, P(AlignedBaseC), _i64]),
    "poa_graph_add_node": (ctypes.c_int, [_vp, _vp, _i64, P(_i64)]),
    "poa_graph_add_edge": (ctypes.c_int, [_vp, _vp, _i64, _i64]),
    "poa_graph_toposort": (ctypes.c_int, [_vp, _vp, _i32]),
    "poa_graph_consensus": (ctypes.c_int, [_vp, _cp, _vp, P(_u8p), P(P(_i64)), P(P(_i64)), P(_i64)]),
    "poa_graph_msa": (ctypes.c_int, [_vp, _cp, _vp, _i64, _ccp, _ccp, P(ctypes.c_char_p), P(_i64)]),
    "poa_graph_gfa": (ctypes.c_int, [_vp, _cp, _vp, _i64, _ccp, P(ctypes.c_char_p), P(_i64)]),
    "poa_graph_sizes_get": (ctypes.c_int, [_vp, _vp, P(GraphSizes)]),
    "poa_graph_export": (ctypes.c_int, [_vp, _vp] + [P(_i64)] * 10),
    "poa_batch_create": (ctypes.c_int, [_vp, _cp, _i64, P(_i64), P(_u8p), P(_i64), P(_vp)]),
    "poa_batch_run": (ctypes.c_int, [_vp, _vp, _i32, P(BatchStats)]),
    "poa_batch_status": (ctypes.c_int, [_vp, _vp, _i64, P(ctypes.c_char_p)]),
    "poa_batch_output": (ctypes.c_int, [_vp, _vp, _i64, _i32, _ccp, _ccp, P(ctypes.c_char_p), P(_i64)]),
    "poa_batch_output_all": (ctypes.c_int, [_vp, _vp, _i32, P(ctypes.c_char_p), P(_i64)]),
    "poa_batch_graph": (ctypes.c_int, [_vp, _vp, _i64, P(_vp)]),
    "poa_batch_free": (None, [_vp]),
    "poa_batch_tune": (ctypes.c_int, [_vp, _vp, _i32, _u64]),
    "poa_batch_autotune": (ctypes.c_int, [_vp, _vp, P(BatchTuning)]),
    "poa_batch_tuning_get": (ctypes.c_int, [_vp, _vp, P(BatchTuning)]),
    "poa_probe_int_peak": (ctypes.c_int, [_i32, P(ctypes.c_double)]),
    "poa_align_noalloc": (ctypes.c_int, [_vp, _cp, _vp, _vp, _i64, _vp, _i64, _vp]),
    "poa_batch_transfer_bytes": (ctypes.c_int, [_vp, _vp, P(_u64), P(_u64)]),
    "poa_server_create": (ctypes.c_int, [_vp, _cp, _u64, _i32, P(_vp)]),
    "poa_server_submit": (ctypes.c_int, [_vp, _vp, _i64, P(_u8p), P(_i64), P(_i64)]),
    "poa_server_submit_gfa": (ctypes.c_int, [_vp, _vp, ctypes.c_char_p, _i64, _i64, P(_u8p), P(_i64), P(_i64)]),
    "poa_server_wait": (ctypes.c_int, [_vp, _vp, _i64, ctypes.c_double, P(_i32)]),
    "poa_server_job_info": (ctypes.c_int, [_vp, _vp, _i64, P(ServerJobInfo)]),
    "poa_server_output": (ctypes.c_int, [_vp, _vp, _i64, _i32, _ccp, _ccp, P(ctypes.c_char_p), P(_i64)]),
    "poa_server_release": (ctypes.c_int, [_vp, _vp, _i64]),
    "poa_server_stats_get": (ctypes.c_int, [_vp, _vp, P(ServerStats)]),
    "poa_server_tune": (ctypes.c_int, [_vp, _vp, ctypes.c_double]),
    "poa_seed_sketch": (ctypes.c_int, [_u8p, _i64, _i64, _i64, P(P(MinimizerC)), P(_i64)]),
    "poa_seed_repeat_intervals": (ctypes.c_int, [P(MinimizerC), _i64, _i64, _i64, P(P(_i64)), P(_i64)]),
    "poa_seed_collect_anchors": (ctypes.c_int, [_cp, _u8p, _i64, _u8p, _i64, P(P(AnchorC)), P(_i64)]),
    "poa_seed_chain": (ctypes.c_int, [P(AnchorC), _i64, _i64, P(P(AnchorC)), P(_i64)]),
    "poa_seed_partition_windows": (ctypes.c_int, [P(AnchorC), _i64, _i64, _i64, _i64, _i64, P(P(AnchorC)), P(_i64),
                                                  P(_i32)]),
    "poa_seed_anchor_windows": (ctypes.c_int, [_cp, _u8p, _i64, _u8p, _i64, P(P(AnchorC)), P(_i64), P(_i32)]),
    "poa_seed_guide_order": (ctypes.c_int, [_cp, _i64, P(_u8p), P(_i64), P(P(_i64))]),
    "poa_server_destroy": (None, [_vp]),
}

_lib = None


def load():
    """Loads the library (raises OSError/RuntimeError when it is missing)."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise RuntimeError(
                f"{LIB_PATH} is missing: build it with `make -C minipoa-rs_b200` "
                "(there is no CPU fallback)")
        L = ctypes.CDLL(LIB_PATH)
        for name, (res, args) in SIGNATURES.items():
            fn = getattr(L, name)
            fn.restype = res
            fn.argtypes = args
        _lib = L
    return _lib
