"""ctypes binding of liborsp.so (the C ABI in include/orsp.h).

The library is the only compute path: importing a function that needs it on
a machine where it is missing raises immediately; nothing falls back to CPU.
"""
from __future__ import annotations

import ctypes
import os
from pathlib import Path

_PKG = Path(__file__).resolve().parent
LIB_PATH = Path(os.environ.get("ORSP_LIBRARY", _PKG / "liborsp.so"))

ORSP_OK = 0
ORSP_NO_PATH = 1
ORSP_ERR_ARG = -1
ORSP_ERR_CUDA = -2
ORSP_ERR_TIMEOUT = -3
ORSP_ERR_OVERFLOW = -4
ORSP_ERR_NOMEM = -5
ORSP_ERR_INTERNAL = -6


class OrspError(RuntimeError):
    def __init__(self, status: int, where: str, msg: str):
        super().__init__(f"{where}: status {status}: {msg}")
        self.status = status


_P = ctypes.c_void_p
_i32 = ctypes.c_int32
_i64 = ctypes.c_int64
_f32 = ctypes.c_float
_u = ctypes.c_size_t  # uintptr_t stream

# name -> (restype, argtypes)
_SIGS = {
    "orsp_abi_version": (ctypes.c_int, []),
    "orsp_status_string": (ctypes.c_char_p, [ctypes.c_int]),
    "orsp_last_error": (ctypes.c_char_p, []),
    "orsp_profile_enable": (ctypes.c_int, [ctypes.c_int]),
    "orsp_profile_last": (ctypes.c_int, [ctypes.POINTER(_f32)]),
    "orsp_profile_counters": (ctypes.c_int, [ctypes.POINTER(_i64)]),
    "orsp_graph_create": (ctypes.c_int, [_i32, _i64, _P, _P, _i32, _i32, _i32, ctypes.c_int, ctypes.POINTER(_P)]),
    "orsp_graph_destroy": (ctypes.c_int, [_P]),
    "orsp_graph_csr": (ctypes.c_int, [_P, ctypes.POINTER(_P), ctypes.POINTER(_P)]),
    "orsp_graph_max_degree": (ctypes.c_int, [_P, ctypes.POINTER(_i32)]),
    "orsp_graph_is_lattice": (ctypes.c_int, [_P, ctypes.POINTER(_i32)]),
    "orsp_lattice_max_layers": (ctypes.c_int, [_i32, ctypes.POINTER(_i32)]),
    "orsp_graph_cost_generation": (ctypes.c_int, [_P, _P, ctypes.c_uint64]),
    "orsp_sssp": (ctypes.c_int, [_P, _P, _i32, _P, _P, _i32, _P, _f32, _P, _P, _i32,
                                 ctypes.POINTER(_i32), ctypes.POINTER(_i32), _u]),
    "orsp_sssp_box": (ctypes.c_int, [_P, _P, _i32, _P, _P, _i32, _P, _f32, _P, _P, _i32,
                                     ctypes.POINTER(_i32), ctypes.POINTER(_i32), _u]),
    "orsp_sssp_sources": (ctypes.c_int, [_P, _P, _i32, _P, _P, _i32, _u]),
    "orsp_sssp_roi_nodes": (ctypes.c_int, [_P, _P, _i32, _i32, _P, _i64, _P, _i32, ctypes.POINTER(_i32), _u]),
    "orsp_batch_set_plan": (ctypes.c_int, [_P, _i32, _P, _P, _P, _P, _P]),
    "orsp_warm_conv3d": (ctypes.c_int, [_P, _P, _P, _P, _P, _P, _i32, _i32, _i32, _i32, _i32, _i32, _u]),
    "orsp_warm_conv3d_tc": (ctypes.c_int, [_P, _P, _P, _P, _P, _P, _i32, _i32, _i32, _i32, _i32, _i32, _u]),
    "orsp_warm_tc_status": (ctypes.c_int, [ctypes.POINTER(_i32)]),
    "orsp_warm_wgrad_tc": (ctypes.c_int, [_P, _P, _P, _P, _P, _i32, _i32, _i32, _i32, _i32, _u]),
    "orsp_warm_wgrad": (ctypes.c_int, [_P, _P, _P, _P, _P, _i32, _i32, _i32, _i32, _i32, _u]),
    "orsp_warm_pool": (ctypes.c_int, [_P, _P, _i32, _i32, _i32, _i32, _u]),
    "orsp_warm_spread": (ctypes.c_int, [_P, _P, _i32, _i32, _i32, _i32, _f32, _u]),
    "orsp_warm_gather4": (ctypes.c_int, [_P, _P, _i32, _i32, _i32, _i32, _u]),
    "orsp_warm_add": (ctypes.c_int, [_P, _P, _P, _i64, _u]),
    "orsp_warm_mse": (ctypes.c_int, [_P, _P, _P, _P, _P, _i64, _i32, _i32, _f32, _u]),
    "orsp_warm_adam": (ctypes.c_int, [_P, _P, _P, _P, _i64, _f32, _f32, _f32, _f32, _f32, _u]),
    "orsp_warm_pack_weights": (ctypes.c_int, [_P, _P, _i32, _i32, _i32, _u]),
    "orsp_node_owner": (ctypes.c_int, [_P, _i32, _P, _P, _P, _i32, _P, _P, _P, _u]),
    "orsp_barrel_conflicts": (ctypes.c_int, [_P, _i32, _P, _P, _P, _P, _P, ctypes.POINTER(_i64), _u]),
    "orsp_barrel_penalty": (ctypes.c_int, [_i64, _P, _P, _f32, _u]),
    "orsp_net_scores": (ctypes.c_int, [_P, _i32, _P, _P, _P, _P, _P, _P, _P, _P, ctypes.POINTER(_i64), _u]),
    "orsp_emit_geometry": (ctypes.c_int, [_P, _i32, _P, _P, _P, _P, _P, _P, _P, _u]),
    "orsp_route_nets": (ctypes.c_int, [_P, _i32, _P, _P, _P, _i32, _P, _i32, _P, _P, _P, _i32, _P, _P, _P, _P, _P,
                                       _P, _P, _f32, _f32, _f32, _f32, _i32, _u]),
    "orsp_route_nets_snapshot": (ctypes.c_int, [_P, _i32, _P, _P, _P, _i32, _P, _i32, _P, _i32, _P, _P, _i32, _P,
                                                _P, _P, _P, _P, _P, _P, _f32, _f32, _f32, _f32, _i32,
                                                ctypes.POINTER(_i64), _u]),
    "orsp_sssp_multi": (ctypes.c_int, [_P, _P, _i32, _P, _P, _i32, _P, _P, _P, _f32, _P, _i32,
                                       ctypes.POINTER(_i32), ctypes.POINTER(_i32), _u]),
    "orsp_roi_from_bitmap": (ctypes.c_int, [_P, _P, _P, _u]),
    "orsp_sssp_batch_bbox": (ctypes.c_int, [_P, _P, _i32, _P, _P, _P, _P, _f32, _P, _P, _i32, _P, _u]),
    "orsp_sssp_batch_ranges": (ctypes.c_int, [_P, _P, _i32, _P, _P, _P, _P, _f32, _P, _P, _i32, _P, _u]),
    "orsp_roi_bfs": (ctypes.c_int, [_P, _i32, _i32, _i32, _i32, _P, _P, ctypes.POINTER(_i32), _u]),
    "orsp_roi_bfs_noalloc": (ctypes.c_int, [_P, _i32, _i32, _i32, _i32, _P, _P, ctypes.POINTER(_i32), _u]),
    "orsp_roi_bfs_keep": (ctypes.c_int, [_P, _i32, _i32, _i32, _i32, _P, _i32, _P, _P, ctypes.POINTER(_i32), _u]),
    "orsp_roi_box_map": (ctypes.c_int, [_P, _P, _P, _u]),
    "orsp_path_to_edges": (ctypes.c_int, [_P, _P, _i32, _P, ctypes.POINTER(_i32), _u]),
    "orsp_update_costs": (ctypes.c_int, [_i64, _P, _P, _P, _P, _P, _P, _P, _f32, _f32, _f32, _f32,
                                         ctypes.c_int, _P, _u]),
    "orsp_update_costs_live": (ctypes.c_int, [_i64, _P, _i64, _P, _P, _P, _P, _f32, _f32, _f32, _f32,
                                              ctypes.c_int, _P, _u]),
    "orsp_update_costs_live_paths": (ctypes.c_int, [_i32, _P, _P, _i32, _P, _P, _P, _P, _f32, _f32, _f32,
                                                    _f32, ctypes.c_int, _P, _u]),
    "orsp_via_usage": (ctypes.c_int, [_P, _i32, _P, _P, _i32, _P, _P, _u]),
    "orsp_via_present": (ctypes.c_int, [_i64, _i32, _P, _P, _P, _P, _P, _P, _P, _f32, _f32, _u]),
    "orsp_via_penalties": (ctypes.c_int, [_P, _P, _P, _P, ctypes.c_int, ctypes.c_double, _f32, _f32, _f32, _P, _u]),
    "orsp_via_hard_block": (ctypes.c_int, [_P, _P, _P, _P, _P, _P, _u]),
    "orsp_update_present_ema": (ctypes.c_int, [_i64, _P, _P, _f32, _f32, _u]),
    "orsp_update_history": (ctypes.c_int, [_i64, _P, _P, _P, _P, _f32, _f32, _f32, _u]),
    "orsp_overuse": (ctypes.c_int, [_i64, _P, _P, _P, _P, _u]),
    "orsp_present_from_usage": (ctypes.c_int, [_i64, _P, _P, _u]),
    "orsp_commit_edges": (ctypes.c_int, [_i64, _P, _P, _P, _i32, _u]),
    "orsp_commit_batch": (ctypes.c_int, [_i32, _P, _P, _i32, _P, _P, _i32, _u]),
}

_lib = None


def load() -> ctypes.CDLL:
    """Loads liborsp.so; raises if it has not been built."""
    global _lib
    if _lib is not None:
        return _lib
    if not LIB_PATH.exists():
        raise RuntimeError(
            f"liborsp.so not found at {LIB_PATH}; build it with "
            "`python -c 'import __graft_entry__ as g; g.build()'` (nvcc, sm_100a)"
        )
    lib = ctypes.CDLL(str(LIB_PATH))
    for name, (res, args) in _SIGS.items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    _lib = lib
    return lib


def exported_symbols():
    return list(_SIGS)


def check(status: int, where: str) -> int:
    """Raises OrspError for negative statuses; returns ORSP_OK / ORSP_NO_PATH."""
    if status < 0:
        lib = load()
        msg = lib.orsp_last_error().decode(errors="replace")
        raise OrspError(status, where, msg)
    return status


def ptr(t) -> ctypes.c_void_p:
    """Device (torch) or host (numpy) array -> void*; None -> NULL."""
    if t is None:
        return None
    if hasattr(t, "data_ptr"):
        return ctypes.c_void_p(t.data_ptr())
    return t.ctypes.data_as(ctypes.c_void_p)
