"""ctypes binding of libb12g.so (the C ABI in include/b12g.h).

The shared library is built in-tree (``b12_b200/libb12g.so``) by ``b12_b200.build``;
importing this module never falls back to anything else: a missing library raises.
"""
from __future__ import annotations

import ctypes as C
import os

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libb12g.so")

MAX_DIM = 4
LEAF_DEPTH = 255
INVALID_INDEX = 0xFFFFFFFF

# statuses
OK, ERR_INVALID, ERR_OOM, ERR_CUDA, ERR_TIMEOUT, ERR_MIXED_DEPTH, ERR_CAPACITY, ERR_NO_DEVICE = range(8)
STATUS_NAMES = {0: "OK", 1: "INVALID", 2: "OOM", 3: "CUDA", 4: "TIMEOUT", 5: "UNSUPPORTED_MIXED_DEPTH",
                6: "CAPACITY", 7: "NO_DEVICE"}

# flags (Flags.h:10-23)
NONE, HIT, INS, EXPD, SD, EQU, ENTR, EXTR, ALL = 0x00, 0x01, 0x02, 0x04, 0x08, 0x10, 0x20, 0x40, 0xFF

MAP_HENON, MAP_LORENZ, MAP_COUPLED_DUFFING, MAP_FORCED_DUFFING = 1, 2, 3, 4
ARITH_STRICT, ARITH_FMA = 0, 1
GRID_INNER, GRID_FULL, GRID_PHILOX = 1, 2, 3


class Domain(C.Structure):
    _fields_ = [("dim", C.c_uint32), ("pad", C.c_uint32),
                ("center", C.c_double * MAX_DIM), ("radius", C.c_double * MAX_DIM)]


class Map(C.Structure):
    _fields_ = [("kind", C.c_uint32), ("arith", C.c_uint32), ("steps", C.c_uint32), ("pad", C.c_uint32),
                ("h", C.c_double), ("p", C.c_double * 6)]


class Grid(C.Structure):
    _fields_ = [("kind", C.c_uint32), ("n", C.c_uint32), ("points", C.c_uint64), ("seed", C.c_uint64),
                ("eps", C.c_double)]


class Scheme(C.Structure):
    _fields_ = [("map", Map), ("grid", Grid), ("depth", C.c_uint8), ("flags_to_check", C.c_uint8),
                ("pad", C.c_uint8 * 6)]


class Job(C.Structure):
    _fields_ = [("domain", Domain), ("map", Map), ("grid", Grid), ("depth", C.c_uint32), ("pad", C.c_uint32)]


class JobInfo(C.Structure):
    _fields_ = [("state", C.c_uint32), ("depth", C.c_uint32), ("n_boxes", C.c_uint32), ("pad", C.c_uint32),
                ("nnz", C.c_uint64), ("t_submit", C.c_double), ("t_start", C.c_double), ("t_done", C.c_double)]


JOB_WAITING, JOB_RUNNING, JOB_DONE, JOB_FAILED = 0, 1, 2, 3


class B12gError(RuntimeError):
    def __init__(self, status: int, where: str, message: str):
        super().__init__(f"{where}: {STATUS_NAMES.get(status, status)}: {message}")
        self.status = status


_lib = None

# name -> (restype, argtypes)
_SIGS = {
    "b12g_last_error": (C.c_char_p, []),
    "b12g_version": (C.c_char_p, []),
    "b12g_tree_create": (C.c_int, [C.POINTER(Domain), C.POINTER(C.c_void_p)]),
    "b12g_tree_destroy": (C.c_int, [C.c_void_p]),
    "b12g_tree_reserve": (C.c_int, [C.c_void_p, C.c_uint64]),
    "b12g_count": (C.c_int, [C.c_void_p, C.c_uint8, C.POINTER(C.c_uint32)]),
    "b12g_depth": (C.c_int, [C.c_void_p, C.POINTER(C.c_uint8)]),
    "b12g_leaves": (C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p]),
    "b12g_load_leaves": (C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_uint32]),
    "b12g_set_flags": (C.c_int, [C.c_void_p, C.c_uint8, C.c_uint8, C.POINTER(C.c_uint32)]),
    "b12g_unset_flags": (C.c_int, [C.c_void_p, C.c_uint8, C.c_uint8, C.POINTER(C.c_uint32)]),
    "b12g_change_flags": (C.c_int, [C.c_void_p, C.c_uint8, C.c_uint8, C.c_uint8, C.POINTER(C.c_uint32)]),
    "b12g_subdivide": (C.c_int, [C.c_void_p, C.c_uint8, C.POINTER(C.c_uint32)]),
    "b12g_remove": (C.c_int, [C.c_void_p, C.c_uint8, C.POINTER(C.c_uint32)]),
    "b12g_delete_depth": (C.c_int, [C.c_void_p, C.c_uint8, C.POINTER(C.c_uint32)]),
    "b12g_unsubdivide": (C.c_int, [C.c_void_p, C.c_uint8, C.POINTER(C.c_uint32)]),
    "b12g_set_flags_by_image": (C.c_int, [C.c_void_p, C.POINTER(Scheme), C.c_uint8, C.c_uint8,
                                          C.POINTER(C.c_uint32)]),
    "b12g_search_by_image": (C.c_int, [C.c_void_p, C.POINTER(Scheme), C.c_uint8, C.c_void_p, C.c_uint64,
                                       C.POINTER(C.c_uint64)]),
    "b12g_insert_points": (C.c_int, [C.c_void_p, C.c_void_p, C.c_uint64, C.c_uint8, C.c_uint8, C.c_uint8,
                                     C.POINTER(C.c_uint32)]),
    "b12g_insert_by_image": (C.c_int, [C.c_void_p, C.POINTER(Scheme), C.c_uint8, C.c_uint8, C.c_uint8,
                                       C.POINTER(C.c_uint32)]),
    "b12g_transition_matrix": (C.c_int, [C.c_void_p, C.POINTER(Scheme), C.c_int, C.c_int, C.POINTER(C.c_void_p)]),
    "b12g_image_point_boxes": (C.c_int, [C.c_void_p, C.POINTER(Scheme), C.c_void_p, C.c_void_p, C.c_uint64,
                                         C.POINTER(C.c_uint64)]),
    "b12g_image_distinct_point_boxes": (C.c_int, [C.c_void_p, C.POINTER(Scheme), C.c_uint8, C.c_void_p,
                                                  C.c_void_p, C.c_uint64, C.POINTER(C.c_uint64)]),
    "b12g_search_point_boxes": (C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p, C.c_uint64, C.c_void_p]),
    "b12g_set_flags_by_point_boxes": (C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p, C.c_uint64, C.c_uint8,
                                                C.POINTER(C.c_uint32)]),
    "b12g_transition_rows": (C.c_int, [C.c_void_p, C.c_void_p, C.c_uint32, C.c_uint32, C.c_int, C.c_int,
                                       C.POINTER(C.c_void_p)]),
    "b12g_load_leaves_device": (C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_uint32]),
    "b12g_csr_shape": (C.c_int, [C.c_void_p, C.POINTER(C.c_uint32), C.POINTER(C.c_uint32), C.POINTER(C.c_uint64)]),
    "b12g_csr_copy": (C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p]),
    "b12g_csr_destroy": (C.c_int, [C.c_void_p]),
    "b12g_invariant_measure": (C.c_int, [C.c_void_p, C.c_uint32, C.c_void_p]),
    "b12g_route_point_boxes": (C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p, C.c_uint64, C.c_void_p, C.c_void_p,
                                         C.c_uint32, C.c_uint32, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p]),
    "b12g_leaf_at": (C.c_int, [C.c_void_p, C.c_uint32, C.POINTER(C.c_uint64), C.POINTER(C.c_uint8),
                               C.POINTER(C.c_uint8)]),
    "b12g_invariant_measure_tol": (C.c_int, [C.c_void_p, C.c_double, C.c_uint32, C.c_uint32, C.c_void_p,
                                             C.POINTER(C.c_uint32), C.POINTER(C.c_double)]),
    "b12g_csr_measure": (C.c_int, [C.c_void_p, C.c_void_p]),
    "b12g_invariant_measure_noalloc": (C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p, C.c_uint32, C.c_uint32,
                                                 C.c_void_p, C.c_void_p]),
    "b12g_subdivision_run": (C.c_int, [C.c_void_p, C.POINTER(Scheme), C.c_uint32, C.c_void_p]),
    "b12g_continuation_run": (C.c_int, [C.c_void_p, C.POINTER(Scheme), C.c_void_p, C.c_uint64, C.c_uint8,
                                        C.c_uint32, C.c_void_p, C.POINTER(C.c_uint32)]),
    "b12g_batch_create": (C.c_int, [C.POINTER(Domain), C.POINTER(Scheme), C.c_uint32, C.c_void_p, C.c_void_p,
                                    C.POINTER(C.c_void_p)]),
    "b12g_batch_destroy": (C.c_int, [C.c_void_p]),
    "b12g_batch_run": (C.c_int, [C.c_void_p]),
    "b12g_batch_counts": (C.c_int, [C.c_void_p, C.c_uint32, C.c_void_p]),
    "b12g_batch_leaves": (C.c_int, [C.c_void_p, C.c_uint32, C.c_void_p, C.c_void_p, C.POINTER(C.c_uint32),
                                    C.POINTER(C.c_uint8)]),
    "b12g_batch_transition_matrices": (C.c_int, [C.c_void_p, C.c_int, C.c_int]),
    "b12g_batch_csr": (C.c_int, [C.c_void_p, C.c_uint32, C.c_void_p, C.c_void_p, C.c_void_p,
                                 C.POINTER(C.c_uint32), C.POINTER(C.c_uint64)]),
    "b12g_batch_info": (C.c_int, [C.c_void_p, C.POINTER(C.c_uint64), C.POINTER(C.c_uint64), C.POINTER(C.c_uint64),
                                  C.POINTER(C.c_uint32), C.POINTER(C.c_uint32), C.POINTER(C.c_uint32)]),
    "b12g_batch_stream": (C.c_int, [C.c_void_p, C.POINTER(C.c_void_p)]),
    "b12g_csr_strong_components": (C.c_int, [C.c_void_p, C.c_void_p, C.POINTER(C.c_uint32)]),
    "b12g_set_flags_by_components": (C.c_int, [C.c_void_p, C.c_void_p, C.c_uint32, C.c_uint8,
                                               C.POINTER(C.c_uint32)]),
    "b12g_set_flags_by_measure": (C.c_int, [C.c_void_p, C.c_void_p, C.c_double, C.c_uint8, C.POINTER(C.c_uint32)]),
    "b12g_chain_recurrent_run": (C.c_int, [C.c_void_p, C.POINTER(Scheme), C.c_uint32, C.c_void_p]),
    "b12g_nim_run": (C.c_int, [C.c_void_p, C.POINTER(Scheme), C.c_uint32, C.c_uint32, C.c_void_p]),
    "b12g_nim_run_tol": (C.c_int, [C.c_void_p, C.POINTER(Scheme), C.c_uint32, C.c_double, C.c_uint32, C.c_void_p]),
    "b12g_set_flags_by_self_hit": (C.c_int, [C.c_void_p, C.POINTER(Scheme), C.c_uint8, C.POINTER(C.c_uint32)]),
    "b12g_fixed_boxes_run": (C.c_int, [C.c_void_p, C.POINTER(Scheme), C.c_uint32, C.c_void_p]),
    "b12g_tree_save_json": (C.c_int, [C.c_void_p, C.c_char_p]),
    "b12g_tree_load_json": (C.c_int, [C.c_char_p, C.POINTER(C.c_void_p)]),
    "b12g_csr_save_json": (C.c_int, [C.c_void_p, C.c_char_p]),
    "b12g_csr_load_json": (C.c_int, [C.c_char_p, C.POINTER(C.c_void_p)]),
    "b12g_json_write_leaves": (C.c_int, [C.c_char_p, C.POINTER(Domain), C.c_void_p, C.c_void_p, C.c_void_p,
                                         C.c_uint64]),
    "b12g_json_read_leaves": (C.c_int, [C.c_char_p, C.POINTER(Domain), C.c_void_p, C.c_void_p, C.c_void_p,
                                        C.POINTER(C.c_uint64)]),
    "b12g_json_write_coo": (C.c_int, [C.c_char_p, C.c_uint32, C.c_uint32, C.c_void_p, C.c_void_p, C.c_void_p]),
    "b12g_json_read_coo": (C.c_int, [C.c_char_p, C.POINTER(C.c_uint32), C.POINTER(C.c_uint32), C.c_void_p,
                                     C.c_void_p, C.c_void_p, C.POINTER(C.c_uint64)]),
    "b12g_server_create": (C.c_int, [C.c_uint64, C.POINTER(C.c_void_p)]),
    "b12g_server_destroy": (C.c_int, [C.c_void_p]),
    "b12g_server_submit": (C.c_int, [C.c_void_p, C.POINTER(Job), C.POINTER(C.c_uint64)]),
    "b12g_server_poll": (C.c_int, [C.c_void_p, C.c_void_p, C.c_uint32, C.POINTER(C.c_uint32), C.c_double]),
    "b12g_server_job": (C.c_int, [C.c_void_p, C.c_uint64, C.POINTER(JobInfo)]),
    "b12g_server_result": (C.c_int, [C.c_void_p, C.c_uint64, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p,
                                     C.c_void_p]),
    "b12g_server_release": (C.c_int, [C.c_void_p, C.c_uint64]),
    "b12g_server_stats": (C.c_int, [C.c_void_p, C.POINTER(C.c_uint64), C.POINTER(C.c_uint64),
                                    C.POINTER(C.c_uint64), C.POINTER(C.c_uint64), C.POINTER(C.c_uint32),
                                    C.POINTER(C.c_uint32)]),
    "b12g_server_engine_stats": (C.c_int, [C.c_void_p, C.c_uint32, C.POINTER(C.c_uint32), C.POINTER(C.c_uint64),
                                           C.POINTER(C.c_uint64), C.POINTER(C.c_double), C.POINTER(C.c_double)]),
    "b12g_tree_stream": (C.c_int, [C.c_void_p, C.POINTER(C.c_void_p)]),
    "b12g_profile_enable": (C.c_int, [C.c_void_p, C.c_int]),
    "b12g_profile_read": (C.c_int, [C.c_void_p, C.c_uint32, C.POINTER(C.c_double), C.POINTER(C.c_uint64), C.c_int]),
    "b12g_launch_count": (C.c_int, [C.POINTER(C.c_uint64)]),
    "b12g_probe_fp64_fma": (C.c_int, [C.c_double, C.POINTER(C.c_double), C.POINTER(C.c_double)]),
}

# symbols the header declares (tests check that the library exports all of them)
DECLARED = sorted(_SIGS)


def lib():
    """Load libb12g.so; raises if it has not been built."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise ImportError(f"{LIB_PATH} is missing: build it with `python -m b12_b200.build`")
        L = C.CDLL(LIB_PATH)
        for name, (res, args) in _SIGS.items():
            f = getattr(L, name)
            f.restype = res
            f.argtypes = args
        _lib = L
    return _lib


def check(status: int, where: str) -> None:
    if status != OK:
        msg = lib().b12g_last_error()
        raise B12gError(status, where, msg.decode() if msg else "")
