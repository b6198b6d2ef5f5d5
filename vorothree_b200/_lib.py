"""ctypes binding of libvoronoid_b200.so (the C ABI in include/voronoid_b200.h).

The library is loaded from this package directory.  There is no CPU
fallback: if the library is missing, or no CUDA device is usable, every
compute call raises.
"""
from __future__ import annotations

import ctypes as C
import os

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "libvoronoid_b200.so")

VD_OK = 0
VD_EINVAL = 1
VD_ENOMEM = 2
VD_EOVERFLOW = 3
VD_ETIMEOUT = 4
VD_ECUDA = 5
VD_ESTATE = 6
VD_EIO = 7
VD_ECANCELED = 8
VD_PREC_FP64 = 0
VD_PREC_MIXED = 1
VD_FAST_SLOTS = 0
VD_FAST_FULL = 1
FAST_LAYOUTS = {"slots": VD_FAST_SLOTS, "full": VD_FAST_FULL}


class Tuning(C.Structure):
    """vd_tuning: launch choices that change no result (0 = default)."""
    _fields_ = [("fast_layout", C.c_int), ("fast_blocks_per_sm", C.c_int), ("huge_direct_max", C.c_int),
                ("huge_blocks_max", C.c_int), ("huge_narrow_max", C.c_int), ("noop_run", C.c_int)]

STATUS_NAMES = {VD_EINVAL: "VD_EINVAL", VD_ENOMEM: "VD_ENOMEM", VD_EOVERFLOW: "VD_EOVERFLOW",
                VD_ETIMEOUT: "VD_ETIMEOUT", VD_ECUDA: "VD_ECUDA", VD_ESTATE: "VD_ESTATE", VD_EIO: "VD_EIO",
                VD_ECANCELED: "VD_ECANCELED"}

# every symbol the header declares, with its ctypes signature
_d = C.POINTER(C.c_double)
_vp = C.c_void_p
_i32p = C.POINTER(C.c_int32)
_i64p = C.POINTER(C.c_int64)
_u32p = C.POINTER(C.c_uint32)
_u64p = C.POINTER(C.c_uint64)
_szp = C.POINTER(C.c_size_t)
SIGNATURES = {
    "vd_tess_create": (C.c_int, [_d, _d, C.c_int, C.c_int, C.c_int, C.POINTER(_vp)]),
    "vd_tess_destroy": (C.c_int, [_vp]),
    "vd_tess_reset": (C.c_int, [_vp, _d, _d, C.c_int, C.c_int, C.c_int]),
    "vd_last_error": (C.c_char_p, [_vp]),
    "vd_tess_add_wall_plane": (C.c_int, [_vp, _d, _d, C.c_int]),
    "vd_tess_add_wall_sphere": (C.c_int, [_vp, _d, C.c_double, C.c_int]),
    "vd_tess_add_wall_cylinder": (C.c_int, [_vp, _d, _d, C.c_double, C.c_int]),
    "vd_tess_add_wall_cone": (C.c_int, [_vp, _d, _d, C.c_double, C.c_int]),
    "vd_tess_add_wall_torus": (C.c_int, [_vp, _d, _d, C.c_double, C.c_double, C.c_int]),
    "vd_tess_add_wall_polyhedron": (C.c_int, [_vp, _d, _d, C.c_int, C.c_int]),
    "vd_tess_clear_walls": (C.c_int, [_vp]),
    "vd_tess_set_generators": (C.c_int, [_vp, _d, C.c_size_t, _szp]),
    "vd_tess_set_generators_device": (C.c_int, [_vp, _vp, C.c_size_t, _szp]),
    "vd_tess_set_generator": (C.c_int, [_vp, C.c_size_t, _d]),
    "vd_tess_random_generators": (C.c_int, [_vp, C.c_size_t, C.c_uint64, _szp]),
    "vd_tess_read_generators": (C.c_int, [_vp, C.c_char_p, C.c_size_t, _szp]),
    "vd_tess_import_generators": (C.c_int, [_vp, C.c_char_p, _szp]),
    "vd_parse_generators": (C.c_int, [C.c_char_p, C.c_size_t, _d, C.c_size_t, _szp]),
    "vd_tess_count_generators": (C.c_int, [_vp, _szp]),
    "vd_tess_get_generators": (C.c_int, [_vp, _d]),
    "vd_tess_set_precision": (C.c_int, [_vp, C.c_int]),
    "vd_tess_set_fast_layout": (C.c_int, [_vp, C.c_int]),
    "vd_tess_set_tuning": (C.c_int, [_vp, _vp]),
    "vd_tess_get_tuning": (C.c_int, [_vp, _vp]),
    "vd_tess_calculate": (C.c_int, [_vp]),
    "vd_tess_calculate_range": (C.c_int, [_vp, C.c_size_t, C.c_size_t]),
    "vd_tess_calculate_strided": (C.c_int, [_vp, C.c_size_t, C.c_size_t, C.c_size_t, C.c_size_t, C.c_size_t]),
    "vd_tess_relax": (C.c_int, [_vp]),
    "vd_tess_calculate_sealed": (C.c_int, [_vp]),
    "vd_tess_prune_boundaries": (C.c_int, [_vp]),
    "vd_tess_seal_log": (C.c_int, [_vp, _vp, _szp]),
    "vd_tess_prune_log": (C.c_int, [_vp, _vp, _szp, _vp, _szp]),
    "vd_tess_count_cells": (C.c_int, [_vp, _szp]),
    "vd_tess_get_cell_summaries": (C.c_int, [_vp, _vp, _vp, _vp]),
    "vd_tess_total_faces": (C.c_int, [_vp, _i64p]),
    "vd_tess_get_neighbors": (C.c_int, [_vp, _vp, _vp]),
    "vd_tess_get_face_areas": (C.c_int, [_vp, _vp, _vp]),
    "vd_tess_get_cell": (C.c_int, [_vp, C.c_size_t, _i32p, _i32p, _i32p, _vp, _vp, _vp, _vp]),
    "vd_wall_contains": (C.c_int, [_vp, _d, C.POINTER(C.c_int)]),
    "vd_wall_cut": (C.c_int, [_vp, _d, _d, _d, C.c_int, C.POINTER(C.c_int)]),
    "vd_search_order": (C.c_int, [_d, _d, C.c_int, C.c_int, C.c_int, C.c_int, _i32p, _d, C.c_size_t, _szp,
                                  C.POINTER(C.c_int), _d]),
    "vd_grid_bin_index": (C.c_int, [_d, _d, C.c_int, C.c_int, C.c_int, _d, _szp]),
    "vd_tess_export_cells": (C.c_int, [_vp, C.c_size_t, C.c_size_t, _i64p, _i64p, _i64p, _vp, _vp, _vp, _vp]),
    "vd_tess_device_results": (C.c_int, [_vp, C.POINTER(_vp), C.POINTER(_vp), C.POINTER(_vp)]),
    "vd_tess_device_neighbors": (C.c_int, [_vp, C.POINTER(_vp), C.POINTER(_vp), C.POINTER(_vp), C.POINTER(C.c_int64)]),
    "vd_tess_stream": (C.c_int, [_vp, C.POINTER(_vp)]),
    "vd_tess_timings": (C.c_int, [_vp, C.POINTER(C.c_float)]),
    "vd_tess_counters": (C.c_int, [_vp, _u64p]),
    "vd_tess_set_instrumentation": (C.c_int, [_vp, C.c_int]),
    "vd_tess_fallback_counts": (C.c_int, [_vp, _u64p]),
    "vd_launch_count": (C.c_int, [_u64p]),
    "vd_host_alloc": (C.c_int, [C.c_size_t, C.POINTER(_vp)]),
    "vd_host_free": (C.c_int, [_vp]),
    "vd_measure_fma_peak": (C.c_int, [C.c_int, _d]),
    "vd_batch_create": (C.c_int, [C.POINTER(_vp)]),
    "vd_batch_destroy": (C.c_int, [_vp]),
    "vd_batch_last_error": (C.c_char_p, [_vp]),
    "vd_batch_add": (C.c_int, [_vp, _d, _d, C.c_int, C.c_int, C.c_int, _vp, C.c_int, _d, C.c_size_t,
                               C.POINTER(C.c_int)]),
    "vd_batch_set_precision": (C.c_int, [_vp, C.c_int]),
    "vd_batch_set_fast_layout": (C.c_int, [_vp, C.c_int]),
    "vd_batch_set_instrumentation": (C.c_int, [_vp, C.c_int]),
    "vd_batch_reset": (C.c_int, [_vp]),
    "vd_batch_commit": (C.c_int, [_vp]),
    "vd_batch_calculate": (C.c_int, [_vp]),
    "vd_batch_lloyd": (C.c_int, [_vp, C.c_int]),
    "vd_batch_count": (C.c_int, [_vp, C.POINTER(C.c_int)]),
    "vd_batch_count_cells": (C.c_int, [_vp, C.c_int, _szp]),
    "vd_batch_total_cells": (C.c_int, [_vp, _szp]),
    "vd_batch_get_generators": (C.c_int, [_vp, C.c_int, _d]),
    "vd_batch_get_summaries": (C.c_int, [_vp, C.c_int, _vp, _vp, _vp]),
    "vd_batch_timing": (C.c_int, [_vp, C.POINTER(C.c_float)]),
    "vd_batch_counters": (C.c_int, [_vp, _u64p]),
    "vd_batch_stream": (C.c_int, [_vp, C.POINTER(_vp)]),
    "vd_server_create": (C.c_int, [C.c_int, C.c_size_t, C.c_int, C.POINTER(_vp)]),
    "vd_server_destroy": (C.c_int, [_vp]),
    "vd_server_last_error": (C.c_char_p, [_vp]),
    "vd_server_submit": (C.c_int, [_vp, _d, _d, C.c_int, C.c_int, C.c_int, _vp, C.c_int, _d, C.c_size_t,
                                   C.POINTER(C.c_uint64)]),
    "vd_server_submit_text": (C.c_int, [_vp, _d, _d, C.c_int, C.c_int, C.c_int, _vp, C.c_int, C.c_char_p,
                                        C.c_size_t, C.POINTER(C.c_uint64)]),
    "vd_server_wait": (C.c_int, [_vp, C.c_uint64, _szp, _d]),
    "vd_server_take": (C.c_int, [_vp, C.c_uint64, _vp, _vp, _vp]),
    "vd_server_stats": (C.c_int, [_vp, _u64p, _u64p, _d, _d, _szp]),
    "vd_server_reset_stats": (C.c_int, [_vp]),
    "vd_server_concurrency": (C.c_int, [_vp, C.POINTER(C.c_int), C.POINTER(C.c_int)]),
    "vd_server_set_face_results": (C.c_int, [_vp, C.c_int]),
    "vd_server_total_faces": (C.c_int, [_vp, C.c_uint64, C.POINTER(C.c_int64)]),
    "vd_server_take_faces": (C.c_int, [_vp, C.c_uint64, _vp, _vp, _vp, _vp, _vp, _vp]),
    "vd_server_cancel": (C.c_int, [_vp, C.c_uint64]),
    "vd_server_set_merging": (C.c_int, [_vp, C.c_int, C.c_size_t, C.c_size_t]),
    "vd_server_merge_stats": (C.c_int, [_vp, _u64p, _u64p]),
    "vd_debug_fail_allocations": (C.c_int, [C.c_int]),
    "vd_cell_last_error": (C.c_char_p, [_vp]),
    "vd_cell_create_box": (C.c_int, [C.c_size_t, _d, _d, C.POINTER(_vp)]),
    "vd_cell_create": (C.c_int, [C.c_size_t, C.c_int32, C.c_int32, _vp, _vp, _vp, _vp, C.POINTER(_vp)]),
    "vd_cell_destroy": (C.c_int, [_vp]),
    "vd_cell_id": (C.c_int, [_vp, _szp]),
    "vd_cell_clip": (C.c_int, [_vp, _d, _d, C.c_int32, _d, C.POINTER(C.c_int), _d]),
    "vd_cell_max_radius_sq": (C.c_int, [_vp, _d, _d]),
    "vd_cell_measure": (C.c_int, [_vp, _d, _d, _i32p, _vp, _vp]),
    "vd_cell_get": (C.c_int, [_vp, _i32p, _i32p, _i32p, _vp, _vp, _vp, _vp]),
    "vd_calculate_noalloc": (C.c_int, [_d, _d, C.c_int, C.c_int, C.c_int, _vp, C.c_size_t, _vp, _vp, _vp,
                                       _vp]),
}

_lib = None


class VoronoidError(RuntimeError):
    def __init__(self, code: int, msg: str):
        super().__init__(f"{STATUS_NAMES.get(code, code)}: {msg}")
        self.code = code


def load():
    """Load the library (building it first if this checkout has nvcc)."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        from . import build as _build
        _build.build()
    L = C.CDLL(LIB_PATH)
    for name, (res, args) in SIGNATURES.items():
        f = getattr(L, name)
        f.restype = res
        f.argtypes = args
    _lib = L
    return L


def check(rc: int, handle=None):
    if rc != VD_OK:
        msg = load().vd_last_error(handle)
        raise VoronoidError(rc, msg.decode() if msg else "")
