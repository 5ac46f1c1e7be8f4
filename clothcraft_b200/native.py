"""Loader of the CUDA library (libclothcraft_b200.so) and its ctypes signatures.

There is no fallback: if the library is missing or no CUDA device is usable,
the solver classes raise instead of computing anything on the CPU.
"""
from __future__ import annotations

import ctypes as C
import os
from pathlib import Path

from .abi import (c_double_p, c_uint32_p, cc_candidates, cc_contacts, cc_grab, cc_mesh, cc_metrics,
                  cc_newton_report, cc_ogc_settings, cc_surface, cc_vbd_settings)

LIB_PATH = Path(__file__).resolve().parent / "_lib" / "libclothcraft_b200.so"
_LIB = None

# name -> (restype, argtypes); mirrors include/clothcraft.h
SIGNATURES = {
    "cc_abi_version": (C.c_int32, []),
    "cc_global_last_error": (C.c_int32, [C.c_char_p, C.c_uint64]),
    "cc_last_error": (C.c_int32, [C.c_void_p, C.c_char_p, C.c_uint64]),
    "cc_world_last_error": (C.c_int32, [C.c_void_p, C.c_char_p, C.c_uint64]),
    "cc_set_device": (C.c_int32, [C.c_int32]),
    "cc_solver_create": (C.c_int32, [C.POINTER(cc_mesh), C.POINTER(cc_surface), c_double_p, c_double_p, C.c_uint64,
                                     C.POINTER(C.c_void_p)]),
    "cc_solver_destroy": (None, [C.c_void_p]),
    "cc_solver_step": (C.c_int32, [C.c_void_p, c_double_p, c_double_p, c_double_p, C.POINTER(cc_vbd_settings),
                                   C.POINTER(cc_grab), C.POINTER(cc_metrics)]),
    "cc_solver_set_state": (C.c_int32, [C.c_void_p, c_double_p, c_double_p, C.c_double]),
    "cc_solver_get_state": (C.c_int32, [C.c_void_p, c_double_p, c_double_p, c_double_p]),
    "cc_solver_step_resident": (C.c_int32, [C.c_void_p, C.POINTER(cc_vbd_settings), C.POINTER(cc_grab),
                                            C.POINTER(cc_metrics)]),
    "cc_solver_moving": (C.c_uint64, [C.c_void_p]),
    "cc_solver_total": (C.c_uint64, [C.c_void_p]),
    "cc_solver_world": (C.c_void_p, [C.c_void_p]),
    "cc_solver_stream": (C.c_void_p, [C.c_void_p]),
    "cc_solver_set_profiling": (C.c_int32, [C.c_void_p, C.c_int32]),
    "cc_solver_set_graphs": (C.c_int32, [C.c_void_p, C.c_int32]),
    "cc_solver_set_lanes": (C.c_int32, [C.c_void_p, C.c_int32]),
    "cc_solver_get_lanes": (C.c_int32, [C.c_void_p]),
    "cc_solver_set_lanes32": (C.c_int32, [C.c_void_p, C.c_int32]),
    "cc_solver_get_lanes32": (C.c_int32, [C.c_void_p]),
    "cc_solver_colors": (C.c_int32, [C.c_void_p, c_double_p, C.c_double, C.POINTER(cc_ogc_settings),
                                     C.POINTER(cc_grab), c_uint32_p, c_uint32_p]),
    "cc_solver_local_blocks": (C.c_int32, [C.c_void_p, c_double_p, C.c_double, C.POINTER(cc_vbd_settings),
                                           C.POINTER(cc_grab), c_double_p, c_double_p, c_double_p, c_double_p,
                                           c_double_p]),
    "cc_solver_newton_step": (C.c_int32, [C.c_void_p, c_double_p, c_double_p, C.POINTER(cc_vbd_settings),
                                          C.c_uint32, C.c_uint32, C.c_double, C.c_double, c_double_p,
                                          C.POINTER(cc_newton_report)]),
    "cc_world_create": (C.c_int32, [c_double_p, C.c_uint64, c_uint32_p, C.c_uint64, C.c_uint64, c_uint32_p,
                                    C.c_uint64, C.POINTER(C.c_void_p)]),
    "cc_world_destroy": (None, [C.c_void_p]),
    "cc_world_validate_start": (C.c_int32, [C.c_void_p, c_double_p]),
    "cc_world_detect": (C.c_int32, [C.c_void_p, c_double_p, C.c_double, C.POINTER(cc_ogc_settings),
                                    C.POINTER(cc_contacts)]),
    "cc_world_candidates": (C.c_int32, [C.c_void_p, c_double_p, C.c_double, C.POINTER(cc_candidates)]),
    "cc_world_edges": (C.c_uint64, [C.c_void_p, c_uint32_p]),
    "cc_world_set_tree_rebuild_period": (C.c_int32, [C.c_void_p, C.c_int32]),
    "cc_batch_create": (C.c_int32, [C.POINTER(cc_mesh), C.POINTER(cc_surface), C.POINTER(c_double_p),
                                    C.POINTER(c_double_p), C.c_uint64, C.POINTER(C.c_void_p)]),
    "cc_batch_instances": (C.c_uint64, [C.c_void_p, C.POINTER(C.c_uint64), C.POINTER(C.c_uint64), C.c_uint64]),
    "cc_mlp_create": (C.c_int32, [C.c_uint64, C.POINTER(C.c_void_p)]),
    "cc_mlp_destroy": (None, [C.c_void_p]),
    "cc_mlp_last_error": (C.c_int32, [C.c_void_p, C.c_char_p, C.c_uint64]),
    "cc_mlp_parameter_count": (C.c_uint64, []),
    "cc_mlp_set_parameters": (C.c_int32, [C.c_void_p, C.POINTER(C.c_float), C.c_uint64]),
    "cc_mlp_get_parameters": (C.c_int32, [C.c_void_p, C.POINTER(C.c_float), C.c_uint64]),
    "cc_mlp_forward": (C.c_int32, [C.c_void_p, C.c_void_p, C.c_uint64, C.c_void_p, C.c_int32]),
    "cc_mlp_gradients": (C.c_int32, [C.c_void_p, C.c_void_p, C.c_void_p, C.c_uint64, C.POINTER(C.c_float),
                                     C.POINTER(C.c_float)]),
    "cc_mlp_train": (C.c_int32, [C.c_void_p, C.c_void_p, C.c_void_p, C.c_uint64, C.c_uint32, C.c_uint32,
                                 C.c_float, C.c_uint64, C.POINTER(C.c_float)]),
    "cc_solver_set_mlp": (C.c_int32, [C.c_void_p, C.c_void_p, C.c_int32]),
    "cc_solver_free_vertices": (C.c_uint64, [C.c_void_p]),
    "cc_solver_last_step_trace": (C.c_int32, [C.c_void_p, c_double_p, c_uint32_p, C.c_uint32]),
    "cc_solver_step_sample": (C.c_int32, [C.c_void_p, C.POINTER(cc_vbd_settings), C.POINTER(cc_grab), C.c_void_p,
                                          C.c_void_p, C.POINTER(cc_metrics)]),
    "cc_ogc_radii_noalloc": (C.c_int32, [C.c_void_p, C.c_uint64, C.c_uint64, C.c_void_p, C.c_uint64, C.c_void_p,
                                         C.c_uint64, C.c_void_p, C.c_uint64, C.c_void_p, C.c_uint64, C.c_double,
                                         C.c_double, C.c_void_p, C.c_void_p, C.c_void_p]),
}


class LibraryMissing(RuntimeError):
    pass


def load(path: str | os.PathLike | None = None):
    """Load the library (building it first if it is absent and nvcc exists)."""
    global _LIB
    if _LIB is not None:
        return _LIB
    p = Path(path) if path else LIB_PATH
    if not p.exists():
        try:
            from .build import build
            build()
        except Exception as e:  # no toolchain: fail loudly, never fall back
            raise LibraryMissing("libclothcraft_b200.so is not built and could not be built: %s" % e) from e
    L = C.CDLL(str(p))
    for name, (res, args) in SIGNATURES.items():
        fn = getattr(L, name)
        fn.restype = res
        fn.argtypes = args
    _LIB = L
    return L
