"""Loads the in-tree CUDA library (nricp_b200/libnricp_b200.so) and declares
its C ABI.  There is no fallback: a missing or unloadable library raises."""

from __future__ import annotations

import ctypes as C
import os
from pathlib import Path

from . import _abi

_HERE = Path(__file__).resolve().parent
# NRICP_B200_LIBRARY may name another build of the same library (the
# measurement variant of build.build_fp32_reductions); it is never built here.
LIB_PATH = Path(os.environ["NRICP_B200_LIBRARY"]) if os.environ.get("NRICP_B200_LIBRARY") else \
    _HERE / "libnricp_b200.so"
_lib: C.CDLL | None = None


class NativeLibraryMissing(RuntimeError):
    pass


def load(build_if_missing: bool = True) -> C.CDLL:
    global _lib
    if _lib is not None:
        return _lib
    if (not LIB_PATH.exists() and build_if_missing and os.environ.get("NRICP_NO_BUILD") != "1"
            and not os.environ.get("NRICP_B200_LIBRARY")):
        from . import build as _build  # compiles with nvcc for sm_100a
        _build.build()
    if not LIB_PATH.exists():
        raise NativeLibraryMissing(
            f"{LIB_PATH} is not built; run `python -m nricp_b200.build` (nvcc, sm_100a). "
            "The wrapping path has no CPU fallback.")
    lib = C.CDLL(str(LIB_PATH))
    _declare(lib)
    _lib = lib
    return lib


def _declare(lib: C.CDLL) -> None:
    P = C.POINTER
    i32p, dp, u32p, fp = P(C.c_int32), P(C.c_double), P(C.c_uint32), P(C.c_float)
    desc_p, result_p = P(_abi.SolveDesc), P(_abi.Result)
    sig = {
        "nricp_last_error": (C.c_char_p, []),
        "nricp_transfer_counters": (C.c_int, [P(C.c_ulonglong), P(C.c_ulonglong), C.c_int]),
        "nricp_device_info": (C.c_int, [P(C.c_int), C.c_char_p, C.c_size_t]),
        "nricp_plan": (C.c_int, [desc_p, i32p, C.c_int, P(C.c_int)]),
        "nricp_solve": (C.c_int, [desc_p, result_p]),
        "nricp_session_create": (C.c_int, [desc_p, P(C.c_void_p)]),
        "nricp_session_step": (C.c_int, [C.c_void_p, P(_abi.Progress)]),
        "nricp_session_run": (C.c_int, [C.c_void_p]),
        "nricp_session_finished": (C.c_int, [C.c_void_p, P(C.c_int)]),
        "nricp_session_vertices": (C.c_int, [C.c_void_p, dp]),
        "nricp_session_result": (C.c_int, [C.c_void_p, result_p]),
        "nricp_session_ticks": (C.c_int, [C.c_void_p, P(C.c_long), P(C.c_long)]),
        "nricp_session_destroy": (None, [C.c_void_p]),
        "nricp_session_inspect": (C.c_int, [C.c_void_p, P(_abi.Inspect)]),
        "nricp_batch_create": (C.c_int, [desc_p, C.c_int, P(C.c_void_p)]),
        "nricp_batch_reset": (C.c_int, [C.c_void_p]),
        "nricp_batch_run": (C.c_int, [C.c_void_p]),
        "nricp_batch_result": (C.c_int, [C.c_void_p, C.c_int, result_p]),
        "nricp_batch_counters": (C.c_int, [C.c_void_p, P(C.c_long), P(C.c_long)]),
        "nricp_batch_profile": (C.c_int, [C.c_void_p, dp, dp, dp, P(C.c_long)]),
        "nricp_batch_destroy": (None, [C.c_void_p]),
        "nricp_batch_step": (C.c_int, [C.c_void_p, dp]),
        "nricp_batch_tune": (C.c_int, [C.c_void_p, C.c_int, P(C.c_int)]),
        "nricp_batch_tick_records": (C.c_int, [C.c_void_p, P(_abi.TickRecord), C.c_int, P(C.c_int)]),
        "nricp_batch_level_sizes": (C.c_int, [C.c_void_p, C.c_int, C.c_int, i32p]),
        "nricp_batch_solve": (C.c_int, [desc_p, C.c_int, result_p]),
        "nricp_template_graph_level": (C.c_int, [dp, C.c_int, C.c_int, C.c_int, C.c_int, C.c_int,
                                                 C.c_int, C.c_int, dp, dp, i32p, dp, i32p, dp, i32p,
                                                 i32p, C.c_int, P(C.c_int), C.c_int]),
        "nricp_closest_points": (C.c_int, [dp, C.c_int, i32p, C.c_int, dp, C.c_int, dp, dp, dp, i32p]),
        "nricp_fit_rigid": (C.c_int, [dp, dp, dp, C.c_int, dp, dp]),
        "nricp_farthest_point_seeds": (C.c_int, [dp, C.c_int, C.c_int, C.c_int, i32p, P(C.c_int)]),
        "nricp_bind_vertices": (C.c_int, [dp, C.c_int, dp, C.c_int, C.c_int, i32p, dp, i32p]),
        "nricp_vertex_normals": (C.c_int, [dp, C.c_int, i32p, C.c_int, dp]),
        "nricp_lbvh_export": (C.c_int, [dp, C.c_int, i32p, C.c_int, u32p, u32p, i32p, i32p, fp]),
        "nricp_lbvh_export_static": (C.c_int, [C.c_void_p, C.c_int, C.c_void_p, C.c_int,
                                               C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p,
                                               C.c_void_p, C.c_void_p]),
        "nricp_server_default_config": (None, [P(_abi.ServerConfig)]),
        "nricp_server_create": (C.c_int, [P(_abi.ServerConfig), P(C.c_void_p)]),
        "nricp_server_submit": (C.c_int, [C.c_void_p, desc_p, P(C.c_long)]),
        "nricp_server_poll": (C.c_int, [C.c_void_p, C.c_long, P(C.c_int), P(C.c_double)]),
        "nricp_server_phases": (C.c_int, [C.c_void_p, C.c_long, P(C.c_double)]),
        "nricp_server_wait": (C.c_int, [C.c_void_p, C.c_long, C.c_double]),
        "nricp_server_result": (C.c_int, [C.c_void_p, C.c_long, result_p]),
        "nricp_server_stats": (C.c_int, [C.c_void_p, P(_abi.ServerStats)]),
        "nricp_server_destroy": (None, [C.c_void_p]),
        "nricp_default_desc": (None, [desc_p]),
        "nricp_default_level": (None, [P(_abi.LevelSettings)]),
    }
    for name, (restype, argtypes) in sig.items():
        fn = getattr(lib, name)
        fn.restype = restype
        fn.argtypes = argtypes


def check(status: int) -> None:
    """Turns a status into the exception the reference raises for it."""
    if status == _abi.OK:
        return
    message = load().nricp_last_error().decode()
    if status == _abi.ERR_INVALID:
        raise ValueError(message)
    raise RuntimeError(message)
