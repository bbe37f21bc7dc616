"""ctypes binding of ``libm3lb.so`` (declarations in ``include/m3lb.h``).

The library is built in-tree (``python -m m3lb_b200.build``).  Loading fails
loudly when it is missing: there is no fallback implementation.
"""
from __future__ import annotations

import ctypes as C
from pathlib import Path

LIB_PATH = Path(__file__).resolve().parent / "libm3lb.so"
HEADER = Path(__file__).resolve().parent.parent / "include" / "m3lb.h"

OK = 0
ERR_INVALID = -1
ERR_UNSUPPORTED = -2
ERR_CUDA = -3
ERR_MEMORY = -4

OP_NONE, OP_BGK, OP_TRT, OP_MRT, OP_CM = 0, 1, 2, 3, 4
EQ_SECOND_ORDER, EQ_PRODUCT_FORM = 0, 1
STORE_F32, STORE_F16, STORE_BF16, STORE_F64, STORE_F16C = 0, 1, 2, 3, 4
OPT_NODE_KERNEL = 1
OPT_KERNEL = 2
OPT_WAIT_CYCLES = 3  # test only: shorten the row kernel's wait for its copies
KERNEL_AUTO, KERNEL_NODES, KERNEL_PAIRS, KERNEL_STREAM, KERNEL_ROWS = 0, 1, 2, 3, 4
MAP_AUTO, MAP_CHUNKS, MAP_DENSE, MAP_TUNE, MAP_ROWS = 0, 1, 2, 3, 4

STORAGE_NAMES = {"f32": STORE_F32, "f16": STORE_F16, "bf16": STORE_BF16, "f64": STORE_F64,
                 "f16c": STORE_F16C}
STORAGE_BYTES = {STORE_F32: 4, STORE_F16: 2, STORE_BF16: 2, STORE_F64: 8, STORE_F16C: 2}


class M3lbError(RuntimeError):
    def __init__(self, code: int, msg: str):
        super().__init__(f"m3lb error {code}: {msg}")
        self.code = code


class ServeConfig(C.Structure):
    """m3lb_serve_config."""
    _fields_ = [("hbm_budget", C.c_size_t), ("max_resident", C.c_int),
                ("round_steps", C.c_int), ("storage", C.c_int), ("keep_fields", C.c_int),
                ("mapping", C.c_int)]


class Request(C.Structure):
    """m3lb_request."""
    _fields_ = [("id", C.c_longlong), ("arrival", C.c_double), ("n", C.c_int), ("op", C.c_int),
                ("steps", C.c_int), ("u0", C.c_double), ("omega", C.c_double),
                ("omega2", C.c_double)]


class Result(C.Structure):
    """m3lb_result."""
    _fields_ = [("id", C.c_longlong), ("arrival", C.c_double), ("admitted", C.c_double),
                ("finished", C.c_double), ("n", C.c_int), ("op", C.c_int), ("steps", C.c_int),
                ("status", C.c_int), ("node_steps", C.c_longlong), ("mass", C.c_double),
                ("momentum", C.c_double * 3), ("energy", C.c_double)]


class ServeStats(C.Structure):
    """m3lb_serve_stats."""
    _fields_ = [("rounds", C.c_longlong), ("launches", C.c_longlong),
                ("graph_captures", C.c_longlong), ("graph_launches", C.c_longlong),
                ("finished", C.c_longlong), ("node_steps", C.c_longlong),
                ("makespan", C.c_double), ("dense_launches", C.c_longlong),
                ("tuned_mapping", C.c_int), ("tuned_chunks_mlups", C.c_double),
                ("tuned_dense_mlups", C.c_double), ("rows_launches", C.c_longlong),
                ("tuned_rows_mlups", C.c_double)]


_vp = C.c_void_p
_i = C.c_int
_d = C.c_double
_pp = C.POINTER(C.c_void_p)

# name -> (restype, argtypes); every entry point of include/m3lb.h
SIGNATURES = {
    "m3lb_last_error": (C.c_char_p, []),
    "m3lb_footprint": (_i, [_i] * 8 + [C.POINTER(C.c_size_t)]),
    "m3lb_create": (_i, [_i] * 12 + [_pp]),
    "m3lb_destroy": (_i, [_vp]),
    "m3lb_set_params": (_i, [_vp] + [_d] * 5),
    "m3lb_set_flags": (_i, [_vp, _vp]),
    "m3lb_set_specular_walls": (_i, [_vp, _vp]),
    "m3lb_set_specular_nodes": (_i, [_vp, _vp]),
    "m3lb_set_regularized_walls": (_i, [_vp, _vp, _vp]),
    "m3lb_set_wall_velocity_scale": (_i, [_vp, _d]),
    "m3lb_set_wall_density": (_i, [_vp, _d]),
    "m3lb_set_wall_velocity_field": (_i, [_vp, _vp]),
    "m3lb_set_wall_velocity_field_scale": (_i, [_vp, _d]),
    "m3lb_set_fd_corners": (_i, [_vp, _i]),
    "m3lb_set_force_correction": (_i, [_vp, _i]),
    "m3lb_set_outflow_order": (_i, [_vp, _i]),
    "m3lb_set_outflow_density": (_i, [_vp, _d]),
    "m3lb_set_buoyancy": (_i, [_vp, _vp] + [_d] * 6),
    "m3lb_set_buoyancy_host": (_i, [_vp, _vp] + [_d] * 6),
    "m3lb_stream_order": (_i, [_vp, _vp]),
    "m3lb_scalar_set_velocity_host": (_i, [_vp] * 4),
    "m3lb_scalar_get_stream": (_i, [_vp, _pp]),
    "m3lb_macro_pointers": (_i, [_vp] + [_pp] * 4),
    "m3lb_get_stream": (_i, [_vp, _pp]),
    "m3lb_scalar_create": (_i, [_i] * 9 + [_pp]),
    "m3lb_scalar_destroy": (_i, [_vp]),
    "m3lb_scalar_set_params": (_i, [_vp] + [_d] * 3),
    "m3lb_scalar_set_stream": (_i, [_vp, _vp]),
    "m3lb_scalar_set_cells": (_i, [_vp, _vp]),
    "m3lb_scalar_set_wall_values": (_i, [_vp, _vp]),
    "m3lb_scalar_set_specular_walls": (_i, [_vp, _vp]),
    "m3lb_scalar_set_specular_nodes": (_i, [_vp, _vp]),
    "m3lb_scalar_set_omega_field": (_i, [_vp, _vp]),
    "m3lb_scalar_set_velocity_device": (_i, [_vp] * 4),
    "m3lb_scalar_finalize_geometry": (_i, [_vp]),
    "m3lb_scalar_init": (_i, [_vp, _d]),
    "m3lb_scalar_init_field": (_i, [_vp, _vp]),
    "m3lb_scalar_step": (_i, [_vp, _i]),
    "m3lb_scalar_add_source": (_i, [_vp, _vp]),
    "m3lb_scalar_add_source_device": (_i, [_vp, _vp]),
    "m3lb_scalar_compute_field": (_i, [_vp]),
    "m3lb_scalar_field": (_i, [_vp, _vp]),
    "m3lb_scalar_field_device": (_i, [_vp, _pp]),
    "m3lb_scalar_total": (_i, [_vp, C.POINTER(C.c_double)]),
    "m3lb_scalar_gather": (_i, [_vp, _vp]),
    "m3lb_scalar_info": (_i, [_vp] + [C.POINTER(C.c_longlong)] * 3),
    "m3lb_scalar_sync": (_i, [_vp]),
    "m3lb_couple_thermal": (_i, [_vp, _vp] + [_d] * 6),
    "m3lb_init_eq": (_i, [_vp] + [_d] * 4),
    "m3lb_init_field_f32": (_i, [_vp] + [_vp] * 4),
    "m3lb_init_field_f64": (_i, [_vp] + [_vp] * 4),
    "m3lb_init_field_device": (_i, [_vp] + [_vp] * 4),
    "m3lb_step": (_i, [_vp, _i, _i]),
    "m3lb_macro_f32": (_i, [_vp] + [_vp] * 4),
    "m3lb_macro_f64": (_i, [_vp] + [_vp] * 4),
    "m3lb_stored_macro_f64": (_i, [_vp] + [_vp] * 4),
    "m3lb_macro_device": (_i, [_vp] + [_pp] * 4),
    "m3lb_reduce": (_i, [_vp, _vp]),
    "m3lb_diagnostics": (_i, [_vp, _vp]),
    "m3lb_gather": (_i, [_vp, _vp]),
    "m3lb_gather_raw": (_i, [_vp, _vp]),
    "m3lb_scatter": (_i, [_vp, _vp]),
    "m3lb_scatter_raw": (_i, [_vp, _vp]),
    "m3lb_timestep": (_i, [_vp, C.POINTER(C.c_longlong)]),
    "m3lb_dims": (_i, [_vp, C.POINTER(C.c_int)]),
    "m3lb_populations": (_i, [_vp, _pp, C.POINTER(C.c_size_t)]),
    "m3lb_set_stream": (_i, [_vp, _vp]),
    "m3lb_sync": (_i, [_vp]),
    "m3lb_set_option": (_i, [_vp, _i, _i]),
    "m3lb_launch_count": (_i, [_vp, C.POINTER(C.c_longlong)]),
    "m3lb_reduce_static": (_i, [_i] * 11 + [_d] * 3 + [_vp, _vp, C.c_longlong, _vp, _vp]),
    "m3lb_serve_create": (_i, [C.POINTER(ServeConfig), _pp]),
    "m3lb_serve_submit": (_i, [_vp, C.POINTER(Request)]),
    "m3lb_serve_run": (_i, [_vp, _d]),
    "m3lb_serve_results": (_i, [_vp, C.POINTER(Result), _i, C.POINTER(_i)]),
    "m3lb_serve_fields": (_i, [_vp, C.c_longlong] + [_vp] * 4),
    "m3lb_serve_get_stats": (_i, [_vp, C.POINTER(ServeStats)]),
    "m3lb_serve_destroy": (_i, [_vp]),
    "m3lb_tgv_field": (_i, [_i, _d] + [_vp] * 4 + [_vp]),
}

_lib = None


def lib():
    """Load libm3lb.so once; raise if it is not built."""
    global _lib
    if _lib is None:
        if not LIB_PATH.exists():
            raise FileNotFoundError(
                f"{LIB_PATH} is not built; run `python -m m3lb_b200.build` (nvcc, sm_100a)")
        L = C.CDLL(str(LIB_PATH))
        for name, (res, args) in SIGNATURES.items():
            fn = getattr(L, name)
            fn.restype = res
            fn.argtypes = args
        _lib = L
    return _lib


def last_error() -> str:
    return lib().m3lb_last_error().decode()


def check(rc: int) -> None:
    if rc != OK:
        raise M3lbError(rc, last_error())


def footprint(lattice, nx, ny, nz, px=True, py=True, pz=True, storage=STORE_F32) -> int:
    out = C.c_size_t(0)
    check(lib().m3lb_footprint(lattice, nx, ny, nz, int(px), int(py), int(pz), storage,
                               C.byref(out)))
    return int(out.value)
