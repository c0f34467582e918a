"""ctypes binding of the C ABI in include/itr_gpu.h (lib/libitr_gpu.so).

The structures below are field-for-field copies of the header's structs. Loading fails
loudly: there is no CPU fallback for the batched forward operator.
"""
from __future__ import annotations

import ctypes as C
import os

HERE = os.path.dirname(os.path.abspath(__file__))
PKG = os.path.dirname(HERE)
LIB_PATH = os.environ.get("ITR_GPU_LIB") or os.path.join(PKG, "lib", "libitr_gpu.so")

ITR_OK, ITR_UNSUPPORTED, ITR_INVALID_ARG, ITR_DEVICE_ERROR, ITR_DEVICE_TIMEOUT = 0, 1, 2, 3, 4
BC_WALL, BC_TRANSMISSIVE, BC_STAGE, BC_INFLOW = 0, 1, 2, 3
FACE_SIGNED, FACE_CREST = 0, 1
RUN_OK, RUN_GUARD_ABORT, RUN_INCUMBENT_ABORT, RUN_UNHEALTHY = 0, 1, 2, 3

_dp = C.POINTER(C.c_double)
_fp = C.POINTER(C.c_float)
_u8p = C.POINTER(C.c_uint8)
_i32p = C.POINTER(C.c_int32)
_u32p = C.POINTER(C.c_uint32)


class Params(C.Structure):
    _fields_ = [
        ("duration_s", C.c_double), ("sync_interval_s", C.c_double), ("cfl", C.c_double),
        ("dt_max_s", C.c_double), ("h_dry", C.c_double), ("h_eps", C.c_double),
        ("rain_t", _dp), ("rain_rate", _dp), ("n_rain", C.c_int32),
        ("infil_capacity", C.c_double), ("initial_depth", C.c_double), ("skip_dry", C.c_int32),
        ("inflow_scale", C.c_double),
    ]


class Grid(C.Structure):
    _fields_ = [
        ("nx", C.c_int32), ("ny", C.c_int32), ("dx", C.c_double), ("dy", C.c_double), ("g", C.c_double),
        ("mode", C.c_int32), ("wet", _fp), ("gn2", _fp), ("bc", _u8p), ("wet_count", C.c_int64),
        ("bc_stage", _dp), ("bc_hydro", _i32p), ("bc_inv_len", _dp), ("n_hydro", C.c_int32),
        ("hydro_off", _i32p), ("hydro_t", _dp), ("hydro_q", _dp),
    ]


class Design(C.Structure):
    _fields_ = [
        ("dzx", _fp), ("dzy", _fp), ("dzx2", _fp), ("dzy2", _fp), ("h0", _fp),
        ("cut_m3", C.c_double), ("fill_m3", C.c_double), ("z_edge", _dp),
    ]


class Objective(C.Structure):
    _fields_ = [
        ("n_assets", C.c_int32), ("asset_off", _i32p), ("asset_pos", _i32p),
        ("asset_threshold", _dp), ("asset_weight", _dp),
        ("n_guard", C.c_int32), ("guard_pos", _i32p), ("baseline_max", _dp),
        ("guard_tolerance", C.c_double), ("tau", C.c_double), ("cut_cost", C.c_double),
        ("fill_cost", C.c_double), ("earth_weight", C.c_double),
        ("require_no_worsening", C.c_int32), ("guard_abort", C.c_int32),
        ("has_incumbent", C.c_int32), ("incumbent", C.c_double),
    ]


class Result(C.Structure):
    _fields_ = [
        ("monitor_max", _dp), ("peak", _fp), ("depth", _fp), ("ledger", _dp), ("max_rows", C.c_int32),
        ("steps", C.c_uint64), ("cell_updates", C.c_uint64), ("t_end", C.c_double),
        ("sync_count", C.c_uint32), ("status", C.c_int32), ("breach_cell", C.c_uint32),
        ("breach_sync", C.c_uint32), ("violation", C.c_double), ("lower_bound", C.c_double),
        ("j", C.c_double), ("feasible", C.c_int32), ("n_rows", C.c_int32),
        ("volume_m3", C.c_double), ("rel_residual", C.c_double), ("warm_start_steps", C.c_uint64),
        ("dt_fallback_t", C.c_double), ("rows_skipped", C.c_uint64),
    ]


class Primitive(C.Structure):
    _fields_ = [
        ("kind", C.c_int32), ("cx", C.c_double), ("cy", C.c_double), ("length", C.c_double), ("width", C.c_double),
        ("angle_deg", C.c_double), ("height", C.c_double),
    ]


class DesignSpace(C.Structure):
    _fields_ = [
        ("origin_x", C.c_double), ("origin_y", C.c_double), ("z", _dp), ("wall", _u8p), ("editable", _u8p),
        ("z_wall", C.c_double), ("max_abs_dz", C.c_double),
    ]


class SceneView(C.Structure):
    _fields_ = [
        ("cam_pos", C.c_float * 3), ("cam_fwd", C.c_float * 3), ("cam_right", C.c_float * 3), ("cam_up", C.c_float * 3),
        ("focal", C.c_float), ("domain", C.c_float * 3), ("z_lo", C.c_float), ("z_span", C.c_float), ("up", C.c_float),
        ("depth_span", C.c_float), ("ve", C.c_float), ("time", C.c_float), ("rain", C.c_float), ("wet", C.c_float),
        ("overcast", C.c_float), ("vel_max", C.c_float), ("base", C.c_float), ("ortho", C.c_int32), ("debug", C.c_int32),
    ]


class Group(C.Structure):
    _fields_ = [
        ("grid", C.POINTER(Grid)), ("n_designs", C.c_int32), ("designs", C.POINTER(Design)),
        ("monitors", C.POINTER(C.c_uint32)), ("n_mon", C.c_int32), ("obj", C.POINTER(Objective)),
    ]


# Every symbol the header declares, with its signature.
SIGNATURES = {
    "itr_gpu_create": (C.c_void_p, [C.c_int, C.c_char_p, C.c_size_t]),
    "itr_gpu_destroy": (None, [C.c_void_p]),
    "itr_gpu_last_error": (C.c_char_p, [C.c_void_p]),
    "itr_gpu_info": (C.c_int, [C.c_void_p, C.c_char_p, C.c_size_t]),
    "itr_gpu_run_batch": (C.c_int, [C.c_void_p, C.POINTER(Params), C.POINTER(Grid), C.c_int32, C.POINTER(Design),
                                    _u32p, C.c_int32, C.POINTER(Objective), C.POINTER(Result)]),
    "itr_gpu_set_option": (C.c_int, [C.c_void_p, C.c_char_p, C.c_int64]),
    "itr_gpu_set_locked_dt": (C.c_int, [C.c_void_p, _dp, C.c_uint64, C.c_double]),
    "itr_gpu_last_timing": (C.c_int, [C.c_void_p, _dp, _dp, C.POINTER(C.c_uint64), _i32p]),
    "itr_gpu_rerun_resident": (C.c_int, [C.c_void_p]),
    "itr_gpu_run_ladder": (C.c_int, [C.c_void_p, C.POINTER(Params), C.c_int32, C.POINTER(Group), C.POINTER(Result)]),
    "itr_gpu_vjp": (C.c_int, [C.c_void_p, C.POINTER(Params), C.POINTER(Grid), C.c_int32, C.POINTER(Design), _u32p,
                              C.c_int32, C.POINTER(Objective), C.c_int32, C.POINTER(Result), _dp, _dp]),
    "itr_gpu_vjp_crest": (C.c_int, [C.c_void_p, C.POINTER(Params), C.POINTER(Grid), C.c_int32, C.POINTER(Design), _u32p,
                                    C.c_int32, C.POINTER(Objective), C.c_int32, C.POINTER(Result), _dp, _dp, _dp, _dp]),
    "itr_gpu_last_vjp_timing": (C.c_int, [C.c_void_p, _dp, _dp]),
    "itr_gpu_render_map": (C.c_int, [C.c_void_p, C.c_int32, C.c_int32, C.c_double, _fp, _fp, _fp, C.c_int32, C.c_float,
                                     C.c_int32, _u8p]),
    "itr_gpu_render_scene": (C.c_int, [C.c_void_p, _u8p, C.c_int32, C.c_int32, _u8p, _u8p, C.c_int32, C.c_int32,
                                       C.POINTER(SceneView), C.c_int32, C.c_int32, _u8p]),
    "itr_gpu_record_baseline": (C.c_int, [C.c_void_p, C.POINTER(Params), C.POINTER(Grid), C.POINTER(Design), _u32p,
                                          C.c_int32, C.c_int32, C.POINTER(Result)]),
    "itr_gpu_run_primitives": (C.c_int, [C.c_void_p, C.POINTER(Params), C.POINTER(Grid), C.POINTER(DesignSpace), C.c_int32,
                                         _i32p, C.POINTER(Primitive), _u32p, C.c_int32, C.POINTER(Objective),
                                         C.POINTER(Result), _dp, _dp]),
    "itr_gpu_vjp_primitives": (C.c_int, [C.c_void_p, C.POINTER(Params), C.POINTER(Grid), C.POINTER(DesignSpace), C.c_int32,
                                         _i32p, C.POINTER(Primitive), _u32p, C.c_int32, C.POINTER(Objective), C.c_int32,
                                         C.POINTER(Result), _dp, _dp, _dp]),
    "itr_gpu_run_plain_static": (C.c_int, [C.c_int, C.POINTER(Params), C.POINTER(Grid), C.POINTER(Design), _u32p,
                                           C.c_int32, C.POINTER(Result), C.c_char_p, C.c_size_t]),
}

_LIB = None


def load(path: str | None = None) -> C.CDLL:
    """Load lib/libitr_gpu.so and declare every entry point. Raises if it is missing."""
    global _LIB
    if _LIB is not None and path is None:
        return _LIB
    p = path or LIB_PATH
    if not os.path.exists(p):
        raise RuntimeError(f"itr_gpu: CUDA library {p} is not built (run __graft_entry__.build() or make -C inverse-terrain-engine_b200)")
    lib = C.CDLL(p)
    for name, (res, args) in SIGNATURES.items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    if path is None:
        _LIB = lib
    return lib
