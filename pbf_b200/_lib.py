"""ctypes bindings to the C ABI in include/pbf.h (libpbf_b200.so, built in-tree).

The library is the only compute path: when it is missing or fails to load, the
import raises instead of falling back to anything else.
"""
from __future__ import annotations

import ctypes as C
import os

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "libpbf_b200.so")

PBF_OK = 0
PBF_ERR_INVALID = -1
PBF_ERR_CUDA = -2
PBF_ERR_ALLOC = -3
PBF_ERR_DEVICE = -4
PBF_ERR_STATE = -5
PBF_ERR_NONFINITE = -6

PBF_DEVERR_SCAN_TIMEOUT = 1
PBF_DEVERR_BAD_INDEX = 2
PBF_DEVERR_NONFINITE = 4
PBF_DEVERR_MLP_TIMEOUT = 8

PBF_FLAG_CLAMP_C = 1
PBF_FLAG_XSPH_RHO = 2
PBF_FLAG_WALL_DENSITY = 4

FIELD = {
    "x": 0, "v": 1, "xold": 2, "xpred": 3, "xl": 4, "rho": 5, "dp": 6, "curl": 7, "vort": 8,
    "visc": 9, "cell": 10, "cell_start": 11, "perm": 12, "ncnt": 13, "nbr": 14, "hash": 15,
    "lambda0": 16, "features": 17, "lambda_total": 18,
}
FLOAT4_FIELDS = {"x", "v", "xold", "xpred", "xl", "dp", "curl", "vort", "visc"}
FLOAT_FIELDS = {"rho", "lambda0", "lambda_total"}
MLP_NUM_WEIGHTS = 9280
MLP_NUM_BIASES = 226


class SolverParameter(C.Structure):
    """Same layout as the reference SolverParameter (include/solverBase.h:16-40)."""

    _fields_ = [
        ("h", C.c_float), ("nParticles", C.c_int), ("restRho", C.c_float), ("epsilon", C.c_float),
        ("k", C.c_float), ("n", C.c_float), ("deltaq", C.c_float), ("c", C.c_float),
        ("dt", C.c_float), ("invDt", C.c_float), ("iterations", C.c_int),
        ("vorticityConfinementEpilon", C.c_float), ("radius", C.c_float),
    ]


class ExtParams(C.Structure):
    """pbf_ext_params (include/pbf.h)."""

    _fields_ = [
        ("gravity", C.c_float * 3), ("grid_dims", C.c_int * 3), ("cell_scale", C.c_float),
        ("wall_jitter", C.c_float), ("grad_rmin", C.c_float), ("max_neighbors", C.c_int),
        ("cell_order", C.c_int), ("flags", C.c_uint), ("scorr_scale", C.c_float),
        ("sphere", C.c_float * 4), ("adaptive", C.c_int), ("density_tol", C.c_float),
        ("max_iterations", C.c_int), ("measure_error", C.c_int), ("debug", C.c_int),
        ("warm_start", C.c_int), ("profile", C.c_int), ("block_size", C.c_int), ("record_features", C.c_int), ("warm_clamp", C.c_float), ("pair_lanes", C.c_int), ("persistent", C.c_int), ("warm_unfused", C.c_int), ("warm_floor", C.c_int),
    ]


STAGES = ["hash", "scan", "scatter", "reorder", "neighbors", "lambda", "dp", "velocity", "curl", "vort", "copy",
          "measure", "mlp"]


class SceneDesc(C.Structure):
    """pbf_scene_desc (include/pbf.h)."""

    _fields_ = [
        ("grid_space", C.c_float * 6), ("boundary", C.c_float * 6), ("grid_dims", C.c_int * 3),
        ("nparticles", C.c_int), ("sphere", C.c_float * 4),
    ]


class Camera(C.Structure):
    """pbf_camera (include/pbf.h)."""

    _fields_ = [
        ("view", C.c_float * 16), ("proj", C.c_float * 16), ("cam_pos", C.c_float * 3), ("radius", C.c_float),
        ("point_coeff", C.c_float), ("tan_half_fov", C.c_float), ("light_pos", C.c_float * 3),
        ("light_diffuse", C.c_float * 3), ("roi", C.c_float), ("room_light_pos", C.c_float * 3),
        ("room_light_diffuse", C.c_float * 3), ("room", C.c_float * 6), ("smooth_iterations", C.c_int),
        ("reserved", C.c_int * 5),
    ]


IMAGE = {"depth_raw": 0, "depth": 1, "thickness": 2, "normal": 3, "room": 4, "color": 5}
IMAGE_CHANNELS = {"depth_raw": 1, "depth": 1, "thickness": 1, "normal": 4, "room": 4, "color": 4}


class Stats(C.Structure):
    _fields_ = [
        ("substeps", C.c_longlong), ("total_iterations", C.c_longlong), ("fallbacks", C.c_longlong),
        ("last_iterations", C.c_int), ("error_bits", C.c_int), ("max_density_error", C.c_double),
        ("mean_density_error", C.c_double),
    ]


# (name, restype, argtypes) for every function include/pbf.h declares
_PROTOS = [
    ("pbf_abi_version", C.c_int, []),
    ("pbf_struct_size", C.c_size_t, [C.c_int]),
    ("pbf_last_error", C.c_char_p, []),
    ("pbf_ext_params_default", None, [C.POINTER(ExtParams)]),
    ("pbf_create", C.c_int, [C.POINTER(SolverParameter), C.POINTER(C.c_float), C.POINTER(C.c_float),
                             C.POINTER(ExtParams), C.POINTER(C.c_void_p)]),
    ("pbf_create_batch", C.c_int, [C.POINTER(SolverParameter), C.c_int, C.POINTER(SceneDesc),
                                   C.POINTER(ExtParams), C.POINTER(C.c_void_p)]),
    ("pbf_get_scene_layout", C.c_int, [C.c_void_p, C.c_int, C.POINTER(C.c_int), C.POINTER(C.c_int),
                                       C.POINTER(C.c_int), C.POINTER(C.c_int)]),
    ("pbf_destroy", C.c_int, [C.c_void_p]),
    ("pbf_upload", C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p, C.c_int]),
    ("pbf_upload_device", C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p, C.c_int, C.c_void_p]),
    ("pbf_bind_position", C.c_int, [C.c_void_p, C.c_void_p]),
    ("pbf_step", C.c_int, [C.c_void_p, C.c_int, C.c_void_p]),
    ("pbf_download", C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p]),
    ("pbf_download_device", C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p]),
    ("pbf_step_host", C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_int, C.c_void_p]),
    ("pbf_host_fence", C.c_int, [C.c_void_p, C.c_void_p]),
    ("pbf_debug_fail_staging_alloc", C.c_int, [C.c_int]),
    ("pbf_debug_expire_wait", C.c_int, [C.c_int, C.POINTER(C.c_int)]),
    ("pbf_measure_fp32_peak", C.c_int, [C.POINTER(C.c_double), C.POINTER(C.c_double)]),
    ("pbf_resize", C.c_int, [C.c_void_p, C.c_int]),
    ("pbf_set_parameter", C.c_int, [C.c_void_p, C.POINTER(SolverParameter)]),
    ("pbf_download_sorted_device", C.c_int, [C.c_void_p] + [C.c_void_p] * 5 + [C.c_void_p]),
    ("pbf_get_stats", C.c_int, [C.c_void_p, C.POINTER(Stats)]),
    ("pbf_fetch", C.c_int, [C.c_void_p, C.c_int, C.c_void_p, C.c_size_t]),
    ("pbf_field_bytes", C.c_size_t, [C.c_void_p, C.c_int]),
    ("pbf_build_grid", C.c_int, [C.c_void_p, C.c_void_p]),
    ("pbf_get_layout", C.c_int, [C.c_void_p, C.POINTER(C.c_int), C.POINTER(C.c_int), C.POINTER(C.c_int)]),
    ("pbf_stage_times", C.c_int, [C.c_void_p, C.POINTER(C.c_float), C.c_int]),
    ("pbf_graph_kernel_count", C.c_int, [C.c_void_p]),
    ("pbf_measure_density_error", C.c_int, [C.c_void_p, C.POINTER(C.c_double), C.POINTER(C.c_double), C.c_void_p]),
    ("pbf_set_warm_start", C.c_int, [C.c_void_p, C.c_void_p, C.c_size_t, C.c_void_p, C.c_size_t]),
    ("pbf_gather_training_rows", C.c_int, [C.c_void_p, C.c_void_p, C.c_int, C.c_void_p, C.c_void_p, C.c_void_p]),
    ("pbf_mlp_trainer_create", C.c_int, [C.c_int, C.c_void_p, C.c_void_p, C.POINTER(C.c_void_p)]),
    ("pbf_mlp_trainer_destroy", C.c_int, [C.c_void_p]),
    ("pbf_mlp_gradients", C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p, C.c_int, C.c_void_p, C.c_void_p,
                                    C.c_void_p, C.c_void_p]),
    ("pbf_mlp_train_step", C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p, C.c_int, C.c_float, C.c_void_p,
                                     C.c_void_p]),
    ("pbf_mlp_get_params", C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p]),
    ("pbf_mlp_forward", C.c_int, [C.c_void_p, C.c_void_p, C.c_int, C.c_void_p, C.c_void_p]),
    ("pbf_tc_gemm_bf16", C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p, C.c_int, C.c_int, C.c_void_p]),
    ("pbf_scan_workspace_bytes", C.c_size_t, [C.c_int]),
    ("pbf_scan_exclusive_i32", C.c_int, [C.c_void_p, C.c_void_p, C.c_int, C.c_void_p, C.c_size_t, C.c_void_p]),
    ("pbf_scan_exclusive_i32_noalloc", C.c_int, [C.c_void_p, C.c_void_p, C.c_int, C.c_void_p]),
    ("pbf_render_create", C.c_int, [C.c_int, C.c_int, C.POINTER(C.c_void_p)]),
    ("pbf_render_destroy", C.c_int, [C.c_void_p]),
    ("pbf_render_frame", C.c_int, [C.c_void_p, C.c_void_p, C.c_int, C.c_int, C.POINTER(Camera), C.c_void_p]),
    ("pbf_render_frame_solver", C.c_int, [C.c_void_p, C.c_void_p, C.POINTER(Camera), C.c_void_p]),
    ("pbf_render_read", C.c_int, [C.c_void_p, C.c_int, C.c_void_p, C.c_size_t]),
]


class PBFError(RuntimeError):
    def __init__(self, code: int, msg: str):
        super().__init__(f"pbf error {code}: {msg}")
        self.code = code


_lib = None


def lib() -> C.CDLL:
    """Load libpbf_b200.so once; raise if it is not built."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise ImportError(f"{LIB_PATH} is not built; run pbf_b200.build.build() (nvcc, sm_100a)")
        L = C.CDLL(LIB_PATH)
        for name, res, args in _PROTOS:
            f = getattr(L, name)
            f.restype = res
            f.argtypes = args
        _lib = L
    return _lib


def check(rc: int) -> None:
    if rc != PBF_OK:
        raise PBFError(rc, lib().pbf_last_error().decode(errors="replace"))


def declared_symbols() -> list[str]:
    return [p[0] for p in _PROTOS]
