"""ctypes view of the C ABI in include/discrete_adjoint.h and include/da_mesh.h.

The shared library is built in-tree (discrete_adjoint_b200/libda_b200.so).  Loading fails
loudly if it is missing: there is no CPU fallback for the device path.
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "libda_b200.so")

DA_MAX_MATERIALS = 16
DA_MAX_PILES = 8

DA_OK = 0
DA_ERR_INVALID = -1
DA_ERR_CUDA = -2
DA_ERR_NAN = -3
DA_ERR_NEG_DEPTH = -4
DA_ERR_EIGEN = -5
DA_ERR_TIMEOUT = -6
DA_ERR_NO_MESH = -7
DA_ERR_OOM = -8
DA_ERR_NO_DEVICE = -9
DA_ERR_UNSUPPORTED = -10
DA_ERR_IO = -11

DA_PREC_FP64 = 0
DA_PREC_FP32_SPLIT = 1

DA_JAC_EXACT = 0
DA_JAC_REFERENCE = 1

PD = C.POINTER(C.c_double)
PF = C.POINTER(C.c_float)
PI32 = C.POINTER(C.c_int32)


class da_params(C.Structure):
    _fields_ = [
        ("precision", C.c_int32),
        ("device", C.c_int32),
        ("epsilon", C.c_double),
        ("gravity_scale", C.c_double),
        ("gamma", C.c_double),
        ("intfrict", C.c_double),
        ("n_materials", C.c_int32),
        ("frict_tiny_iters", C.c_int32),
        ("bedfrict", C.c_double * DA_MAX_MATERIALS),
        ("frict_tiny_early", C.c_double),
        ("frict_tiny_late", C.c_double),
        ("max_time", C.c_double),
        ("next_output", C.c_double),
        ("next_save", C.c_double),
        ("influx_dt", C.c_double),
        ("fp32_sign_floor", C.c_double),
        ("tile_culling", C.c_int32),
        ("grid_blocks", C.c_int32),
        ("blocks_per_sm", C.c_int32),
        ("tile_staging", C.c_int32),
        ("jacobian_mode", C.c_int32),
        ("pad_mode", C.c_int32),
    ]


class da_restart_header(C.Structure):
    _fields_ = [
        ("min_dx", C.c_double * 2), ("min_gen", C.c_double),
        ("maxh_iter", C.c_int32), ("maxh_hmax", C.c_double),
        ("iter", C.c_int32), ("adjiter", C.c_int32), ("time", C.c_double),
        ("solrec_last_step", C.c_int32),
        ("n_nodes", C.c_int32), ("n_elements", C.c_int32), ("n_unresolved", C.c_int32),
        ("xrange", C.c_double * 2), ("yrange", C.c_double * 2),
    ]


class da_restart_cells(C.Structure):
    _fields_ = [
        ("keys", C.POINTER(C.c_uint32)), ("nbr", C.POINTER(C.c_int32)),
        ("level", C.POINTER(C.c_int32)), ("material", C.POINTER(C.c_int32)),
        ("x", C.POINTER(C.c_double)), ("y", C.POINTER(C.c_double)), ("dx", C.POINTER(C.c_double)),
        ("dy", C.POINTER(C.c_double)), ("elevation", C.POINTER(C.c_double)),
        ("zeta", C.POINTER(C.c_double)), ("curvature", C.POINTER(C.c_double)),
        ("d_gravity", C.POINTER(C.c_double)), ("gravity", C.POINTER(C.c_double)),
        ("h", C.POINTER(C.c_double)), ("hu", C.POINTER(C.c_double)), ("hv", C.POINTER(C.c_double)),
    ]


class da_mesh_soa(C.Structure):
    _fields_ = [
        ("n_cells", C.c_int32),
        ("nbr", PI32),
        ("x", PD), ("y", PD),
        ("dx", PD), ("dy", PD),
        ("gravity", PD),
        ("d_gravity", PD),
        ("curvature", PD),
        ("material", PI32),
    ]


DA_TUNE_MAX = 8
DA_TRACE_KINDS = 11


class da_tune_result(C.Structure):
    _fields_ = [("n", C.c_int32), ("best", C.c_int32), ("grid", C.c_int32 * DA_TUNE_MAX),
                ("blocks_per_sm", C.c_int32 * DA_TUNE_MAX), ("ms_per_step", C.c_double * DA_TUNE_MAX)]


class da_step_stats(C.Structure):
    _fields_ = [
        ("dt", C.c_double),
        ("time", C.c_double),
        ("volume", C.c_double),
        ("hmax", C.c_double),
        ("iter", C.c_int64),
    ]


class da_dem(C.Structure):
    _fields_ = [
        ("nrows", C.c_int32), ("ncols", C.c_int32),
        ("xmin", C.c_double), ("ymin", C.c_double), ("res", C.c_double),
        ("elev", PF),
        ("mat", PI32),
    ]


class da_pile_spec(C.Structure):
    _fields_ = [
        ("xc", C.c_double), ("yc", C.c_double),
        ("height", C.c_double),
        ("major", C.c_double), ("minor", C.c_double),
        ("rot_deg", C.c_double),
        ("vx", C.c_double), ("vy", C.c_double),
    ]


class da_mesh_spec(C.Structure):
    _fields_ = [
        ("xmin", C.c_double), ("ymin", C.c_double),
        ("dx0", C.c_double), ("dy0", C.c_double),
        ("nx0", C.c_int32), ("ny0", C.c_int32),
        ("max_level", C.c_int32), ("uniform", C.c_int32),
        ("refine_margin", C.c_double),
        ("n_boxes", C.c_int32),
        ("boxes", PD),
        ("random_frac", C.c_double),
        ("seed", C.c_uint64),
        ("extra_level", C.c_int32),
        ("pad", C.c_int32),
    ]


class da_mesh_host(C.Structure):
    _fields_ = [
        ("n_cells", C.c_int32), ("max_level", C.c_int32), ("n_piles", C.c_int32),
        ("level", PI32), ("ix", PI32), ("iy", PI32),
        ("nbr", PI32),
        ("x", PD), ("y", PD), ("dx", PD), ("dy", PD),
        ("elevation", PD),
        ("zeta", PD),
        ("curvature", PD),
        ("gravity", PD),
        ("d_gravity", PD),
        ("material", PI32),
        ("h0", PD), ("hu0", PD), ("hv0", PD),
        ("dh0_dpile", PD),
    ]


class da_functional(C.Structure):
    _fields_ = [("kind", C.c_int32), ("pad", C.c_int32), ("box", C.c_double * 4)]


class da_gradient(C.Structure):
    _fields_ = [
        ("J", C.c_double),
        ("dJ_dbedfrict", C.c_double * DA_MAX_MATERIALS),
        ("dJ_dintfrict", C.c_double),
        ("dJ_dpile", C.c_double * DA_MAX_PILES),
        ("forward_steps", C.c_int64),
        ("snapshots", C.c_int32),
        ("pad", C.c_int32),
        ("device_ms", C.c_double),
    ]


DA_FUNC_H2_BOX = 1


DA_MAX_PLANES = 16


class da_stats_props(C.Structure):
    _fields_ = [("heightifreach", C.c_double), ("xyifreach", C.c_double * 2), ("hxyminmax", C.c_double),
                ("min_height", C.c_double), ("vslump", C.c_double), ("n_planes", C.c_int32), ("pad", C.c_int32),
                ("planes", PD)]


class da_stats(C.Structure):
    _fields_ = [(k, C.c_double) for k in ("xcen", "ycen", "xvar", "yvar", "rmean", "area", "vmean", "umean",
                                          "vxmean", "vymean", "slopemean", "statvolume", "piler", "hmax", "vmax",
                                          "umax", "vstar")] + \
               [("xyminmax", C.c_double * 4), ("testpoint_reach", C.c_int32), ("pad", C.c_int32),
                ("energy", C.c_double)]


class da_member(C.Structure):
    _fields_ = [
        ("mesh", da_mesh_soa),
        ("h0", PD), ("hu0", PD), ("hv0", PD),
        ("dh0_dpile", PD),
        ("n_materials", C.c_int32),
        ("pad", C.c_int32),
        ("bedfrict", C.c_double * DA_MAX_MATERIALS),
        ("intfrict", C.c_double),
        ("box", C.c_double * 4),
    ]

# name -> (restype, argtypes) for every symbol the headers declare
SIGNATURES = {
    "da_abi_version": (C.c_int, []),
    "da_selftest_barrier": (C.c_int, [C.c_void_p, C.c_int32]),
    "da_set_owned": (C.c_int, [C.c_void_p, C.c_int32]),
    "da_get_stream": (C.c_int, [C.c_void_p, C.POINTER(C.c_void_p)]),
    "da_step_bounds": (C.c_int, [C.c_void_p, C.c_void_p]),
    "da_step_apply": (C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p]),
    "da_halo_pack": (C.c_int, [C.c_void_p, C.c_void_p, C.c_int32, C.c_void_p]),
    "da_halo_unpack": (C.c_int, [C.c_void_p, C.c_void_p, C.c_int32, C.c_void_p]),
    "da_sync": (C.c_int, [C.c_void_p]),
    "da_strerror": (C.c_char_p, [C.c_int]),
    "da_params_default": (None, [C.POINTER(da_params)]),
    "da_create": (C.c_void_p, [C.POINTER(da_params), C.POINTER(C.c_int)]),
    "da_destroy": (None, [C.c_void_p]),
    "da_last_error": (C.c_char_p, [C.c_void_p]),
    "da_set_params": (C.c_int, [C.c_void_p, C.POINTER(da_params)]),
    "da_set_time": (C.c_int, [C.c_void_p, C.c_double, C.c_int64]),
    "da_upload_mesh": (C.c_int, [C.c_void_p, C.POINTER(da_mesh_soa), C.c_int32]),
    "da_set_state": (C.c_int, [C.c_void_p, PD, PD, PD]),
    "da_get_state": (C.c_int, [C.c_void_p, PD, PD, PD]),
    "da_forward_step": (C.c_int, [C.c_void_p, C.POINTER(da_step_stats)]),
    "da_forward_run": (C.c_int, [C.c_void_p, C.c_int32, C.POINTER(da_step_stats)]),
    "da_forward_run_timed": (C.c_int, [C.c_void_p, C.c_int32, C.POINTER(da_step_stats), PD]),
    "da_adjoint_run": (C.c_int, [C.c_void_p, C.POINTER(da_functional), C.c_int32, C.c_int32, PD, C.c_int32,
                                 C.POINTER(da_gradient), PD]),
    "da_adjoint_run_seeded": (C.c_int, [C.c_void_p, PD, C.c_int32, C.c_int32, PD, C.c_int32,
                                        C.POINTER(da_gradient), PD]),
    "da_adjoint_run_dwr": (C.c_int, [C.c_void_p, C.POINTER(da_functional), C.c_int32, C.c_int32, PD, C.c_int32,
                                     C.POINTER(da_gradient), PD, PD, PD]),
    "da_adjoint_step": (C.c_int, [C.c_void_p, PD, PD, C.POINTER(da_gradient)]),
    "da_set_dt_replay": (C.c_int, [C.c_void_p, PD, C.c_int32, C.c_int64]),
    "da_forward_step_noalloc": (C.c_int, [C.POINTER(da_params), C.POINTER(da_mesh_soa), PD, PD, PD, PD, PD, PD,
                                          C.c_double, C.c_int64, C.c_void_p, C.POINTER(da_step_stats)]),
    "da_forward_profile": (C.c_int, [C.c_void_p, C.c_int32, PD]),
    "da_forward_kernel_name": (C.c_char_p, [C.c_int32]),
    "da_set_tracing": (C.c_int, [C.c_void_p, C.c_int32]),
    "da_trace_read": (C.c_int, [C.c_void_p, C.c_int32, PD, C.POINTER(C.c_int64)]),
    "da_trace_name": (C.c_char_p, [C.c_int32]),
    "da_trace_steps": (C.c_int, [C.c_void_p, C.c_int32, C.POINTER(C.c_int64)]),
    "da_autotune": (C.c_int, [C.c_void_p, C.c_int32, C.POINTER(da_tune_result)]),
    "da_compute_stats": (C.c_int, [C.c_void_p, C.POINTER(da_stats_props), C.c_double, C.POINTER(da_stats), PD]),
    "da_refine_info": (C.c_int, [C.c_void_p, PD, C.POINTER(C.c_uint8), PD]),
    "da_outline_init": (C.c_int, [C.c_void_p, PD, PD, PD]),
    "da_outline_update": (C.c_int, [C.c_void_p]),
    "da_outline_read": (C.c_int, [C.c_void_p, C.POINTER(C.c_int32), C.POINTER(C.c_int32), PD]),
    "da_dwr_setup": (C.c_int, [C.c_void_p, C.POINTER(da_mesh_soa), PI32, PI32, PD]),
    "da_dwr_step": (C.c_int, [C.c_void_p, PD, PD, PD, PD]),
    "da_ensemble_upload": (C.c_int, [C.c_void_p, C.POINTER(da_member), C.c_int32]),
    "da_ensemble_restart": (C.c_int, [C.c_void_p]),
    "da_ensemble_forward": (C.c_int, [C.c_void_p, C.c_int32, C.POINTER(C.c_double)]),
    "da_ensemble_stats": (C.c_int, [C.c_void_p, C.POINTER(da_step_stats)]),
    "da_ensemble_get_state": (C.c_int, [C.c_void_p, C.c_int32, PD, PD, PD]),
    "da_ensemble_adjoint": (C.c_int, [C.c_void_p, C.c_int32, C.c_int32, C.POINTER(da_gradient), C.POINTER(C.c_double)]),
    "da_mesh_build": (C.c_int, [C.POINTER(da_mesh_spec), C.POINTER(da_dem), C.POINTER(da_pile_spec), C.c_int32,
                                C.c_double, C.c_double, C.POINTER(C.POINTER(da_mesh_host))]),
    "da_mesh_free": (None, [C.POINTER(da_mesh_host)]),
    "da_mesh_view": (C.c_int, [C.POINTER(da_mesh_host), C.POINTER(da_mesh_soa)]),
    "da_cell_keys": (C.c_int, [C.c_int32, PD, PD, PD, PD, C.POINTER(C.c_uint32)]),
    "da_write_solution": (C.c_int, [C.c_char_p, C.c_int32, C.POINTER(C.c_uint32), PD, PD, PD]),
    "da_read_solution": (C.c_int, [C.c_char_p, C.c_int32, C.POINTER(C.c_uint32), PD, PD, PD,
                                   C.POINTER(C.c_int32)]),
    "da_write_restart": (C.c_int, [C.c_char_p, C.POINTER(da_restart_header), PD, C.c_int32, C.POINTER(da_mesh_soa),
                                   PI32, PI32, PI32, PD, PD, PD, PD, PD, PD]),
    "da_read_restart": (C.c_int, [C.c_char_p, C.POINTER(da_restart_header), C.POINTER(C.c_int32),
                                  C.POINTER(C.c_int32), PD, C.POINTER(da_restart_cells)]),
    "da_write_outline": (C.c_int, [C.c_char_p, PD, PD, PD, C.c_int32, C.c_int32, PD]),
}

_lib = None


def load(path: str = LIB_PATH) -> C.CDLL:
    """Loads libda_b200.so and binds every declared symbol (raises if any is missing)."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(path):
        raise RuntimeError(
            f"{path} is missing: build it with `python -m discrete_adjoint_b200._build` "
            "(there is no CPU fallback for the device path)")
    lib = C.CDLL(path)
    for name, (res, args) in SIGNATURES.items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    _lib = lib
    return lib


class DAError(RuntimeError):
    def __init__(self, code: int, msg: str):
        super().__init__(f"{msg} (code {code})")
        self.code = code


def dptr(a: np.ndarray):
    assert a.dtype == np.float64 and a.flags.c_contiguous
    return a.ctypes.data_as(PD)


def fptr(a: np.ndarray):
    assert a.dtype == np.float32 and a.flags.c_contiguous
    return a.ctypes.data_as(PF)


def iptr(a: np.ndarray):
    assert a.dtype == np.int32 and a.flags.c_contiguous
    return a.ctypes.data_as(PI32)
