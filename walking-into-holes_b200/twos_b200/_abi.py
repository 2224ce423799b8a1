"""ctypes binding of libtwos.so (include/twos.h).

The structures mirror the C declarations field for field; their sizes are
checked at load time.  Loading fails loudly when the library is missing:
there is no CPU fallback.
"""
from __future__ import annotations

import ctypes
from pathlib import Path

PKG_ROOT = Path(__file__).resolve().parent.parent
LIB_PATH = PKG_ROOT / "_build" / "libtwos.so"
BIN_DIR = PKG_ROOT / "_build"

ABI_VERSION = 2  # TWOS_ABI_VERSION of include/twos.h
OK, ERR_RUNTIME, ERR_USAGE = 0, 1, 2
MODE_COMPLIANCE, MODE_PAIRED, MODE_HOT = 0, 1, 2
PREC_FP64, PREC_MIXED = 0, 1
SOURCE_CENTER, SOURCE_GREEN, SOURCE_EXACT = 0, 1, 2
TERM_CONST, TERM_LINEAR, TERM_GAUSS, TERM_BUMP, TERM_BOX, TERM_BALL, TERM_QUAD = range(7)
MAX_TERMS = 8
DEVERR_QUERY, DEVERR_STACK, DEVERR_ITER, DEVERR_CONFIG = 1, 2, 4, 8

EXPORTED = [
    "twos_abi_version", "twos_last_error", "twos_mesh_open", "twos_mesh_open_ply", "twos_mesh_close",
    "twos_mesh_get_info", "twos_mesh_set_stream", "twos_closest_point", "twos_mesh_distance_bound", "twos_estimate",
    "twos_estimate_device",
    "twos_estimate_batch", "twos_design_loop", "twos_walk_samples", "twos_inside", "twos_topk_device",
    "twos_estimate_noalloc", "twos_mesh_set_tuning", "twos_mesh_get_tuning", "twos_diffwos",
    "twos_ball_green_integral", "twos_validate", "twos_estimate_gradient", "twos_rqmc", "twos_finalize_samples",
    "twos_l2_read_gbs", "twos_trace_grid_steps", "twos_sobol_directions",
]
RQMC_MC, RQMC_ARRAY, RQMC_NEIGHBOUR, RQMC_SOBOL = 0, 1, 2, 3


class SourceTerm(ctypes.Structure):
    _fields_ = [
        ("kind", ctypes.c_int32), ("axis", ctypes.c_int32),
        ("amp", ctypes.c_double), ("offset", ctypes.c_double), ("div", ctypes.c_double),
        ("c", ctypes.c_double * 3), ("w", ctypes.c_double * 3),
    ]


class Request(ctypes.Structure):
    _fields_ = [
        ("mode", ctypes.c_int32), ("precision", ctypes.c_int32),
        ("walks", ctypes.c_int32), ("max_steps", ctypes.c_int32),
        ("seed", ctypes.c_uint64), ("repeat", ctypes.c_uint32), ("stream", ctypes.c_uint32),
        ("epsilon", ctypes.c_double), ("cavity_radius", ctypes.c_double), ("query_radius", ctypes.c_double),
        ("green", ctypes.c_int32), ("n_source", ctypes.c_int32), ("n_adjoint", ctypes.c_int32),
        ("skip_cavity_sites", ctypes.c_int32), ("site_offset", ctypes.c_uint32), ("n_boundary", ctypes.c_uint32),
        ("source", SourceTerm * MAX_TERMS), ("adjoint", SourceTerm * MAX_TERMS), ("boundary", SourceTerm * MAX_TERMS),
    ]


class SiteResult(ctypes.Structure):
    _fields_ = [
        ("u", ctypes.c_double), ("p", ctypes.c_double), ("score", ctypes.c_double),
        ("score_se", ctypes.c_double), ("same_index", ctypes.c_double),
        ("steps", ctypes.c_uint64), ("caps", ctypes.c_uint64),
    ]


class Summary(ctypes.Structure):
    _fields_ = [
        ("kernel_seconds", ctypes.c_double), ("walk_seconds", ctypes.c_double),
        ("total_seconds", ctypes.c_double),
        ("paths", ctypes.c_uint64), ("steps", ctypes.c_uint64), ("caps", ctypes.c_uint64),
        ("queries", ctypes.c_uint64), ("h2d_bytes", ctypes.c_uint64), ("d2h_bytes", ctypes.c_uint64),
        ("launches", ctypes.c_uint32), ("error_flags", ctypes.c_uint32),
        ("node_tests", ctypes.c_uint64), ("plane_tests", ctypes.c_uint64), ("triangle_tests", ctypes.c_uint64),
        ("grid_steps", ctypes.c_uint64),
    ]


class MeshInfo(ctypes.Structure):
    _fields_ = [
        ("vertices", ctypes.c_uint64), ("faces", ctypes.c_uint64), ("bvh_nodes", ctypes.c_uint64),
        ("bvh_depth", ctypes.c_uint32), ("device", ctypes.c_uint32),
        ("bounds_min", ctypes.c_double * 3), ("bounds_max", ctypes.c_double * 3),
        ("center", ctypes.c_double * 3), ("mixed_delta", ctypes.c_double),
        ("build_seconds", ctypes.c_double), ("device_bytes", ctypes.c_uint64),
        ("grid_dims", ctypes.c_uint32 * 3), ("grid_pad", ctypes.c_uint32), ("grid_spacing", ctypes.c_double),
    ]


class Tuning(ctypes.Structure):
    _fields_ = [("block", ctypes.c_int32), ("refill", ctypes.c_int32), ("step_threshold", ctypes.c_int32),
                ("blocks_per_sm", ctypes.c_int32), ("grid_threshold", ctypes.c_float), ("units", ctypes.c_int32),
                ("entry", ctypes.c_int32), ("grid_fp64", ctypes.c_int32), ("bvh_width", ctypes.c_int32),
                ("lane_walks", ctypes.c_int32), ("wavefront", ctypes.c_int32)]


class DesignParams(ctypes.Structure):
    _fields_ = [
        ("iterations", ctypes.c_uint32), ("shortlist", ctypes.c_uint32),
        ("cavity_radius", ctypes.c_double), ("z", ctypes.c_double), ("accept_threshold", ctypes.c_double),
        ("outer_clearance", ctypes.c_double), ("pair_gap", ctypes.c_double),
        ("use_graph", ctypes.c_int32), ("reserved", ctypes.c_int32),
    ]


class DesignStep(ctypes.Structure):
    _fields_ = [
        ("chosen", ctypes.c_uint32), ("accepted", ctypes.c_uint32),
        ("scout_score", ctypes.c_double), ("score", ctypes.c_double), ("score_se", ctypes.c_double),
        ("lower", ctypes.c_double), ("slot", ctypes.c_uint32), ("n_cavities", ctypes.c_uint32),
    ]


class RqmcParams(ctypes.Structure):
    _fields_ = [("method", ctypes.c_int32), ("batches", ctypes.c_uint32), ("n_u_boundary", ctypes.c_uint32),
                ("n_p_boundary", ctypes.c_uint32), ("u_boundary", SourceTerm * MAX_TERMS),
                ("p_boundary", SourceTerm * MAX_TERMS), ("walk_first", ctypes.c_void_p),
                ("walk_u", ctypes.c_void_p), ("walk_p", ctypes.c_void_p), ("site_radius", ctypes.c_void_p)]


class ValidateParams(ctypes.Structure):
    _fields_ = [("radius_cap", ctypes.c_double), ("value_cap", ctypes.c_double)]


GRADIENT_DTYPE = [("u", "f8"), ("p", "f8"), ("grad_u", "f8", (3,)), ("grad_p", "f8", (3,)), ("cross", "f8"),
                  ("cross_se", "f8"), ("steps", "u8"), ("caps", "u8"), ("u_se", "f8"), ("p_se", "f8")]

VALIDATE_MAX_STAGES = 5
CERT_SAMPLE_DTYPE = [("value", "f8"), ("steps", "u4"), ("capped", "u1"), ("clipped", "u1"), ("contained", "u1"),
                     ("pad", "u1")]
VALIDATE_STAGE_DTYPE = [("site", "u4"), ("n", "u4"), ("mean", "f8"), ("mean_steps", "f8"), ("clipped", "u8"),
                        ("path_caps", "u8"), ("center_clearance_lower", "f8"), ("center_distance", "f8")]

# twos_diff_result / twos_diff_stats as numpy record layouts.
DIFF_DTYPE = [("dc", "f8", (3,)), ("dc_se", "f8", (3,)), ("dR", "f8"), ("dR_se", "f8")]
DIFF_STATS_DTYPE = [("outer_steps", "u8"), ("nested_steps", "u8"), ("cavity_terminations", "u8"),
                    ("near_seam", "u8"), ("segment_unsafe", "u8"), ("unsafe_offset", "u8"), ("limits", "u8")]

DESIGN_DTYPE = [("chosen", "u4"), ("accepted", "u4"), ("scout_score", "f8"), ("score", "f8"),
                ("score_se", "f8"), ("lower", "f8"), ("slot", "u4"), ("n_cavities", "u4")]

assert ctypes.sizeof(SourceTerm) == 80
assert ctypes.sizeof(SiteResult) == 56

SITE_DTYPE = [("u", "f8"), ("p", "f8"), ("score", "f8"), ("score_se", "f8"), ("same_index", "f8"),
              ("steps", "u8"), ("caps", "u8")]

_lib = None


class TwosError(RuntimeError):
    def __init__(self, code: int, message: str):
        super().__init__(message)
        self.code = code


def load(path: Path | str | None = None):
    """Load libtwos.so (once).  Raises if it has not been built."""
    global _lib
    if _lib is not None:
        return _lib
    p = Path(path) if path else LIB_PATH
    if not p.exists():
        raise RuntimeError(f"libtwos.so not built ({p}); run walking-into-holes_b200/build.py")
    L = ctypes.CDLL(str(p))
    vp, u64, u32, i32, dbl = ctypes.c_void_p, ctypes.c_uint64, ctypes.c_uint32, ctypes.c_int, ctypes.c_double
    L.twos_abi_version.restype = ctypes.c_int
    L.twos_last_error.restype = ctypes.c_char_p
    L.twos_mesh_open.argtypes = [vp, u64, vp, u64, i32, ctypes.POINTER(vp)]
    L.twos_mesh_open_ply.argtypes = [ctypes.c_char_p, i32, ctypes.POINTER(vp)]
    L.twos_mesh_close.argtypes = [vp]
    L.twos_mesh_close.restype = None
    L.twos_mesh_get_info.argtypes = [vp, ctypes.POINTER(MeshInfo)]
    L.twos_mesh_set_stream.argtypes = [vp, vp]
    L.twos_closest_point.argtypes = [vp, i32, vp, u64, dbl, vp, vp]
    L.twos_mesh_distance_bound.argtypes = [vp, vp, u64, vp]
    L.twos_estimate.argtypes = [vp, ctypes.POINTER(Request), vp, u32, vp, u32, vp, ctypes.POINTER(Summary)]
    L.twos_estimate_device.argtypes = [vp, ctypes.POINTER(Request), vp, u32, vp, u32, vp, ctypes.POINTER(Summary)]
    L.twos_mesh_set_tuning.argtypes = [vp, ctypes.POINTER(Tuning)]
    L.twos_mesh_get_tuning.argtypes = [vp, ctypes.POINTER(Tuning)]
    L.twos_estimate_noalloc.argtypes = [vp, ctypes.POINTER(Request), vp, u32, vp, u32, vp, ctypes.POINTER(Summary)]
    L.twos_estimate_batch.argtypes = [vp, ctypes.POINTER(Request), u32, vp, vp, vp, vp, vp, ctypes.POINTER(Summary)]
    L.twos_design_loop.argtypes = [vp, ctypes.POINTER(Request), ctypes.POINTER(Request), vp, u32, vp, u32,
                                   ctypes.POINTER(DesignParams), vp, vp, ctypes.POINTER(u32), ctypes.POINTER(Summary)]
    L.twos_walk_samples.argtypes = [vp, ctypes.POINTER(Request), vp, u32, vp, u32, vp, vp, vp]
    L.twos_inside.argtypes = [vp, vp, u64, vp]
    L.twos_finalize_samples.argtypes = [vp, i32, i32, vp, vp, vp, u32, u32, vp]
    L.twos_l2_read_gbs.argtypes = [i32, u64, u32, ctypes.POINTER(ctypes.c_double)]
    L.twos_trace_grid_steps.argtypes = [vp, ctypes.POINTER(Request), vp, u32, u64, vp, vp, ctypes.POINTER(u64)]
    L.twos_ball_green_integral.argtypes = [vp, u32, vp, i32]
    L.twos_rqmc.argtypes = [vp, ctypes.POINTER(Request), ctypes.POINTER(RqmcParams), vp, u32, vp, vp, vp,
                            ctypes.POINTER(Summary)]
    L.twos_estimate_gradient.argtypes =[vp, ctypes.POINTER(Request), vp, u32, vp, u32, vp, ctypes.POINTER(Summary)]
    L.twos_validate.argtypes = [vp, ctypes.POINTER(Request), ctypes.POINTER(ValidateParams), vp, u32, vp, u32, vp,
                                vp, ctypes.POINTER(u32), ctypes.POINTER(Summary)]
    L.twos_diffwos.argtypes = [vp, ctypes.POINTER(Request), dbl, i32, vp, u32, vp, u32, vp, vp,
                               ctypes.POINTER(Summary)]
    L.twos_topk_device.argtypes = [vp, vp, u32, u32, vp]
    L.twos_sobol_directions.argtypes = [u32, u32, vp]
    for name in EXPORTED:
        if name not in ("twos_mesh_close", "twos_last_error"):
            getattr(L, name).restype = ctypes.c_int
    if L.twos_abi_version() != ABI_VERSION:
        raise RuntimeError("libtwos.so ABI version mismatch")
    _lib = L
    return L


def check(rc: int) -> None:
    if rc != OK:
        raise TwosError(rc, load().twos_last_error().decode(errors="replace"))
