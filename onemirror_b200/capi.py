"""ctypes binding of the qmcrt C-ABI (include/qmcrt.h).

This is the binding a Python caller of the library uses; the structures
mirror the header field for field.  Loading fails loudly when the in-tree
library has not been built: there is no fallback implementation.
"""
import ctypes as C
import os

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "lib", "libqmcrt.so")

# status codes
OK, ERR_INVALID_ARGUMENT, ERR_CUDA, ERR_OUT_OF_MEMORY, ERR_NOT_SUPPORTED, ERR_TIMEOUT, ERR_SAMPLING, ERR_INTERNAL = range(8)

QUIRK_SKIP_ORIGIN_CELL = 1 << 0
QUIRK_AABB_RADIUS = 1 << 1
QUIRK_SELF_HIT = 1 << 2
QUIRK_PREV_PERTURB = 1 << 3
QUIRK_ZENITH_FRAME = 1 << 4
QUIRK_PIXEL_EDGE = 1 << 5
QUIRKS_REFERENCE = 0x3F

RECEIVER_FLAT, RECEIVER_CYLINDER = 0, 1
POINTS_POISSON, POINTS_GRID = 0, 1
DEPOSIT_NEAREST, DEPOSIT_BILINEAR = 0, 1
ATTEN_NONE, ATTEN_POLY_EXP = 0, 1
CAND_CAP = 32  # QMCRT_CAND_CAP: occluder candidates kept per heliostat and walk
TRIM_SORTED, TRIM_HEAPS = 0, 1
SMOOTH_COUNTS, SMOOTH_ENERGY = 0, 1
TIMING_TRACE, TIMING_SETUP, TIMING_FINALIZE, TIMING_ALL = 1, 2, 4, 7
RAY_SHADOWED, RAY_BLOCKED, RAY_HIT, RAY_OFFMAP = 1, 2, 4, 8

fp = C.POINTER(C.c_float)
dp = C.POINTER(C.c_double)
i32p = C.POINTER(C.c_int32)
u32p = C.POINTER(C.c_uint32)


class Field(C.Structure):
    _fields_ = [("n", C.c_int32), ("pos", fp), ("size", fp), ("aim", fp), ("normal", fp),
                ("slope_sigma", fp), ("sigma", C.c_float), ("tilt", fp)]


class Receiver(C.Structure):
    _fields_ = [("type", C.c_int32), ("pos", C.c_float * 3), ("size", C.c_float * 3),
                ("normal", C.c_float * 3), ("face", C.c_int32), ("res_x", C.c_int32), ("res_y", C.c_int32)]


class GridParams(C.Structure):
    _fields_ = [("cell", C.c_float * 3), ("margin", C.c_float), ("explicit_bounds", C.c_int32),
                ("origin", C.c_float * 3), ("extent", C.c_float * 3), ("fine_div", C.c_int32)]


class Sun(C.Structure):
    _fields_ = [("dir", C.c_float * 3), ("dni", C.c_float), ("csr", C.c_float)]


class TraceParams(C.Structure):
    _fields_ = [("seed", C.c_uint64), ("rays", C.c_uint64), ("rays_per_point", C.c_int32),
                ("point_mode", C.c_int32), ("point_spacing", C.c_float), ("reflectivity", C.c_float),
                ("quirks", C.c_uint32), ("deposit", C.c_int32), ("accumulate", C.c_int32),
                ("kernel_variant", C.c_int32), ("item", C.c_uint32), ("attenuation", C.c_int32),
                ("ray_begin", C.c_uint64), ("ray_end", C.c_uint64)]


class Outputs(C.Structure):
    _fields_ = [("d_counts", C.c_void_p), ("d_energy", C.c_void_p), ("d_flux", C.c_void_p),
                ("d_ray_flags", C.c_void_p), ("d_ray_pixel", C.c_void_p)]


class TraceStats(C.Structure):
    _fields_ = [("rays", C.c_uint64), ("shadowed", C.c_uint64), ("blocked", C.c_uint64), ("hit", C.c_uint64),
                ("offmap", C.c_uint64), ("rect_tests", C.c_uint64), ("dda_cells", C.c_uint64),
                ("total_power", C.c_double), ("intercepted_power", C.c_double), ("intercept_ratio", C.c_double)]


class TableInputs(C.Structure):
    _fields_ = [("d_sun_local", C.c_void_p), ("d_turb_local", C.c_void_p), ("table_size", C.c_int64),
                ("d_start", C.c_void_p), ("d_point_xz", C.c_void_p), ("d_point_helio", C.c_void_p),
                ("points", C.c_int64), ("rays_per_point", C.c_int32)]


class GridInfo(C.Structure):
    _fields_ = [("origin", C.c_float * 3), ("cell", C.c_float * 3), ("dims", C.c_int32 * 3),
                ("cells", C.c_int64), ("entries", C.c_int64), ("fine_div", C.c_int32)]


class BatchItem(C.Structure):
    _fields_ = [("scene", C.c_int32), ("sun", Sun)]


class BatchTuning(C.Structure):
    _fields_ = [("chunk_rays", C.c_int32), ("ctas_per_sm", C.c_int32), ("tile", C.c_int32), ("ms", C.c_float)]


class SmoothParams(C.Structure):
    _fields_ = [("radius", C.c_int32), ("ratio", C.c_float), ("method", C.c_int32), ("source", C.c_int32)]


class Timing(C.Structure):
    _fields_ = [("setup_ms", C.c_float), ("trace_kernel_ms", C.c_float), ("finalize_ms", C.c_float)]


class FacetParams(C.Structure):
    _fields_ = [("a", C.c_float), ("b", C.c_float), ("normal", C.c_float * 3), ("centre", C.c_float * 3),
                ("rows", C.c_int32), ("cols", C.c_int32), ("facet", C.c_float), ("gap", C.c_float),
                ("thickness", C.c_float), ("reference_frame", C.c_int32)]


class LayoutParams(C.Structure):
    _fields_ = [("n", C.c_int32), ("helio_w", C.c_float), ("helio_h", C.c_float), ("thickness", C.c_float),
                ("r_min", C.c_float), ("r_max", C.c_float), ("az_center_deg", C.c_float),
                ("az_span_deg", C.c_float), ("spacing", C.c_float), ("jitter", C.c_float),
                ("mount_height", C.c_float), ("seed", C.c_uint64)]


# name -> (restype, argtypes); every symbol declared in include/qmcrt.h
PROTOTYPES = {
    "qmcrt_version": (C.c_char_p, []),
    "qmcrt_status_string": (C.c_char_p, [C.c_int]),
    "qmcrt_last_error": (C.c_char_p, []),
    "qmcrt_sun_direction": (C.c_int, [C.c_float, C.c_float, fp]),
    "qmcrt_solar_declination": (C.c_float, [C.c_int32]),
    "qmcrt_solar_position": (C.c_int, [C.c_float, C.c_float, C.c_float, fp, fp]),
    "qmcrt_batch_create": (C.c_int, [C.POINTER(C.c_void_p), C.c_int32, C.POINTER(BatchItem), C.c_int32,
                                     C.POINTER(TraceParams), C.POINTER(C.c_void_p)]),
    "qmcrt_batch_destroy": (C.c_int, [C.c_void_p]),
    "qmcrt_batch_autotune": (C.c_int, [C.c_void_p, C.POINTER(BatchTuning), C.c_void_p]),
    "qmcrt_batch_set_tuning": (C.c_int, [C.c_void_p, C.POINTER(BatchTuning)]),
    "qmcrt_batch_run": (C.c_int, [C.c_void_p, C.c_void_p]),
    "qmcrt_batch_capture": (C.c_int, [C.c_void_p]),
    "qmcrt_batch_launch": (C.c_int, [C.c_void_p, C.c_void_p]),
    "qmcrt_batch_maps": (C.c_int, [C.c_void_p, C.c_int32, C.POINTER(C.c_void_p), C.POINTER(C.c_void_p)]),
    "qmcrt_batch_read": (C.c_int, [C.c_void_p, C.c_int32, u32p, fp, C.POINTER(TraceStats), C.c_void_p]),
    "qmcrt_buie_table": (C.c_int, [C.c_float, fp, fp, fp, fp]),
    "qmcrt_layout_radial_staggered": (C.c_int, [C.POINTER(LayoutParams), fp, C.c_int32, i32p]),
    "qmcrt_scn_parse": (C.c_int, [C.c_char_p, C.POINTER(Receiver), C.POINTER(GridParams), fp, fp, C.c_int32, i32p]),
    "qmcrt_layout_paraboloid_facets": (C.c_int, [C.POINTER(FacetParams), fp, fp, fp, C.c_int32, i32p]),
    "qmcrt_write_flux_csv": (C.c_int, [C.c_char_p, fp, C.c_int32, C.c_int32, C.c_int32, C.c_int32]),
    "qmcrt_write_intercept_ratio": (C.c_int, [C.c_char_p, fp, C.c_int32, C.c_int32, C.c_float, C.c_int32, fp]),
    "qmcrt_scene_create": (C.c_int, [C.POINTER(Field), C.POINTER(Receiver), C.POINTER(GridParams), C.POINTER(C.c_void_p)]),
    "qmcrt_scene_destroy": (C.c_int, [C.c_void_p]),
    "qmcrt_scene_set_field": (C.c_int, [C.c_void_p, C.POINTER(Field), C.c_void_p]),
    "qmcrt_scene_set_sun": (C.c_int, [C.c_void_p, C.POINTER(Sun), C.c_uint32, C.c_void_p]),
    "qmcrt_scene_grid_info": (C.c_int, [C.c_void_p, C.POINTER(GridInfo)]),
    "qmcrt_scene_read_grid": (C.c_int, [C.c_void_p, i32p, i32p, C.c_void_p]),
    "qmcrt_scene_read_geometry": (C.c_int, [C.c_void_p, dp, dp, C.c_void_p]),
    "qmcrt_scene_read_candidates": (C.c_int, [C.c_void_p, C.c_int32, i32p, i32p, C.c_void_p]),
    "qmcrt_fp64_recip_probe": (C.c_int, [C.c_void_p, C.c_int64, C.c_void_p, C.c_void_p, C.c_void_p]),
    "qmcrt_scene_sample_points": (C.c_int, [C.c_void_p, C.POINTER(TraceParams), C.POINTER(C.c_int64), C.c_void_p]),
    "qmcrt_scene_read_points": (C.c_int, [C.c_void_p, fp, i32p, C.c_void_p]),
    "qmcrt_sample_points_noalloc": (C.c_int, [fp, C.c_int32, C.c_int64, C.c_float, C.c_uint64, C.c_void_p,
                                              C.c_void_p, C.c_void_p]),
    "qmcrt_trace": (C.c_int, [C.c_void_p, C.POINTER(Sun), C.POINTER(TraceParams), C.POINTER(Outputs),
                              C.POINTER(TraceStats), C.c_void_p]),
    "qmcrt_trace_tables": (C.c_int, [C.c_void_p, C.POINTER(Sun), C.POINTER(TableInputs), C.POINTER(TraceParams),
                                     C.POINTER(Outputs), C.POINTER(TraceStats), C.c_void_p]),
    "qmcrt_trace_host": (C.c_int, [C.c_void_p, C.POINTER(Field), C.POINTER(Sun), C.POINTER(TraceParams), u32p, fp,
                                   C.POINTER(TraceStats), C.c_void_p]),
    "qmcrt_results_host": (C.c_int, [C.c_void_p, C.POINTER(Field), C.POINTER(Sun), C.POINTER(TraceParams),
                                     C.POINTER(SmoothParams), u32p, fp, fp, C.POINTER(TraceStats), C.c_void_p]),
    "qmcrt_smooth_trimmed_u32": (C.c_int, [C.c_void_p, C.c_void_p, C.c_int32, C.c_int32, C.c_int32, C.c_float,
                                           C.c_int32, C.c_void_p]),
    "qmcrt_smooth_trimmed_f32": (C.c_int, [C.c_void_p, C.c_void_p, C.c_int32, C.c_int32, C.c_int32, C.c_float,
                                           C.c_int32, C.c_void_p]),
    "qmcrt_scene_timing": (C.c_int, [C.c_void_p, C.c_void_p]),
    "qmcrt_scene_set_timing": (C.c_int, [C.c_void_p, C.c_uint32]),
    "qmcrt_adjoint_forward": (C.c_int, [C.c_void_p, C.POINTER(Sun), C.POINTER(TraceParams), C.c_void_p, C.c_uint64,
                                        C.c_void_p, C.POINTER(C.c_double), C.POINTER(C.c_void_p), C.c_void_p]),
    "qmcrt_adjoint_backward": (C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p]),
    "qmcrt_adjoint_replay": (C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p, C.POINTER(C.c_double), C.c_void_p]),
    "qmcrt_tape_loss": (C.c_int, [C.c_void_p, C.POINTER(C.c_double), C.c_void_p]),
    "qmcrt_tape_energy": (C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p]),
    "qmcrt_buie_sample_probe": (C.c_int, [C.c_float, C.c_void_p, C.c_int64, C.c_void_p, C.c_void_p]),
    "qmcrt_adjoint_loss": (C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.POINTER(C.c_double),
                                     C.c_void_p]),
    "qmcrt_tape_free": (C.c_int, [C.c_void_p]),
    "qmcrt_fp32_peak_probe": (C.c_int, [C.c_void_p, C.c_int32, dp, C.c_void_p]),
    "qmcrt_philox_blocks": (C.c_int, [u32p, u32p, C.c_int64, C.c_void_p, C.c_void_p]),
}

_lib = None


class QmcrtError(RuntimeError):
    def __init__(self, status, msg):
        super().__init__("qmcrt status %d: %s" % (status, msg))
        self.status = status


def lib():
    """The loaded library (raises if it was not built)."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise RuntimeError("libqmcrt.so is not built (run __graft_entry__.build()); "
                               "there is no CPU fallback for the tracer")
        L = C.CDLL(LIB_PATH)
        for name, (res, args) in PROTOTYPES.items():
            f = getattr(L, name)
            f.restype = res
            f.argtypes = args
        _lib = L
    return _lib


def check(status):
    if status != OK:
        raise QmcrtError(status, lib().qmcrt_last_error().decode())
    return status


def as_fp(a):
    return a.ctypes.data_as(fp) if a is not None else None


def as_i32p(a):
    return a.ctypes.data_as(i32p) if a is not None else None


def as_u32p(a):
    return a.ctypes.data_as(u32p) if a is not None else None
