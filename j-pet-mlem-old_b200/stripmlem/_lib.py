"""ctypes binding of the C ABI in include/stripmlem.h (lib/libstripmlem.so).

The library is the product: if it is missing the import fails loudly; there
is no CPU fallback.
"""
import ctypes
import os

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(os.path.dirname(_HERE), "lib", "libstripmlem.so")

STRIP_OK = 0
STRIP_E_INVALID = -1
STRIP_E_CUDA = -2
STRIP_E_NOMEM = -3
STRIP_E_STATE = -4
STRIP_E_KERNEL = -5
STRIP_E_NODEVICE = -6

MODE_CPU = 0
MODE_GPU = 1
ACCUM_FP32 = 0
ACCUM_KAHAN = 1
ACCUM_FP64 = 2

ERROR_NAMES = {
    STRIP_E_INVALID: "invalid argument",
    STRIP_E_CUDA: "CUDA error",
    STRIP_E_NOMEM: "out of memory",
    STRIP_E_STATE: "call out of order",
    STRIP_E_KERNEL: "kernel error",
    STRIP_E_NODEVICE: "no CUDA device",
}


class Geometry(ctypes.Structure):
    _fields_ = [
        ("radius", ctypes.c_double),
        ("scintillator_length", ctypes.c_double),
        ("n_y_pixels", ctypes.c_int32),
        ("n_z_pixels", ctypes.c_int32),
        ("pixel_height", ctypes.c_double),
        ("pixel_width", ctypes.c_double),
        ("sigma_z", ctypes.c_double),
        ("sigma_dl", ctypes.c_double),
        ("center_y", ctypes.c_double),
        ("center_z", ctypes.c_double),
    ]


REGION_ELLIPSE, REGION_RECTANGLE, REGION_POINT = 0, 1, 2


class Region(ctypes.Structure):
    _fields_ = [("kind", ctypes.c_int32), ("reserved", ctypes.c_int32),
                ("z", ctypes.c_double), ("y", ctypes.c_double), ("a", ctypes.c_double),
                ("b", ctypes.c_double), ("angle_deg", ctypes.c_double),
                ("intensity", ctypes.c_double)]


class Simulation(ctypes.Structure):
    _fields_ = [("additive", ctypes.c_int32), ("uniform_angle", ctypes.c_int32),
                ("count_emitted", ctypes.c_int32), ("reserved", ctypes.c_int32),
                ("d_emitted", ctypes.c_void_p), ("d_detected", ctypes.c_void_p),
                ("pixel_size", ctypes.c_double), ("origin_z", ctypes.c_double),
                ("origin_y", ctypes.c_double)]


class Tuning(ctypes.Structure):
    _fields_ = [("tile", ctypes.c_int32), ("grab", ctypes.c_int32), ("ms", ctypes.c_double)]


class Stats(ctypes.Structure):
    _fields_ = [
        ("n_events", ctypes.c_int64),
        ("n_empty", ctypes.c_int64),
        ("n_overflow", ctypes.c_int64),
        ("n_tiles_z", ctypes.c_int32),
        ("n_tiles_y", ctypes.c_int32),
        ("tile_z", ctypes.c_int32),
        ("tile_y", ctypes.c_int32),
        ("halo_z", ctypes.c_int32),
        ("halo_y", ctypes.c_int32),
        ("n_work_items", ctypes.c_int32),
        ("n_subsets", ctypes.c_int32),
        ("max_box_w", ctypes.c_int32),
        ("max_box_h", ctypes.c_int32),
        ("smem_bytes", ctypes.c_int32),
        ("kernel_launches", ctypes.c_int32),
        ("last_iterate_ms", ctypes.c_double),
        ("last_setup_ms", ctypes.c_double),
        ("last_tile_ms", ctypes.c_double),
        ("n_fallback", ctypes.c_int64),
        ("max_item_events", ctypes.c_int32),
        ("reserved", ctypes.c_int32),
        ("last_upload_ms", ctypes.c_double),
    ]


class Ellipse(ctypes.Structure):
    _fields_ = [
        ("z", ctypes.c_double),
        ("y", ctypes.c_double),
        ("a", ctypes.c_double),
        ("b", ctypes.c_double),
        ("angle_deg", ctypes.c_double),
        ("activity", ctypes.c_double),
    ]


PROGRESS_CB = ctypes.CFUNCTYPE(ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_void_p)

_P = ctypes.POINTER
_f = _P(ctypes.c_float)
_d = _P(ctypes.c_double)
_ctx = ctypes.c_void_p

# name -> (restype, argtypes); every symbol include/stripmlem.h declares.
SIGNATURES = {
    "strip_ctx_create": (ctypes.c_int, [_P(Geometry), ctypes.c_int, _P(ctypes.c_void_p)]),
    "strip_ctx_destroy": (ctypes.c_int, [_ctx]),
    "strip_last_error": (ctypes.c_int, [_ctx, ctypes.c_char_p, ctypes.c_size_t]),
    "strip_device_name": (ctypes.c_int, [_ctx, ctypes.c_char_p, ctypes.c_size_t]),
    "strip_set_accumulation": (ctypes.c_int, [_ctx, ctypes.c_int]),
    "strip_get_stats": (ctypes.c_int, [_ctx, _P(Stats)]),
    "strip_set_events": (ctypes.c_int, [_ctx, _f, _f, _f, ctypes.c_int64, ctypes.c_int]),
    "strip_set_responses": (ctypes.c_int, [_ctx, _f, ctypes.c_int64, ctypes.c_int]),
    "strip_set_events_device": (
        ctypes.c_int,
        [_ctx, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int64, ctypes.c_int],
    ),
    "strip_set_image": (ctypes.c_int, [_ctx, _f]),
    "strip_get_image": (ctypes.c_int, [_ctx, _f]),
    "strip_get_sensitivity": (ctypes.c_int, [_ctx, ctypes.c_int, _f]),
    "strip_iterate": (
        ctypes.c_int,
        [_ctx, ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_int, PROGRESS_CB, ctypes.c_void_p],
    ),
    "strip_set_accumulator": (ctypes.c_int, [_ctx, ctypes.c_void_p]),
    "strip_accumulate": (ctypes.c_int, [_ctx, ctypes.c_int, ctypes.c_int, ctypes.c_int]),
    "strip_update": (ctypes.c_int, [_ctx, ctypes.c_double]),
    "strip_forward": (ctypes.c_int, [_ctx, _f, ctypes.c_double, ctypes.c_double, ctypes.c_int, _d]),
    "strip_adjoint": (ctypes.c_int, [_ctx, _d, ctypes.c_double, ctypes.c_double, ctypes.c_int, _d]),
    "strip_grad_sigma": (
        ctypes.c_int,
        [_ctx, _f, _d, ctypes.c_double, ctypes.c_double, _d, _d],
    ),
    "strip_forward_device": (
        ctypes.c_int,
        [_ctx, ctypes.c_void_p, ctypes.c_double, ctypes.c_double, ctypes.c_int, ctypes.c_void_p],
    ),
    "strip_adjoint_device": (
        ctypes.c_int,
        [_ctx, ctypes.c_void_p, ctypes.c_double, ctypes.c_double, ctypes.c_int, ctypes.c_void_p],
    ),
    "strip_grad_sigma_device": (
        ctypes.c_int,
        [_ctx, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_double, ctypes.c_double,
         ctypes.c_void_p],
    ),
    "strip_batch_create": (
        ctypes.c_int, [_P(ctypes.c_void_p), ctypes.c_int, ctypes.c_int, _P(ctypes.c_void_p)]),
    "strip_batch_iterate": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_int]),
    "strip_batch_stats": (
        ctypes.c_int,
        [ctypes.c_void_p, _d, _P(ctypes.c_int64), _P(ctypes.c_int32), _P(ctypes.c_int32)]),
    "strip_batch_last_error": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_char_p, ctypes.c_size_t]),
    "strip_batch_destroy": (ctypes.c_int, [ctypes.c_void_p]),
    "strip_autotune": (ctypes.c_int, [_ctx, ctypes.c_int, _P(Tuning)]),
    "strip_set_schedule": (ctypes.c_int, [_ctx, ctypes.c_int, ctypes.c_int]),
    "strip_set_item_events": (ctypes.c_int, [_ctx, ctypes.c_int]),
    "strip_load_responses_file": (ctypes.c_int, [_ctx, ctypes.c_char_p, ctypes.c_int64,
                                                 ctypes.c_int64, ctypes.c_int,
                                                 _P(ctypes.c_int64)]),
    "strip_debug_pixel_sets": (
        ctypes.c_int,
        [_ctx, _f, _f, _f, ctypes.c_int64, _P(ctypes.c_int32), _P(ctypes.c_int32), _P(ctypes.c_uint64)],
    ),
    "strip_debug_scale_item_stats": (ctypes.c_int, [_ctx, ctypes.c_float]),
    "strip_iterate_noalloc": (
        ctypes.c_int,
        [_P(Geometry), ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int64,
         ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int, ctypes.c_void_p],
    ),
    "strip_probe_fp32_peak": (ctypes.c_int, [ctypes.c_int, _d]),
    "strip_count_work": (
        ctypes.c_int,
        [_ctx, _P(ctypes.c_int64), _P(ctypes.c_int64), _P(ctypes.c_int64)],
    ),
    "strip_generate_events": (
        ctypes.c_int,
        [_P(Geometry), _P(Ellipse), ctypes.c_int, ctypes.c_uint64, ctypes.c_int64, _f, _f, _f],
    ),
    "strip_generate_events_device": (
        ctypes.c_int,
        [_P(Geometry), _P(Ellipse), ctypes.c_int, ctypes.c_uint64, ctypes.c_int64,
         ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p],
    ),
    "strip_generate_events_image_device": (
        ctypes.c_int,
        [_P(Geometry), _f, ctypes.c_uint64, ctypes.c_int64, ctypes.c_int,
         ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p],
    ),
    "strip_simulate_device": (
        ctypes.c_int,
        [_P(Geometry), _P(Region), ctypes.c_int, _P(Simulation), ctypes.c_uint64,
         ctypes.c_int64, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p,
         _P(ctypes.c_int64), _P(ctypes.c_int64)],
    ),
    "strip_simulate": (
        ctypes.c_int,
        [_P(Geometry), _P(Region), ctypes.c_int, _P(Simulation), ctypes.c_uint64,
         ctypes.c_int64, ctypes.c_int, _f, _f, _f, _P(ctypes.c_uint32), _P(ctypes.c_uint32),
         _P(ctypes.c_int64), _P(ctypes.c_int64)],
    ),
    "strip_generate_events_image": (
        ctypes.c_int,
        [_P(Geometry), _f, ctypes.c_uint64, ctypes.c_int64, ctypes.c_int, _f, _f, _f],
    ),
}



class HybridSetup(ctypes.Structure):
    """hybrid_setup of include/hybridmlem.h."""
    _fields_ = [
        ("n_columns", ctypes.c_int32),
        ("n_rows", ctypes.c_int32),
        ("n_planes", ctypes.c_int32),
        ("reserved", ctypes.c_int32),
        ("pixel_size", ctypes.c_double),
        ("z_left", ctypes.c_double),
        ("length", ctypes.c_double),
        ("sigma_z", ctypes.c_double),
        ("sigma_dl", ctypes.c_double),
    ]


class HybridStats(ctypes.Structure):
    """hybrid_stats of include/hybridmlem.h."""
    _fields_ = [
        ("n_responses", ctypes.c_int64),
        ("n_events", ctypes.c_int64),
        ("n_lors", ctypes.c_int64),
        ("n_pixel_infos", ctypes.c_int64),
        ("used_pixels", ctypes.c_int64),
        ("used_voxels", ctypes.c_int64),
        ("iterations", ctypes.c_int32),
        ("reserved", ctypes.c_int32),
        ("last_iteration_ms", ctypes.c_double),
    ]


class HybridCylinder(ctypes.Structure):
    """hybrid_cylinder of include/hybridmlem.h."""
    _fields_ = [(k, ctypes.c_double) for k in
                ("x", "y", "z", "radius", "half_length", "activity")]


HYBRID_SENS_CALCULATE, HYBRID_SENS_ONE, HYBRID_SENS_EXTERNAL, HYBRID_SENS_GIVEN = 0, 1, 2, 3
HYBRID_PROGRESS_CB = ctypes.CFUNCTYPE(None, ctypes.c_int32, ctypes.c_int32, ctypes.c_void_p)
_vp = ctypes.c_void_p

# every symbol include/hybridmlem.h declares
SIGNATURES.update({
    "hybrid_ctx_create": (ctypes.c_int, [_P(HybridSetup), ctypes.c_int32, _P(ctypes.c_void_p)]),
    "hybrid_ctx_destroy": (ctypes.c_int, [_ctx]),
    "hybrid_last_error": (ctypes.c_char_p, [_ctx]),
    "hybrid_set_geometry_from_matrix": (
        ctypes.c_int,
        [_ctx, ctypes.c_int32, _vp, ctypes.c_int64, _vp, _vp, _vp, _vp, _vp, ctypes.c_uint32,
         _vp, ctypes.c_int32]),
    "hybrid_get_geometry": (ctypes.c_int, [_ctx, _vp, _vp, _vp, _vp, _vp, _vp]),
    "hybrid_set_geometry_soa": (
        ctypes.c_int, [_ctx, ctypes.c_int32, _vp, ctypes.c_int64, _vp, _vp, _vp, _vp, _vp]),
    "hybrid_set_frames": (ctypes.c_int, [_ctx, ctypes.c_int64] + [_vp] * 9),
    "hybrid_set_sensitivity": (ctypes.c_int, [_ctx, ctypes.c_int32, _vp]),
    "hybrid_get_sensitivity": (ctypes.c_int, [_ctx, _vp]),
    "hybrid_set_responses": (ctypes.c_int, [_ctx, _vp, _vp, _vp, _vp, _vp, ctypes.c_int64]),
    "hybrid_get_frames": (ctypes.c_int, [_ctx, _vp, _vp, _vp, _vp, _vp, _vp]),
    "hybrid_iterate": (ctypes.c_int, [_ctx, ctypes.c_int32, HYBRID_PROGRESS_CB, _vp]),
    "hybrid_set_image": (ctypes.c_int, [_ctx, _vp]),
    "hybrid_set_accumulator": (ctypes.c_int, [_ctx, _vp]),
    "hybrid_accumulate": (ctypes.c_int, [_ctx]),
    "hybrid_update": (ctypes.c_int, [_ctx]),
    "hybrid_get_image": (ctypes.c_int, [_ctx, _vp]),
    "hybrid_get_stats": (ctypes.c_int, [_ctx, _P(HybridStats)]),
    "hybrid_debug_atan2": (ctypes.c_int, [ctypes.c_int32, _vp, _vp, ctypes.c_int64,
                                          ctypes.c_int32, _vp]),
    "hybrid_smear_responses": (ctypes.c_int, [ctypes.c_int64, ctypes.c_double, ctypes.c_double,
                                              ctypes.c_int64, _vp, _vp, _vp]),
    "hybrid_parse_responses_text": (ctypes.c_int, [ctypes.c_char_p, ctypes.c_int64,
                                                   ctypes.c_int64] + [_vp] * 5
                                    + [_P(ctypes.c_int64)]),
    "hybrid_generate_responses": (
        ctypes.c_int,
        [ctypes.c_int32, _vp, _P(HybridCylinder), ctypes.c_int32, ctypes.c_double,
         ctypes.c_double, ctypes.c_double, ctypes.c_uint64, ctypes.c_int64, ctypes.c_int32,
         _vp, _vp, _vp, _vp, _vp]),
})

_lib = None


def load():
    """Loads lib/libstripmlem.so (raises OSError when it was not built)."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise OSError(
            f"{LIB_PATH} is missing: build it with `make -C j-pet-mlem-old_b200` "
            "(there is no CPU fallback)")
    lib = ctypes.CDLL(LIB_PATH)
    for name, (res, args) in SIGNATURES.items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    _lib = lib
    return lib
