"""ctypes declarations of include/gpsb200.h and the loader of libgpsb200.so.

The library is built in-tree (gps-pbvr-web_b200/build.py). Loading fails loudly when it is
missing: there is no CPU fallback of the renderer.
"""
import ctypes as C
import os

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libgpsb200.so")

GPSB_OK = 0
STATUS_NAMES = {0: "OK", 1: "INVALID_ARGUMENT", 2: "LIMIT", 3: "CUDA", 4: "OUT_OF_MEMORY", 5: "TIMEOUT",
                6: "STATE", 7: "PARSE"}


class Gaussian(C.Structure):
    _fields_ = [("pos_opacity", C.c_float * 4), ("log_scale", C.c_float * 4), ("rot_wxyz", C.c_float * 4),
                ("color", C.c_float * 4)]


class Camera(C.Structure):
    _fields_ = [("view_rot", C.c_double * 9), ("view_pos", C.c_double * 3), ("focal_x", C.c_double),
                ("focal_y", C.c_double), ("cx", C.c_double), ("cy", C.c_double), ("low_pass", C.c_double)]


class PbvrParamsC(C.Structure):
    _fields_ = [("calibration", C.c_uint32), ("radial_correction", C.c_uint32), ("centre_depth", C.c_uint32),
                ("low_pass_jitter", C.c_uint32), ("base_k", C.c_float), ("reference_pixel_length", C.c_float)]


class ParamsC(C.Structure):
    _fields_ = [("spp_side", C.c_uint32), ("density_scale", C.c_float), ("max_points_per_splat", C.c_uint32),
                ("near_z", C.c_float), ("background", C.c_float * 3), ("exposure", C.c_float),
                ("srgb_output", C.c_uint32), ("exact_radius", C.c_uint32), ("sh_degree", C.c_uint32),
                ("path", C.c_uint32), ("method", C.c_uint32), ("pbvr", PbvrParamsC)]


class StatsC(C.Structure):
    _fields_ = [("points", C.c_uint64), ("truncated_splats", C.c_uint64), ("dropped_points", C.c_uint64),
                ("visible_splats", C.c_uint64), ("orphan_subpixels", C.c_uint64), ("candidates", C.c_uint64),
                ("undercovered_splats", C.c_uint64), ("skipped_ensembles", C.c_uint64), ("ensembles", C.c_uint64),
                ("probe_demand", C.c_uint64), ("issue", C.c_uint32), ("_pad", C.c_uint32),
                ("subpixel_writes", C.c_uint64), ("list_entries", C.c_uint64), ("particles", C.c_uint64)]


class ProfileC(C.Structure):
    _fields_ = [("launches", C.c_uint64 * 8), ("ms", C.c_double * 8), ("total_launches", C.c_uint64)]


class TuningC(C.Structure):
    _fields_ = [("sort_digit_bits", C.c_uint32), ("blend_tile_w", C.c_uint32), ("blend_tile_h", C.c_uint32),
                ("particle_items", C.c_uint32), ("particle_blocks_per_sm", C.c_uint32), ("ensemble_batch", C.c_uint32)]


class SessionStateC(C.Structure):
    _fields_ = [("sorted_active", C.c_uint32), ("sorted_ok", C.c_uint32), ("moving_prefers_gps", C.c_uint32),
                ("lod_moving", C.c_uint32), ("effective_per_frame", C.c_uint32), ("lod_n", C.c_uint32),
                ("auto_density", C.c_float), ("history_epoch", C.c_uint32), ("frames_since_reset", C.c_uint32),
                ("next_seed", C.c_uint32), ("ensemble_counter", C.c_uint32), ("slow_frames", C.c_uint32),
                ("last_demand", C.c_uint64), ("ema_ms", C.c_double)]


# gpsb_session_backend: the renderer calls of a frame-loop session
BE_RENDER = C.CFUNCTYPE(C.c_int, C.c_void_p, C.c_void_p, C.c_void_p, C.c_uint32, C.c_uint32)
BE_SORTED = C.CFUNCTYPE(C.c_int, C.c_void_p, C.c_void_p, C.c_void_p, C.c_uint32)
BE_PROBE = C.CFUNCTYPE(C.c_int, C.c_void_p, C.c_void_p, C.c_void_p)
BE_CALL = C.CFUNCTYPE(C.c_int, C.c_void_p)
BE_STATS = C.CFUNCTYPE(C.c_int, C.c_void_p, C.c_void_p)
BE_U32 = C.CFUNCTYPE(C.c_uint32, C.c_void_p)


class SessionBackendC(C.Structure):
    _fields_ = [("render_ensembles", BE_RENDER), ("render_sorted", BE_SORTED), ("probe_demand", BE_PROBE),
                ("request_stats", BE_CALL), ("latest_stats", BE_STATS), ("stats_issued", BE_U32),
                ("accumulated", BE_U32), ("submitted", BE_U32), ("reset_accum", BE_CALL), ("reset_stats", BE_CALL),
                ("gaussian_count", BE_U32)]


STAGES = ["geometry", "count_scan", "particles", "resolve", "clear", "primitive", "sorted", "composite"]


P = C.c_void_p
U32 = C.c_uint32
SZ = C.c_size_t
ST = C.c_int
U64 = C.c_uint64

# name -> (restype, argtypes); every function declared in include/gpsb200.h
SIGNATURES = {
    "gpsb_params_default": (None, [P]),
    "gpsb_version": (C.c_char_p, []),
    "gpsb_last_error": (C.c_char_p, [P]),
    "gpsb_camera_look_at": (ST, [P, P, P, C.c_double, U32, U32, P]),
    "gpsb_orbit_camera": (ST, [P, C.c_double, C.c_double, C.c_double, P, C.c_double, U32, U32, P]),
    "gpsb_robust_sphere": (ST, [P, SZ, P, P]),
    "gpsb_radius_lut": (ST, [P]),
    "gpsb_estimate_memory": (None, [U32, U32, U32, SZ, P, P, P]),
    "gpsb_create": (ST, [C.c_int, U32, U32, U32, P]),
    "gpsb_destroy": (None, [P]),
    "gpsb_set_stream": (ST, [P, P]),
    "gpsb_set_feature_accum": (ST, [P, P]),
    "gpsb_set_footprint": (ST, [P, U32, C.c_float, U32, U32]),
    "gpsb_set_fast_decisions": (ST, [P, U32]),
    "gpsb_debug_fast_counts": (ST, [P, P]),
    "gpsb_debug_fast_bounds": (ST, [P, P]),
    "gpsb_set_gaussians": (ST, [P, P, SZ]),
    "gpsb_set_gaussians_sh": (ST, [P, P, SZ, P, SZ, U32]),
    "gpsb_set_gaussians_sh_device": (ST, [P, P, SZ, P, SZ, U32]),
    "gpsb_resize": (ST, [P, U32, U32, U32]),
    "gpsb_reset_accum": (ST, [P]),
    "gpsb_reset_stats": (ST, [P]),
    "gpsb_render_ensembles": (ST, [P, P, P, U32, U32]),
    "gpsb_render_trajectory": (ST, [P, P, U32, P, U32, U32, P]),
    "gpsb_render_trajectory_graph": (ST, [P, P, U32, P, U32, U32, P]),
    "gpsb_render_sorted": (ST, [P, P, P, U32]),
    "gpsb_probe_demand": (ST, [P, P, P]),
    "gpsb_read_accum": (ST, [P, P]),
    "gpsb_accum_device_ptr": (ST, [P, P]),
    "gpsb_read_stats": (ST, [P, P]),
    "gpsb_request_stats": (ST, [P]),
    "gpsb_latest_stats": (ST, [P, P]),
    "gpsb_stats_issued": (U32, [P]),
    "gpsb_read_sorted": (ST, [P, P, P]),
    "gpsb_accumulated": (U32, [P]),
    "gpsb_submitted": (U32, [P]),
    "gpsb_sync": (ST, [P]),
    "gpsb_composite_rgba8": (ST, [P, P, U32, U32, P]),
    "gpsb_size": (None, [P, P, P, P]),
    "gpsb_gaussian_count": (U32, [P]),
    "gpsb_sh_max_degree": (U32, [P]),
    "gpsb_sh_bytes": (C.c_uint64, [P]),
    "gpsb_debug_read_counts": (ST, [P, U32, P]),
    "gpsb_debug_read_subpixels": (ST, [P, U32, P]),
    "gpsb_debug_error_word": (U32, [P]),
    "gpsb_debug_particle_seeds": (ST, [P, U32, U64, U32, P]),
    "gpsb_debug_fmath": (ST, [U32, P, P, U64]),
    "gpsb_load_ply": (ST, [P, SZ, P, P, P, P]),
    "gpsb_load_ply_device": (ST, [P, SZ, P, P, P, P, P]),
    "gpsb_ply_last_error": (C.c_char_p, []),
    "gpsb_profile_enable": (ST, [P, C.c_int]),
    "gpsb_profile_read": (ST, [P, P]),
    "gpsb_sort_pairs_noalloc": (ST, [P, P, P, P, U32, U32, P, P]),
    "gpsb_set_tuning": (ST, [P, P]),
    "gpsb_scan_u32": (ST, [P, P, P, U32, P]),
    "gpsb_sort_pairs": (ST, [P, P, P, P, P, U32, U32]),
    "gpsb_p0_sample": (ST, [P, U32, U32, U32, U32, P]),
    "gpsb_get_tuning": (ST, [P, P]),
    "gpsb_session_create": (ST, [P, P]),
    "gpsb_session_create_with_backend": (ST, [P, P, P]),
    "gpsb_session_destroy": (None, [P]),
    "gpsb_session_configure": (ST, [P, P, U32, U32]),
    "gpsb_session_set_lod": (ST, [P, C.c_int, C.c_double, U32]),
    "gpsb_session_set_point_budget": (ST, [P, C.c_double]),
    "gpsb_session_set_render_path": (ST, [P, U32, C.c_double]),
    "gpsb_session_set_camera": (ST, [P, P, C.c_int]),
    "gpsb_session_reset": (ST, [P]),
    "gpsb_session_frame": (ST, [P, C.c_double, P]),
    "gpsb_session_read_state": (ST, [P, P]),
    # denoiser kernels (return cudaError_t codes)
    "gpsb_dn_conv_fwd": (ST, [P, ST, ST, ST, ST, ST, ST, P, ST, ST, P, P, ST, ST, ST, ST, P, P]),
    "gpsb_dn_conv3_weight_bytes": (C.c_ulonglong, [ST, ST]),
    "gpsb_dn_channel_sum": (ST, [P, ST, ST, ST, P, P]),
    "gpsb_dn_mean_rgb": (ST, [P, ST, P, P]),
    "gpsb_denoiser_create": (ST, [ST, P]),
    "gpsb_denoiser_destroy": (None, [P]),
    "gpsb_denoiser_last_error": (C.c_char_p, [P]),
    "gpsb_denoiser_layer_shape": (ST, [U32, P, P, P]),
    "gpsb_denoiser_set_layer": (ST, [P, U32, P, P]),
    "gpsb_denoiser_set_gate": (ST, [P, C.c_float]),
    "gpsb_denoiser_forward": (ST, [P, P, P, U32, U32, P, P]),
    "gpsb_denoiser_graph_state": (C.c_int, [P]),
    "gpsb_render_denoised": (ST, [P, P, P, P, U32, U32, C.c_float, U32, P, P, P]),
    "gpsb_dn_conv3_weights": (ST, [P, ST, ST, ST, P, P]),
    "gpsb_dn_conv3": (ST, [P, ST, ST, ST, ST, ST, ST, P, ST, P, P, ST, ST, ST, ST, P, P]),
    "gpsb_dn_conv_dw": (ST, [P, ST, P, ST, ST, ST, ST, ST, ST, ST, ST, P, P, P]),
    "gpsb_dn_flip": (ST, [P, ST, ST, ST, P, ST, ST, P]),
    "gpsb_dn_relu_bwd": (ST, [P, ST, ST, P, ST, ST, ST, ST, ST, P, ST, P]),
    "gpsb_dn_up2": (ST, [P, ST, ST, ST, ST, ST, P, ST, ST, P]),
    "gpsb_dn_up2_bwd": (ST, [P, ST, ST, ST, ST, ST, ST, P, P]),
    "gpsb_dn_pool2": (ST, [P, ST, ST, ST, ST, ST, ST, P, P]),
    "gpsb_dn_pool2_bwd_add": (ST, [P, ST, ST, ST, ST, P, ST, ST, P]),
    "gpsb_dn_bias_grad": (ST, [P, ST, ST, ST, ST, P, P]),
    "gpsb_dn_l1": (ST, [P, P, P, ST, P, P, C.c_float, P]),
    "gpsb_dn_residual": (ST, [P, P, ST, P, P]),
    "gpsb_dn_adam": (ST, [P, P, P, P, ST, C.c_float, C.c_float, C.c_float, C.c_float, ST, P, P]),
    "gpsb_dn_to_bf16": (ST, [P, ST, ST, ST, P, ST, P]),
    "gpsb_dn_pack": (ST, [P, P, ST, P, P, P]),
    "gpsb_dn_crop": (ST, [P, P, P, ST, ST, ST, P, ST, ST, ST, P, P, P, P, P]),
}

_lib = None


def lib():
    """The loaded renderer library (raises if it was not built)."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise RuntimeError(f"{LIB_PATH} is missing: build it with `python gps-pbvr-web_b200/build.py` "
                               "(the renderer has no CPU fallback)")
        L = C.CDLL(LIB_PATH)
        for name, (res, args) in SIGNATURES.items():
            f = getattr(L, name)
            f.restype = res
            f.argtypes = args
        _lib = L
    return _lib


def header_functions(header_path=None):
    """Function names declared in include/gpsb200.h (for the export check)."""
    import re
    path = header_path or os.path.join(os.path.dirname(HERE), "include", "gpsb200.h")
    text = open(path).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    # function names are followed by "(", function-pointer members of a struct by "(*"
    return sorted(set(re.findall(r"\b(gpsb_[a-z0-9_]+)\s*\((?!\s*\*)", text)))
