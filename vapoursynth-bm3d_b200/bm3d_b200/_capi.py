"""ctypes declarations of include/bm3d_b200.h (the library's C ABI)."""
import ctypes as C
import os

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(os.path.dirname(_HERE), "lib", "libbm3d_b200.so")

BM3D_OK, BM3D_ERR_ARG, BM3D_ERR_CUDA, BM3D_ERR_UNSUPPORTED, BM3D_ERR_STATE = 0, 1, 2, 3, 4
GRAY, RGB, YUV = 1, 2, 3
INTEGER, FLOAT = 0, 1
MEM_HOST, MEM_DEVICE = 0, 1

# every symbol the header declares
EXPORTS = [
    "bm3d_map_create", "bm3d_map_free", "bm3d_map_set_int", "bm3d_map_set_float", "bm3d_map_set_data",
    "bm3d_map_set_clip", "bm3d_create", "bm3d_output_info", "bm3d_frame_window", "bm3d_get_frames",
    "bm3d_get_frames_async", "bm3d_set_stream", "bm3d_synchronize", "bm3d_free", "bm3d_get_error",
    "bm3d_set_log_callback", "bm3d_debug_matches", "bm3d_debug_slow_blocks", "bm3d_debug_dct3d",
    "bm3d_set_profiling", "bm3d_debug_stage_times", "bm3d_debug_launch_count", "bm3d_basic_noalloc",
    "bm3d_debug_reference_fp64", "bm3d_debug_bm_tc_counts", "bm3d_proposal_default_weights",
    "bm3d_proposal_descriptors", "bm3d_proposal_gradients", "bm3d_proposal_train", "bm3d_proposal_match",
    "bm3d_debug_proposal_sets", "bm3d_debug_threshold_rechecks", "bm3d_debug_set_recheck_band",
    "bm3d_debug_retained_counts",
]


class VideoInfo(C.Structure):
    _fields_ = [("color_family", C.c_int), ("sample_type", C.c_int), ("bits_per_sample", C.c_int),
                ("subsampling_w", C.c_int), ("subsampling_h", C.c_int), ("width", C.c_int),
                ("height", C.c_int), ("num_frames", C.c_int)]


class Frame(C.Structure):
    _fields_ = [("data", C.c_void_p * 3), ("stride", C.c_int64 * 3), ("memory", C.c_int),
                ("prop_bm3d_opp", C.c_int64), ("prop_range", C.c_int64), ("prop_matrix", C.c_int64),
                ("prop_v_radius", C.c_int64), ("prop_v_process", C.c_int64 * 3),
                ("prop_v_process_count", C.c_int)]


LOG_FN = C.CFUNCTYPE(None, C.c_int, C.c_char_p, C.c_void_p)

_lib = None


def lib():
    """Loads the in-tree library (raises if it has not been built)."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise RuntimeError("libbm3d_b200.so not built; run vapoursynth-bm3d_b200/build.py")
    L = C.CDLL(LIB_PATH)
    P = C.POINTER
    L.bm3d_map_create.restype = C.c_void_p
    L.bm3d_map_free.argtypes = [C.c_void_p]
    L.bm3d_map_set_int.argtypes = [C.c_void_p, C.c_char_p, C.c_int64]
    L.bm3d_map_set_float.argtypes = [C.c_void_p, C.c_char_p, C.c_double]
    L.bm3d_map_set_data.argtypes = [C.c_void_p, C.c_char_p, C.c_char_p]
    L.bm3d_map_set_clip.argtypes = [C.c_void_p, C.c_char_p, P(VideoInfo)]
    L.bm3d_create.argtypes = [C.c_char_p, C.c_void_p, P(C.c_void_p)]
    L.bm3d_output_info.argtypes = [C.c_void_p, P(VideoInfo)]
    L.bm3d_frame_window.argtypes = [C.c_void_p, C.c_int, C.c_int, P(C.c_int), P(C.c_int)]
    L.bm3d_get_frames.argtypes = [C.c_void_p, C.c_int, C.c_int, P(P(Frame)), P(P(Frame)), P(P(Frame))]
    L.bm3d_get_frames_async.argtypes = L.bm3d_get_frames.argtypes
    L.bm3d_set_stream.argtypes = [C.c_void_p, C.c_void_p]
    L.bm3d_synchronize.argtypes = [C.c_void_p]
    L.bm3d_free.argtypes = [C.c_void_p]
    L.bm3d_get_error.restype = C.c_char_p
    L.bm3d_set_log_callback.argtypes = [LOG_FN, C.c_void_p]
    L.bm3d_debug_matches.argtypes = [C.c_void_p, C.c_int, P(C.c_int), P(C.c_int), P(C.c_int), P(C.c_int),
                                     P(C.c_float), C.c_int]
    L.bm3d_debug_slow_blocks.argtypes = [C.c_void_p]
    L.bm3d_debug_slow_blocks.restype = C.c_int64
    L.bm3d_debug_bm_tc_counts.argtypes = [C.c_void_p, P(C.c_int64), P(C.c_int64)]
    L.bm3d_proposal_default_weights.argtypes = [P(C.c_float), C.c_int]
    L.bm3d_proposal_descriptors.argtypes = [P(C.c_float), C.c_int, C.c_int, P(C.c_float), P(C.c_float)]
    L.bm3d_proposal_gradients.argtypes = [P(C.c_float), C.c_int, C.c_int, P(C.c_float), P(C.c_int), C.c_int,
                                          P(C.c_float), P(C.c_float)]
    L.bm3d_proposal_train.argtypes = [P(C.c_float), C.c_int, C.c_int, C.c_int, C.c_int, C.c_int, C.c_float, C.c_uint64,
                                      P(C.c_float), P(C.c_float)]
    L.bm3d_proposal_match.argtypes = [P(C.c_float), C.c_int, C.c_int, P(C.c_float), C.c_int, C.c_int, C.c_int,
                                      C.c_float, C.c_int, P(C.c_int), P(C.c_int), P(C.c_int), C.c_int]
    L.bm3d_debug_proposal_sets.argtypes = [P(C.c_float), C.c_int, C.c_int, P(C.c_float), C.c_int, C.c_int, C.c_int,
                                           P(C.c_uint32), P(C.c_int64), C.c_int]
    L.bm3d_debug_threshold_rechecks.argtypes = [C.c_void_p, P(C.c_int64), P(C.c_int64)]
    L.bm3d_debug_set_recheck_band.argtypes = [C.c_void_p, C.c_float]
    L.bm3d_debug_retained_counts.argtypes = [C.c_void_p, C.c_int, P(C.c_int), C.c_int]
    L.bm3d_set_profiling.argtypes = [C.c_void_p, C.c_int]
    L.bm3d_debug_stage_times.argtypes = [C.c_void_p, P(C.c_double), C.c_int]
    L.bm3d_debug_launch_count.restype = C.c_int64
    L.bm3d_debug_reference_fp64.argtypes = [C.c_void_p, C.c_int, P(C.c_double), C.c_int64]
    L.bm3d_debug_dct3d.argtypes = [P(C.c_float), C.c_int, C.c_int, C.c_int, C.c_int, C.c_int]
    L.bm3d_basic_noalloc.argtypes = [C.c_void_p, C.c_void_p, C.c_int, C.c_int, C.c_int64, C.c_char_p, C.c_double,
                                     C.c_void_p]
    _lib = L
    return L


def last_error():
    return lib().bm3d_get_error().decode()
