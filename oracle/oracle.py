"""ctypes wrapper of the CPU oracle (oracle/liboracle.so) and of the reference's own Block.h
(oracle/_ref/librefblock.so, when built).

TEST INFRASTRUCTURE ONLY: imported by tests/, by __graft_entry__.smoke() and by bench.py's CPU
baseline leg, always as the checker or the timed CPU baseline, never by the product.
"""
import ctypes as C
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB = os.path.join(HERE, "liboracle.so")
REF_LIB = os.path.join(HERE, "_ref", "librefblock.so")

_P = C.POINTER
_F = _P(C.c_float)
_I = _P(C.c_int)
_L = _P(C.c_longlong)

STAT_NAMES = ("groups", "coefficients", "flips_vs_fp64", "near_threshold", "blocks", "tie_blocks")


class Params(C.Structure):
    _fields_ = [("wiener", C.c_int), ("B", C.c_int), ("step", C.c_int), ("G", C.c_int), ("R", C.c_int),
                ("bmstep", C.c_int), ("th_mse", C.c_double), ("lambda_", C.c_double), ("sigma", C.c_double * 3),
                ("matrix", C.c_int), ("process", C.c_int * 3), ("radius", C.c_int), ("psnum", C.c_int),
                ("psrange", C.c_int), ("psstep", C.c_int), ("wiener_mode", C.c_int)]


_lib = None
_ref = None


def build():
    """Builds liboracle.so (and _ref/librefblock.so when the reference checkout is present)."""
    subprocess.run(["make", "-s", "-C", HERE], check=True)


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB):
            build()
        L = C.CDLL(LIB)
        L.oracle_default_params.argtypes = [C.c_int, C.c_int, C.c_char_p, C.c_double, _P(Params)]
        L.oracle_matrix_default.argtypes = [C.c_int, C.c_int]
        L.oracle_matrix_norms.argtypes = [C.c_int, _P(C.c_double)]
        L.oracle_filter_tables.argtypes = [C.c_int, C.c_double, C.c_int, C.c_int, C.c_double, _P(C.c_double), _F, _F]
        L.oracle_bm3d.argtypes = [_P(Params), C.c_int, C.c_int, C.c_int, C.c_int, C.c_int, _F, _F, _F, C.c_int]
        L.oracle_bm3d_ex.argtypes = [_P(Params), C.c_int, C.c_int, C.c_int, C.c_int, C.c_int, _F, _F, _F, C.c_int, _L]
        L.oracle_bm3d_matches.argtypes = [_P(Params), C.c_int, C.c_int, C.c_int, _F, _I, _I, _I, _F]
        L.oracle_bm3d_matches_ex.argtypes = [_P(Params), C.c_int, C.c_int, C.c_int, _F, _I, _I, _I, _F, C.c_int, _L]
        L.oracle_vbm3d_matches.argtypes = [_P(Params), C.c_int, C.c_int, C.c_int, C.c_int, C.c_int, _F, _I, _I, _I, _I, _F]
        L.oracle_vbm3d_matches_ex.argtypes = [_P(Params), C.c_int, C.c_int, C.c_int, C.c_int, C.c_int, _F, _I, _I, _I, _I,
                                              _F, C.c_int, _L]
        L.oracle_vbm3d.argtypes = [_P(Params), C.c_int, C.c_int, C.c_int, C.c_int, C.c_int, C.c_int, C.c_int, _F, _F, _F, C.c_int]
        L.oracle_vbm3d_ex.argtypes = [_P(Params), C.c_int, C.c_int, C.c_int, C.c_int, C.c_int, C.c_int, C.c_int, _F, _F, _F,
                                      C.c_int, _L]
        L.oracle_vaggregate.argtypes = [C.c_int, C.c_int, C.c_int, C.c_int, _I, C.c_int, C.c_int, C.c_int, _F, _F]
        L.oracle_dct3d.argtypes = [_F, C.c_int, C.c_int, C.c_int]
        L.oracle_dct3d_scalar.argtypes = [_F, C.c_int, C.c_int, C.c_int]
        L.oracle_dct_tables.argtypes = [C.c_int, _F, _F, _F]
        L.oracle_int2float.argtypes = [C.c_void_p, C.c_int, C.c_int, C.c_int, C.c_int, C.c_int, C.c_int, C.c_int, C.c_int, _F]
        L.oracle_float2int.argtypes = [_F, C.c_int, C.c_int, C.c_int, C.c_int, C.c_int, C.c_int, C.c_int, C.c_int, C.c_void_p]
        L.oracle_rgb2opp_float.argtypes = [_F, _F, _F, C.c_int, C.c_int, C.c_int, _F, _F, _F]
        L.oracle_opp2rgb_float.argtypes = [_F, _F, _F, C.c_int, C.c_int, C.c_int, _F, _F, _F]
        V = C.c_void_p
        L.oracle_rgb2opp_any.argtypes = [V, V, V, C.c_int, C.c_int, V, V, V, C.c_int, C.c_int, C.c_int, C.c_int,
                                         C.c_int, C.c_int]
        L.oracle_opp2rgb_any.argtypes = L.oracle_rgb2opp_any.argtypes
        L.oracle_rgb2y_any.argtypes = [V, V, V, C.c_int, C.c_int, C.c_int, C.c_int, C.c_int, _F]
        _lib = L
    return _lib


def ref_available():
    return os.path.exists(REF_LIB)


def ref():
    global _ref
    if _ref is None:
        R = C.CDLL(REF_LIB)
        R.ref_bm_range.argtypes = [_F, C.c_int, C.c_int, C.c_int, C.c_int, C.c_int, C.c_int, C.c_int, C.c_int,
                                   C.c_double, C.c_int, _F, _I, _I, C.c_int]
        R.ref_bm_positions.argtypes = [_F, C.c_int, C.c_int, C.c_int, C.c_int, _F, _I, _I, C.c_int, C.c_double,
                                       C.c_int, _F, _I, _I, C.c_int]
        R.ref_gen_search_pos.argtypes = [_I, _I, C.c_int, C.c_int, C.c_int, C.c_int, C.c_int, C.c_int, _I, _I, C.c_int]
        R.ref_vbm3d_match.argtypes = [_P(_F), C.c_int, C.c_int, C.c_int, C.c_int, C.c_int, C.c_int, C.c_int,
                                      C.c_int, C.c_int, C.c_int, C.c_int, C.c_int, C.c_int, C.c_int, C.c_double,
                                      _F, _I, _I, _I, C.c_int]
        R.ref_group_gather.argtypes = [_F, C.c_int, _I, _I, C.c_int, C.c_int, _F]
        R.ref_group_scatter.argtypes = [_F, _I, _I, C.c_int, C.c_int, C.c_float, C.c_float, _F, _F, C.c_int]
        _ref = R
    return _ref


def fp(a):
    return a.ctypes.data_as(_F)


def ip(a):
    return a.ctypes.data_as(_I)


# ---- parameters ------------------------------------------------------------------------------

def default_params(wiener, vbm3d=False, profile="fast", sigma=(10.0, 10.0, 10.0), matrix=None, width=None,
                   height=None, process=None, wiener_mode=0, **over):
    """Profile defaults (A1) with user overrides, as arguments_process resolves them."""
    p = Params()
    s = list(sigma) if hasattr(sigma, "__len__") else [sigma]
    while len(s) < 3:
        s.append(s[-1])
    lib().oracle_default_params(int(wiener), int(vbm3d), profile.encode(), C.c_double(s[0]), C.byref(p))
    p.sigma[:] = s[:3]
    if matrix is None or matrix == 2:
        matrix = lib().oracle_matrix_default(width, height)
    p.matrix = matrix
    p.process[:] = process if process is not None else [1 if v != 0 else 0 for v in s[:3]]
    p.wiener_mode = wiener_mode
    names = {"block_size": "B", "block_step": "step", "group_size": "G", "bm_range": "R", "bm_step": "bmstep",
             "th_mse": "th_mse", "hard_thr": "lambda_", "radius": "radius", "ps_num": "psnum",
             "ps_range": "psrange", "ps_step": "psstep"}
    for k, v in over.items():
        if v is not None:
            setattr(p, names[k], v)
    return p


def matrix_norms(matrix):
    n = (C.c_double * 3)()
    lib().oracle_matrix_norms(matrix, n)
    return list(n)


def scan(extent, B, step):
    out, j, last = [], 0, extent - B
    while True:
        if j >= last + step:
            break
        if j > last:
            j = last
        out.append(j)
        j += step
    return out


# ---- processing ------------------------------------------------------------------------------

def _stats_buf(stats):
    return np.zeros(len(STAT_NAMES), np.int64) if stats else None


def _stats_ptr(buf):
    return buf.ctypes.data_as(_L) if buf is not None else None


def _stats_dict(buf):
    return {k: int(v) for k, v in zip(STAT_NAMES, buf)}


def bm3d(p, src, ref=None, threads=1, stats=False):
    """src/ref: float32 [frames][planes][H][W].  Returns float32 output of the same shape, and with
    stats=True also the counters of STAT_NAMES (threshold decisions flipped against an FP64
    evaluation of the transform, tie events of the block matching)."""
    src = np.ascontiguousarray(src, np.float32)
    ref = src if ref is None else np.ascontiguousarray(ref, np.float32)
    F, P, H, W = src.shape
    dst = np.zeros_like(src)
    sb = _stats_buf(stats)
    lib().oracle_bm3d_ex(C.byref(p), F, P, H, W, W, fp(src), fp(ref), fp(dst), threads, _stats_ptr(sb))
    return (dst, _stats_dict(sb)) if stats else dst


def bm3d_matches(p, refY, threads=1, stats=False):
    refY = np.ascontiguousarray(refY, np.float32)
    H, W = refY.shape
    nb = len(scan(H, p.B, p.step)) * len(scan(W, p.B, p.step))
    cnt = np.zeros(nb, np.int32)
    ys = np.full(nb * p.G, -1, np.int32)
    xs = np.full(nb * p.G, -1, np.int32)
    ks = np.zeros(nb * p.G, np.float32)
    sb = _stats_buf(stats)
    lib().oracle_bm3d_matches_ex(C.byref(p), H, W, W, fp(refY), ip(cnt), ip(ys), ip(xs), fp(ks), threads, _stats_ptr(sb))
    out = (cnt, ys.reshape(nb, p.G), xs.reshape(nb, p.G), ks.reshape(nb, p.G))
    return (out, _stats_dict(sb)) if stats else out


def vbm3d_matches(p, refY_clip, n, threads=1, stats=False):
    clip = np.ascontiguousarray(refY_clip, np.float32)
    F, H, W = clip.shape
    nb = len(scan(H, p.B, p.step)) * len(scan(W, p.B, p.step))
    cnt = np.zeros(nb, np.int32)
    zs = np.full(nb * p.G, -1, np.int32)
    ys = np.full(nb * p.G, -1, np.int32)
    xs = np.full(nb * p.G, -1, np.int32)
    ks = np.zeros(nb * p.G, np.float32)
    sb = _stats_buf(stats)
    lib().oracle_vbm3d_matches_ex(C.byref(p), F, n, H, W, W, fp(clip), ip(cnt), ip(zs), ip(ys), ip(xs), fp(ks),
                                  threads, _stats_ptr(sb))
    g = p.G
    out = (cnt, zs.reshape(nb, g), ys.reshape(nb, g), xs.reshape(nb, g), ks.reshape(nb, g))
    return (out, _stats_dict(sb)) if stats else out


def vbm3d(p, src, ref=None, n0=0, count=None, threads=1, stats=False):
    """src/ref: float32 [F][planes][H][W].  Returns [count][planes][(2r+1)*2*H][W] stacked output."""
    src = np.ascontiguousarray(src, np.float32)
    ref = src if ref is None else np.ascontiguousarray(ref, np.float32)
    F, P, H, W = src.shape
    count = F - n0 if count is None else count
    slots = (2 * p.radius + 1) * 2
    dst = np.zeros((count, P, slots * H, W), np.float32)
    sb = _stats_buf(stats)
    lib().oracle_vbm3d_ex(C.byref(p), F, n0, count, P, H, W, W, fp(src), fp(ref), fp(dst), threads, _stats_ptr(sb))
    return (dst, _stats_dict(sb)) if stats else dst


def vaggregate(radius, stacked, process=(1, 1, 1)):
    """stacked: [F][planes][(2r+1)*2*H][W] float32 -> [F][planes][H][W] float32."""
    stacked = np.ascontiguousarray(stacked, np.float32)
    F, P, HH, W = stacked.shape
    H = HH // ((2 * radius + 1) * 2)
    out = np.zeros((F, P, H, W), np.float32)
    pr = np.array(list(process) + [1, 1, 1], np.int32)[:3]
    for n in range(F):
        lib().oracle_vaggregate(radius, F, n, P, ip(pr), H, W, W, fp(stacked), fp(out[n]))
    return out


def dct3d(groups, inverse=False, scalar=False):
    g = np.ascontiguousarray(groups, np.float32).copy()
    ng, n, B, _ = g.shape
    fn = lib().oracle_dct3d_scalar if scalar else lib().oracle_dct3d
    for k in range(ng):
        fn(fp(g[k]), n, B, int(inverse))
    return g


def rgb2opp(rgb):
    rgb = np.ascontiguousarray(rgb, np.float32)
    H, W = rgb.shape[-2:]
    out = np.zeros_like(rgb)
    lib().oracle_rgb2opp_float(fp(rgb[0]), fp(rgb[1]), fp(rgb[2]), H, W, W, fp(out[0]), fp(out[1]), fp(out[2]))
    return out


def opp2rgb(yuv):
    yuv = np.ascontiguousarray(yuv, np.float32)
    H, W = yuv.shape[-2:]
    out = np.zeros_like(yuv)
    lib().oracle_opp2rgb_float(fp(yuv[0]), fp(yuv[1]), fp(yuv[2]), H, W, W, fp(out[0]), fp(out[1]), fp(out[2]))
    return out


def int2float(plane, bits, full=True, chroma=False):
    plane = np.ascontiguousarray(plane)
    H, W = plane.shape
    out = np.zeros((H, W), np.float32)
    lib().oracle_int2float(plane.ctypes.data, plane.itemsize, bits, int(full), int(chroma), H, W, W, W, fp(out))
    return out


def float2int(plane, bits, full=True, chroma=False):
    plane = np.ascontiguousarray(plane, np.float32)
    H, W = plane.shape
    out = np.zeros((H, W), np.uint8 if bits <= 8 else np.uint16)
    lib().oracle_float2int(fp(plane), out.itemsize, bits, int(full), int(chroma), H, W, W, W, out.ctypes.data)
    return out


# ---- the reference's own Block.h -------------------------------------------------------------

def ref_bm_range(plane, j, i, B, bm_range, bm_step, thmse_norm, G):
    plane = np.ascontiguousarray(plane, np.float32)
    H, W = plane.shape
    k = np.zeros(G, np.float32)
    y = np.zeros(G, np.int32)
    x = np.zeros(G, np.int32)
    n = ref().ref_bm_range(fp(plane), H, W, W, j, i, B, bm_range, bm_step, thmse_norm, G, fp(k), ip(y), ip(x), G)
    return k[:n], y[:n], x[:n]


def ref_vbm3d_match(clip, cur, j, i, B, bm_range, bm_step, G, ps_num, ps_range, ps_step, thmse_norm):
    clip = np.ascontiguousarray(clip, np.float32)
    F, H, W = clip.shape
    arr = (_F * F)(*[C.cast(clip[f].ctypes.data, _F) for f in range(F)])
    cap = G
    k = np.zeros(cap, np.float32)
    z = np.zeros(cap, np.int32)
    y = np.zeros(cap, np.int32)
    x = np.zeros(cap, np.int32)
    n = ref().ref_vbm3d_match(arr, F, cur, H, W, W, j, i, B, bm_range, bm_step, G, ps_num, ps_range, ps_step,
                              thmse_norm, fp(k), ip(z), ip(y), ip(x), cap)
    return k[:n], z[:n], y[:n], x[:n]


def _bits_of(a, bits):
    return 32 if a.dtype == np.float32 else (bits or (8 if a.dtype == np.uint8 else 16))


def rgb2opp_any(rgb, out_dtype=np.float32, in_bits=None, clip=None):
    """MatrixConvert_RGB2YUV (OPP) for any sample types, full range: rgb [3][H][W] uint8/uint16/
    float32 -> [3][H][W] of out_dtype.  clip defaults to "integer output" (RGB2OPP's rule)."""
    rgb = np.ascontiguousarray(rgb)
    H, W = rgb.shape[-2:]
    out = np.zeros((3, H, W), out_dtype)
    clip = (out.dtype != np.float32) if clip is None else clip
    lib().oracle_rgb2opp_any(rgb[0].ctypes.data, rgb[1].ctypes.data, rgb[2].ctypes.data, rgb.itemsize,
                             _bits_of(rgb, in_bits), out[0].ctypes.data, out[1].ctypes.data, out[2].ctypes.data,
                             out.itemsize, _bits_of(out, None), H, W, W, int(clip))
    return out


def opp2rgb_any(yuv, out_dtype=np.float32, in_bits=None, clip=None):
    """MatrixConvert_YUV2RGB (OPP) for any sample types, full range."""
    yuv = np.ascontiguousarray(yuv)
    H, W = yuv.shape[-2:]
    out = np.zeros((3, H, W), out_dtype)
    clip = (out.dtype != np.float32) if clip is None else clip
    lib().oracle_opp2rgb_any(yuv[0].ctypes.data, yuv[1].ctypes.data, yuv[2].ctypes.data, yuv.itemsize,
                             _bits_of(yuv, in_bits), out[0].ctypes.data, out[1].ctypes.data, out[2].ctypes.data,
                             out.itemsize, _bits_of(out, None), H, W, W, int(clip))
    return out


def rgb2y_any(rgb, in_bits=None):
    """ConvertToY (OPP) into float: the Y plane Basic matches on for an RGB ref clip."""
    rgb = np.ascontiguousarray(rgb)
    H, W = rgb.shape[-2:]
    out = np.zeros((H, W), np.float32)
    lib().oracle_rgb2y_any(rgb[0].ctypes.data, rgb[1].ctypes.data, rgb[2].ctypes.data, rgb.itemsize,
                           _bits_of(rgb, in_bits), H, W, W, fp(out))
    return out
