"""bm3d_b200 -- Python mirror of the reference VapourSynth plugin interface over the C ABI.

    from bm3d_b200 import core, source
    clip = source(frames, color_family="RGB")          # numpy (host) or torch CUDA (device) frames
    opp = core.bm3d.RGB2OPP(clip, sample=1)
    basic = core.bm3d.Basic(opp, profile="np", matrix=100)
    final = core.bm3d.Final(opp, basic, profile="np", matrix=100)
    rgb = core.bm3d.OPP2RGB(final, sample=1).numpy()

The functions, argument names, defaults and error messages are those of the reference plugin
(namespace bm3d: RGB2OPP, OPP2RGB, Basic, Final, VBasic, VFinal, VAggregate); every frame is
computed by libbm3d_b200.so on the GPU.  Frames held as torch CUDA tensors stay on the device
between stages; numpy frames are staged through the device by the library.
"""
import ctypes as C

import numpy as np

from . import _capi as capi

GRAY, RGB, YUV = capi.GRAY, capi.RGB, capi.YUV
INTEGER, FLOAT = capi.INTEGER, capi.FLOAT

__all__ = ["core", "source", "Error", "VideoNode", "VideoFrame", "GRAY", "RGB", "YUV", "INTEGER", "FLOAT"]

_FAMILY = {"GRAY": GRAY, "RGB": RGB, "YUV": YUV}
_PROP_KEYS = ("BM3D_OPP", "_Range", "_Matrix", "BM3D_V_radius", "BM3D_V_process")


class Error(Exception):
    """Raised with the library's message (the reference's "bm3d.<Func>: ..." text)."""


def _dtype(sample_type, bits):
    if sample_type == FLOAT:
        return np.float32
    return np.uint8 if bits <= 8 else np.uint16


class VideoFrame:
    """Planes (numpy arrays on the host or torch tensors on the GPU) plus frame properties."""

    def __init__(self, planes, props=None):
        self.planes = list(planes)
        self.props = dict(props or {})

    @property
    def on_device(self):
        return not isinstance(self.planes[0], np.ndarray)

    def numpy(self):
        out = []
        for p in self.planes:
            out.append(p if isinstance(p, np.ndarray) else p.detach().cpu().numpy())
        return np.stack(out)


class VideoNode:
    """Clip: format + dimensions + frames produced on request."""

    def __init__(self, info):
        self.info = info

    color_family = property(lambda s: s.info.color_family)
    sample_type = property(lambda s: s.info.sample_type)
    bits_per_sample = property(lambda s: s.info.bits_per_sample)
    width = property(lambda s: s.info.width)
    height = property(lambda s: s.info.height)
    num_frames = property(lambda s: s.info.num_frames)

    @property
    def num_planes(self):
        return 1 if self.info.color_family == GRAY else 3

    def get_frame(self, n):
        return self.get_frames(n, 1)[0]

    def get_frames(self, n, count):
        raise NotImplementedError

    def numpy(self, batch=None):
        """All frames as an array [frames][planes][height][width] on the host."""
        batch = batch or self.num_frames
        frames = []
        for n in range(0, self.num_frames, batch):
            frames += self.get_frames(n, min(batch, self.num_frames - n))
        return np.stack([f.numpy() for f in frames])


class SourceNode(VideoNode):
    def __init__(self, frames, color_family, sample_type, bits, props, subsampling=(0, 0)):
        nf, npl, h, w = frames.shape
        info = capi.VideoInfo(color_family, sample_type, bits, subsampling[0], subsampling[1], w, h, nf)
        super().__init__(info)
        self._frames = frames
        self._props = props

    def get_frames(self, n, count):
        out = []
        for k in range(n, n + count):
            props = self._props[k] if isinstance(self._props, (list, tuple)) else dict(self._props)
            out.append(VideoFrame([self._frames[k, p] for p in range(self._frames.shape[1])], props))
        return out


def source(frames, color_family="GRAY", bits=None, props=None):
    """Wraps an array [frames][planes][height][width] (numpy uint8/uint16/float32, or a torch CUDA
    tensor of those types) as a clip.  props: one dict for every frame or a list of dicts."""
    cf = _FAMILY[color_family] if isinstance(color_family, str) else int(color_family)
    dt = str(frames.dtype).replace("torch.", "")
    if "float32" in dt:
        st, b = FLOAT, 32
    elif "uint16" in dt:
        st, b = INTEGER, bits or 16
    elif "uint8" in dt:
        st, b = INTEGER, bits or 8
    else:
        raise Error("unsupported sample type " + dt)
    if frames.ndim == 3:
        frames = frames[:, None]
    return SourceNode(frames, cf, st, b, props if props is not None else {})


def _frame_struct(vf, planes_n, memory_host):
    fr = capi.Frame()
    for p in range(planes_n):
        a = vf.planes[p]
        if isinstance(a, np.ndarray):
            fr.data[p] = a.ctypes.data
            fr.stride[p] = a.strides[0]
        else:
            fr.data[p] = a.data_ptr()
            fr.stride[p] = a.stride(0) * a.element_size()
    fr.memory = capi.MEM_HOST if memory_host else capi.MEM_DEVICE
    pr = vf.props
    fr.prop_bm3d_opp = int(pr.get("BM3D_OPP", -1))
    fr.prop_range = int(pr.get("_Range", -1))
    fr.prop_matrix = int(pr.get("_Matrix", -1))
    fr.prop_v_radius = int(pr.get("BM3D_V_radius", -1))
    vp = pr.get("BM3D_V_process")
    if vp is None:
        fr.prop_v_process_count = -1
    else:
        fr.prop_v_process_count = len(vp)
        for i, v in enumerate(list(vp)[:3]):
            fr.prop_v_process[i] = int(v)
    return fr


def _props_from_struct(fr):
    props = {}
    if fr.prop_bm3d_opp >= 0:
        props["BM3D_OPP"] = fr.prop_bm3d_opp
    if fr.prop_range >= 0:
        props["_Range"] = fr.prop_range
    if fr.prop_matrix >= 0:
        props["_Matrix"] = fr.prop_matrix
    if fr.prop_v_radius >= 0:
        props["BM3D_V_radius"] = fr.prop_v_radius
    if fr.prop_v_process_count >= 0:
        props["BM3D_V_process"] = [fr.prop_v_process[i] for i in range(min(3, fr.prop_v_process_count))]
    return props


class FilterNode(VideoNode):
    """A bm3d.* function applied to clips; frames are produced by the library in batches."""

    _POSITIONAL = {
        "RGB2OPP": ("input", "sample"), "OPP2RGB": ("input", "sample"),
        "Basic": ("input", "ref"), "Final": ("input", "ref"),
        "VBasic": ("input", "ref"), "VFinal": ("input", "ref"),
        "VAggregate": ("input", "radius", "sample"),
    }

    def __init__(self, name, *args, **kwargs):
        L = capi.lib()
        for i, a in enumerate(args):
            names = self._POSITIONAL.get(name, ("input",))
            if i >= len(names):
                raise Error(name + ": too many positional arguments")
            kwargs[names[i]] = a
        self.name = name
        self.inputs = {k: v for k, v in kwargs.items() if isinstance(v, VideoNode)}
        m = L.bm3d_map_create()
        try:
            for k, v in kwargs.items():
                if v is None:
                    continue
                key = k.encode()
                if isinstance(v, VideoNode):
                    L.bm3d_map_set_clip(m, key, C.byref(v.info))
                elif isinstance(v, str):
                    L.bm3d_map_set_data(m, key, v.encode())
                elif isinstance(v, (list, tuple)):
                    for e in v:
                        if isinstance(e, float):
                            L.bm3d_map_set_float(m, key, e)
                        else:
                            L.bm3d_map_set_int(m, key, int(e)) if k != "sigma" else L.bm3d_map_set_float(m, key, float(e))
                elif isinstance(v, bool):
                    L.bm3d_map_set_int(m, key, int(v))
                elif isinstance(v, (int, np.integer)):
                    if k in ("sigma", "th_mse", "hard_thr"):
                        L.bm3d_map_set_float(m, key, float(v))
                    else:
                        L.bm3d_map_set_int(m, key, int(v))
                else:
                    L.bm3d_map_set_float(m, key, float(v))
            h = C.c_void_p()
            rc = L.bm3d_create(name.encode(), m, C.byref(h))
        finally:
            L.bm3d_map_free(m)
        if rc != capi.BM3D_OK:
            raise Error(capi.last_error())
        self._h = h
        info = capi.VideoInfo()
        L.bm3d_output_info(h, C.byref(info))
        super().__init__(info)
        self._cache = {}

    def __del__(self):
        h = getattr(self, "_h", None)
        if h:
            try:
                capi.lib().bm3d_free(h)
            except Exception:
                pass
            self._h = None

    def window(self, n, count):
        first, num = C.c_int(), C.c_int()
        if capi.lib().bm3d_frame_window(self._h, n, count, C.byref(first), C.byref(num)) != 0:
            raise Error(capi.last_error())
        return first.value, num.value

    def _alloc(self, like_device):
        info = self.info
        dt = _dtype(info.sample_type, info.bits_per_sample)
        npl = 1 if info.color_family == GRAY else 3
        if like_device:
            import torch
            tdt = {np.float32: torch.float32, np.uint16: torch.uint16, np.uint8: torch.uint8}[dt]
            return VideoFrame([torch.empty((info.height, info.width), dtype=tdt, device="cuda") for _ in range(npl)])
        return VideoFrame([np.zeros((info.height, info.width), dtype=dt) for _ in range(npl)])

    def compute(self, n, count, sync=True):
        """Runs the filter for output frames [n, n+count) and returns them (uncached)."""
        L = capi.lib()
        first, num = self.window(n, count)
        src_node = self.inputs["input"]
        src = src_node.get_frames(first, num)
        ref = self.inputs["ref"].get_frames(first, num) if "ref" in self.inputs else None
        dev = src[0].on_device
        dst = [self._alloc(dev) for _ in range(count)]
        npl_in = src_node.num_planes
        npl_out = 1 if self.info.color_family == GRAY else 3
        s_structs = [_frame_struct(f, npl_in, not dev) for f in src]
        r_structs = [_frame_struct(f, npl_in, not dev) for f in ref] if ref else None
        d_structs = [_frame_struct(f, npl_out, not dev) for f in dst]
        PF = C.POINTER(capi.Frame)
        s_arr = (PF * num)(*[C.pointer(s) for s in s_structs])
        r_arr = (PF * num)(*[C.pointer(s) for s in r_structs]) if r_structs else None
        d_arr = (PF * count)(*[C.pointer(s) for s in d_structs])
        fn = L.bm3d_get_frames if sync else L.bm3d_get_frames_async
        rc = fn(self._h, n, count, s_arr, r_arr, d_arr)
        if rc != 0:
            raise Error(capi.last_error())
        for f, s in zip(dst, d_structs):
            f.props = _props_from_struct(s)
        self._keep = (src, ref, s_structs, r_structs, d_structs, s_arr, r_arr, d_arr)
        return dst

    def get_frames(self, n, count):
        missing = [k for k in range(n, n + count) if k not in self._cache]
        if missing:
            lo, hi = missing[0], missing[-1] + 1
            for k, f in enumerate(self.compute(lo, hi - lo)):
                self._cache[lo + k] = f
        return [self._cache[k] for k in range(n, n + count)]

    def matches(self, k, group_size):
        """Match lists of output frame k of the last computed batch: (counts, z, y, x, keys)."""
        L = capi.lib()
        cap = 1 << 22
        counts = np.zeros(cap, np.int32)
        z = np.zeros(cap * group_size, np.int32)
        y = np.zeros_like(z)
        x = np.zeros_like(z)
        keys = np.zeros(cap * group_size, np.float32)
        P = C.POINTER
        nb = L.bm3d_debug_matches(self._h, k, counts.ctypes.data_as(P(C.c_int)), z.ctypes.data_as(P(C.c_int)),
                                  y.ctypes.data_as(P(C.c_int)), x.ctypes.data_as(P(C.c_int)),
                                  keys.ctypes.data_as(P(C.c_float)), cap)
        if nb < 0:
            raise Error("no match lists available")
        g = group_size
        return (counts[:nb], z[:nb * g].reshape(nb, g), y[:nb * g].reshape(nb, g), x[:nb * g].reshape(nb, g),
                keys[:nb * g].reshape(nb, g))

    def reference_fp64(self, k=0):
        """FP64 GPU oracle of output frame k of the last computed batch (Basic / Final): float64
        [planes][H][W] in the filter's internal float domain (planes not processed are zero)."""
        L = capi.lib()
        info = self.info
        out = np.zeros((3, info.height, info.width), np.float64)
        rc = L.bm3d_debug_reference_fp64(self._h, k, out.ctypes.data_as(C.POINTER(C.c_double)), info.height * info.width)
        if rc != 0:
            raise Error("no FP64 reference for this filter / frame")
        return out

    def slow_blocks(self):
        return int(capi.lib().bm3d_debug_slow_blocks(self._h))

    def threshold_rechecks(self):
        """Precision form, hard threshold, last call: (coefficients recomputed in fp32 because their
        tensor-core value lay near the threshold, keep / zero decisions that changed)."""
        r, c = C.c_int64(0), C.c_int64(0)
        capi.lib().bm3d_debug_threshold_rechecks(self._h, C.byref(r), C.byref(c))
        return int(r.value), int(c.value)

    def set_recheck_band(self, band):
        if capi.lib().bm3d_debug_set_recheck_band(self._h, float(band)) != 0:
            raise Error("not a BM3D / V-BM3D filter")

    def retained_counts(self, k=0):
        """Retained-coefficient count of every group of output frame k of the last computed batch
        (Basic): int32 [3][blocks], -1 for planes not processed."""
        cap = 3 * (1 << 21)
        out = np.zeros(cap, np.int32)
        nb = capi.lib().bm3d_debug_retained_counts(self._h, k, out.ctypes.data_as(C.POINTER(C.c_int)), cap)
        if nb < 0:
            raise Error("no retained counts for this filter / frame")
        return out[:3 * nb].reshape(3, nb)

    def bm_tc_counts(self):
        """Precision-form block matching of the last call: (reference blocks that fell back to
        exact distances for every candidate, CTAs whose tensor-core wait timed out)."""
        fb, to = C.c_int64(0), C.c_int64(0)
        capi.lib().bm3d_debug_bm_tc_counts(self._h, C.byref(fb), C.byref(to))
        return int(fb.value), int(to.value)


class _Namespace:
    def __getattr__(self, name):
        if name not in FilterNode._POSITIONAL:
            raise AttributeError(name)
        return lambda *a, **k: FilterNode(name, *a, **k)


class _Core:
    bm3d = _Namespace()


core = _Core()


def dct3d(groups, inverse=False, fast=False):
    """Runs the library's 3-D transform on groups [g][n][B][B] (float32, host); returns a copy."""
    g = np.ascontiguousarray(groups, dtype=np.float32).copy()
    ng, n, b, _ = g.shape
    rc = capi.lib().bm3d_debug_dct3d(g.ctypes.data_as(C.POINTER(C.c_float)), ng, n, b, int(inverse), int(fast))
    if rc != 0:
        raise Error(capi.last_error())
    return g
