"""CPU tests of the C ABI: the library loads, exports every entry point the header declares, and
rejects bad arguments with the reference plugin's messages (argument processing runs before any
device access).  No compute call is made here."""
import ctypes as C
import os
import re

import pytest

from conftest import HAS_GPU, ROOT

import bm3d_b200
from bm3d_b200 import _capi as capi

HEADER = os.path.join(ROOT, "include", "bm3d_b200.h")


def declared_symbols():
    text = open(HEADER).read()
    return sorted(set(re.findall(r"BM3D_API\s+[\w\s\*]+?\b(bm3d_\w+)\s*\(", text)))


def test_header_declares_the_abi():
    syms = declared_symbols()
    assert "bm3d_create" in syms and "bm3d_get_frames" in syms and len(syms) >= 19
    assert sorted(capi.EXPORTS) == syms


def test_library_exports_every_declared_symbol():
    L = capi.lib()
    for s in declared_symbols():
        assert hasattr(L, s), s
    # nothing else leaks (symbols are hidden by default)
    out = os.popen("nm -D --defined-only " + capi.LIB_PATH).read()
    exported = set(re.findall(r" T (\w+)", out))
    assert exported == set(declared_symbols())


def clip(cf=bm3d_b200.RGB, st=bm3d_b200.FLOAT, bits=32, w=64, h=48, n=3, ssw=0, ssh=0):
    return capi.VideoInfo(cf, st, bits, ssw, ssh, w, h, n)


def create(name, **args):
    L = capi.lib()
    m = L.bm3d_map_create()
    for k, v in args.items():
        vals = v if isinstance(v, list) else [v]
        for e in vals:
            if isinstance(e, capi.VideoInfo):
                L.bm3d_map_set_clip(m, k.encode(), C.byref(e))
            elif isinstance(e, str):
                L.bm3d_map_set_data(m, k.encode(), e.encode())
            elif isinstance(e, float):
                L.bm3d_map_set_float(m, k.encode(), e)
            else:
                L.bm3d_map_set_int(m, k.encode(), e)
    h = C.c_void_p()
    rc = L.bm3d_create(name.encode(), m, C.byref(h))
    L.bm3d_map_free(m)
    if rc == 0:
        L.bm3d_free(h)
    return rc, capi.last_error()


# (function, args, expected message) -- texts of source/BM3D_Base.cpp:46-247,
# source/VBM3D_Base.cpp:117-368, source/BM3D_Basic.cpp:50, source/VAggregate.cpp:44-76,
# include/RGB2OPP.h:64-91, include/OPP2RGB.h:64-91
ERRORS = [
    ("Basic", dict(input=clip(st=0, bits=20)), "bm3d.Basic: Invalid input clip, only 8-16 bit integer or 32 bit float formats supported"),
    ("Basic", dict(input=clip(), ref=clip(cf=bm3d_b200.YUV)), "bm3d.Basic: input clip and clip \"ref\" must be of the same format"),
    ("Basic", dict(input=clip(), ref=clip(w=32)), "bm3d.Basic: input clip and clip \"ref\" must be of the same width and height"),
    ("Basic", dict(input=clip(), ref=clip(n=4)), "bm3d.Basic: input clip and clip \"ref\" must have the same number of frames"),
    ("Basic", dict(input=clip(), profile="fastest"), "bm3d.Basic: Unrecognized \"profile\" specified, should be \"fast\", \"lc\", \"np\", \"high\" or \"vn\""),
    ("Basic", dict(input=clip(), sigma=[10.0, -1.0]), "bm3d.Basic: Invalid \"sigma\" assigned, must be a non-negative floating point number"),
    ("Basic", dict(input=clip(), block_size=65), "bm3d.Basic: Invalid \"block_size\" assigned, must be an integer in [1, 64]"),
    ("Basic", dict(input=clip(w=16, h=12), block_size=13), "bm3d.Basic: Invalid \"block_size\" assigned, must not exceed width or height of the frame"),
    ("Basic", dict(input=clip(), block_step=9), "bm3d.Basic: Invalid \"block_step\" assigned, must be an integer in [1, block_size]"),
    ("Basic", dict(input=clip(), group_size=257), "bm3d.Basic: Invalid \"group_size\" assigned, must be an integer in [1, 256]"),
    ("Basic", dict(input=clip(), bm_range=0), "bm3d.Basic: Invalid \"bm_range\" assigned, must be a positive integer"),
    ("Basic", dict(input=clip(), bm_step=10), "bm3d.Basic: Invalid \"bm_step\" assigned, must be an integer in [1, bm_range]"),
    ("Basic", dict(input=clip(), th_mse=0.0), "bm3d.Basic: Invalid \"th_mse\" assigned, must be a positive floating point number"),
    ("Basic", dict(input=clip(cf=bm3d_b200.YUV), matrix=3), "bm3d.Basic: Unsupported \"matrix\" specified"),
    ("Basic", dict(input=clip(cf=bm3d_b200.YUV, ssw=1, ssh=1)), "bm3d.Basic: input clip: sub-sampled format is not supported when chroma is processed, convert it to YUV444 or RGB first. For the best quality, RGB colorspace is recommended as input."),
    ("Basic", dict(input=clip(), hard_thr=0.0), "bm3d.Basic: Invalid \"hard_thr\" assigned, must be a positive floating point number"),
    ("Basic", dict(input=clip(), precision="fp16"), "bm3d.Basic: Invalid \"precision\" assigned, must be \"fp32\", \"tf32\", \"tf32_match\" or \"learned\""),
    ("VFinal", dict(input=clip(), ref=clip(), precision="bf16"), "bm3d.VFinal: Invalid \"precision\" assigned, must be \"fp32\", \"tf32\", \"tf32_match\" or \"learned\""),
    ("VBasic", dict(input=clip(), aggregate=2), "bm3d.VBasic: Invalid \"aggregate\" assigned, must be 0 (stacked output) or 1 (aggregated output)"),
    ("VFinal", dict(input=clip(), ref=clip(), aggregate=1, sample=2), "bm3d.VFinal: Invalid 'sample' assigned, must be 0 (integer sample type) or 1 (float sample type)"),
    ("Final", dict(input=clip(), ref=clip(), group_size=0), "bm3d.Final: Invalid \"group_size\" assigned, must be an integer in [1, 256]"),
    ("VBasic", dict(input=clip(), radius=17), "bm3d.VBasic: Invalid \"radius\" assigned, must be an integer in [1, 16]"),
    ("VBasic", dict(input=clip(), ps_num=9), "bm3d.VBasic: Invalid \"ps_num\" assigned, must be an integer in [1, group_size]"),
    ("VBasic", dict(input=clip(), ps_range=0), "bm3d.VBasic: Invalid \"ps_range\" assigned, must be a positive integer"),
    ("VFinal", dict(input=clip(), ref=clip(), ps_step=9), "bm3d.VFinal: Invalid \"ps_step\" assigned, must be an integer in [1, ps_range]"),
    ("VAggregate", dict(input=clip(cf=bm3d_b200.YUV, st=0, bits=16)), "bm3d.VAggregate: Invalid input clip, only accept 32 bit float format clip from bm3d.VBasic or bm3d.VFinal"),
    ("VAggregate", dict(input=clip()), "bm3d.VAggregate: Invalid input clip, must be of Gray or YUV color family"),
    ("VAggregate", dict(input=clip(cf=bm3d_b200.YUV), radius=0), "bm3d.VAggregate: Invalid \"radius\" assigned, must be an integer in [1, 16]"),
    ("VAggregate", dict(input=clip(cf=bm3d_b200.YUV), sample=2), "bm3d.VAggregate: Invalid 'sample' assigned, must be 0 (integer sample type) or 1 (float sample type)"),
    ("RGB2OPP", dict(input=clip(cf=bm3d_b200.YUV)), "bm3d.RGB2OPP: Invalid input clip, must be of RGB color family"),
    ("RGB2OPP", dict(input=clip(st=1, bits=16)), "bm3d.RGB2OPP: Invalid input clip, only 8-16 bit int or 32 bit float formats supported"),
    ("OPP2RGB", dict(input=clip()), "bm3d.OPP2RGB: Invalid input clip, must be of YUV color family"),
    ("OPP2RGB", dict(input=clip(cf=bm3d_b200.YUV), sample=3), "bm3d.OPP2RGB: Invalid 'sample' assigned, must be 0 (integer sample type) or 1 (float sample type)"),
]


@pytest.mark.parametrize("name,args,msg", ERRORS)
def test_argument_errors_match_reference_text(name, args, msg):
    rc, err = create(name, **args)
    assert rc == capi.BM3D_ERR_ARG
    assert err == msg


def test_argspec_errors():
    rc, err = create("Basic", input=clip(), bogus=1)
    assert rc == capi.BM3D_ERR_ARG and "bogus" in err
    rc, err = create("Final", input=clip())
    assert rc == capi.BM3D_ERR_ARG and "ref" in err
    rc, err = create("Basic", input=clip(), block_size=8.5)
    assert rc == capi.BM3D_ERR_ARG and "block_size" in err
    # the aggregated-output extension belongs to VBasic / VFinal only
    rc, err = create("Basic", input=clip(), aggregate=1)
    assert rc == capi.BM3D_ERR_ARG and "aggregate" in err


def test_first_error_wins_in_reference_order():
    # block_size is checked before group_size (source/BM3D_Base.cpp:129-165)
    rc, err = create("Basic", input=clip(), block_size=0, group_size=0)
    assert err.endswith("\"block_size\" assigned, must be an integer in [1, 64]")


@pytest.mark.skipif(HAS_GPU, reason="checks the no-device path")
def test_valid_arguments_without_gpu_fail_loudly():
    rc, err = create("Basic", input=clip(), profile="np")
    assert rc == capi.BM3D_ERR_CUDA, err
    # every precision value passes the argument checks (and then needs the device)
    for prec in ("fp32", "tf32", "tf32_match", "learned"):
        rc, err = create("Final", input=clip(), ref=clip(), precision=prec)
        assert rc == capi.BM3D_ERR_CUDA, (prec, err)
    with pytest.raises(bm3d_b200.Error):
        bm3d_b200.core.bm3d.Basic(bm3d_b200.source(__import__("numpy").zeros((1, 3, 48, 64), "float32"), "RGB"))
