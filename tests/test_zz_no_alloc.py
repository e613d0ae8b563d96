"""bm3d_basic_noalloc: the allocation-free Basic entry point, checked against bm3d_get_frames.

The entry point keeps its work buffers in one fixed device array shared by every call, so the GPU
test makes consecutive calls with different sizes and profiles (stale match lists or
accumulators from the previous call would show up as differences) and repeats the first call.
This file is named so that pytest collects it last; it passes alone in a fresh process and after
the other tests.
"""
import ctypes as C

import numpy as np
import pytest

from bm3d_b200 import _capi, core, source, synth

TOL = 1e-4       # float outputs, as in the other parity tests


def _noalloc(src_ptr, dst_ptr, w, h, stride, profile, sigma, stream=None):
    L = _capi.lib()
    return L.bm3d_basic_noalloc(src_ptr, dst_ptr, w, h, stride, profile, sigma, stream)


def test_noalloc_is_exported():
    L = _capi.lib()
    assert hasattr(L, "bm3d_basic_noalloc")


def test_noalloc_rejects_bad_arguments_before_touching_the_device():
    # fake non-null pointers: every one of these calls must fail before any device work
    fake = C.c_void_p(4096)
    r = _noalloc(fake, fake, 3840, 2160, 3840 * 4, b"np", 10.0)
    assert r == _capi.BM3D_ERR_UNSUPPORTED
    msg = _capi.last_error()
    assert "3840x2160" in msg and "48 MiB" in msg and "needs" in msg
    assert _noalloc(fake, fake, 64, 64, 256, b"bogus", 10.0) == _capi.BM3D_ERR_ARG
    assert "Unrecognized \"profile\"" in _capi.last_error()
    assert _noalloc(fake, fake, 64, 64, 256, b"np", -1.0) == _capi.BM3D_ERR_ARG
    assert "sigma" in _capi.last_error()
    assert _noalloc(fake, fake, 64, 64, 255, b"np", 10.0) == _capi.BM3D_ERR_ARG
    assert _noalloc(fake, fake, 64, 64, 128, b"np", 10.0) == _capi.BM3D_ERR_ARG
    assert _noalloc(fake, fake, 7, 64, 256, b"np", 10.0) == _capi.BM3D_ERR_ARG
    assert _noalloc(None, fake, 64, 64, 256, b"np", 10.0) == _capi.BM3D_ERR_STATE


@pytest.mark.gpu
def test_noalloc_matches_basic_on_consecutive_calls():
    import torch
    torch.cuda.set_device(0)
    cases = [  # (seed, height, width, row padding in floats, profile, sigma)
        (31, 144, 250, 7, "np", 10.0),
        (32, 97, 131, 0, "lc", 25.0),
    ]
    expected, bufs = [], []
    for seed, h, w, pad, prof, sigma in cases:
        nz, _ = synth.gray_frames(seed, 1, h, w, sigma)
        # the existing entry point (bm3d_get_frames on a Basic filter, device frames)
        node = core.bm3d.Basic(source(torch.from_numpy(nz).cuda(), "GRAY"), profile=prof, sigma=sigma)
        expected.append(node.get_frames(0, 1)[0].numpy()[0])
        src = torch.full((h, w + pad), 3.0, dtype=torch.float32, device="cuda")
        src[:, :w] = torch.from_numpy(nz[0, 0]).cuda()
        dst = torch.full((h, w + pad), -7.0, dtype=torch.float32, device="cuda")
        bufs.append((src, dst, w, h, (w + pad) * 4, prof.encode(), sigma))
    torch.cuda.synchronize()
    stream = C.c_void_p(torch.cuda.current_stream().cuda_stream)

    def run(i):
        src, dst, w, h, stride, prof, sigma = bufs[i]
        dst.fill_(-7.0)
        r = _noalloc(C.c_void_p(src.data_ptr()), C.c_void_p(dst.data_ptr()), w, h, stride, prof, sigma, stream)
        assert r == _capi.BM3D_OK, _capi.last_error()
        torch.cuda.synchronize()
        out = dst.cpu().numpy()
        assert np.all(out[:, w:] == -7.0), "wrote beyond the plane width"
        return out[:, :w]

    # two calls in a row, different sizes and profiles
    for i in range(2):
        got = run(i)
        err = float(np.abs(got - expected[i]).max())
        assert err <= TOL, f"call {i + 1}: max |noalloc - get_frames| = {err}"
    # the first case again, after the second call left its contents in the shared array; the
    # device's free memory must not change across the call
    free0 = torch.cuda.mem_get_info()[0]
    got = run(0)
    free1 = torch.cuda.mem_get_info()[0]
    assert float(np.abs(got - expected[0]).max()) <= TOL
    assert free1 == free0, f"free device memory changed by {free0 - free1} bytes during the call"


@pytest.mark.gpu
def test_noalloc_sigma_zero_copies_the_plane():
    import torch
    nz, _ = synth.gray_frames(33, 1, 40, 56, 10.0)
    src = torch.from_numpy(nz[0, 0]).cuda()
    dst = torch.zeros_like(src)
    stream = C.c_void_p(torch.cuda.current_stream().cuda_stream)
    r = _noalloc(C.c_void_p(src.data_ptr()), C.c_void_p(dst.data_ptr()), 56, 40, 56 * 4, b"np", 0.0, stream)
    assert r == _capi.BM3D_OK, _capi.last_error()
    torch.cuda.synchronize()
    assert torch.equal(dst, src)
