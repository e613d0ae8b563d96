"""GPU parity tests: the CUDA path (through the C ABI) against the CPU oracle.

Bars: match lists index-identical (positions, order, and keys bit for bit); 3-D transforms bit
for bit; outputs within max abs 1e-4 for float and 1 LSB for 16-bit (aggregation order differs:
float atomics on the GPU versus the reference's sequential sums).
"""
import numpy as np
import pytest

import bm3d_b200
from bm3d_b200 import core, source, synth

pytestmark = pytest.mark.gpu

TOL = 1e-4


def gray(img):
    return source(np.ascontiguousarray(img, np.float32)[None, None], "GRAY")


def assert_lists_equal(node, k, oracle_lists, G):
    cnt, z, y, x, keys = node.matches(k, G)
    ocnt, oy, ox, ok = oracle_lists
    assert np.array_equal(cnt, ocnt)
    for b in range(len(cnt)):
        n = cnt[b]
        assert np.array_equal(y[b, :n], oy[b, :n]), b
        assert np.array_equal(x[b, :n], ox[b, :n]), b
        assert np.array_equal(keys[b, :n].view(np.int32), ok[b, :n].view(np.int32)), b


# ---- transforms ---------------------------------------------------------------------------------

@pytest.mark.parametrize("n", [8, 16, 32])
def test_fast_dct_bit_exact(orc, n):
    rng = np.random.default_rng(n)
    g = rng.normal(0, 1, (64, n, 8, 8)).astype(np.float32)
    for inv in (False, True):
        got = bm3d_b200.dct3d(g, inverse=inv, fast=True)
        exp = orc.dct3d(g, inverse=inv)
        assert np.array_equal(got.view(np.int32), exp.view(np.int32))


@pytest.mark.parametrize("n,B", [(1, 8), (3, 8), (5, 8), (12, 8), (16, 8), (7, 11), (4, 5), (64, 8), (2, 16)])
def test_generic_dct_bit_exact(orc, n, B):
    rng = np.random.default_rng(n * 31 + B)
    g = rng.normal(0, 1, (8, n, B, B)).astype(np.float32)
    for inv in (False, True):
        got = bm3d_b200.dct3d(g, inverse=inv, fast=False)
        exp = orc.dct3d(g, inverse=inv)
        assert np.array_equal(got.view(np.int32), exp.view(np.int32))


# ---- block matching against the reference's own Block.h (golden vectors) -----------------------

GOLDEN_BM = ["fast_noisy", "np_basic_noisy", "np_final_noisy", "ties_np", "ties_final", "ties_step2",
             "vn_final_b11", "b5_ties", "b16", "b8_g64"]


@pytest.mark.parametrize("name", GOLDEN_BM)
def test_block_matching_golden(golden, name):
    B, step, G, R, bms = [int(v) for v in golden[f"bm/{name}/params"]]
    th = float(golden[f"bm/{name}/th_mse"])
    img = golden[f"bm/{name}/img"]
    node = core.bm3d.Basic(gray(img), block_size=B, block_step=step, group_size=G, bm_range=R, bm_step=bms,
                           th_mse=th, matrix=6)
    node.get_frames(0, 1)
    exp = (golden[f"bm/{name}/count"], golden[f"bm/{name}/y"], golden[f"bm/{name}/x"], golden[f"bm/{name}/key"])
    assert_lists_equal(node, 0, exp, G)


# ---- Basic / Final outputs -----------------------------------------------------------------------

def test_basic_config1_640x480(orc):
    """bm3d.Basic, profile 'fast', hard_thr 2.2, sigma 10, one gray float 640x480 frame."""
    nz, _ = synth.gray_frames(0, 1, 480, 640, 10.0)
    node = core.bm3d.Basic(source(nz, "GRAY"), profile="fast", sigma=10.0, hard_thr=2.2)
    out = node.numpy()
    p = orc.default_params(0, False, "fast", 10.0, width=640, height=480, hard_thr=2.2)
    exp = orc.bm3d(p, nz)
    assert_lists_equal(node, 0, orc.bm3d_matches(p, nz[0, 0]), p.G)
    assert np.abs(out - exp).max() <= TOL


@pytest.mark.parametrize("profile", ["np", "lc", "high"])
def test_basic_then_final_gray(orc, profile):
    nz, _ = synth.gray_frames(1, 2, 96, 128, 15.0)
    b = core.bm3d.Basic(source(nz, "GRAY"), profile=profile, sigma=15.0)
    pb = orc.default_params(0, False, profile, 15.0, width=128, height=96)
    ob = orc.bm3d(pb, nz)
    gb = b.numpy()
    assert np.abs(gb - ob).max() <= TOL
    # Final with the oracle's basic estimate as ref on both sides, so matching sees identical input
    f = core.bm3d.Final(source(nz, "GRAY"), source(ob, "GRAY"), profile=profile, sigma=15.0)
    gf = f.numpy()
    pf = orc.default_params(1, False, profile, 15.0, width=128, height=96)
    of = orc.bm3d(pf, nz, ob)
    for k in range(2):
        assert_lists_equal(f, k, orc.bm3d_matches(pf, ob[k, 0]), pf.G)
    assert np.abs(gf - of).max() <= TOL


def test_rgb_pipeline_float(orc):
    """RGB2OPP -> Basic('np') -> Final('np', ref=basic) -> OPP2RGB on float RGB frames."""
    nz, _ = synth.rgb_frames(2, 2, 72, 96, 10.0)
    src = source(nz, "RGB")
    opp = core.bm3d.RGB2OPP(src, sample=1)
    basic = core.bm3d.Basic(opp, profile="np", matrix=100)
    final = core.bm3d.Final(opp, basic, profile="np", matrix=100)
    rgb = core.bm3d.OPP2RGB(final, sample=1)
    g_opp, g_basic, g_rgb = opp.numpy(), basic.numpy(), rgb.numpy()
    o_opp = np.stack([orc.rgb2opp(nz[k]) for k in range(2)])
    assert np.array_equal(g_opp.view(np.int32), o_opp.view(np.int32))
    pb = orc.default_params(0, False, "np", 10.0, matrix=100)
    o_basic = orc.bm3d(pb, o_opp)
    assert np.abs(g_basic - o_basic).max() <= TOL
    pf = orc.default_params(1, False, "np", 10.0, matrix=100)
    o_final = orc.bm3d(pf, o_opp, g_basic)          # the GPU basic estimate as ref on both sides
    o_rgb = np.stack([orc.opp2rgb(o_final[k]) for k in range(2)])
    assert np.abs(g_rgb - o_rgb).max() <= 2 * TOL
    assert final.get_frame(0).props.get("BM3D_OPP") == 1
    assert rgb.get_frame(0).props.get("_Matrix") == 0 and "BM3D_OPP" not in rgb.get_frame(0).props


def test_rgb_input_direct(orc):
    """RGB input to Basic converts to OPP internally and back (source/BM3D_Base.cpp:663-749)."""
    nz, _ = synth.rgb_frames(3, 1, 48, 64, 10.0)
    g = core.bm3d.Basic(source(nz, "RGB"), profile="lc").numpy()
    p = orc.default_params(0, False, "lc", 10.0, matrix=100)
    o = orc.opp2rgb(orc.bm3d(p, orc.rgb2opp(nz[0])[None])[0])
    assert np.abs(g[0] - o).max() <= 2 * TOL


def test_tie_heavy_input_exact_lists(orc):
    rng = np.random.default_rng(11)
    img = (np.round(rng.random((64, 80)) * 3) / 255.0).astype(np.float32)
    node = core.bm3d.Basic(gray(img), profile="np", th_mse=3000.0, matrix=6)
    out = node.numpy()
    p = orc.default_params(0, False, "np", 10.0, matrix=6, th_mse=3000.0)
    assert_lists_equal(node, 0, orc.bm3d_matches(p, img), p.G)
    assert node.slow_blocks() > 0
    assert np.abs(out - orc.bm3d(p, img[None, None])).max() <= TOL


def test_edges_and_odd_sizes(orc):
    rng = np.random.default_rng(5)
    for (h, w, prof) in [(53, 67, "np"), (8, 40, "fast"), (17, 9, "lc")]:
        img = (0.5 + 0.05 * rng.normal(size=(h, w))).astype(np.float32)
        node = core.bm3d.Basic(gray(img), profile=prof, matrix=6)
        out = node.numpy()
        p = orc.default_params(0, False, prof, 10.0, matrix=6)
        assert_lists_equal(node, 0, orc.bm3d_matches(p, img), p.G)
        assert np.abs(out - orc.bm3d(p, img[None, None])).max() <= TOL


def test_yuv444_16bit(orc):
    nz, _ = synth.rgb_frames(4, 1, 40, 56, 15.0)
    yuv = np.stack([synth.to_u16(np.clip(nz[0, c], 0, 1)) for c in range(3)])[None]
    node = core.bm3d.Basic(source(yuv, "YUV"), profile="fast", sigma=[15.0, 15.0, 15.0])
    g = node.numpy()
    p = orc.default_params(0, False, "fast", 15.0, width=56, height=40)
    f = np.stack([orc.int2float(yuv[0, c], 16, True, c > 0) for c in range(3)])[None]
    o = orc.bm3d(p, f)
    oi = np.stack([orc.float2int(o[0, c], 16, True, c > 0) for c in range(3)])
    assert np.abs(g[0].astype(np.int64) - oi.astype(np.int64)).max() <= 1


def test_unprocessed_planes_copied():
    nz, _ = synth.rgb_frames(5, 1, 40, 48, 10.0)
    yuv = nz.astype(np.float32)
    g = core.bm3d.Basic(source(yuv, "YUV"), sigma=[10.0, 0.0, 0.0]).numpy()
    assert np.array_equal(g[0, 1], yuv[0, 1]) and np.array_equal(g[0, 2], yuv[0, 2])


def test_device_frames_match_host_frames():
    import torch
    nz, _ = synth.rgb_frames(6, 2, 48, 64, 10.0)
    host = core.bm3d.OPP2RGB(core.bm3d.Basic(core.bm3d.RGB2OPP(source(nz, "RGB"), sample=1), matrix=100), sample=1).numpy()
    dev_src = source(torch.from_numpy(nz).cuda(), "RGB")
    dev = core.bm3d.OPP2RGB(core.bm3d.Basic(core.bm3d.RGB2OPP(dev_src, sample=1), matrix=100), sample=1)
    frames = dev.get_frames(0, 2)
    assert frames[0].on_device
    d = np.stack([f.numpy() for f in frames])
    assert np.abs(d - host).max() <= TOL


# ---- V-BM3D ----------------------------------------------------------------------------------

def test_vbm3d_golden_lists(golden):
    for name in ["vbasic_fast", "vfinal_ties_r2"]:
        B, step, G, R, bms, rad, psn, psr, pss = [int(v) for v in golden[f"vbm/{name}/params"]]
        th = float(golden[f"vbm/{name}/th_mse"])
        clip = golden[f"vbm/{name}/clip"]
        node = core.bm3d.VBasic(source(clip[:, None], "GRAY"), block_size=B, block_step=step, group_size=G,
                                bm_range=R, bm_step=bms, radius=rad, ps_num=psn, ps_range=psr, ps_step=pss,
                                th_mse=th, matrix=6)
        for n in range(clip.shape[0]):
            node.compute(n, 1)
            cnt, z, y, x, keys = node.matches(0, G)
            assert np.array_equal(cnt, golden[f"vbm/{name}/count"][n])
            for b in range(len(cnt)):
                m = cnt[b]
                assert np.array_equal(z[b, :m], golden[f"vbm/{name}/z"][n, b, :m])
                assert np.array_equal(y[b, :m], golden[f"vbm/{name}/y"][n, b, :m])
                assert np.array_equal(x[b, :m], golden[f"vbm/{name}/x"][n, b, :m])
                assert np.array_equal(keys[b, :m].view(np.int32), golden[f"vbm/{name}/key"][n, b, :m].view(np.int32))


def test_vbasic_vaggregate_yuv_float(orc):
    nz, _ = synth.motion_frames(7, 5, 40, 56, 15.0, planes=3)
    yuv = nz.astype(np.float32)
    vb = core.bm3d.VBasic(source(yuv, "YUV"), radius=1, sigma=15.0)
    stacked = vb.numpy()
    p = orc.default_params(0, True, "fast", 15.0, width=56, height=40, radius=1)
    o_st = orc.vbm3d(p, yuv)
    # compare the used slots only (unused slots are left unspecified by the reference)
    agg = core.bm3d.VAggregate(vb, radius=1, sample=1).numpy()
    o_agg = orc.vaggregate(1, o_st)
    assert np.abs(agg - o_agg).max() <= TOL
    assert vb.get_frame(0).props["BM3D_V_radius"] == 1
    assert "BM3D_V_radius" not in core.bm3d.VAggregate(vb, radius=1, sample=1).get_frame(0).props
    H = 40
    for n in range(5):
        for s in range(3):
            if 0 <= n - 1 + s < 5:
                num = slice(2 * s * H, (2 * s + 1) * H)
                assert np.abs(stacked[n, :, num] - o_st[n, :, num]).max() <= TOL
    # match lists of the last batch (all five frames)
    for n in range(5):
        cnt, z, y, x, keys = vb.matches(n, p.G)
        ocnt, oz, oy, ox, ok = orc.vbm3d_matches(p, yuv[:, 0], n)
        assert np.array_equal(cnt, ocnt)
        for b in range(len(cnt)):
            m = cnt[b]
            assert np.array_equal(z[b, :m], oz[b, :m]) and np.array_equal(y[b, :m], oy[b, :m])
            assert np.array_equal(x[b, :m], ox[b, :m])


def test_vfinal_16bit_pipeline(orc):
    """Config-3 style chain on a small clip: VBasic -> VAggregate -> VFinal -> VAggregate, 16-bit."""
    nz, _ = synth.motion_frames(8, 4, 40, 48, 15.0, planes=3)
    yuv = np.stack([np.stack([synth.to_u16(np.clip(nz[f, c], 0, 1))
                              for c in range(3)]) for f in range(4)])
    src = source(yuv, "YUV")
    basic = core.bm3d.VAggregate(core.bm3d.VBasic(src, radius=1, ps_num=2, ps_range=4, sigma=15.0), radius=1)
    final = core.bm3d.VAggregate(core.bm3d.VFinal(src, basic, radius=1, sigma=15.0), radius=1)
    g_basic = basic.numpy()
    p = orc.default_params(0, True, "fast", 15.0, width=48, height=40, radius=1, ps_num=2, ps_range=4)
    f = np.stack([np.stack([orc.int2float(yuv[k, c], 16, True, c > 0) for c in range(3)]) for k in range(4)])
    o_basic_f = orc.vaggregate(1, orc.vbm3d(p, f))
    o_basic = np.stack([np.stack([orc.float2int(o_basic_f[k, c], 16, True, c > 0) for c in range(3)]) for k in range(4)])
    assert np.abs(g_basic.astype(np.int64) - o_basic.astype(np.int64)).max() <= 1
    g_final = final.numpy()
    pf = orc.default_params(1, True, "fast", 15.0, width=48, height=40, radius=1)
    rf = np.stack([np.stack([orc.int2float(g_basic[k, c], 16, True, c > 0) for c in range(3)]) for k in range(4)])
    o_final_f = orc.vaggregate(1, orc.vbm3d(pf, f, rf))
    o_final = np.stack([np.stack([orc.float2int(o_final_f[k, c], 16, True, c > 0) for c in range(3)]) for k in range(4)])
    assert np.abs(g_final.astype(np.int64) - o_final.astype(np.int64)).max() <= 1


# ---- aggregated V-BM3D output (no stacked clip) -------------------------------------------------

@pytest.mark.parametrize("sample", [1, 0])
def test_vbasic_vfinal_aggregate_equals_chain(sample):
    """VBasic / VFinal with aggregate=1 give VAggregate(radius, sample) of their stacked output,
    for whole-clip batches and for single-frame requests (which filter the neighbouring reference
    frames too)."""
    nz, _ = synth.motion_frames(9, 5, 40, 56, 15.0, planes=3)
    if sample == 1:
        src = source(nz.astype(np.float32), "YUV")
    else:
        src = source(np.stack([np.stack([synth.to_u16(np.clip(nz[f, c], 0, 1)) for c in range(3)]) for f in range(5)]), "YUV")
    chain_b = core.bm3d.VAggregate(core.bm3d.VBasic(src, radius=2, sigma=15.0), radius=2, sample=sample)
    fused_b = core.bm3d.VBasic(src, radius=2, sigma=15.0, aggregate=1, sample=sample)
    assert fused_b.height == 40 and fused_b.bits_per_sample == (32 if sample else 16)
    cb = chain_b.numpy()
    tol = TOL if sample == 1 else 1
    for batch in (None, 1):
        fb = core.bm3d.VBasic(src, radius=2, sigma=15.0, aggregate=1, sample=sample).numpy(batch)
        assert np.abs(fb.astype(np.float64) - cb.astype(np.float64)).max() <= tol
    f0 = fused_b.get_frame(0)
    assert "BM3D_V_radius" not in f0.props and "BM3D_V_process" not in f0.props
    ref = source(cb, "YUV")
    chain_f = core.bm3d.VAggregate(core.bm3d.VFinal(src, ref, radius=2, sigma=15.0), radius=2, sample=sample).numpy()
    fused_f = core.bm3d.VFinal(src, ref, radius=2, sigma=15.0, aggregate=1, sample=sample).numpy(2)
    assert np.abs(fused_f.astype(np.float64) - chain_f.astype(np.float64)).max() <= tol


# ---- the mvsfunc wrapper's call sequence ----------------------------------------------------------

def test_mvsfunc_bm3d_call_pattern(orc):
    """mvsfunc.BM3D(src, sigma=3.0, profile1="fast") on RGB float input (README.md:329-335), as the
    wrapper issues it: RGB2OPP(sample=1) -> Basic(sigma=[3,3,3], profile='fast', matrix=100) ->
    Final(opp, basic, same) -> OPP2RGB(sample=1)."""
    nz, _ = synth.rgb_frames(17, 2, 72, 96, 3.0)
    src = source(nz, "RGB")
    opp = core.bm3d.RGB2OPP(src, 1)
    basic = core.bm3d.Basic(opp, sigma=[3.0, 3.0, 3.0], profile="fast", matrix=100)
    final = core.bm3d.Final(opp, basic, sigma=[3.0, 3.0, 3.0], profile="fast", matrix=100)
    out = core.bm3d.OPP2RGB(final, 1)
    g_basic, g_out = basic.numpy(), out.numpy()
    o_opp = np.stack([orc.rgb2opp(nz[k]) for k in range(2)])
    pb = orc.default_params(0, False, "fast", 3.0, matrix=100)
    assert np.abs(g_basic - orc.bm3d(pb, o_opp)).max() <= TOL
    pf = orc.default_params(1, False, "fast", 3.0, matrix=100)
    o_final = orc.bm3d(pf, o_opp, g_basic)
    o_out = np.stack([orc.opp2rgb(o_final[k]) for k in range(2)])
    assert np.abs(g_out - o_out).max() <= 2 * TOL
    assert out.color_family == bm3d_b200.RGB and out.bits_per_sample == 32
