"""GPU parity at the full sizes of the reference workloads, and the input/output formats the
drop-in has to reproduce.

* 1080p RGB float, 2 frames: RGB2OPP -> Basic('np') -> Final('np') -> OPP2RGB (the benchmark's
  pipeline).  Match lists of every reference block of both frames are index-identical to the
  oracle's (Final with the oracle's Basic estimate as ref on both sides, so matching sees the same
  input); outputs within max abs 1e-4 (2e-4 after OPP2RGB, which sums three planes).
* 1080p YUV444 16-bit, 3 frames: VBasic(radius 1, ps_num 2, ps_range 4) -> VAggregate -> VFinal
  -> VAggregate, within 1 LSB; VBasic match lists of the middle frame index-identical.
* 8-bit input, limited-range input (_Range = 0: chroma without clip, output rounding +0.5),
  integer RGB through Basic's internal OPP path, RGB2OPP / OPP2RGB with sample = 0, the 'vn'
  Final (block size 11, generic filter kernel), group_size 64 / 128, bm_step / ps_step 2.

Every test prints the tie events and hard-threshold flip counts of the oracle next to the GPU's
exact tie-path block count (run pytest with -s to see them).
"""
import os

import numpy as np
import pytest

from bm3d_b200 import core, source, synth

pytestmark = pytest.mark.gpu

TOL = 1e-4
THREADS = max(1, os.cpu_count() or 1)


def lists_equal(node, k, exp, G):
    """Index-identical lists: counts, positions and keys (bit for bit) of every block."""
    cnt, z, y, x, keys = node.matches(k, G)
    ocnt, oy, ox, ok = exp
    assert np.array_equal(cnt, ocnt)
    mask = np.arange(G)[None, :] < cnt[:, None]
    assert np.array_equal(np.where(mask, y, -1), np.where(mask, oy, -1))
    assert np.array_equal(np.where(mask, x, -1), np.where(mask, ox, -1))
    assert np.array_equal(np.where(mask, keys.view(np.int32), 0), np.where(mask, ok.view(np.int32), 0))


def report(name, **kv):
    print(f"\n[{name}] " + " ".join(f"{k}={v}" for k, v in kv.items()))


# ---- 1920x1080 RGB float, Basic + Final --------------------------------------------------------

@pytest.fixture(scope="module")
def cfg2(orc):
    nz, clean = synth.rgb_frames(2, 2, 1080, 1920, 10.0)
    opp = np.stack([orc.rgb2opp(nz[k]) for k in range(2)])
    pb = orc.default_params(0, False, "np", 10.0, matrix=100)
    o_basic, st_b = orc.bm3d(pb, opp, threads=THREADS, stats=True)
    return dict(nz=nz, clean=clean, opp=opp, pb=pb, o_basic=o_basic, st_b=st_b)


def test_1080p_rgb_basic_lists_and_outputs(orc, cfg2):
    nz, opp, pb = cfg2["nz"], cfg2["opp"], cfg2["pb"]
    src = source(nz, "RGB")
    g_opp = core.bm3d.RGB2OPP(src, sample=1)
    basic = core.bm3d.Basic(g_opp, profile="np", matrix=100)
    gb = basic.numpy()
    assert np.array_equal(g_opp.numpy().view(np.int32), opp.view(np.int32))
    ties = 0
    for k in range(2):
        exp, st = orc.bm3d_matches(pb, opp[k, 0], threads=THREADS, stats=True)
        lists_equal(basic, k, exp, pb.G)
        ties += st["tie_blocks"]
    err = float(np.abs(gb - cfg2["o_basic"]).max())
    st = cfg2["st_b"]
    report("1080p Basic np", max_abs=f"{err:.3g}", oracle_tie_blocks=ties, gpu_tie_path_blocks=basic.slow_blocks(),
           flips_fp32_vs_fp64=st["flips_vs_fp64"], decisions=st["coefficients"], near_threshold=st["near_threshold"])
    assert err <= TOL


def test_1080p_rgb_final_lists_and_outputs(orc, cfg2):
    nz, opp, o_basic = cfg2["nz"], cfg2["opp"], cfg2["o_basic"]
    g_opp = core.bm3d.RGB2OPP(source(nz, "RGB"), sample=1)
    ref = source(o_basic, "YUV", props={"BM3D_OPP": 1})
    final = core.bm3d.Final(g_opp, ref, profile="np", matrix=100)
    rgb = core.bm3d.OPP2RGB(final, sample=1)
    g_rgb = rgb.numpy()
    g_final = np.stack([f.numpy() for f in final.get_frames(0, 2)])
    pf = orc.default_params(1, False, "np", 10.0, matrix=100)
    o_final, st = orc.bm3d(pf, opp, o_basic, threads=THREADS, stats=True)
    ties = 0
    for k in range(2):
        exp, sm = orc.bm3d_matches(pf, o_basic[k, 0], threads=THREADS, stats=True)
        lists_equal(final, k, exp, pf.G)
        ties += sm["tie_blocks"]
    err = float(np.abs(g_final - o_final).max())
    o_rgb = np.stack([orc.opp2rgb(o_final[k]) for k in range(2)])
    err_rgb = float(np.abs(g_rgb - o_rgb).max())
    # the reference's shipped x86 build takes the Wiener weight through _mm_rcp_ps
    o_rcp = orc.bm3d(orc.default_params(1, False, "np", 10.0, matrix=100, wiener_mode=1), opp, o_basic,
                     threads=THREADS)
    rcp_dev = float(np.abs(o_rcp - o_final).max())
    psnr = lambda a: 10 * np.log10(1.0 / np.mean((a.astype(np.float64) - cfg2["clean"]) ** 2))
    report("1080p Final np", max_abs=f"{err:.3g}", max_abs_rgb=f"{err_rgb:.3g}", oracle_tie_blocks=ties,
           gpu_tie_path_blocks=final.slow_blocks(), rcpps_vs_exact_max_abs=f"{rcp_dev:.3g}",
           psnr_gpu=f"{psnr(g_rgb):.4f}", psnr_oracle_rcpps=f"{psnr(np.stack([orc.opp2rgb(o_rcp[k]) for k in range(2)])):.4f}")
    assert err <= TOL
    assert err_rgb <= 2 * TOL


# ---- 1920x1080 YUV444 16-bit V-BM3D ------------------------------------------------------------

def test_1080p_yuv16_vbm3d_pipeline(orc):
    F = 3
    nz, _ = synth.motion_frames(3, F, 1080, 1920, 15.0, planes=3)
    yuv = np.stack([np.stack([synth.to_u16(np.clip(nz[f, c], 0, 1)) for c in range(3)]) for f in range(F)])
    src = source(yuv, "YUV")
    vb = core.bm3d.VBasic(src, radius=1, ps_num=2, ps_range=4, sigma=15.0)
    basic = core.bm3d.VAggregate(vb, radius=1)
    final = core.bm3d.VAggregate(core.bm3d.VFinal(src, basic, radius=1, sigma=15.0), radius=1)
    g_basic = basic.numpy()
    g_final = final.numpy()
    p = orc.default_params(0, True, "fast", 15.0, width=1920, height=1080, radius=1, ps_num=2, ps_range=4)
    fl = np.stack([np.stack([orc.int2float(yuv[k, c], 16, True, c > 0) for c in range(3)]) for k in range(F)])
    o_st, st_b = orc.vbm3d(p, fl, threads=THREADS, stats=True)
    o_basic_f = orc.vaggregate(1, o_st)
    o_basic = np.stack([np.stack([orc.float2int(o_basic_f[k, c], 16, True, c > 0) for c in range(3)]) for k in range(F)])
    d_basic = int(np.abs(g_basic.astype(np.int64) - o_basic.astype(np.int64)).max())
    pf = orc.default_params(1, True, "fast", 15.0, width=1920, height=1080, radius=1)
    rf = np.stack([np.stack([orc.int2float(g_basic[k, c], 16, True, c > 0) for c in range(3)]) for k in range(F)])
    o_final_f = orc.vaggregate(1, orc.vbm3d(pf, fl, rf, threads=THREADS))
    o_final = np.stack([np.stack([orc.float2int(o_final_f[k, c], 16, True, c > 0) for c in range(3)]) for k in range(F)])
    d_final = int(np.abs(g_final.astype(np.int64) - o_final.astype(np.int64)).max())
    # VBasic match lists of the middle frame (a batch of that frame alone)
    vb.compute(1, 1)
    cnt, z, y, x, keys = vb.matches(0, p.G)
    (ocnt, oz, oy, ox, ok), sm = orc.vbm3d_matches(p, fl[:, 0], 1, threads=THREADS, stats=True)
    assert np.array_equal(cnt, ocnt)
    mask = np.arange(p.G)[None, :] < cnt[:, None]
    for a, b in ((z, oz), (y, oy), (x, ox)):
        assert np.array_equal(np.where(mask, a, -1), np.where(mask, b, -1))
    assert np.array_equal(np.where(mask, keys.view(np.int32), 0), np.where(mask, ok.view(np.int32), 0))
    report("1080p V-BM3D u16", basic_max_lsb=d_basic, final_max_lsb=d_final, oracle_tie_blocks=sm["tie_blocks"],
           gpu_tie_path_blocks=vb.slow_blocks(), flips_fp32_vs_fp64=st_b["flips_vs_fp64"],
           decisions=st_b["coefficients"])
    assert d_basic <= 1 and d_final <= 1


# ---- formats -----------------------------------------------------------------------------------

def test_gray_8bit(orc):
    nz, _ = synth.gray_frames(11, 2, 64, 80, 12.0)
    u8 = np.clip(np.round(nz * 255.0), 0, 255).astype(np.uint8)
    g = core.bm3d.Basic(source(u8, "GRAY"), profile="np", sigma=12.0).numpy()
    p = orc.default_params(0, False, "np", 12.0, width=80, height=64)
    f = np.stack([orc.int2float(u8[k, 0], 8, True, False) for k in range(2)])[:, None]
    o = orc.bm3d(p, f)
    oi = np.stack([orc.float2int(o[k, 0], 8, True, False) for k in range(2)])[:, None]
    assert g.dtype == np.uint8
    assert np.abs(g.astype(np.int64) - oi.astype(np.int64)).max() <= 1


@pytest.mark.parametrize("bits", [8, 16])
def test_limited_range_yuv(orc, bits):
    """_Range = 0: limited-range quantisation both ways (Int2Float / Float2Int with full = false)."""
    nz, _ = synth.rgb_frames(12, 1, 48, 64, 10.0)
    lo, hi_y, hi_c = 16 << (bits - 8), 235 << (bits - 8), 240 << (bits - 8)
    dt = np.uint8 if bits == 8 else np.uint16
    planes = [np.clip(np.round(lo + nz[0, 0] * (hi_y - lo)), lo, hi_y)]
    for c in (1, 2):
        planes.append(np.clip(np.round((1 << (bits - 1)) + (nz[0, c] - 0.5) * (hi_c - lo)), lo, hi_c))
    yuv = np.stack(planes).astype(dt)[None]
    node = core.bm3d.Basic(source(yuv, "YUV", props={"_Range": 0}), profile="fast", sigma=10.0)
    g = node.numpy()
    p = orc.default_params(0, False, "fast", 10.0, width=64, height=48)
    f = np.stack([orc.int2float(yuv[0, c], bits, False, c > 0) for c in range(3)])[None]
    o = orc.bm3d(p, f)
    oi = np.stack([orc.float2int(o[0, c], bits, False, c > 0) for c in range(3)])
    assert np.abs(g[0].astype(np.int64) - oi.astype(np.int64)).max() <= 1
    assert node.get_frame(0).props.get("_Range") == 0


@pytest.mark.parametrize("bits", [8, 16])
def test_rgb_integer_basic(orc, bits):
    """Integer RGB into Basic: RGB2FloatYUV -> filter in OPP -> FloatYUV2RGB with clipping
    (source/BM3D_Base.cpp:663-749)."""
    nz, _ = synth.rgb_frames(13, 1, 48, 64, 10.0)
    dt = np.uint8 if bits == 8 else np.uint16
    rgb = np.clip(np.round(nz * ((1 << bits) - 1)), 0, (1 << bits) - 1).astype(dt)
    g = core.bm3d.Basic(source(rgb, "RGB"), profile="lc", sigma=10.0).numpy()
    p = orc.default_params(0, False, "lc", 10.0, matrix=100)
    opp = orc.rgb2opp_any(rgb[0], np.float32, clip=False)
    o = orc.bm3d(p, opp[None])[0]
    exp = orc.opp2rgb_any(o, dt)
    assert g.dtype == dt
    assert np.abs(g[0].astype(np.int64) - exp.astype(np.int64)).max() <= 1


@pytest.mark.parametrize("bits", [8, 16])
def test_rgb2opp_opp2rgb_sample0(orc, bits):
    """RGB2OPP / OPP2RGB with sample = 0 (16-bit integer output, clipped): bit-exact."""
    nz, _ = synth.rgb_frames(14, 2, 40, 56, 10.0)
    dt = np.uint8 if bits == 8 else np.uint16
    rgb = np.clip(np.round(nz * ((1 << bits) - 1)), 0, (1 << bits) - 1).astype(dt)
    opp = core.bm3d.RGB2OPP(source(rgb, "RGB"), sample=0)
    g_opp = opp.numpy()
    assert g_opp.dtype == np.uint16
    o_opp = np.stack([orc.rgb2opp_any(rgb[k], np.uint16) for k in range(2)])
    assert np.array_equal(g_opp, o_opp)
    assert opp.get_frame(0).props.get("BM3D_OPP") == 1
    back = core.bm3d.OPP2RGB(opp, sample=0).numpy()
    o_back = np.stack([orc.opp2rgb_any(o_opp[k], np.uint16) for k in range(2)])
    assert back.dtype == np.uint16 and np.array_equal(back, o_back)
    # float OPP in, 16-bit RGB out
    fopp = core.bm3d.RGB2OPP(source(rgb, "RGB"), sample=1)
    back_f = core.bm3d.OPP2RGB(fopp, sample=0).numpy()
    o_f = np.stack([orc.opp2rgb_any(orc.rgb2opp_any(rgb[k], np.float32), np.uint16) for k in range(2)])
    assert np.array_equal(back_f, o_f)


def test_vn_final_block11(orc):
    """profile 'vn': Final with block_size 11 (generic filter kernel, non-power-of-two DCT)."""
    nz, _ = synth.gray_frames(15, 2, 72, 96, 20.0)
    pb = orc.default_params(0, False, "vn", 20.0, width=96, height=72)
    ob = orc.bm3d(pb, nz)
    gb = core.bm3d.Basic(source(nz, "GRAY"), profile="vn", sigma=20.0).numpy()
    assert np.abs(gb - ob).max() <= TOL
    pf = orc.default_params(1, False, "vn", 20.0, width=96, height=72)
    assert pf.B == 11
    f = core.bm3d.Final(source(nz, "GRAY"), source(ob, "GRAY"), profile="vn", sigma=20.0)
    gf = f.numpy()
    of = orc.bm3d(pf, nz, ob)
    for k in range(2):
        lists_equal(f, k, orc.bm3d_matches(pf, ob[k, 0]), pf.G)
    assert np.abs(gf - of).max() <= TOL


@pytest.mark.parametrize("G", [64, 128])
@pytest.mark.parametrize("wiener", [0, 1])
def test_large_group_sizes(orc, wiener, G):
    nz, _ = synth.gray_frames(16, 1, 64, 72, 10.0)
    pb = orc.default_params(0, False, "np", 10.0, width=72, height=64, group_size=G)
    ob = orc.bm3d(pb, nz)
    if not wiener:
        node = core.bm3d.Basic(source(nz, "GRAY"), profile="np", group_size=G)
        g = node.numpy()
        lists_equal(node, 0, orc.bm3d_matches(pb, nz[0, 0]), G)
        assert np.abs(g - ob).max() <= TOL
    else:
        pf = orc.default_params(1, False, "np", 10.0, width=72, height=64, group_size=G)
        node = core.bm3d.Final(source(nz, "GRAY"), source(ob, "GRAY"), profile="np", group_size=G)
        g = node.numpy()
        lists_equal(node, 0, orc.bm3d_matches(pf, ob[0, 0]), G)
        assert np.abs(g - orc.bm3d(pf, nz, ob)).max() <= TOL


def test_search_steps_above_one(orc):
    """bm_step = 2 (range-form lattice) and ps_step = 2 (predictive windows) outputs."""
    nz, _ = synth.gray_frames(18, 1, 72, 96, 12.0)
    pb = orc.default_params(0, False, "lc", 12.0, width=96, height=72, bm_step=2)
    node = core.bm3d.Basic(source(nz, "GRAY"), profile="lc", sigma=12.0, bm_step=2)
    g = node.numpy()
    lists_equal(node, 0, orc.bm3d_matches(pb, nz[0, 0]), pb.G)
    assert np.abs(g - orc.bm3d(pb, nz)).max() <= TOL
    mz, _ = synth.motion_frames(19, 4, 40, 56, 12.0, planes=1)
    clip = mz.astype(np.float32)
    pv = orc.default_params(0, True, "lc", 12.0, width=56, height=40, ps_step=2, bm_step=2)
    vb = core.bm3d.VBasic(source(clip, "GRAY"), profile="lc", sigma=12.0, ps_step=2, bm_step=2)
    agg = core.bm3d.VAggregate(vb, radius=pv.radius, sample=1).numpy()
    o_agg = orc.vaggregate(pv.radius, orc.vbm3d(pv, clip), process=(1, 0, 0))
    assert np.abs(agg[:, 0] - o_agg[:, 0]).max() <= TOL
