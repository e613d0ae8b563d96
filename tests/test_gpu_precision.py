"""Precision form (precision="tf32"): tensor-core transforms against the plain FP32 path.

The plain path is the oracle-exact drop-in; the precision form computes the 3-D DCTs of full
groups as tf32 matrix products, so its output differs slightly (hard-threshold decisions near
the threshold can flip).  Bars: PSNR against the clean frames within 0.05 dB of the plain path's;
RMS deviation from the plain output below 10 % of the noise level, maximum below the noise level.
"""
import os

import numpy as np
import pytest

from bm3d_b200 import core, source, synth

pytestmark = pytest.mark.gpu

PSNR_TOL_DB = 0.05


def check_close(tc, plain, clean, sigma, what):
    s = sigma / 255.0
    d = tc.astype(np.float64) - plain
    dpsnr = psnr(tc, clean) - psnr(plain, clean)
    rms, mx = float(np.sqrt(np.mean(d * d))), float(np.abs(d).max())
    print(f"{what}: psnr delta {dpsnr:+.4f} dB, rms dev {rms:.2e}, max dev {mx:.2e}")
    assert np.isfinite(tc).all()
    assert abs(dpsnr) <= PSNR_TOL_DB, what
    assert rms <= 0.1 * s, what
    assert mx <= s, what


def psnr(x, clean):
    return 10 * np.log10(1.0 / np.mean((x.astype(np.float64) - clean) ** 2))


def run_gray(nz, profile, sigma, precision):
    clip = source(nz, "GRAY")
    basic = core.bm3d.Basic(clip, profile=profile, sigma=sigma, precision=precision)
    final = core.bm3d.Final(clip, basic, profile=profile, sigma=sigma, precision=precision)
    return basic.numpy(), final.numpy()


@pytest.mark.parametrize("profile,sigma", [("np", 10.0), ("lc", 25.0), ("fast", 5.0), ("vn", 30.0)])
def test_tf32_gray_close_to_plain(profile, sigma):
    nz, clean = synth.gray_frames(51, 2, 160, 224, sigma)
    b0, f0 = run_gray(nz, profile, sigma, "fp32")
    b1, f1 = run_gray(nz, profile, sigma, "tf32")
    check_close(b1, b0, clean, sigma, f"basic {profile}")
    check_close(f1, f0, clean, sigma, f"final {profile}")


def test_tf32_rgb_pipeline_psnr():
    nz, clean = synth.rgb_frames(52, 2, 144, 200, 10.0)
    out = {}
    for prec in ("fp32", "tf32"):
        opp = core.bm3d.RGB2OPP(source(nz, "RGB"), sample=1)
        b = core.bm3d.Basic(opp, profile="np", matrix=100, precision=prec)
        f = core.bm3d.Final(opp, b, profile="np", matrix=100, precision=prec)
        out[prec] = core.bm3d.OPP2RGB(f, sample=1).numpy()
    check_close(out["tf32"], out["fp32"], clean, 10.0, "rgb pipeline")


def test_tf32_vbm3d_close_to_plain():
    nz, clean = synth.motion_frames(53, 4, 96, 128, 15.0, planes=1)
    nz = nz.astype(np.float32)
    out = {}
    for prec in ("fp32", "tf32"):
        clip = source(nz, "GRAY")
        vb = core.bm3d.VAggregate(core.bm3d.VBasic(clip, radius=1, sigma=15.0, precision=prec), radius=1, sample=1)
        vf = core.bm3d.VAggregate(core.bm3d.VFinal(clip, vb, radius=1, sigma=15.0, precision=prec), radius=1, sample=1)
        out[prec] = vf.numpy()
    check_close(out["tf32"], out["fp32"], clean, 15.0, "v-bm3d")


def test_precision_argument_is_validated():
    nz, _ = synth.gray_frames(54, 1, 32, 32, 10.0)
    with pytest.raises(Exception) as e:
        core.bm3d.Basic(source(nz, "GRAY"), precision="fp16")
    assert "precision" in str(e.value)


def flips(node_tc, node_plain, k):
    """Sum over groups of |retained count (precision form) - retained count (plain path)|: a
    lower bound of the keep / zero decisions that differ (exact unless one group flips both
    ways)."""
    a, b = node_tc.retained_counts(k), node_plain.retained_counts(k)
    assert (a >= 0).sum() == (b >= 0).sum() > 0
    m = b >= 0
    return int(np.abs(a[m].astype(np.int64) - b[m]).sum()), int(b[m].sum())


@pytest.mark.parametrize("sigma", [5.0, 10.0, 30.0])
def test_hard_threshold_flips_counted(orc, sigma):
    """Hard-threshold decisions of the precision form against the plain path, on the same match
    lists (the tensor-core matching is exact), for a sweep of the recheck band.  Without the
    recheck the tf32 coefficients flip some decisions; with it every coefficient within the band
    is recomputed from the pixels in double precision, so the decisions left differing from the
    plain path are those the plain FP32 transform itself takes against exact arithmetic (the
    oracle counts them on the same frames)."""
    nz, _ = synth.gray_frames(55, 2, 540, 960, sigma)
    clip = source(nz, "GRAY")
    plain = core.bm3d.Basic(clip, profile="np", sigma=sigma)
    plain.numpy()
    tc = core.bm3d.Basic(clip, profile="np", sigma=sigma, precision="tf32")
    res = {}
    for band in (0.0, 1.0 / 4096, 1.0 / 1024, 1.0 / 256, 1.0 / 64):
        tc.set_recheck_band(band)
        tc.compute(0, 2)
        res[band] = (sum(flips(tc, plain, k)[0] for k in range(2)),) + tc.threshold_rechecks()
    pb = orc.default_params(0, False, "np", sigma, width=960, height=540)
    _, st = orc.bm3d(pb, nz, threads=max(1, os.cpu_count() or 1), stats=True)
    kept = sum(int(plain.retained_counts(k)[0].sum()) for k in range(2))
    print(f"\nsigma {sigma}: decisions {st['coefficients']}, retained {kept}, plain FP32 vs FP64 flips "
          f"(oracle) {st['flips_vs_fp64']}; band -> (flips vs plain, recomputed, changed): "
          + ", ".join(f"1/{int(round(1 / b)) if b else 0}: {v}" for b, v in res.items()))
    f_raw, f_tc = res[0.0][0], res[1.0 / 64][0]
    assert f_raw > 0
    assert f_tc <= 2 * st["flips_vs_fp64"] + 4


def list_agreement(a, b, k, G):
    ca, _, ya, xa, _ = a.matches(k, G)
    cb, _, yb, xb, _ = b.matches(k, G)
    m = np.arange(G)[None, :] < ca[:, None]
    same = (ca == cb) & np.all(~m | ((ya == yb) & (xa == xb)), axis=1)
    return float(same.mean())


@pytest.mark.parametrize("sigma", [5.0, 15.0, 30.0])
def test_precision_form_2160p(sigma):
    """Gray float 3840x2160, 4 frames, profile 'np': the precision form against the plain path --
    PSNR delta against the clean frames, match-list agreement, hard-threshold flips, and the error
    of each stage's output against the FP64 recomputation of frame 0."""
    nz, clean = synth.gray_frames(4, 4, 2160, 3840, sigma)
    clip = source(nz, "GRAY")
    res = {}
    for prec in ("fp32", "tf32"):
        b = core.bm3d.Basic(clip, profile="np", sigma=sigma, precision=prec)
        f = core.bm3d.Final(clip, b, profile="np", sigma=sigma, precision=prec)
        ob, of = b.numpy(), f.numpy()
        eb = ob[0, 0].astype(np.float64) - b.reference_fp64(0)[0]
        ef = of[0, 0].astype(np.float64) - f.reference_fp64(0)[0]
        res[prec] = dict(b=b, f=f, ob=ob, of=of, eb=eb, ef=ef)
    # the Final match lists with the plain Basic estimate as ref on both sides
    ref = source(res["fp32"]["ob"], "GRAY")
    fp = core.bm3d.Final(clip, ref, profile="np", sigma=sigma)
    ft = core.bm3d.Final(clip, ref, profile="np", sigma=sigma, precision="tf32")
    fp.compute(0, 1)
    ft.compute(0, 1)
    agree_b = list_agreement(res["tf32"]["b"], res["fp32"]["b"], 0, 16)
    agree_f = list_agreement(ft, fp, 0, 32)
    fl = sum(flips(res["tf32"]["b"], res["fp32"]["b"], k)[0] for k in range(4))
    d_basic = psnr(res["tf32"]["ob"], clean) - psnr(res["fp32"]["ob"], clean)
    d_final = psnr(res["tf32"]["of"], clean) - psnr(res["fp32"]["of"], clean)
    stat = lambda e: f"rms {np.sqrt(np.mean(e * e)):.2e} max {np.abs(e).max():.2e}"
    print(f"\n2160p sigma {sigma}: psnr plain {psnr(res['fp32']['of'], clean):.3f} dB, delta basic {d_basic:+.4f} "
          f"final {d_final:+.4f} dB; list agreement basic {agree_b:.4f} final {agree_f:.4f}; flips {fl}; "
          f"vs FP64 basic plain [{stat(res['fp32']['eb'])}] tf32 [{stat(res['tf32']['eb'])}], "
          f"final plain [{stat(res['fp32']['ef'])}] tf32 [{stat(res['tf32']['ef'])}]")
    assert agree_b == 1.0 and agree_f == 1.0
    assert abs(d_final) <= PSNR_TOL_DB
    # decisions left differing from the plain path: of the order of the plain path's own FP32
    # flips against exact arithmetic (about 1e-8 of the decisions at 1080p)
    decisions = 4 * res["fp32"]["b"].retained_counts(0).shape[1] * 16 * 64
    assert fl <= 1e-7 * decisions


def test_tf32_final_short_groups():
    """Final on the tensor cores when most groups are shorter than group_size (a small th_mse
    leaves few candidates under the distance threshold): a short group takes the transforms of
    its own length in its rows of the z-stage matrices.  Against the plain Final (same Basic
    estimate as ref): PSNR within 0.05 dB and max deviation 2e-3 (the Wiener filter has no
    keep / zero decisions, so only tf32 rounding separates the two)."""
    sigma = 20.0
    nz, clean = synth.gray_frames(56, 2, 160, 224, sigma)
    clip = source(nz, "GRAY")
    basic = core.bm3d.Basic(clip, profile="np", sigma=sigma).numpy()
    out, short = {}, {}
    for prec in ("fp32", "tf32"):
        node = core.bm3d.Final(clip, source(basic, "GRAY"), profile="np", sigma=sigma,
                               th_mse=100.0, precision=prec)
        out[prec] = node.numpy()
        cnt = node.matches(0, 32)[0]
        short[prec] = float(np.mean(cnt < 32))
    assert short["tf32"] == short["fp32"]          # the same lists
    print(f"short groups: {short['tf32']:.3f}")
    assert short["tf32"] > 0.5
    check_close(out["tf32"], out["fp32"], clean, sigma, "final, short groups")
    assert float(np.abs(out["tf32"].astype(np.float64) - out["fp32"]).max()) <= 2e-3


def test_tf32_match_output_is_plain():
    """precision="tf32_match": the tensor-core matching (the plain kernel's lists) with the plain
    transforms, so Basic and Final give the "fp32" output up to the order of the aggregation's
    float atomics (which makes the plain path itself vary in the last bits): lists identical,
    outputs within 1e-5.  Both Finals take the same ref (a last-bit difference of the ref can
    reorder near-equal candidates)."""
    nz, _ = synth.gray_frames(57, 2, 144, 176, 10.0)
    clip = source(nz, "GRAY")
    ref = source(core.bm3d.Basic(clip, profile="np", sigma=10.0).numpy(), "GRAY")
    out, lists = {}, {}
    for prec in ("fp32", "tf32_match"):
        basic = core.bm3d.Basic(clip, profile="np", sigma=10.0, precision=prec)
        final = core.bm3d.Final(clip, ref, profile="np", sigma=10.0, precision=prec)
        out[prec] = (basic.numpy(), final.numpy())
        lists[prec] = basic.matches(0, 16)[:4] + final.matches(0, 32)[:4]
    for u, v in zip(lists["tf32_match"], lists["fp32"]):
        assert np.array_equal(u, v)
    for u, v in zip(out["tf32_match"], out["fp32"]):
        assert float(np.abs(u.astype(np.float64) - v).max()) <= 1e-5
