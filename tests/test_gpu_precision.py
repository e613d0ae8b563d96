"""Precision form (precision="tf32"): tensor-core transforms against the plain FP32 path.

The plain path is the oracle-exact drop-in; the precision form computes the 3-D DCTs of full
groups as tf32 matrix products, so its output differs slightly (hard-threshold decisions near
the threshold can flip).  Bars: PSNR against the clean frames within 0.05 dB of the plain path's;
RMS deviation from the plain output below 10 % of the noise level, maximum below the noise level.
"""
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
def test_hard_threshold_flips_counted(sigma):
    """Hard-threshold decisions of the precision form against the plain path, on the same match
    lists (the tensor-core matching is exact): without the near-threshold recheck the tf32
    coefficients flip some decisions; with it every coefficient within the band is recomputed in
    fp32 from the pixels and no decision differs."""
    nz, _ = synth.gray_frames(55, 2, 540, 960, sigma)
    clip = source(nz, "GRAY")
    plain = core.bm3d.Basic(clip, profile="np", sigma=sigma)
    plain.numpy()
    raw = core.bm3d.Basic(clip, profile="np", sigma=sigma, precision="tf32")
    raw.set_recheck_band(0.0)
    raw.numpy()
    tc = core.bm3d.Basic(clip, profile="np", sigma=sigma, precision="tf32")
    tc.numpy()
    f_raw = sum(flips(raw, plain, k)[0] for k in range(2))
    f_tc, dec = 0, 0
    for k in range(2):
        f, d = flips(tc, plain, k)
        f_tc += f
    rechecked, changed = tc.threshold_rechecks()
    kept = sum(int(plain.retained_counts(k)[0].sum()) for k in range(2))
    print(f"sigma {sigma}: retained {kept}, flips without recheck {f_raw}, with recheck {f_tc}; "
          f"recomputed {rechecked}, changed {changed}")
    assert f_tc == 0
