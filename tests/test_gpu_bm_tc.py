"""Precision-form block matching (precision="tf32"): bf16 tensor-core distance estimates with an
error-bounded short list and exact re-ranking.

Bar: the match lists are the plain kernel's lists exactly (positions, order, keys bit for bit),
on ordinary noisy frames, on clipped windows of small frames, on frames full of exact ties
(piecewise-constant, noise-free), and against the oracle for one configuration.  The number of
reference blocks that needed the exact fallback is reported; no tensor-core wait may time out.
"""
import numpy as np
import pytest

from bm3d_b200 import core, source, synth

pytestmark = pytest.mark.gpu


def lists(node, k, G):
    cnt, z, y, x, keys = node.matches(k, G)
    return cnt, y, x, keys


def assert_same_lists(a, b, what):
    ca, ya, xa, ka = a
    cb, yb, xb, kb = b
    assert np.array_equal(ca, cb), what
    for i in range(len(ca)):
        n = ca[i]
        assert np.array_equal(ya[i, :n], yb[i, :n]), (what, i)
        assert np.array_equal(xa[i, :n], xb[i, :n]), (what, i)
        assert np.array_equal(ka[i, :n].view(np.int32), kb[i, :n].view(np.int32)), (what, i)


def basic_lists(nz, profile, sigma, precision, **kw):
    node = core.bm3d.Basic(source(nz, "GRAY"), profile=profile, sigma=sigma, precision=precision, **kw)
    node.get_frames(0, nz.shape[0])
    return node


def final_lists(nz, ref, profile, sigma, precision):
    node = core.bm3d.Final(source(nz, "GRAY"), source(ref, "GRAY"), profile=profile, sigma=sigma, precision=precision)
    node.get_frames(0, nz.shape[0])
    return node


@pytest.mark.parametrize("profile,sigma", [("np", 10.0), ("lc", 25.0), ("high", 15.0)])
@pytest.mark.parametrize("h,w", [(160, 224), (40, 56)])
def test_tc_matching_equals_plain(profile, sigma, h, w):
    nz, _ = synth.gray_frames(61, 2, h, w, sigma)
    p = basic_lists(nz, profile, sigma, "fp32")
    t = basic_lists(nz, profile, sigma, "tf32")
    G = 16 if profile != "vn" else 32
    for k in range(2):
        assert_same_lists(lists(t, k, G), lists(p, k, G), f"basic {profile} {h}x{w} frame {k}")
    fb, to = t.bm_tc_counts()
    print(f"basic {profile} {h}x{w}: exact fallbacks {fb}, time-outs {to}")
    assert to == 0
    ref = p.numpy()
    pf = final_lists(nz, ref, profile, sigma, "fp32")
    tf = final_lists(nz, ref, profile, sigma, "tf32")
    Gf = 32 if profile in ("np", "high") else 16
    for k in range(2):
        assert_same_lists(lists(tf, k, Gf), lists(pf, k, Gf), f"final {profile} {h}x{w} frame {k}")
    fb, to = tf.bm_tc_counts()
    print(f"final {profile} {h}x{w}: exact fallbacks {fb}, time-outs {to}")
    assert to == 0


def test_tc_matching_ties_fall_back_exactly():
    """Noise-free piecewise-constant frames: many zero and equal distances, so the estimates
    cannot settle most lists; the fallback must reproduce the plain lists (tie order included)."""
    rng = np.random.default_rng(62)
    img = np.zeros((1, 1, 96, 128), np.float32)
    for _ in range(12):
        y0, x0 = rng.integers(0, 80), rng.integers(0, 110)
        img[0, 0, y0:y0 + rng.integers(8, 40), x0:x0 + rng.integers(8, 40)] = rng.integers(0, 8) / 8.0
    p = basic_lists(img, "np", 10.0, "fp32")
    t = basic_lists(img, "np", 10.0, "tf32")
    assert_same_lists(lists(t, 0, 16), lists(p, 0, 16), "piecewise constant")
    fb, to = t.bm_tc_counts()
    print(f"piecewise constant: exact fallbacks {fb} of {len(lists(t, 0, 16)[0])} blocks, time-outs {to}")
    assert fb > 0 and to == 0


def test_tc_matching_matches_oracle(orc):
    nz, _ = synth.gray_frames(63, 1, 96, 128, 15.0)
    t = basic_lists(nz, "np", 15.0, "tf32")
    pb = orc.default_params(0, False, "np", 15.0, width=128, height=96)
    ocnt, oy, ox, ok = orc.bm3d_matches(pb, nz[0, 0])
    assert_same_lists(lists(t, 0, pb.G), (ocnt, oy, ox, ok), "oracle")
