"""Learned block-matching proposal (precision="learned"): the network's GPU forward and backward
against the NumPy restatement (oracle/proposal_ref.py), training, group recall of the proposals
against the exhaustive search, the ablation with untrained weights, and the filter's PSNR.
"""
import ctypes as C

import numpy as np
import pytest

import proposal_ref as pr
from bm3d_b200 import _capi as capi
from bm3d_b200 import core, source, synth

pytestmark = pytest.mark.gpu
P = C.POINTER


def fptr(a):
    return a.ctypes.data_as(P(C.c_float))


def iptr(a):
    return a.ctypes.data_as(P(C.c_int))


def default_weights():
    w = np.zeros(pr.NW, np.float32)
    assert capi.lib().bm3d_proposal_default_weights(fptr(w), pr.NW) == pr.NW
    return w


def descriptors(x, w):
    H, W = x.shape
    out = np.zeros((H - 7, W - 7, 16), np.float32)
    assert capi.lib().bm3d_proposal_descriptors(fptr(x), W, H, fptr(w), fptr(out)) == 0
    return out


def gpu_grad(x, w, trip):
    H, W = x.shape
    t = np.ascontiguousarray(np.asarray(trip, np.int32).ravel())
    loss = np.zeros(1, np.float32)
    g = np.zeros(pr.NW, np.float32)
    assert capi.lib().bm3d_proposal_gradients(fptr(x), W, H, fptr(w), iptr(t), len(trip), fptr(loss), fptr(g)) == 0
    return float(loss[0]), g


def match(x, w, step, G, R, th, nprop):
    H, W = x.shape
    cap = 1 << 16
    cnt = np.zeros(cap, np.int32)
    ys = np.zeros(cap * G, np.int32)
    xs = np.zeros(cap * G, np.int32)
    n = capi.lib().bm3d_proposal_match(fptr(x), W, H, fptr(w) if w is not None else None, step, G, R, C.c_float(th),
                                        nprop, iptr(cnt), iptr(ys), iptr(xs), cap)
    assert n > 0
    return cnt[:n], ys[:n * G].reshape(n, G), xs[:n * G].reshape(n, G)


def recall(got, ref):
    """Mean over reference blocks of |proposal list ∩ exhaustive list| / |exhaustive list|."""
    (cg, yg, xg), (cr, yr, xr) = got, ref
    r = []
    for b in range(len(cr)):
        a = set(zip(yr[b, :cr[b]].tolist(), xr[b, :cr[b]].tolist()))
        s = set(zip(yg[b, :cg[b]].tolist(), xg[b, :cg[b]].tolist()))
        r.append(len(a & s) / len(a))
    return float(np.mean(r))


def test_descriptors_match_restatement():
    x = synth.gray_frames(70, 1, 40, 52, 10.0)[0][0, 0].astype(np.float32)
    w = default_weights()
    got = descriptors(x, w)
    _, _, ref = pr.forward(x, w, bf=True)
    tol = 2.0 ** -7 * np.abs(ref) + 1e-3 * np.abs(ref).max()        # one bf16 step, plus summation order
    assert np.all(np.abs(got - ref) <= tol)


def test_gradients_match_restatement():
    rng = np.random.default_rng(71)
    x = synth.gray_frames(71, 1, 36, 44, 10.0)[0][0, 0].astype(np.float32)
    w = default_weights()
    trip = [tuple(int(v) for v in (rng.integers(0, 29), rng.integers(0, 37), rng.integers(0, 29), rng.integers(0, 37),
                                   rng.integers(0, 29), rng.integers(0, 37))) for _ in range(64)]
    Lg, gg = gpu_grad(x, w, trip)
    Lr, gr = pr.loss_and_grad(x, w, trip, bf=True)
    print(f"loss gpu {Lg:.6f} restatement {Lr:.6f}; gradient norm {np.linalg.norm(gr):.4g}, "
          f"max abs diff {np.abs(gg - gr).max():.3g}")
    assert abs(Lg - Lr) <= 1e-3 * max(1.0, abs(Lr))
    assert np.linalg.norm(gg - gr) <= 2e-2 * np.linalg.norm(gr)
    cos = float(np.dot(gg, gr) / (np.linalg.norm(gg) * np.linalg.norm(gr)))
    assert cos > 0.999


def test_training_lowers_the_loss():
    frames = np.ascontiguousarray(np.stack([synth.gray_frames(72 + k, 1, 96, 96, 10.0)[0][0, 0] for k in range(2)]),
                                  np.float32)
    import train_proposal
    w0 = train_proposal.init_weights(3)
    w, losses = train_proposal.train(frames, 60, 512, 3e-3, 3, w0)
    print(f"loss first 10 {losses[:10].mean():.4f}, last 10 {losses[-10:].mean():.4f}")
    assert np.isfinite(losses).all()
    assert losses[-10:].mean() < 0.9 * losses[:10].mean()


def test_recall_and_ablation():
    """Group recall of the learned proposals (64 of the 1,089 window candidates; the filter uses
    96) against the exhaustive search, at two noise levels; the untrained network (He
    initialisation) must do clearly worse, a random choice of 64 would find 5.9 %."""
    import train_proposal
    for seed, sigma, bar in ((73, 10.0, 0.72), (75, 25.0, 0.62)):
        x = synth.gray_frames(seed, 1, 160, 224, sigma)[0][0, 0].astype(np.float32)
        ref = match(x, None, 4, 16, 16, 3.0e38, 64)
        r_trained = recall(match(x, default_weights(), 4, 16, 16, 3.0e38, 64), ref)
        r_untrained = recall(match(x, train_proposal.init_weights(1), 4, 16, 16, 3.0e38, 64), ref)
        print(f"sigma {sigma}: recall of the 16-lists with 64 proposals: trained {r_trained:.4f}, "
              f"untrained {r_untrained:.4f}, random {64 / 1089:.4f}")
        assert r_trained >= bar
        assert r_trained >= r_untrained + 0.05


def test_learned_filter_psnr():
    """Basic + Final with learned proposals against the exhaustive search of the tf32 form: the
    lists lose some of their best matches, so the output loses PSNR; bounded here at 0.3 dB on this
    small frame pair (the measured loss is reported; on the 1080p benchmark it is 0.046 dB)."""
    nz, clean = synth.gray_frames(74, 2, 160, 224, 10.0)

    def run(prec):
        clip = source(nz, "GRAY")
        b = core.bm3d.Basic(clip, profile="np", sigma=10.0, precision=prec)
        f = core.bm3d.Final(clip, b, profile="np", sigma=10.0, precision=prec)
        return f.numpy()

    def psnr(o):
        return 10 * np.log10(1.0 / np.mean((o.astype(np.float64) - clean) ** 2))

    p_exh, p_learn = psnr(run("tf32")), psnr(run("learned"))
    print(f"PSNR exhaustive (tf32) {p_exh:.4f} dB, learned proposals {p_learn:.4f} dB")
    assert np.isfinite(p_learn)
    assert p_learn >= p_exh - 0.3


def proposal_sets(x, w, step, R, nprop):
    H, W = x.shape
    cap = 1 << 14
    sets = np.zeros(cap * nprop, np.uint32)
    ovf = C.c_int64(0)
    n = capi.lib().bm3d_debug_proposal_sets(fptr(x), W, H, fptr(w), step, R, nprop,
                                            sets.ctypes.data_as(P(C.c_uint32)), C.byref(ovf), cap)
    assert n > 0
    return sets[:n * nprop].reshape(n, nprop), int(ovf.value)


@pytest.mark.parametrize("kind", ["noisy", "flat"])
def test_proposal_sets_are_the_best_nprop(kind):
    """Every block's proposal set holds the nprop best candidates by descriptor distance (the
    trailing default (0, 0) candidate included, the block itself excluded): no candidate outside
    the set scores lower than one inside.  The flat frame makes the scores nearly equal (the
    number of blocks that needed the exact bisection of the cut is printed)."""
    H, W, R, step, nprop = 56, 72, 16, 4, 96
    if kind == "noisy":
        x = synth.gray_frames(21, 1, H, W, 20.0)[0][0, 0]
    else:
        x = np.full((H, W), 0.5, np.float32) + 1e-4 * np.random.default_rng(3).normal(size=(H, W)).astype(np.float32)
    w = default_weights()
    d = descriptors(x, w).astype(np.float64)
    sets, ovf = proposal_sets(x, w, step, R, nprop)
    print(f"\n{kind}: blocks whose proposal cut needed the exact bisection: {ovf} of {len(sets)}")
    ys, xs = synth_scan(H, step), synth_scan(W, step)
    b = 0
    for j in ys:
        for i in xs:
            t, bo = max(0, j - R), min(H - 8, j + R)
            l, r = max(0, i - R), min(W - 8, i + R)
            cy, cx = np.mgrid[t:bo + 1, l:r + 1]
            cy = np.append(cy.ravel(), 0)
            cx = np.append(cx.ravel(), 0)
            sc = ((d[cy, cx] - d[j, i]) ** 2).sum(axis=1)
            sc[:-1][(cy[:-1] == j) & (cx[:-1] == i)] = np.inf
            got = sets[b][sets[b] != 0xFFFFFFFF].astype(np.int64)
            assert len(got) == min(nprop, len(sc)) and len(set(got.tolist())) == len(got)
            inside = np.zeros(len(sc), bool)
            inside[got] = True
            if (~inside).any():
                assert sc[inside].max() <= sc[~inside].min() + 1e-5 * (1.0 + sc[~inside].min())
            b += 1


def synth_scan(extent, step, B=8):
    out, j, last = [], 0, extent - B
    while j < last + step:
        out.append(min(j, last))
        j += step
    return out


def list_recall(got, ref, G):
    """Mean fraction of the exhaustive list's entries (z, y, x) that the other list also holds."""
    cg, zg, yg, xg, _ = got
    cr, zr, yr, xr, _ = ref
    kg = (zg.astype(np.int64) << 32) | (yg.astype(np.int64) << 16) | xg
    kr = (zr.astype(np.int64) << 32) | (yr.astype(np.int64) << 16) | xr
    hits = 0.0
    for b in range(len(cr)):
        hits += len(set(kr[b, :cr[b]].tolist()) & set(kg[b, :cg[b]].tolist())) / cr[b]
    return hits / len(cr)


def test_learned_vbm3d_1080p_30_frames():
    """V-BM3D with learned proposals in every frame of the window (the current frame's full search
    and the other frames' predictive search): VBasic + VFinal, radius 2, 1920x1080 YUV444 float,
    30 frames, sigma 20; group recall of the VBasic lists against the exhaustive search and PSNR of
    the aggregated output against the exhaustive forms."""
    F, H, W, sigma = 30, 1080, 1920, 20.0
    nz, clean = synth.motion_frames(5, F, H, W, sigma, planes=3)
    src = source(nz.astype(np.float32), "YUV")
    clean = clean.astype(np.float64)
    out, vb = {}, {}
    for prec in ("fp32", "tf32", "learned"):
        basic = core.bm3d.VBasic(src, radius=2, sigma=sigma, precision=prec, aggregate=1, sample=1)
        final = core.bm3d.VFinal(src, basic, radius=2, sigma=sigma, precision=prec, aggregate=1, sample=1)
        out[prec] = final.numpy(10)
        v = core.bm3d.VBasic(src, radius=2, sigma=sigma, precision=prec)
        v.compute(F // 2, 1)
        vb[prec] = v.matches(0, 8)
    ps = {k: 10 * np.log10(1.0 / np.mean((v.astype(np.float64) - clean) ** 2)) for k, v in out.items()}
    rec = list_recall(vb["learned"], vb["fp32"], 8)
    rec_tc = list_recall(vb["tf32"], vb["fp32"], 8)
    print(f"\nlearned V-BM3D 1080p x{F}: PSNR fp32 {ps['fp32']:.3f}, tf32 {ps['tf32']:.3f}, learned {ps['learned']:.3f} dB "
          f"(input {10 * np.log10(1.0 / np.mean((nz - clean) ** 2)):.3f}); VBasic group recall vs exhaustive: "
          f"learned {rec:.4f}, tf32 {rec_tc:.4f}")
    assert rec_tc == 1.0
    assert rec >= 0.8
    assert ps["learned"] - ps["fp32"] >= -0.1
