"""CPU tests of the oracle: pinned to the reference's own Block.h (committed golden vectors and,
where the reference checkout exists, a live build), the DCT checked against its definition."""
import math

import numpy as np
import pytest

BM_NAMES = ["fast_noisy", "np_basic_noisy", "np_final_noisy", "ties_np", "ties_final", "ties_step2",
            "vn_final_b11", "b5_ties", "b16", "b8_g64"]
VBM_NAMES = ["vbasic_fast", "vfinal_ties_r2"]


def oracle_params_bm(orc, golden, name):
    B, step, G, R, bms = [int(v) for v in golden[f"bm/{name}/params"]]
    th = float(golden[f"bm/{name}/th_mse"])
    return orc.default_params(0, False, "np", 10.0, matrix=6, block_size=B, block_step=step, group_size=G,
                              bm_range=R, bm_step=bms, th_mse=th)


@pytest.mark.parametrize("name", BM_NAMES)
def test_block_matching_matches_reference_golden(orc, golden, name):
    p = oracle_params_bm(orc, golden, name)
    img = golden[f"bm/{name}/img"]
    cnt, ys, xs, ks = orc.bm3d_matches(p, img)
    exp_cnt = golden[f"bm/{name}/count"]
    assert np.array_equal(cnt, exp_cnt)
    for b in range(len(cnt)):
        n = cnt[b]
        assert np.array_equal(ys[b, :n], golden[f"bm/{name}/y"][b, :n])
        assert np.array_equal(xs[b, :n], golden[f"bm/{name}/x"][b, :n])
        assert np.array_equal(ks[b, :n].view(np.int32), golden[f"bm/{name}/key"][b, :n].view(np.int32))


def test_golden_has_ties_and_duplicate_origin(golden):
    # the tie-heavy cases really exercise equal keys inside the kept lists, and the reference's
    # trailing (0, 0) candidate appears in lists of blocks that are not at (0, 0)
    k = golden["bm/ties_np/key"]
    c = golden["bm/ties_np/count"]
    ties = sum(len(np.unique(k[b, 1:c[b]])) < c[b] - 1 for b in range(len(c)))
    assert ties > 10
    y, x = golden["bm/ties_np/y"], golden["bm/ties_np/x"]
    origin = sum(((y[b, 1:c[b]] == 0) & (x[b, 1:c[b]] == 0)).sum() for b in range(len(c)))
    assert origin > 0


@pytest.mark.parametrize("name", VBM_NAMES)
def test_vbm3d_grouping_matches_reference_golden(orc, golden, name):
    B, step, G, R, bms, rad, psn, psr, pss = [int(v) for v in golden[f"vbm/{name}/params"]]
    th = float(golden[f"vbm/{name}/th_mse"])
    p = orc.default_params(0, True, "np", 10.0, matrix=6, block_size=B, block_step=step, group_size=G,
                           bm_range=R, bm_step=bms, th_mse=th, radius=rad, ps_num=psn, ps_range=psr, ps_step=pss)
    clip = golden[f"vbm/{name}/clip"]
    for n in range(clip.shape[0]):
        cnt, zs, ys, xs, ks = orc.vbm3d_matches(p, clip, n)
        assert np.array_equal(cnt, golden[f"vbm/{name}/count"][n])
        for b in range(len(cnt)):
            m = cnt[b]
            assert np.array_equal(zs[b, :m], golden[f"vbm/{name}/z"][n, b, :m])
            assert np.array_equal(ys[b, :m], golden[f"vbm/{name}/y"][n, b, :m])
            assert np.array_equal(xs[b, :m], golden[f"vbm/{name}/x"][n, b, :m])
            assert np.array_equal(ks[b, :m].view(np.int32), golden[f"vbm/{name}/key"][n, b, :m].view(np.int32))


def test_block_matching_matches_live_reference(orc):
    if not orc.ref_available():
        pytest.skip("reference Block.h not built here (oracle/_ref)")
    rng = np.random.default_rng(7)
    norm = orc.matrix_norms(6)[0]
    for trial in range(6):
        H, W = int(rng.integers(20, 50)), int(rng.integers(20, 50))
        B = int(rng.choice([3, 4, 8, 9, 12]))
        if B > min(H, W):
            continue
        step = int(rng.integers(1, B + 1))
        G = int(rng.choice([2, 5, 8, 16, 31, 33]))
        R = int(rng.integers(2, 12))
        bms = int(rng.integers(1, 3))
        img = (np.round(rng.random((H, W)) * rng.integers(1, 5)) / 255.0).astype(np.float32)
        th = 2000.0
        p = orc.default_params(0, False, "np", 10.0, matrix=6, block_size=B, block_step=step, group_size=G,
                               bm_range=R, bm_step=bms, th_mse=th)
        cnt, ys, xs, ks = orc.bm3d_matches(p, img)
        b = 0
        for j in orc.scan(H, B, step):
            for i in orc.scan(W, B, step):
                k, y, x = orc.ref_bm_range(img, j, i, B, R, bms, th * norm, G)
                assert cnt[b] == len(k)
                assert np.array_equal(ys[b, :len(k)], y) and np.array_equal(xs[b, :len(k)], x)
                assert np.array_equal(ks[b, :len(k)].view(np.int32), k.view(np.int32))
                b += 1


def dct_definition(x, inverse):
    """FFTW REDFT10 / REDFT01 along every axis of a [n][B][B] array, in float64."""
    y = x.astype(np.float64)
    for axis in range(3):
        N = y.shape[axis]
        j = np.arange(N)
        if not inverse:
            M = 2.0 * np.cos(np.pi * np.outer(j, 2 * j + 1) / (2 * N))           # [k][j]
        else:
            M = 2.0 * np.cos(np.pi * np.outer(2 * j + 1, j) / (2 * N))           # [k][j]
            M[:, 0] = 1.0
        y = np.moveaxis(np.tensordot(M, np.moveaxis(y, axis, 0), axes=(1, 0)), 0, axis)
    return y


@pytest.mark.parametrize("n,B", [(1, 8), (2, 8), (3, 8), (5, 8), (8, 8), (16, 8), (32, 8), (12, 11), (7, 5), (4, 16)])
def test_dct_against_definition(orc, n, B):
    rng = np.random.default_rng(n * 100 + B)
    g = rng.normal(0, 1, (2, n, B, B)).astype(np.float32)
    for inverse in (False, True):
        got = orc.dct3d(g, inverse)
        exp = np.stack([dct_definition(g[k], inverse) for k in range(2)])
        scale = np.abs(exp).max()
        assert np.abs(got - exp).max() <= 2e-6 * scale * math.sqrt(n * B * B)


@pytest.mark.parametrize("n,B", [(1, 8), (5, 8), (16, 8), (32, 8), (7, 11), (4, 5), (3, 16), (256, 2)])
def test_vector_dct_equals_scalar_dct(orc, n, B):
    # the lane-parallel transform performs the scalar operation sequence bit for bit
    rng = np.random.default_rng(n + 7 * B)
    g = rng.normal(0, 1, (3, n, B, B)).astype(np.float32)
    for inverse in (False, True):
        a = orc.dct3d(g, inverse)
        b = orc.dct3d(g, inverse, scalar=True)
        assert np.array_equal(a.view(np.int32), b.view(np.int32))


def test_dct_round_trip_amplification(orc):
    # inverse(forward(x)) = 2n * 2B * 2B * x (finalAMP of source/BM3D.cpp:155)
    rng = np.random.default_rng(3)
    for n, B in [(16, 8), (9, 8), (32, 8)]:
        g = rng.normal(0, 1, (1, n, B, B)).astype(np.float32)
        rt = orc.dct3d(orc.dct3d(g, False), True)
        amp = 2 * n * 2 * B * 2 * B
        assert np.allclose(rt / amp, g, atol=1e-5)


def test_profile_defaults(orc):
    # README.md profile tables (bm3d.Basic / bm3d.Final / bm3d.VBasic / bm3d.VFinal)
    table = {  # profile: (B, step, G, R) for Basic, Final, VBasic, VFinal
        "fast": [(8, 8, 8, 9), (8, 7, 8, 9), (8, 8, 8, 7), (8, 7, 8, 7)],
        "lc": [(8, 6, 16, 9), (8, 5, 16, 9), (8, 6, 8, 9), (8, 5, 8, 9)],
        "np": [(8, 4, 16, 16), (8, 3, 32, 16), (8, 4, 8, 12), (8, 3, 8, 12)],
        "high": [(8, 3, 16, 16), (8, 2, 32, 16), (8, 3, 8, 16), (8, 2, 8, 16)],
        "vn": [(8, 4, 32, 16), (11, 6, 32, 16), (8, 4, 16, 12), (11, 6, 16, 12)],
    }
    vtable = {"fast": (1, 2, 4, 5), "lc": (2, 2, 4, 5), "np": (3, 2, 5, 6), "high": (4, 2, 7, 8), "vn": (4, 2, 5, 6)}
    for prof, rows in table.items():
        for idx, (wiener, v) in enumerate([(0, False), (1, False), (0, True), (1, True)]):
            p = orc.default_params(wiener, v, prof, 10.0, matrix=100)
            assert (p.B, p.step, p.G, p.R) == rows[idx], (prof, idx)
            assert p.bmstep == 1
            if v:
                r, psn, psr_b, psr_f = vtable[prof]
                assert (p.radius, p.psnum, p.psrange, p.psstep) == (r, psn, psr_f if wiener else psr_b, 1)
        # th_mse defaults: sigma*80+400 / sigma*10+200, vn sigma*150+1000 / sigma*40+400; hard_thr 2.7 (vn 2.8)
        b = orc.default_params(0, False, prof, 10.0, matrix=100)
        f = orc.default_params(1, False, prof, 10.0, matrix=100)
        assert b.th_mse == (2500.0 if prof == "vn" else 1200.0)
        assert f.th_mse == (800.0 if prof == "vn" else 300.0)
        assert b.lambda_ == (2.8 if prof == "vn" else 2.7)


def test_matrix_norms(orc):
    y, u, v = orc.matrix_norms(100)
    assert abs(y - 0.57735) < 1e-5 and abs(u - 0.70711) < 1e-5 and abs(v - 0.61237) < 1e-5
    assert abs(orc.matrix_norms(6)[0] - 0.66856) < 1e-5
    assert abs(orc.matrix_norms(1)[0] - 0.74961) < 1e-5
    assert abs(orc.matrix_norms(9)[0] - 0.72953) < 1e-5


def test_integer_conversions_round_trip(orc):
    rng = np.random.default_rng(1)
    for bits in (8, 10, 16):
        plane = rng.integers(0, 1 << bits, (17, 23)).astype(np.uint8 if bits == 8 else np.uint16)
        for chroma in (False, True):
            f = orc.int2float(plane, bits, True, chroma)
            back = orc.float2int(f, bits, True, chroma)
            assert np.array_equal(back, plane)
