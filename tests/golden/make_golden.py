"""Generates tests/golden/block_matching.npz: match lists produced by the reference plugin's own
include/Block.h (compiled unmodified through oracle/ref_block_shim.cpp into
oracle/_ref/librefblock.so) on small seeded inputs.  Run here, where the reference checkout
exists:  python tests/golden/make_golden.py

Cases cover the BM3D range search (include/Block.h:683-729) with several block sizes, steps,
group sizes and tie-heavy quantised inputs (libstdc++ partial_sort tie order), and the V-BM3D
grouping (source/VBM3D_Base.cpp:540-659) restated on the reference's primitives.
"""
import os
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, os.path.join(ROOT, "oracle"))
import oracle  # noqa: E402

OUT = os.path.join(os.path.dirname(os.path.abspath(__file__)), "block_matching.npz")


def smooth_noisy(rng, h, w, sigma):
    yy, xx = np.mgrid[0:h, 0:w]
    img = 0.4 + 0.2 * np.sin(xx / 7.0) * np.cos(yy / 5.0) + 0.1 * (xx > w // 2)
    return (img + rng.normal(0, sigma / 255.0, (h, w))).astype(np.float32)


def quantised(rng, h, w, levels):
    return (np.round(rng.random((h, w)) * levels) / 255.0).astype(np.float32)


BM_CASES = [
    # name, image maker, B, step, G, R, bm_step, th_mse, matrix norm source (W, H)
    ("fast_noisy", lambda r: smooth_noisy(r, 48, 64, 10), 8, 8, 8, 9, 1, 1200.0),
    ("np_basic_noisy", lambda r: smooth_noisy(r, 53, 67, 10), 8, 4, 16, 16, 1, 1200.0),
    ("np_final_noisy", lambda r: smooth_noisy(r, 53, 67, 10), 8, 3, 32, 16, 1, 300.0),
    ("ties_np", lambda r: quantised(r, 48, 64, 3), 8, 4, 16, 16, 1, 1200.0),
    ("ties_final", lambda r: quantised(r, 40, 45, 2), 8, 3, 32, 12, 1, 1200.0),
    ("ties_step2", lambda r: quantised(r, 40, 45, 2), 8, 3, 8, 9, 2, 400.0),
    ("vn_final_b11", lambda r: smooth_noisy(r, 40, 45, 20), 11, 6, 32, 16, 1, 1200.0),
    ("b5_ties", lambda r: quantised(r, 30, 37, 2), 5, 2, 12, 7, 1, 4000.0),
    ("b16", lambda r: smooth_noisy(r, 40, 48, 10), 16, 8, 16, 8, 1, 1200.0),
    ("b8_g64", lambda r: quantised(r, 32, 40, 2), 8, 4, 64, 8, 1, 1200.0),
]

VBM_CASES = [
    # name, clip maker, B, step, G, R, bm_step, radius, ps_num, ps_range, ps_step, th_mse
    ("vbasic_fast", lambda r: np.stack([smooth_noisy(r, 40, 48, 10) for _ in range(4)]), 8, 8, 8, 7, 1, 1, 2, 4, 1, 1200.0),
    ("vfinal_ties_r2", lambda r: np.stack([quantised(r, 40, 48, 3) for _ in range(5)]), 8, 5, 16, 9, 1, 2, 3, 5, 2, 1200.0),
]


def main():
    if not oracle.ref_available():
        raise SystemExit("oracle/_ref/librefblock.so missing: build it with `make -C oracle` where the reference exists")
    data = {}
    norm = oracle.matrix_norms(6)[0]   # smpte170m, the default for these sizes
    data["normY"] = np.array(norm)
    for ci, (name, mk, B, step, G, R, bms, th) in enumerate(BM_CASES):
        rng = np.random.default_rng(1000 + ci)
        img = mk(rng)
        H, W = img.shape
        ys_, xs_ = oracle.scan(H, B, step), oracle.scan(W, B, step)
        nb = len(ys_) * len(xs_)
        cnt = np.zeros(nb, np.int32)
        ky = np.zeros((nb, G), np.float32)
        py = np.full((nb, G), -1, np.int32)
        px = np.full((nb, G), -1, np.int32)
        b = 0
        for j in ys_:
            for i in xs_:
                if G == 1:
                    k, y, x = np.zeros(1, np.float32), np.array([j]), np.array([i])
                else:
                    k, y, x = oracle.ref_bm_range(img, j, i, B, R, bms, th * norm, G)
                cnt[b] = len(k)
                ky[b, :len(k)] = k
                py[b, :len(k)] = y
                px[b, :len(k)] = x
                b += 1
        data[f"bm/{name}/img"] = img
        data[f"bm/{name}/params"] = np.array([B, step, G, R, bms], np.int32)
        data[f"bm/{name}/th_mse"] = np.array(th)
        data[f"bm/{name}/count"] = cnt
        data[f"bm/{name}/key"] = ky
        data[f"bm/{name}/y"] = py
        data[f"bm/{name}/x"] = px
    for ci, (name, mk, B, step, G, R, bms, rad, psn, psr, pss, th) in enumerate(VBM_CASES):
        rng = np.random.default_rng(2000 + ci)
        clip = mk(rng)
        F, H, W = clip.shape
        ys_, xs_ = oracle.scan(H, B, step), oracle.scan(W, B, step)
        nb = len(ys_) * len(xs_)
        cnt = np.zeros((F, nb), np.int32)
        kz = np.zeros((F, nb, G), np.float32)
        pz = np.full((F, nb, G), -1, np.int32)
        py = np.full((F, nb, G), -1, np.int32)
        px = np.full((F, nb, G), -1, np.int32)
        for n in range(F):
            boff, foff = -min(n, rad), min(F - 1 - n, rad)
            win = clip[n + boff:n + foff + 1]
            b = 0
            for j in ys_:
                for i in xs_:
                    k, z, y, x = oracle.ref_vbm3d_match(win, -boff, j, i, B, R, bms, G, psn, psr, pss, th * norm)
                    cnt[n, b] = len(k)
                    kz[n, b, :len(k)] = k
                    pz[n, b, :len(k)] = z
                    py[n, b, :len(k)] = y
                    px[n, b, :len(k)] = x
                    b += 1
        data[f"vbm/{name}/clip"] = clip
        data[f"vbm/{name}/params"] = np.array([B, step, G, R, bms, rad, psn, psr, pss], np.int32)
        data[f"vbm/{name}/th_mse"] = np.array(th)
        data[f"vbm/{name}/count"] = cnt
        data[f"vbm/{name}/key"] = kz
        data[f"vbm/{name}/z"] = pz
        data[f"vbm/{name}/y"] = py
        data[f"vbm/{name}/x"] = px
    np.savez_compressed(OUT, **data)
    print("wrote", OUT, os.path.getsize(OUT), "bytes")


if __name__ == "__main__":
    main()
