"""Test infrastructure only: NumPy restatement of the learned block-matching proposal network
(the GPU code is vapoursynth-bm3d_b200/csrc/proposal.cuh) -- forward pass, logistic ranking loss
and the analytic backward pass -- used to check the GPU gradients and, by finite differences, the
backward formulas themselves.  No reference counterpart (the reference searches exhaustively).

Weight vector (2480): w1[16][9], b1[16], w2[16][16][9], b2[16]; tap k = 3 dy + dx over offsets
dy, dx in {-1, 0, 1}; zero padding.  `bf16=True` rounds the hidden layer, the features and the
descriptors to bf16 (round to nearest even) exactly where the GPU stores them.  Descriptor:
channel c of the features averaged over quadrant c % 4 (rows 4 (q // 2) .., columns 4 (q % 2) ..)
of the 8x8 block.
"""
import numpy as np

NW = 2480


def unpack(w):
    w = np.asarray(w, np.float64)
    return (w[0:144].reshape(16, 9), w[144:160], w[160:2464].reshape(16, 16, 9), w[2464:2480])


def bf16(a):
    a32 = np.ascontiguousarray(a, np.float32)
    u = a32.view(np.uint32).astype(np.uint64)
    u = (u + 0x7FFF + ((u >> 16) & 1)) & 0xFFFF0000
    return u.astype(np.uint32).view(np.float32).astype(np.float64)


def shifted(img, dy, dx):
    """out[y, x] = img[y + dy, x + dx] (zero outside)."""
    H, W = img.shape[-2:]
    out = np.zeros_like(img)
    ys, ye = max(0, -dy), min(H, H - dy)
    xs, xe = max(0, -dx), min(W, W - dx)
    out[..., ys:ye, xs:xe] = img[..., ys + dy:ye + dy, xs + dx:xe + dx]
    return out


def forward(x, w, bf=True):
    """x: [H][W] -> (hidden [16][H][W], features [16][H][W], descriptors [H-7][W-7][16])."""
    w1, b1, w2, b2 = unpack(w)
    x = np.asarray(x, np.float64)
    taps = [shifted(x, k // 3 - 1, k % 3 - 1) for k in range(9)]
    pre = np.einsum('ck,kyx->cyx', w1, np.stack(taps)) + b1[:, None, None]
    h = np.maximum(pre, 0.0)
    if bf:
        h = bf16(h)
    htaps = np.stack([shifted(h, k // 3 - 1, k % 3 - 1) for k in range(9)])      # [9][16][H][W]
    f = np.einsum('cik,kiyx->cyx', w2, htaps) + b2[:, None, None]
    if bf:
        f = bf16(f)
    H, W = x.shape
    cs = np.cumsum(np.cumsum(np.pad(f, ((0, 0), (1, 0), (1, 0))), axis=1), axis=2)
    box4 = cs[:, 4:, 4:] - cs[:, :-4, 4:] - cs[:, 4:, :-4] + cs[:, :-4, :-4]     # 4x4 sums [16][H-3][W-3]
    d = np.zeros((H - 7, W - 7, 16))
    for c in range(16):
        qy, qx = 4 * ((c % 4) // 2), 4 * (c % 2)
        d[:, :, c] = box4[c, qy:qy + H - 7, qx:qx + W - 7] / 16.0
    if bf:
        d = bf16(d)
    return h, f, d


def loss_and_grad(x, w, triplets, bf=True):
    """Mean softplus(s_ap - s_an) over triplets [T][6] (ay, ax, py, px, ny, nx) and d/dw."""
    w1, b1, w2, b2 = unpack(w)
    x = np.asarray(x, np.float64)
    h, f, d = forward(x, w, bf)
    T = len(triplets)
    gd = np.zeros_like(d)
    L = 0.0
    for ay, ax, py, px, ny, nx in triplets:
        a, p, n = d[ay, ax], d[py, px], d[ny, nx]
        z = np.sum((a - p) ** 2) - np.sum((a - n) ** 2)
        L += np.logaddexp(0.0, z) / T
        g = 1.0 / (1.0 + np.exp(-z)) / T
        gd[ay, ax] += g * (2 * (a - p) - 2 * (a - n))
        gd[py, px] += -g * 2 * (a - p)
        gd[ny, nx] += g * 2 * (a - n)
    H, W = x.shape
    gdc = np.moveaxis(gd, -1, 0)                                                 # [16][H-7][W-7]
    df = np.zeros((16, H, W))
    for c in range(16):
        qy, qx = 4 * ((c % 4) // 2), 4 * (c % 2)
        for u in range(4):
            for v in range(4):
                df[c, qy + u:qy + u + H - 7, qx + v:qx + v + W - 7] += gdc[c]
    df /= 16.0
    htaps = np.stack([shifted(h, k // 3 - 1, k % 3 - 1) for k in range(9)])
    gw2 = np.einsum('cyx,kiyx->cik', df, htaps)
    gb2 = df.sum(axis=(1, 2))
    dh = np.zeros_like(h)
    for k in range(9):
        dy, dx = k // 3 - 1, k % 3 - 1
        dh += np.einsum('ci,cyx->iyx', w2[:, :, k], shifted(df, -dy, -dx))
    dh *= (h > 0)
    taps = np.stack([shifted(x, k // 3 - 1, k % 3 - 1) for k in range(9)])
    gw1 = np.einsum('cyx,kyx->ck', dh, taps)
    gb1 = dh.sum(axis=(1, 2))
    grad = np.concatenate([gw1.ravel(), gb1, gw2.ravel(), gb2])
    return L, grad
