"""Seeded synthetic frames for the benchmarks and tests (no dataset is involved).

Clean image (values in about [0, 1]):
  * background: linear gradient of random direction between two levels drawn in [0.1, 0.9];
  * structure: 40 axis-aligned rectangles with uniform values U[0.1, 0.9], random corners,
    painted in order onto a 0.5 canvas, blended 50/50 with the gradient;
  * texture: 6 rectangular patches of sinusoids, period U[4, 16] px, amplitude 0.1, random
    orientation and phase, added.
RGB frames: each channel is sqrt(0.6) * S + sqrt(0.4) * I_c on zero-mean structure/texture fields
(S shared, I_c independent per channel), plus the shared gradient -- cross-channel correlation 0.6.
Motion clips: frame k samples a frame-0 image generated with a 6-pixel margin at a random
sub-pixel translation |v| <= 3 px (bilinear).
Noise: i.i.d. N(0, (sigma/255)^2), unclipped for float; 16-bit = clip(round(65535 x)).
Seeds: config * 1000 + frame * 10 + channel.
"""
import numpy as np


def _rng(seed):
    return np.random.Generator(np.random.PCG64(seed))


def _gradient(rng, h, w):
    theta = rng.uniform(0.0, 2.0 * np.pi)
    lo, hi = np.sort(rng.uniform(0.1, 0.9, 2))
    yy, xx = np.mgrid[0:h, 0:w].astype(np.float64)
    t = xx * np.cos(theta) + yy * np.sin(theta)
    t = (t - t.min()) / max(t.max() - t.min(), 1e-9)
    return lo + (hi - lo) * t


def _structure(rng, h, w):
    canvas = np.full((h, w), 0.5)
    for _ in range(40):
        y0, y1 = np.sort(rng.integers(0, h + 1, 2))
        x0, x1 = np.sort(rng.integers(0, w + 1, 2))
        canvas[y0:y1, x0:x1] = rng.uniform(0.1, 0.9)
    tex = np.zeros((h, w))
    yy, xx = np.mgrid[0:h, 0:w].astype(np.float64)
    for _ in range(6):
        ph, pw = int(rng.integers(max(h // 8, 8), max(h // 2, 9))), int(rng.integers(max(w // 8, 8), max(w // 2, 9)))
        y0, x0 = int(rng.integers(0, max(h - ph, 1))), int(rng.integers(0, max(w - pw, 1)))
        period = rng.uniform(4.0, 16.0)
        ang = rng.uniform(0.0, np.pi)
        phase = rng.uniform(0.0, 2.0 * np.pi)
        wave = 0.1 * np.sin(2.0 * np.pi * (xx * np.cos(ang) + yy * np.sin(ang)) / period + phase)
        tex[y0:y0 + ph, x0:x0 + pw] += wave[y0:y0 + ph, x0:x0 + pw]
    return canvas, tex


def clean_gray(h, w, seed):
    rng = _rng(seed)
    grad = _gradient(rng, h, w)
    canvas, tex = _structure(rng, h, w)
    return (0.5 * grad + 0.5 * canvas + tex).astype(np.float64)


def clean_rgb(h, w, seed, corr=0.6):
    rng = _rng(seed)
    grad = _gradient(rng, h, w)
    cs, ts = _structure(rng, h, w)
    shared = 0.5 * (cs - cs.mean()) + ts
    out = []
    for c in range(3):
        ci, ti = _structure(_rng(seed * 7 + 13 + c), h, w)
        own = 0.5 * (ci - ci.mean()) + ti
        out.append(0.5 * grad + 0.25 + np.sqrt(corr) * shared + np.sqrt(1.0 - corr) * own)
    return np.stack(out)


def _shift(img, vy, vx, margin):
    h, w = img.shape[-2] - 2 * margin, img.shape[-1] - 2 * margin
    yy, xx = np.mgrid[0:h, 0:w].astype(np.float64)
    sy, sx = yy + margin + vy, xx + margin + vx
    y0, x0 = np.floor(sy).astype(int), np.floor(sx).astype(int)
    fy, fx = sy - y0, sx - x0
    a = img[..., y0, x0]
    b = img[..., y0, x0 + 1]
    c = img[..., y0 + 1, x0]
    d = img[..., y0 + 1, x0 + 1]
    return (1 - fy) * ((1 - fx) * a + fx * b) + fy * ((1 - fx) * c + fx * d)


def noisy(clean, sigma, seed):
    rng = _rng(seed)
    return clean + rng.normal(0.0, sigma / 255.0, clean.shape)


def to_u16(x):
    return np.clip(np.round(65535.0 * x), 0, 65535).astype(np.uint16)


def gray_frames(config, nframes, h, w, sigma, first=0):
    """[nframes][1][h][w] float32 noisy frames first..first+nframes-1 of a clip, and their clean
    counterparts."""
    fr = range(first, first + nframes)
    clean = np.stack([clean_gray(h, w, config * 1000 + f * 10)[None] for f in fr])
    nz = np.stack([noisy(clean[i], sigma, config * 1000 + f * 10 + 5) for i, f in enumerate(fr)])
    return nz.astype(np.float32), clean.astype(np.float32)


def rgb_frames(config, nframes, h, w, sigma, first=0):
    """[nframes][3][h][w] float32 noisy RGB frames first..first+nframes-1 of a clip (correlated
    channels), and their clean counterparts."""
    fr = range(first, first + nframes)
    clean = np.stack([clean_rgb(h, w, config * 1000 + f * 10) for f in fr])
    nz = np.stack([np.stack([noisy(clean[i, c], sigma, config * 1000 + f * 10 + c) for c in range(3)])
                   for i, f in enumerate(fr)])
    return nz.astype(np.float32), clean.astype(np.float32)


def motion_frames(config, nframes, h, w, sigma, planes=3, max_shift=3.0):
    """[nframes][planes][h][w] float64 clean frames of a translating scene and noisy versions."""
    m = 6
    base = clean_rgb(h + 2 * m, w + 2 * m, config * 1000) if planes == 3 else clean_gray(h + 2 * m, w + 2 * m, config * 1000)[None]
    rng = _rng(config * 1000 + 999)
    clean = []
    for f in range(nframes):
        r = rng.uniform(0.0, max_shift)
        a = rng.uniform(0.0, 2.0 * np.pi)
        clean.append(_shift(base, r * np.sin(a), r * np.cos(a), m))
    clean = np.stack(clean)
    nz = np.stack([np.stack([noisy(clean[f, c], sigma, config * 1000 + f * 10 + c) for c in range(planes)])
                   for f in range(nframes)])
    return nz, clean
