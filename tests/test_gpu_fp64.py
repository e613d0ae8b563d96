"""FP64 GPU oracle: per-stage error of the plain FP32 path and of the tf32 precision form.

bm3d_debug_reference_fp64 recomputes a Basic or Final frame in double precision on the GPU from
the filter's own match lists (transforms, shrinkage, aggregation, normalisation).  Stages checked:
  * transform: the FP32 register DCT of the plain path against a float64 evaluation of the
    REDFT10 definition (relative to the coefficient scale);
  * output: plain FP32 and tf32 outputs against the FP64 recomputation.
The bars are loose ceilings; the measured figures are printed (pytest -s) and kept in the design
notes.
"""
import numpy as np
import pytest

import bm3d_b200
from bm3d_b200 import core, source, synth

pytestmark = pytest.mark.gpu


def dct1_f64(x, axis):
    n = x.shape[axis]
    k = np.arange(n)[:, None]
    j = np.arange(n)[None, :]
    m = 2.0 * np.cos(np.pi * (2 * j + 1) * k / (2.0 * n))
    return np.moveaxis(np.tensordot(m, np.moveaxis(x, axis, 0), axes=(1, 0)), 0, axis)


def test_transform_stage_error():
    rng = np.random.default_rng(7)
    g = rng.uniform(0, 1, (256, 32, 8, 8)).astype(np.float32)
    got = bm3d_b200.dct3d(g, inverse=False, fast=True).astype(np.float64)
    ref = dct1_f64(dct1_f64(dct1_f64(g.astype(np.float64), 3), 2), 1)
    scale = np.abs(ref).max()
    err = np.abs(got - ref) / scale
    print(f"transform (FP32 register DCT, n=32): max rel {err.max():.2e}, rms rel {np.sqrt(np.mean(err ** 2)):.2e}")
    assert err.max() < 1e-5


@pytest.mark.parametrize("profile,sigma", [("np", 10.0), ("fast", 25.0)])
def test_output_stage_error(profile, sigma):
    nz, clean = synth.gray_frames(61, 1, 96, 128, sigma)
    clip = source(nz, "GRAY")
    for prec in ("fp32", "tf32"):
        basic = core.bm3d.Basic(clip, profile=profile, sigma=sigma, precision=prec)
        b = basic.get_frames(0, 1)[0].numpy()[0].astype(np.float64)
        rb = basic.reference_fp64(0)[0]
        final = core.bm3d.Final(clip, basic, profile=profile, sigma=sigma, precision=prec)
        f = final.get_frames(0, 1)[0].numpy()[0].astype(np.float64)
        rf = final.reference_fp64(0)[0]
        for name, out, ref in (("basic", b, rb), ("final", f, rf)):
            d = out - ref
            rms, mx = float(np.sqrt(np.mean(d * d))), float(np.abs(d).max())
            print(f"{profile} {prec} {name} vs FP64: rms {rms:.2e}, max {mx:.2e}")
            assert np.isfinite(ref).all()
            assert rms < 0.05 * sigma / 255.0
            assert mx < sigma / 255.0
