"""CPU check of the learned proposal network's backward formulas (oracle/proposal_ref.py, the
restatement the GPU gradients are compared with): central finite differences of the float64
forward pass against the analytic gradient."""
import numpy as np

import proposal_ref as pr


def test_backward_matches_finite_differences():
    rng = np.random.default_rng(5)
    x = rng.random((20, 22))
    w = rng.normal(0.0, 0.4, pr.NW)
    trip = []
    for _ in range(12):
        ay, ax, py, px, ny, nx = (int(v) for v in rng.integers(0, 13, 6))
        trip.append((ay, ax, py, px, ny, nx))
    L, g = pr.loss_and_grad(x, w, trip, bf=False)
    idx = np.concatenate([rng.choice(160, 20, replace=False), 160 + rng.choice(2320, 30, replace=False)])
    eps = 1e-6
    for i in idx:
        wp, wm = w.copy(), w.copy()
        wp[i] += eps
        wm[i] -= eps
        num = (pr.loss_and_grad(x, wp, trip, bf=False)[0] - pr.loss_and_grad(x, wm, trip, bf=False)[0]) / (2 * eps)
        assert abs(num - g[i]) <= 1e-6 + 1e-5 * abs(num), (i, num, g[i])


def test_bf16_rounding_is_nearest_even():
    v = np.array([1.0, 1.0 + 2 ** -8, 1.0 + 3 * 2 ** -8, -2.5, 0.0], np.float32)
    r = pr.bf16(v)
    assert r[0] == 1.0 and r[1] == 1.0 and r[2] == 1.0 + 2 ** -6 and r[3] == -2.5 and r[4] == 0.0
