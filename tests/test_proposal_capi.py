"""CPU checks of the learned-proposal entry points' host logic (no GPU needed): the built-in
weights are the trained ones in their documented layout, and bad arguments fail with an error
code and a message before any device work."""
import ctypes as C

import numpy as np

from bm3d_b200 import _capi as capi

P = C.POINTER


def fptr(a):
    return a.ctypes.data_as(P(C.c_float))


def iptr(a):
    return a.ctypes.data_as(P(C.c_int))


def test_default_weights_layout():
    L = capi.lib()
    w = np.zeros(2480, np.float32)
    assert L.bm3d_proposal_default_weights(fptr(w), 2480) == 2480
    assert np.isfinite(w).all()
    w1, b1, w2, b2 = w[:144], w[144:160], w[160:2464], w[2464:]
    assert np.abs(w1).max() > 0 and np.abs(w2).max() > 0
    # trained, not the zero-bias He initialisation
    assert np.abs(b1).max() > 0 or np.abs(b2).max() > 0
    small = np.zeros(100, np.float32)
    assert L.bm3d_proposal_default_weights(fptr(small), 100) != 0
    assert "too small" in capi.last_error()


def test_bad_arguments_are_rejected():
    L = capi.lib()
    x = np.zeros((16, 16), np.float32)
    w = np.zeros(2480, np.float32)
    cnt = np.zeros(64, np.int32)
    ys = np.zeros(64 * 16, np.int32)
    xs = np.zeros(64 * 16, np.int32)
    # nprop beyond the kernel's 128, group size beyond 32, a plane smaller than a block
    assert L.bm3d_proposal_match(fptr(x), 16, 16, fptr(w), 4, 16, 4, C.c_float(1.0), 129, iptr(cnt), iptr(ys), iptr(xs), 64) != 0
    assert L.bm3d_proposal_match(fptr(x), 16, 16, fptr(w), 4, 33, 4, C.c_float(1.0), 32, iptr(cnt), iptr(ys), iptr(xs), 64) != 0
    assert L.bm3d_proposal_match(fptr(x), 4, 4, fptr(w), 4, 16, 4, C.c_float(1.0), 32, iptr(cnt), iptr(ys), iptr(xs), 64) != 0
    loss = np.zeros(1, np.float32)
    g = np.zeros(2480, np.float32)
    t = np.zeros(6, np.int32)
    assert L.bm3d_proposal_gradients(fptr(x), 16, 16, fptr(w), iptr(t), 0, fptr(loss), fptr(g)) != 0
    assert L.bm3d_proposal_train(fptr(x), 1, 16, 16, 1, 1, C.c_float(1e-3), C.c_uint64(1), fptr(w), fptr(loss)) != 0
    assert capi.last_error()
