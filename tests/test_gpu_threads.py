"""Two host threads, each with its own filter instances (own stream), request disjoint frame ranges
concurrently, as a frame server's worker threads do; the frames must equal those of one call over
the whole clip (up to the order of the float atomics in the aggregation)."""
import threading

import numpy as np
import pytest

from bm3d_b200 import core, source, synth

pytestmark = pytest.mark.gpu


def _run_threads(make, ranges):
    outs, errors = {}, []

    def worker(lo, cnt):
        try:
            node = make()
            outs[lo] = np.stack([f.numpy() for f in node.compute(lo, cnt)])
        except Exception as e:  # noqa: BLE001 -- re-raised on the main thread
            errors.append(e)

    ts = [threading.Thread(target=worker, args=r) for r in ranges]
    for t in ts:
        t.start()
    for t in ts:
        t.join()
    if errors:
        raise errors[0]
    return np.concatenate([outs[lo] for lo, _ in ranges])


@pytest.mark.parametrize("precision", ["fp32", "tf32"])
def test_basic_final_two_threads(precision):
    nz, _ = synth.gray_frames(7, 4, 240, 320, 10.0)
    clip = source(nz, "GRAY")
    kw = dict(profile="np", sigma=10.0, precision=precision)
    whole_b = core.bm3d.Basic(clip, **kw).numpy()
    split_b = _run_threads(lambda: core.bm3d.Basic(clip, **kw), [(0, 2), (2, 2)])
    assert np.abs(split_b - whole_b).max() <= 1e-5
    # Final against a fixed reference clip: with the Basic estimate recomputed, its last bits
    # (float atomics in any order) can change near-equal matching distances, hence lists, hence
    # the Final output by up to ~1e-3 from run to run, threads or not
    ref = source(np.ascontiguousarray(whole_b[:, 0]), "GRAY")
    whole_f = core.bm3d.Final(clip, ref, **kw).numpy()
    split_f = _run_threads(lambda: core.bm3d.Final(clip, ref, **kw), [(0, 2), (2, 2)])
    assert split_f.shape == whole_f.shape
    assert np.abs(split_f - whole_f).max() <= 1e-5


def test_vbasic_two_threads():
    nz, _ = synth.gray_frames(9, 6, 160, 224, 15.0)
    clip = source(nz, "GRAY")

    def make():
        return core.bm3d.VAggregate(core.bm3d.VBasic(clip, sigma=15.0, radius=1), radius=1)

    whole = make().numpy()
    split = _run_threads(make, [(0, 3), (3, 3)])
    # 16-bit output: the float sums before the rounding differ in their last bits at most
    assert np.abs(split.astype(np.int64) - whole.astype(np.int64)).max() <= 1
