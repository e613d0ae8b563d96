"""Trains the learned block-matching proposal network on the GPU and writes its weights as
csrc/proposal_weights.h (the built-in weights of precision="learned").

Network (csrc/proposal.cuh): 3x3 conv 1 -> 16 channels, ReLU, 3x3 conv 16 -> 16; the 16-channel
feature map averaged over each 8x8 block is that block position's descriptor, and candidates are
proposed by descriptor distance.  Training data: seeded synthetic gray frames of the library's
generator (bm3d_b200/synth.py; seeds 900.. here, disjoint from the tests' and the benchmark's),
noise sigma drawn from {5, 10, 15, 25}.  Targets: the exhaustive 32-lists of the exact SSD
(block step 4, range 16).  Loss: logistic ranking loss on (reference, one of its 15 best, a later
list entry or a uniform window candidate) triplets, Adam.

    python train_proposal.py [--iters 600] [--batch 2048] [--lr 3e-3] [--seed 1] [--out PATH]
    python train_proposal.py --init-only      # untrained (He-initialised) weights, no GPU needed
"""
import argparse
import ctypes as C
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, HERE)

NW = 2480  # w1[16][9], b1[16], w2[16][16][9], b2[16]


def init_weights(seed):
    """He-normal initialisation, zero biases."""
    rng = np.random.default_rng(seed)
    w = np.zeros(NW, np.float32)
    w[0:144] = rng.normal(0.0, np.sqrt(2.0 / 9.0), 144)
    w[160:2464] = rng.normal(0.0, np.sqrt(2.0 / (16 * 9)), 2304)
    return w


def write_header(w, path, note):
    lines = ["// proposal_weights.h -- built-in weights of the learned block-matching proposal network",
             "// (layout: w1[16][9], b1[16], w2[16][16][9], b2[16]; see proposal.cuh).",
             f"// Generated by train_proposal.py: {note}",
             "#pragma once", "", f"constexpr int kProposalWeightCount = {NW};",
             "static const float kProposalWeights[kProposalWeightCount] = {"]
    vals = [f"{float(v):.9e}f" for v in w]
    for i in range(0, NW, 8):
        lines.append("    " + ", ".join(vals[i:i + 8]) + ",")
    lines.append("};")
    with open(path, "w") as f:
        f.write("\n".join(lines) + "\n")


def training_frames(n, h, w):
    from bm3d_b200 import synth
    frames = []
    for k in range(n):
        sigma = (5.0, 10.0, 15.0, 25.0)[k % 4]
        nz, _ = synth.gray_frames(900 + k, 1, h, w, sigma)
        frames.append(nz[0, 0])
    return np.ascontiguousarray(np.stack(frames), np.float32)


def train(frames, iters, batch, lr, seed, w0):
    from bm3d_b200 import _capi as capi
    L = capi.lib()
    w = np.ascontiguousarray(w0.copy(), np.float32)
    losses = np.zeros(iters, np.float32)
    n, h, wd = frames.shape
    P = C.POINTER
    rc = L.bm3d_proposal_train(frames.ctypes.data_as(P(C.c_float)), n, wd, h, iters, batch, C.c_float(lr),
                               C.c_uint64(seed), w.ctypes.data_as(P(C.c_float)), losses.ctypes.data_as(P(C.c_float)))
    if rc != 0:
        raise RuntimeError(capi.lib().bm3d_get_error().decode())
    return w, losses


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--iters", type=int, default=600)
    ap.add_argument("--batch", type=int, default=2048)
    ap.add_argument("--lr", type=float, default=3e-3)
    ap.add_argument("--seed", type=int, default=1)
    ap.add_argument("--frames", type=int, default=8)
    ap.add_argument("--size", type=int, default=192)
    ap.add_argument("--out", default=os.path.join(HERE, "csrc", "proposal_weights.h"))
    ap.add_argument("--init-only", action="store_true")
    args = ap.parse_args()
    w0 = init_weights(args.seed)
    if args.init_only:
        write_header(w0, args.out, f"untrained He initialisation, seed {args.seed}")
        return
    frames = training_frames(args.frames, args.size, args.size)
    w, losses = train(frames, args.iters, args.batch, args.lr, args.seed, w0)
    k = max(1, args.iters // 10)
    print("loss per tenth:", " ".join(f"{float(losses[i:i + k].mean()):.4f}" for i in range(0, args.iters, k)))
    write_header(w, args.out, f"--iters {args.iters} --batch {args.batch} --lr {args.lr} --seed {args.seed} "
                              f"--frames {args.frames} --size {args.size}; final mean loss "
                              f"{float(losses[-k:].mean()):.4f} (initial {float(losses[:k].mean()):.4f})")


if __name__ == "__main__":
    main()
