#!/usr/bin/env python
"""bench.py -- 1080p Basic+Final Mpix/s of the plain FP32 path on B200.

Workload (one step): 8 synthetic RGB float32 1920x1080 frames per GPU through
    RGB2OPP(sample=1) -> Basic(profile='np', matrix=100) -> Final(ref=basic, profile='np',
    matrix=100) -> OPP2RGB(sample=1), sigma 10,
the full-pipeline configuration of the reference plugin's benchmark (8 frames, 1080p RGB).
Four forms run: the plain FP32 path (precision="fp32", the oracle-exact drop-in), the precision
form (precision="tf32": tensor-core transforms, tensor-core matching estimates with exact
re-rank), the same with Basic at precision="tf32_match" ("tf32_final": Basic's matching on the
tensor cores but its hard-threshold filter on the plain transform, the Final filter on the tensor
cores) and the learned-proposal form
(precision="learned": as tf32, but matching re-ranks only the proposals of the learned descriptor
network).  `value` is the fastest of the tensor-core forms whose output PSNR against the clean
frames stays within 0.05 dB of the plain path's (else the plain path's); `forms` gives all four.  `value` times the device-resident pipeline (frames
already in HBM); `e2e` times the same calls with pinned host frames (host->device and
device->host copies inside the timed region), made as a frame server makes them: four host threads,
each with its own filter instances and stream, request a quarter of the frames each, so that one
quarter's copies overlap the other quarters' kernels.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

Multi-GPU: one process per GPU (torchrun), each rank processes its own 8 frames (frame sharding,
no collective on the data path; weak scaling); barrier + max over ranks of the device time.
--impl reference times the CPU oracle (the reference's path restated in C++; the reference plugin
itself needs FFTW and VapourSynth, absent here) on the host cores.
"""
import argparse
import ctypes as C
import json
import os
import statistics
import subprocess
import sys
import threading
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(ROOT, "vapoursynth-bm3d_b200"))

W, H, NFR, SIGMA = 1920, 1080, 8, 10.0
METRIC = "1080p Basic+Final Mpix/s: plain FP32 vs TC+learned-BM form at ≤0.05 dB PSNR loss"
WORKLOAD = "RGB float32 1920x1080 x8 frames/GPU: RGB2OPP(sample=1) -> Basic(np, matrix=100) -> Final(np, matrix=100, ref=basic) -> OPP2RGB(sample=1), sigma 10"


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--frames", type=int, default=NFR)
    ap.add_argument("--width", type=int, default=W)
    ap.add_argument("--height", type=int, default=H)
    ap.add_argument("--workload", default="bm3d", choices=["bm3d", "vbm3d"],
                    help="bm3d: the headline Basic+Final pipeline; vbm3d: the V-BM3D pipeline of YUV444 16-bit "
                         "clips (VBasic -> VAggregate -> VFinal -> VAggregate), stacked and aggregated forms")
    return ap.parse_args()


def dist_env():
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return rank, world, local


# ---- CPU side (oracle) ---------------------------------------------------------------------------

def cpu_sample(threads, frames, width, rows):
    """Times the CPU oracle on `threads` frames cropped to `rows` rows (one frame per thread, as
    VapourSynth's fmParallel does).  Returns (Mpix/s, seconds, sample description)."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import numpy as np
    import oracle
    from bm3d_b200 import synth
    nz, _ = synth.rgb_frames(1, frames, rows, width, SIGMA)
    t0 = time.perf_counter()
    opp = np.stack([oracle.rgb2opp(nz[k]) for k in range(frames)])
    pb = oracle.default_params(0, False, "np", SIGMA, matrix=100)
    basic = oracle.bm3d(pb, opp, threads=threads)
    pf = oracle.default_params(1, False, "np", SIGMA, matrix=100)
    final = oracle.bm3d(pf, opp, basic, threads=threads)
    _ = [oracle.opp2rgb(final[k]) for k in range(frames)]
    dt = time.perf_counter() - t0
    mpix = frames * width * rows / dt / 1e6
    return mpix, dt, f"{frames} frame crops of {width}x{rows} (rows 0..{rows - 1} of the config frames), one per thread"


def workload_config(frames, width, height, world):
    """The workload as both arms report it (the form that produced the number is a separate key)."""
    mb = frames * width * height * 3 * 4 / 1e6
    l2 = (f"inputs larger than L2 ({mb:.0f} MB of input frames, ~{10 * mb / 1e3:.0f} GB working set per step)"
          if mb > 126 else f"inputs smaller than L2 ({mb:.0f} MB of input frames): a short run, not the headline size")
    return {"workload": WORKLOAD, "frames_per_gpu": frames, "width": width, "height": height,
            "parallelism": f"frame-sharded replicas x{world}", "l2": l2}


def reference_arm(args):
    rank, world, _ = dist_env()
    if rank != 0:
        return
    threads = min(os.cpu_count() or 1, args.frames)
    rows = 136
    vals = []
    for i in range(args.warmup + args.steps):
        mpix, dt, sample = cpu_sample(threads, threads, args.width, rows)
        if i >= args.warmup:
            vals.append((mpix, dt))
    value = statistics.median(v[0] for v in vals)
    ms = statistics.median(v[1] for v in vals) * 1e3
    line = {
        "impl": "reference", "metric": METRIC, "value": round(value, 4), "unit": "Mpix/s", "n_gpus": args.gpus,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": round(ms, 2), "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
        "config": workload_config(args.frames, args.width, args.height, world),
        "cpu_baseline": {"value": round(value, 4), "unit": "Mpix/s", "cores": threads, "kind": "port",
                         "sample": sample + "; CPU oracle (bm3d_oracle.cpp) restating the reference's path, "
                                            "FFTW replaced by a separable FP32 DCT"},
        "e2e": {"value": round(value, 4), "unit": "Mpix/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


# ---- GPU side ----------------------------------------------------------------------------------

class Clocks:
    """Samples nvidia-smi during the timed region."""

    FIELDS = "index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap"

    def __init__(self, gpu):
        self.gpu = gpu
        self.rows = []
        self.proc = None

    def start(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.gpu), "--query-gpu=" + self.FIELDS,
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except Exception:
            self.proc = None

    def _read(self):
        for line in self.proc.stdout:
            self.rows.append([c.strip() for c in line.split(",")])

    def stop(self):
        if not self.proc:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        rows = [r for r in self.rows if len(r) >= 9]
        sm = [float(r[1]) for r in rows if r[1].replace(".", "").isdigit()]
        mx = [float(r[2]) for r in rows if r[2].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[i] for r in rows for i in range(4) if r[5 + i].lower() == "active"})
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": reasons, "samples": len(rows)}


def fp32_peak_tflops(torch):
    """Measured FP32 (no TF32) cuBLAS SGEMM throughput on this GPU: the SIMT FP32 ceiling."""
    torch.backends.cuda.matmul.allow_tf32 = False
    n = 8192
    a = torch.randn(n, n, device="cuda", dtype=torch.float32)
    b = torch.randn(n, n, device="cuda", dtype=torch.float32)
    for _ in range(2):
        torch.matmul(a, b)
    torch.cuda.synchronize()
    best = 0.0
    for _ in range(5):
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        torch.matmul(a, b)
        e1.record()
        torch.cuda.synchronize()
        best = max(best, 2.0 * n ** 3 / (e0.elapsed_time(e1) * 1e-3) / 1e12)
    del a, b
    return best


def scan(extent, B, step):
    out, j, last = [], 0, extent - B
    while True:
        if j >= last + step:
            break
        if j > last:
            j = last
        out.append(j)
        j += step
    return out


def lattice_count(pos, lim, rng):
    lo = max(0, pos - rng)
    hi = min(lim, pos + rng)
    return hi - lo + 1


def algorithmic_work(width, height, frames, step, G, n_mean, wiener):
    """Algorithmic FLOPs of one call: BM = 3*B^2 per evaluated candidate (sub, mul,
    add per pixel); DCT = dense separable count 2*(n*2B^3 + B^2*n^2) per transform, 2 transforms
    (Basic) or 3 (Final) per group and plane, 3 planes."""
    B, R = 8, 16
    ys, xs = scan(height, B, step), scan(width, B, step)
    cy = sum(lattice_count(y, height - B, R) for y in ys)
    cx = sum(lattice_count(x, width - B, R) for x in xs)
    cands = cy * cx                     # lattice minus self plus the trailing (0,0) candidate
    bm = 3.0 * B * B * cands * frames
    ng = len(ys) * len(xs) * frames
    n = n_mean
    dct = 2.0 * (n * 2 * B ** 3 + B * B * n * n) * (3 if wiener else 2) * 3 * ng
    return bm, dct, ng


class Stage:
    def __init__(self, L, name, args, inputs):
        from bm3d_b200 import _capi as capi
        m = L.bm3d_map_create()
        for k, v in args.items():
            if isinstance(v, capi.VideoInfo):
                L.bm3d_map_set_clip(m, k.encode(), C.byref(v))
            elif isinstance(v, str):
                L.bm3d_map_set_data(m, k.encode(), v.encode())
            elif isinstance(v, float):
                L.bm3d_map_set_float(m, k.encode(), v)
            else:
                L.bm3d_map_set_int(m, k.encode(), v)
        self.h = C.c_void_p()
        rc = L.bm3d_create(name.encode(), m, C.byref(self.h))
        L.bm3d_map_free(m)
        if rc:
            raise RuntimeError(capi.last_error())
        self.info = capi.VideoInfo()
        L.bm3d_output_info(self.h, C.byref(self.info))


def make_frames(capi, planes, memory):
    PF = C.POINTER(capi.Frame)
    structs = []
    for pl in planes:
        fr = capi.Frame()
        for p, a in enumerate(pl):
            if memory == capi.MEM_DEVICE:
                fr.data[p] = a.data_ptr()
                fr.stride[p] = a.stride(0) * a.element_size()
            else:
                fr.data[p] = a.data_ptr()
                fr.stride[p] = a.stride(0) * a.element_size()
        fr.memory = memory
        fr.prop_bm3d_opp = fr.prop_range = fr.prop_matrix = fr.prop_v_radius = -1
        fr.prop_v_process_count = -1
        structs.append(fr)
    arr = (PF * len(structs))(*[C.pointer(s) for s in structs])
    return structs, arr


class Pipeline:
    """RGB2OPP -> Basic -> Final -> OPP2RGB on one stream; `precision` is the argument of Basic
    and Final, or a pair (Basic's, Final's)."""

    def __init__(self, L, capi, vi, stream, precision):
        pb, pf = precision if isinstance(precision, tuple) else (precision, precision)
        common = {"profile": "np", "matrix": 100, "sigma": SIGMA}
        self.opp = Stage(L, "RGB2OPP", {"input": vi, "sample": 1}, None)
        self.basic = Stage(L, "Basic", dict(common, input=self.opp.info, precision=pb), None)
        self.final = Stage(L, "Final", dict(common, input=self.opp.info, ref=self.basic.info, precision=pf), None)
        self.rgb = Stage(L, "OPP2RGB", {"input": self.final.info, "sample": 1}, None)
        for st in (self.opp, self.basic, self.final, self.rgb):
            L.bm3d_set_stream(st.h, C.c_void_p(stream.cuda_stream))
        self.L, self.capi = L, capi

    def run(self, F, a_in, a_opp, a_basic, a_final, a_out, n=0):
        """Output frames [n, n + F); the arrays hold those F frames."""
        for (st, src, ref, dst) in ((self.opp, a_in, None, a_opp), (self.basic, a_opp, None, a_basic),
                                    (self.final, a_opp, a_basic, a_final), (self.rgb, a_final, None, a_out)):
            if self.L.bm3d_get_frames_async(st.h, n, F, src, ref, dst) != 0:
                raise RuntimeError(self.capi.last_error())


def ours_arm(args):
    import numpy as np
    import torch
    from bm3d_b200 import _capi as capi
    from bm3d_b200 import shard, synth

    rank, world, local = dist_env()
    torch.cuda.set_device(local)
    dist = None
    if world > 1:
        import datetime
        import torch.distributed as tdist
        tdist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300))
        dist = tdist

    L = capi.lib()
    F, Wd, Hd = args.frames, args.width, args.height
    # frame sharding: the clip has F frames per rank; this rank filters its contiguous range
    first, count = shard.frame_range(F * world, rank, world)
    nz, clean = synth.rgb_frames(1, count, Hd, Wd, SIGMA, first=first)
    rgb_in = torch.from_numpy(nz).cuda()
    stream = torch.cuda.Stream()
    vi = capi.VideoInfo(capi.RGB, capi.FLOAT, 32, 0, 0, Wd, Hd, F)
    # forms: the plain drop-in; tensor cores in both filters; the hard-threshold filter in FP32
    # (exact decisions, and faster than its tensor-core version) after tensor-core matching, with
    # the tensor-core Final; and the learned proposals
    precisions = {"fp32": "fp32", "tf32": "tf32", "tf32_final": ("tf32_match", "tf32"), "learned": "learned"}
    pipes = {form: Pipeline(L, capi, vi, stream, pr) for form, pr in precisions.items()}

    def planes(n):
        return [[torch.empty((Hd, Wd), dtype=torch.float32, device="cuda") for _ in range(3)] for _ in range(n)]

    f_in = [[rgb_in[k, p] for p in range(3)] for k in range(F)]
    f_opp, f_basic, f_final, f_out = planes(F), planes(F), planes(F), planes(F)
    D = capi.MEM_DEVICE
    _, a_in = make_frames(capi, f_in, D)
    _, a_opp = make_frames(capi, f_opp, D)
    _, a_basic = make_frames(capi, f_basic, D)
    _, a_final = make_frames(capi, f_final, D)
    _, a_out = make_frames(capi, f_out, D)
    # host (pinned) frames for the end-to-end measurement
    h_in = torch.from_numpy(nz).pin_memory()
    h_out = torch.empty_like(h_in).pin_memory()
    H_ = capi.MEM_HOST
    # end to end as a frame server runs it: four host threads, each with its own filter instances on
    # its own stream, request a quarter of the frames each, so that one quarter's copies overlap the
    # other quarters' kernels (the calls with host frames block until their results are on the host)
    nparts = max(1, min(4, F))
    bounds = [F * i // nparts for i in range(nparts + 1)]
    halves = []
    for lo, hi in zip(bounds[:-1], bounds[1:]):
        arrs = tuple(make_frames(capi, fr[lo:hi], kind)[1] for fr, kind in (
            ([[h_in[k, p] for p in range(3)] for k in range(F)], H_), (f_opp, D), (f_basic, D), (f_final, D),
            ([[h_out[k, p] for p in range(3)] for k in range(F)], H_)))
        halves.append((lo, hi - lo, arrs))
    streams2 = [torch.cuda.Stream() for _ in range(len(halves) - 1)]
    pipes2 = {}

    def barrier():
        if dist:
            dist.barrier()
        torch.cuda.synchronize()

    def timed(pipe, steps, warmup, profile=False):
        fn = lambda: pipe.run(F, a_in, a_opp, a_basic, a_final, a_out)  # noqa: E731
        for _ in range(warmup):
            fn()
        torch.cuda.synchronize()
        if profile:
            for st in (pipe.basic, pipe.final):
                L.bm3d_set_profiling(st.h, 1)
        stage = {"basic": [0.0] * 6, "final": [0.0] * 6}
        barrier()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        total = 0.0
        launches0 = L.bm3d_debug_launch_count()
        for _ in range(steps):
            with torch.cuda.stream(stream):
                e0.record(stream)
            fn()
            with torch.cuda.stream(stream):
                e1.record(stream)
            e1.synchronize()
            total += e0.elapsed_time(e1)
            if profile:
                buf = (C.c_double * 6)()
                for name, st in (("basic", pipe.basic), ("final", pipe.final)):
                    if L.bm3d_debug_stage_times(st.h, buf, 6) == 6:
                        for i in range(6):
                            stage[name][i] += buf[i]
        launches = L.bm3d_debug_launch_count() - launches0
        barrier()
        if profile:
            for st in (pipe.basic, pipe.final):
                L.bm3d_set_profiling(st.h, 0)
        ms = total / steps
        if dist:
            t = torch.tensor([ms], device="cuda")
            dist.all_reduce(t, op=dist.ReduceOp.MAX)
            ms = float(t.item())
        return ms, {k: [v / steps for v in vs] for k, vs in stage.items()}, launches // steps

    def timed_e2e(form, steps, warmup):
        """Host frames in and out, a part of the frames per host thread (`halves`); CUDA events on the
        first stream bracket every stream's work."""
        if form not in pipes2:
            pipes2[form] = [Pipeline(L, capi, vi, s2, precisions[form]) for s2 in streams2]
        workers = [pipes[form]] + pipes2[form]
        errors = []

        def half(i):
            n, cnt, arrs = halves[i]
            try:
                workers[i].run(cnt, *arrs, n=n)
            except Exception as e:  # noqa: BLE001 -- reported on the main thread
                errors.append(e)

        def step():
            ts = [threading.Thread(target=half, args=(i,)) for i in range(len(halves))]
            for t in ts:
                t.start()
            for t in ts:
                t.join()
            if errors:
                raise errors[0]

        for _ in range(warmup):
            step()
        barrier()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        total = 0.0
        ebs = [torch.cuda.Event() for _ in streams2]
        for _ in range(steps):
            e0.record(stream)
            for s2 in streams2:
                s2.wait_event(e0)
            step()
            for s2, eb in zip(streams2, ebs):
                eb.record(s2)
                stream.wait_event(eb)
            e1.record(stream)
            e1.synchronize()
            total += e0.elapsed_time(e1)
        barrier()
        ms = total / steps
        if dist:
            t = torch.tensor([ms], device="cuda")
            dist.all_reduce(t, op=dist.ReduceOp.MAX)
            ms = float(t.item())
        return ms

    def psnr_of(out):
        return 10 * np.log10(1.0 / float(np.mean((out.astype(np.float64) - clean) ** 2)))

    peak = fp32_peak_tflops(torch) if rank == 0 else None
    res = {}
    clocks = Clocks(local)
    clocks.start()
    for form, pipe in pipes.items():
        ms, stage, launches = timed(pipe, args.steps, args.warmup, profile=True)
        out = torch.stack([torch.stack(f) for f in f_out]).cpu().numpy()
        ms_plain, _, _ = timed(pipe, args.steps, 1, profile=False)
        ms_e2e = timed_e2e(form, args.steps, args.warmup)
        # one more whole-batch run, so that the instances' counters and lists read below describe
        # the 8-frame step (the end-to-end calls left half a batch in them)
        pipe.run(F, a_in, a_opp, a_basic, a_final, a_out)
        torch.cuda.synchronize()
        res[form] = dict(ms=ms, stage=stage, launches=launches, psnr=psnr_of(out), ms_unprofiled=ms_plain, ms_e2e=ms_e2e)
    clk = clocks.stop()
    psnr_in = psnr_of(nz)
    # the headline form: the tensor-core form when it keeps PSNR within 0.05 dB of the plain path
    dpsnr = res["tf32"]["psnr"] - res["fp32"]["psnr"]
    dpsnr_l = res["learned"]["psnr"] - res["fp32"]["psnr"]
    ok = [f for f in ("tf32", "tf32_final", "learned") if res[f]["psnr"] - res["fp32"]["psnr"] >= -0.05]
    head = min(ok, key=lambda f: res[f]["ms"]) if ok else "fp32"
    R = res[head]
    pipe = pipes[head]

    # group fill of frame 0 (mean n) for the algorithmic work count
    nb_b = len(scan(Hd, 8, 4)) * len(scan(Wd, 8, 4))
    nb_f = len(scan(Hd, 8, 3)) * len(scan(Wd, 8, 3))

    def mean_n(st, G, nb):
        cnt = np.zeros(nb, np.int32)
        z = np.zeros(nb * G, np.int32)
        P = C.POINTER
        rc = L.bm3d_debug_matches(st.h, 0, cnt.ctypes.data_as(P(C.c_int)), z.ctypes.data_as(P(C.c_int)),
                                  z.ctypes.data_as(P(C.c_int)), z.ctypes.data_as(P(C.c_int)),
                                  np.zeros(nb * G, np.float32).ctypes.data_as(P(C.c_float)), nb)
        if rc <= 0:
            return float(G), 1.0
        return float(cnt.mean()), float((cnt == G).mean())

    def lists_of(st, G, nb):
        cnt = np.zeros(nb, np.int32)
        y = np.zeros(nb * G, np.int32)
        x = np.zeros(nb * G, np.int32)
        z = np.zeros(nb * G, np.int32)
        P = C.POINTER
        rc = L.bm3d_debug_matches(st.h, 0, cnt.ctypes.data_as(P(C.c_int)), z.ctypes.data_as(P(C.c_int)),
                                  y.ctypes.data_as(P(C.c_int)), x.ctypes.data_as(P(C.c_int)),
                                  np.zeros(nb * G, np.float32).ctypes.data_as(P(C.c_float)), nb)
        return (cnt, y.reshape(nb, G), x.reshape(nb, G)) if rc > 0 else None

    for pp in pipes.values():
        for st in (pp.basic, pp.final):
            L.bm3d_synchronize(st.h)
    (nb_mean, nb_full), (nf_mean, nf_full) = mean_n(pipe.basic, 16, nb_b), mean_n(pipe.final, 32, nb_f)
    # match-list agreement of the two forms' Basic matching on frame 0 (same input plane): the
    # precision form estimates distances on the tensor cores and re-ranks exactly
    agree = None
    la, lb = lists_of(pipes["fp32"].basic, 16, nb_b), lists_of(pipes["tf32"].basic, 16, nb_b)
    if la is not None and lb is not None:
        same = (la[0] == lb[0])
        for k in range(16):
            same &= ((la[1][:, k] == lb[1][:, k]) & (la[2][:, k] == lb[2][:, k])) | (k >= la[0])
        agree = float(same.mean())
    # the learned form's Basic lists on frame 0 against the exhaustive ones: mean fraction found
    recall_l = None
    ll = lists_of(pipes["learned"].basic, 16, nb_b)
    if la is not None and ll is not None:
        hits = np.zeros(nb_b)
        for k in range(16):
            for k2 in range(16):
                hits += ((la[1][:, k] == ll[1][:, k2]) & (la[2][:, k] == ll[2][:, k2]) & (k < la[0]) & (k2 < ll[0]))
        recall_l = float(np.mean(hits / la[0]))
    tcfb, lcut, rchk = {}, {}, {}
    for name, st in (("basic", pipes["tf32"].basic), ("final", pipes["tf32"].final)):
        fb, to = C.c_int64(0), C.c_int64(0)
        L.bm3d_debug_bm_tc_counts(st.h, C.byref(fb), C.byref(to))
        tcfb[name] = (int(fb.value), int(to.value))
        # learned form: reference blocks whose proposal cut needed the exact radix selection
        L.bm3d_debug_bm_tc_counts(getattr(pipes["learned"], name).h, C.byref(fb), C.byref(to))
        lcut[name] = int(fb.value)
    rc, ch = C.c_int64(0), C.c_int64(0)
    L.bm3d_debug_threshold_rechecks(pipes["tf32"].basic.h, C.byref(rc), C.byref(ch))
    rchk = {"recomputed": int(rc.value), "changed": int(ch.value)}
    bm_b, dct_b, _ = algorithmic_work(Wd, Hd, F, 4, 16, nb_mean, False)
    bm_f, dct_f, _ = algorithmic_work(Wd, Hd, F, 3, 32, nf_mean, True)
    stage = R["stage"]
    cands = {
        "basic_block_matching": (stage["basic"][1], bm_b),
        "basic_collaborative_filter": (stage["basic"][3], dct_b),
        "final_block_matching": (stage["final"][1], bm_f),
        "final_collaborative_filter": (stage["final"][3], dct_f),
    }
    dom = max(cands, key=lambda k: cands[k][0])
    t_dom, w_dom = cands[dom]

    if rank == 0:
        mpix = lambda ms: F * Wd * Hd * world / (ms * 1e-3) / 1e6
        traffic = None
        tpath = os.path.join(ROOT, "profiles", "traffic.json")
        if os.path.exists(tpath):
            try:
                traffic = json.load(open(tpath)).get(dom)
            except Exception:
                traffic = None
        achieved = w_dom / (t_dom * 1e-3) / 1e12 if t_dom > 0 else None
        # the bound of the dominant kernel: FP32 SIMT for the plain form and for block matching;
        # the tensor cores (tf32) for the precision form's collaborative filter
        if head in ("tf32", "tf32_final", "learned") and dom == "final_collaborative_filter":
            try:
                bf16 = json.load(open(os.path.join(ROOT, "MEASURED_PEAKS.json")))["bf16_tflops"]
                r_peak, r_bound = bf16 / 2.0, "tensor"
                r_src = "measured bf16 dense GEMM (MEASURED_PEAKS.json) / 2: the tf32 tensor rate is half the bf16 rate"
            except Exception:
                r_peak, r_bound, r_src = 1590.0 / 2.0, "tensor", "fallback bf16 1590 TFLOP/s / 2 (tf32 rate)"
        else:
            r_peak, r_bound = peak, "fp32"
            r_src = "measured in-process: cuBLAS SGEMM FP32 (TF32 off), 8192^3 best of 5"

        def form_summary(form):
            r = res[form]
            return {"value": round(mpix(r["ms"]), 3), "ms_per_step": round(r["ms"], 3),
                    "e2e": round(mpix(r["ms_e2e"]), 3), "psnr_out_db": round(r["psnr"], 4),
                    "stages_ms": {k: [round(v, 3) for v in vs] for k, vs in r["stage"].items()}}

        line = {
            "metric": METRIC, "value": round(mpix(R["ms"]), 3), "unit": "Mpix/s", "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": round(R["ms"], 3), "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f32" if head == "fp32" else "f32 (tf32 tensor-core transforms)",
            "data": "synthetic",
            "config": workload_config(F, Wd, Hd, world), "form": head,
            "forms": {"fp32": form_summary("fp32"), "tf32": form_summary("tf32"),
                      "tf32_final": form_summary("tf32_final"), "learned": form_summary("learned"),
                      "psnr_delta_db": round(dpsnr, 4), "speedup": round(res["fp32"]["ms"] / res["tf32"]["ms"], 3),
                      "tf32_final_psnr_delta_db": round(res["tf32_final"]["psnr"] - res["fp32"]["psnr"], 4),
                      "tf32_final_speedup": round(res["fp32"]["ms"] / res["tf32_final"]["ms"], 3),
                      "learned_psnr_delta_db": round(dpsnr_l, 4),
                      "learned_speedup": round(res["fp32"]["ms"] / res["learned"]["ms"], 3)},
            "roofline": {"bound": r_bound, "kernel": dom, "achieved": round(achieved, 3) if achieved else None,
                         "peak": round(r_peak, 3) if r_peak else None, "unit": "TFLOP/s",
                         "frac": round(achieved / r_peak, 4) if (achieved and r_peak) else None, "traffic": traffic,
                         "peak_source": r_src, "fp32_simt_peak": round(peak, 3) if peak else None,
                         "work": "algorithmic FLOPs: block matching 3*B^2 per evaluated candidate; transforms 2*(n*2B^3+B^2*n^2) per 3-D DCT of a group of n blocks (2 per group and plane for Basic, 3 for Final)"},
            "stages_ms": {"basic": [round(v, 3) for v in stage["basic"]], "final": [round(v, 3) for v in stage["final"]],
                          "order": ["ingest", "block_matching", "predictive", "collaborative_filter", "normalise", "egress"]},
            "e2e": {"value": round(mpix(R["ms_e2e"]), 3), "unit": "Mpix/s", "h2d_bytes_per_step": int(nz.nbytes),
                    "d2h_bytes_per_step": int(nz.nbytes), "ms_per_step": round(R["ms_e2e"], 3)},
            "ms_per_step_unprofiled": round(R["ms_unprofiled"], 3),
            "groups": {"basic_mean_n": round(nb_mean, 3), "basic_full_fraction": round(nb_full, 4),
                       "final_mean_n": round(nf_mean, 3), "final_full_fraction": round(nf_full, 4),
                       "basic_exact_tie_blocks": int(L.bm3d_debug_slow_blocks(pipe.basic.h)),
                       "final_exact_tie_blocks": int(L.bm3d_debug_slow_blocks(pipe.final.h))},
            "learned_block_matching": {"basic_list_recall_vs_exhaustive": recall_l, "exact_cut_blocks": lcut},
            "tc_threshold_recheck_basic": rchk,
            "tc_block_matching": {"basic_list_agreement_vs_fp32": agree,
                                  "exact_fallback_blocks": {k: v[0] for k, v in tcfb.items()},
                                  "timeouts": {k: v[1] for k, v in tcfb.items()}},
            "gpu_launches": int(R["launches"]),
            "clocks": clk,
            "quality": {"psnr_in_db": round(psnr_in, 3), "psnr_out_db": round(R["psnr"], 3)},
        }
        if not args.no_cpu_baseline:
            threads = min(os.cpu_count() or 1, F)
            mp, dt, sample = cpu_sample(threads, threads, Wd, 136)
            line["cpu_baseline"] = {"value": round(mp, 4), "unit": "Mpix/s", "cores": threads, "kind": "port",
                                    "sample": sample, "seconds": round(dt, 2)}
        print(json.dumps(line), flush=True)
    if dist:
        dist.barrier()
        dist.destroy_process_group()


def vbm3d_arm(args):
    """V-BM3D on a YUV444 16-bit 1920x1080 clip of `frames` frames (default 15), sigma 15, radius 1,
    ps_num 2, ps_range 4: VBasic -> VAggregate -> VFinal(ref) -> VAggregate through the C ABI on
    device-resident frames (the stacked drop-in chain), and the same chain with aggregate=1 (no
    stacked clip).  Prints one JSON line; not the headline metric."""
    import numpy as np
    import torch
    from bm3d_b200 import _capi as capi
    from bm3d_b200 import synth

    rank, world, local = dist_env()
    torch.cuda.set_device(local)
    L = capi.lib()
    F = args.frames if args.frames != NFR else 15
    Wd, Hd, sig, r = args.width, args.height, 15.0, 1
    nz, clean = synth.motion_frames(3, F, Hd, Wd, sig, planes=3)
    yuv = np.stack([np.stack([synth.to_u16(np.clip(nz[f, c], 0, 1)) for c in range(3)]) for f in range(F)])
    # 16-bit samples travel as int16 tensors (same bytes; torch's uint16 support is partial)
    d_in = torch.from_numpy(np.ascontiguousarray(yuv).view(np.int16)).cuda()
    stream = torch.cuda.Stream()
    vi = capi.VideoInfo(capi.YUV, capi.INTEGER, 16, 0, 0, Wd, Hd, F)
    common = {"sigma": sig, "radius": r}
    D = capi.MEM_DEVICE

    def planes(n, h, dt):
        return [[torch.empty((h, Wd), dtype=dt, device="cuda") for _ in range(3)] for _ in range(n)]

    _, a_in = make_frames(capi, [[d_in[k, p] for p in range(3)] for k in range(F)], D)
    # stacked chain
    vb = Stage(L, "VBasic", dict(common, input=vi, ps_num=2, ps_range=4), None)
    ag1 = Stage(L, "VAggregate", {"input": vb.info, "radius": r}, None)
    vf = Stage(L, "VFinal", dict(common, input=vi, ref=ag1.info), None)
    ag2 = Stage(L, "VAggregate", {"input": vf.info, "radius": r}, None)
    st_h = Hd * (2 * r + 1) * 2
    f_vb, f_ag1 = planes(F, st_h, torch.float32), planes(F, Hd, torch.int16)
    f_vf, f_ag2 = planes(F, st_h, torch.float32), planes(F, Hd, torch.int16)
    _, a_vb = make_frames(capi, f_vb, D)
    _, a_ag1 = make_frames(capi, f_ag1, D)
    _, a_vf = make_frames(capi, f_vf, D)
    _, a_ag2 = make_frames(capi, f_ag2, D)
    # aggregated chain
    fb = Stage(L, "VBasic", dict(common, input=vi, ps_num=2, ps_range=4, aggregate=1), None)
    ff = Stage(L, "VFinal", dict(common, input=vi, ref=fb.info, aggregate=1), None)
    f_fb, f_ff = planes(F, Hd, torch.int16), planes(F, Hd, torch.int16)
    _, a_fb = make_frames(capi, f_fb, D)
    _, a_ff = make_frames(capi, f_ff, D)
    for st in (vb, ag1, vf, ag2, fb, ff):
        L.bm3d_set_stream(st.h, C.c_void_p(stream.cuda_stream))

    def call(st, src, ref, dst):
        if L.bm3d_get_frames_async(st.h, 0, F, src, ref, dst) != 0:
            raise RuntimeError(capi.last_error())

    def stacked():
        call(vb, a_in, None, a_vb)
        call(ag1, a_vb, None, a_ag1)
        call(vf, a_in, a_ag1, a_vf)
        call(ag2, a_vf, None, a_ag2)

    def fused():
        call(fb, a_in, None, a_fb)
        call(ff, a_in, a_fb, a_ff)

    def timed(fn):
        for _ in range(args.warmup):
            fn()
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        tot = 0.0
        for _ in range(args.steps):
            with torch.cuda.stream(stream):
                e0.record(stream)
            fn()
            with torch.cuda.stream(stream):
                e1.record(stream)
            e1.synchronize()
            tot += e0.elapsed_time(e1)
        return tot / args.steps

    clocks = Clocks(local)
    clocks.start()
    ms_st = timed(stacked)
    ms_fu = timed(fused)
    clk = clocks.stop()
    out_st = torch.stack([torch.stack(f) for f in f_ag2]).cpu().numpy().view(np.uint16).astype(np.int64)
    out_fu = torch.stack([torch.stack(f) for f in f_ff]).cpu().numpy().view(np.uint16).astype(np.int64)
    # the Basic stage of both chains (VAggregate(VBasic) against VBasic(aggregate=1)): the Final's
    # block matching runs on it, so a last-bit difference there can change a Final match list
    bas_st = torch.stack([torch.stack(f) for f in f_ag1]).cpu().numpy().view(np.uint16).astype(np.int64)
    bas_fu = torch.stack([torch.stack(f) for f in f_fb]).cpu().numpy().view(np.uint16).astype(np.int64)
    dfin = np.abs(out_st - out_fu)

    def psnr16(o):
        return 10 * np.log10(65535.0 ** 2 / np.mean((o - np.clip(np.round(clean * 65535.0), 0, 65535)) ** 2))

    mpix = lambda ms: F * Wd * Hd / (ms * 1e-3) / 1e6
    line = {"metric": "1080p V-BM3D Mpix/s (VBasic -> VAggregate -> VFinal -> VAggregate, YUV444 16-bit, radius 1)",
            "value": round(mpix(ms_st), 3), "unit": "Mpix/s", "n_gpus": 1, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": round(ms_st, 3), "higher_is_better": True, "dtype": "f32", "data": "synthetic",
            "config": {"workload": f"YUV444 u16 {Wd}x{Hd} x{F} frames, translating scene, sigma 15", "radius": r,
                       "ps_num": 2, "ps_range": 4},
            "aggregated": {"value": round(mpix(ms_fu), 3), "ms_per_step": round(ms_fu, 3),
                           "basic_max_lsb_vs_stacked": int(np.abs(bas_st - bas_fu).max()),
                           "max_lsb_vs_stacked": int(dfin.max()),
                           "fraction_over_1_lsb": float(np.mean(dfin > 1))},
            "psnr_db": {"input": round(float(psnr16(yuv.astype(np.int64))), 3), "stacked": round(float(psnr16(out_st)), 3),
                        "aggregated": round(float(psnr16(out_fu)), 3)},
            "clocks": clk}
    print(json.dumps(line), flush=True)


def main():
    args = parse()
    if args.impl == "reference":
        reference_arm(args)
    elif args.workload == "vbm3d":
        vbm3d_arm(args)
    else:
        ours_arm(args)


if __name__ == "__main__":
    main()
