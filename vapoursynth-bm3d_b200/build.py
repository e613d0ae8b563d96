"""Build recipe for the in-tree shared library lib/libbm3d_b200.so (sm_100a).

Compiles csrc/kernels.cu (every kernel), csrc/host.cpp (argument processing, filter objects,
C ABI of include/bm3d_b200.h) and csrc/noalloc.cu (the allocation-free Basic entry point) with
nvcc, linking the CUDA runtime statically so the library only needs the NVIDIA driver at run time.

Where the VapourSynth SDK header (VapourSynth4.h) is installed, also builds the VapourSynth plugin
lib/libbm3d_vs.so from vs/bm3d_vsplugin.cpp (linked against libbm3d_b200.so, found next to it).
"""
import os
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
LIB_DIR = os.path.join(HERE, "lib")
LIB = os.path.join(LIB_DIR, "libbm3d_b200.so")
SOURCES = ["kernels.cu", "host.cpp", "noalloc.cu"]


def deps():
    """Every source and header of csrc/ plus the public header."""
    names = [n for n in os.listdir(CSRC) if n.endswith((".cu", ".cuh", ".cpp", ".h"))]
    return [os.path.join(CSRC, n) for n in names] + [os.path.join(os.path.dirname(HERE), "include", "bm3d_b200.h")]


def nvcc_path():
    for cand in (shutil.which("nvcc"), "/usr/local/cuda/bin/nvcc"):
        if cand and os.path.exists(cand):
            return cand
    raise RuntimeError("nvcc not found")


VS_SRC = os.path.join(HERE, "vs", "bm3d_vsplugin.cpp")
VS_LIB = os.path.join(LIB_DIR, "libbm3d_vs.so")


def vapoursynth_include():
    """Directory holding VapourSynth4.h (pkg-config vapoursynth, then the usual prefixes), or None."""
    try:
        out = subprocess.run(["pkg-config", "--cflags-only-I", "vapoursynth"], capture_output=True, text=True)
        dirs = [d[2:] for d in out.stdout.split() if d.startswith("-I")] if out.returncode == 0 else []
    except OSError:
        dirs = []
    dirs += ["/usr/include/vapoursynth", "/usr/local/include/vapoursynth", "/usr/include", "/usr/local/include"]
    for d in dirs:
        if os.path.exists(os.path.join(d, "VapourSynth4.h")):
            return d
    return None


def build_vs_plugin(verbose=False):
    """Builds lib/libbm3d_vs.so when the VapourSynth SDK is present; returns its path or None."""
    inc = vapoursynth_include()
    if inc is None:
        if verbose:
            print("VapourSynth SDK (VapourSynth4.h) not found: plugin adapter not built", file=sys.stderr)
        return None
    cmd = ["g++", "-std=c++17", "-O2", "-fPIC", "-shared", "-I" + inc,
           "-I" + os.path.join(os.path.dirname(HERE), "include"), "-o", VS_LIB, VS_SRC,
           "-L" + LIB_DIR, "-lbm3d_b200", "-Wl,-rpath,$ORIGIN"]
    if verbose:
        print(" ".join(cmd), file=sys.stderr)
    subprocess.run(cmd, check=True)
    return VS_LIB


def needs_build():
    if not os.path.exists(LIB):
        return True
    t = os.path.getmtime(LIB)
    return any(os.path.getmtime(d) > t for d in deps())


def build(force=False, verbose=False):
    if not force and not needs_build():
        return LIB
    os.makedirs(LIB_DIR, exist_ok=True)
    cmd = [nvcc_path(), "-gencode", "arch=compute_100a,code=sm_100a", "-O3", "-lineinfo", "-std=c++17",
           "-I" + os.path.join(os.path.dirname(HERE), "include"),
           "-Xcompiler", "-fPIC,-fvisibility=hidden", "-shared", "-cudart", "static",
           "-o", LIB + ".tmp"] + [os.path.join(CSRC, s) for s in SOURCES]
    if verbose:
        print(" ".join(cmd), file=sys.stderr)
    subprocess.run(cmd, check=True, cwd=CSRC)
    os.replace(LIB + ".tmp", LIB)
    build_vs_plugin(verbose)
    return LIB


if __name__ == "__main__":
    print(build(force="--force" in sys.argv, verbose=True))
