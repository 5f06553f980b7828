"""Build recipe of libgpsb200.so (the C-ABI renderer) and the gpsb-verify CLI, for sm_100a.

Kernels are compiled with --fmad=false so every multiply-add is rounded as written (bit-exact
parity with the CPU mirror oracle); host C++ with -ffp-contract=off for the same reason.
Objects are rebuilt when a source or header is newer. Usage: python gps-pbvr-web_b200/build.py
"""
import glob
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
OBJ = os.path.join(HERE, "_build")
LIB = os.path.join(HERE, "libgpsb200.so")
CLI = os.path.join(HERE, "gpsb-verify")
ROOT = os.path.dirname(HERE)
CUDA = os.environ.get("CUDA_HOME", "/usr/local/cuda")
NVCC = os.path.join(CUDA, "bin", "nvcc")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
CU_FLAGS = ARCH + ["-O3", "-lineinfo", "--fmad=false", "-std=c++17", "-Xcompiler", "-fPIC,-ffp-contract=off",
                   "-I" + CSRC, "-I" + os.path.join(ROOT, "include")]
CXX_FLAGS = ["-O2", "-std=c++17", "-fPIC", "-ffp-contract=off", "-fno-fast-math", "-I" + os.path.join(CUDA, "include"),
             "-I" + CSRC, "-I" + os.path.join(ROOT, "include")]
# extra nvcc flags for tuning builds (e.g. GPSB_NVCC_EXTRA="-DGPSB_SORT_LOOKAHEAD=16"; rebuild with --force)
CU_FLAGS += os.environ.get("GPSB_NVCC_EXTRA", "").split()
LIB_SOURCES = ["kernels.cu", "sorted.cu", "primitives.cu", "denoise.cu", "conv3x3.cu", "ply_gpu.cu", "renderer.cpp", "denoiser.cpp", "session.cpp", "hostmath.cpp", "ply.cpp"]


def _headers():
    return glob.glob(os.path.join(CSRC, "*.h")) + glob.glob(os.path.join(CSRC, "*.cuh")) + \
        [os.path.join(ROOT, "include", "gpsb200.h")]


def _newer(target, deps):
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(d) > t for d in deps)


def _run(cmd, verbose):
    if verbose:
        print(" ".join(cmd), flush=True)
    subprocess.run(cmd, check=True)


def build(force=False, verbose=False):
    os.makedirs(OBJ, exist_ok=True)
    hdrs = _headers() + [__file__]
    objs = []
    for src in LIB_SOURCES:
        path = os.path.join(CSRC, src)
        obj = os.path.join(OBJ, src + ".o")
        objs.append(obj)
        if force or _newer(obj, [path] + hdrs):
            if src.endswith(".cu"):
                _run([NVCC] + CU_FLAGS + ["-c", path, "-o", obj], verbose)
            else:
                _run(["g++"] + CXX_FLAGS + ["-c", path, "-o", obj], verbose)
    if force or _newer(LIB, objs):
        _run([NVCC] + ARCH + ["-shared", "-o", LIB + ".tmp"] + objs + ["-lcudart"], verbose)
        os.replace(LIB + ".tmp", LIB)
    cli_src = os.path.join(CSRC, "gpsb_verify.cpp")
    if os.path.exists(cli_src) and (force or _newer(CLI, [cli_src, LIB] + hdrs)):
        _run(["g++", "-O2", "-std=c++17", "-I" + os.path.join(ROOT, "include"), cli_src, "-o", CLI, "-L" + HERE,
              "-lgpsb200", "-Wl,-rpath,$ORIGIN", "-pthread"], verbose)
    return LIB


if __name__ == "__main__":
    print(build(force="--force" in sys.argv, verbose=True))
