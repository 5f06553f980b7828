"""Build recipe of the oracle library (test infrastructure only).

Compiles O1 (oracle/o1_core.cpp, f64 restatement of crates/gps-core) and O2
(oracle/o2_mirror.cpp, f32 mirror of shaders/gps_splat.wgsl) into oracle/libgpsoracle.so.
-ffp-contract=off keeps every a*b+c unfused so O2 matches the CUDA kernels bit for bit.
The reference itself is Rust + WGSL and cannot be compiled here (no cargo/rustc, no graphics
stack), so there is no oracle/_ref build.
"""
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
LIB = os.path.join(HERE, "libgpsoracle.so")
SOURCES = ["o1_core.cpp", "o2_mirror.cpp"]
HEADERS = [os.path.join(HERE, "..", "include", "gpsb200.h"),
           os.path.join(HERE, "..", "gps-pbvr-web_b200", "csrc", "fmath.h")]


def _stale() -> bool:
    if not os.path.exists(LIB):
        return True
    t = os.path.getmtime(LIB)
    deps = [os.path.join(HERE, s) for s in SOURCES] + HEADERS + [__file__]
    return any(os.path.getmtime(d) > t for d in deps)


def build(force: bool = False) -> str:
    if force or _stale():
        cmd = ["g++", "-O2", "-std=c++17", "-fPIC", "-shared", "-ffp-contract=off", "-fno-fast-math",
               "-pthread", "-o", LIB + ".tmp"] + [os.path.join(HERE, s) for s in SOURCES]
        subprocess.run(cmd, check=True)
        os.replace(LIB + ".tmp", LIB)
    return LIB


if __name__ == "__main__":
    print(build(force="--force" in sys.argv))
