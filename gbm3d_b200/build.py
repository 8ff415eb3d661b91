"""Build libgbm3d.so in-tree with nvcc for sm_100a.

    python -m gbm3d_b200.build [--verbose]

--fmad=false keeps the compiler from contracting a*b+c into fma: the kernels
write fmaf() where a fused operation is meant, so results are a fixed function
of the inputs (the CPU oracle reproduces them bit for bit).
"""
from __future__ import annotations

import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
SRC = os.path.join(HERE, "csrc")
LIB = os.path.join(HERE, "libgbm3d.so")
SOURCES = ["match.cu", "wavelet.cu", "wiener.cu", "aggregate.cu", "gbm3d_api.cu", "noalloc.cu", "global_match.cu",
           "tc_check.cu", "match_tc.cu", "pilot.cu", "video.cu"]
NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
FLAGS = ["-O3", "-std=c++17", "-lineinfo", "--fmad=false", "-Xcompiler", "-fPIC,-O2",
         "--expt-relaxed-constexpr", "-I", os.path.join(ROOT, "include")]


def _stale() -> bool:
    if not os.path.exists(LIB):
        return True
    t = os.path.getmtime(LIB)
    deps = [os.path.join(SRC, f) for f in os.listdir(SRC)] + [os.path.join(ROOT, "include", "gbm3d.h")]
    return any(os.path.getmtime(p) > t for p in deps)


def build(force: bool = False, verbose: bool = False) -> str:
    if not force and not _stale():
        return LIB
    objdir = os.path.join(HERE, "_build")
    os.makedirs(objdir, exist_ok=True)
    objs = []
    procs = []
    for f in SOURCES:
        obj = os.path.join(objdir, f.replace(".cu", ".o"))
        cmd = [NVCC, *ARCH, *FLAGS, "-c", os.path.join(SRC, f), "-o", obj]
        if verbose:
            cmd += ["-Xptxas", "-v"]
        procs.append((f, subprocess.Popen(cmd, stdout=subprocess.PIPE, stderr=subprocess.STDOUT, text=True)))
        objs.append(obj)
    failed = False
    for f, p in procs:
        out, _ = p.communicate()
        if out and (verbose or p.returncode):
            sys.stderr.write(f"--- {f}\n{out}")
        failed |= p.returncode != 0
    if failed:
        raise RuntimeError("nvcc failed")
    tmp = LIB + ".tmp"
    subprocess.run([NVCC, *ARCH, "-shared", "-o", tmp, *objs], check=True)
    os.replace(tmp, LIB)
    return LIB


if __name__ == "__main__":
    build(force=True, verbose="--verbose" in sys.argv)
    print(LIB)
