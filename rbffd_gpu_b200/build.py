"""Build librbffd_sm100.so in-tree (rbffd_gpu_b200/lib/) with nvcc for sm_100a.

Every CUDA translation unit is compiled with
``-gencode arch=compute_100a,code=sm_100a -lineinfo -O3``; the host-side C++
(input builders, the C++ API layer) with the same nvcc driver so one shared
library carries the whole C ABI declared in include/rbffd_sm100.h.
"""
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
LIBDIR = os.path.join(HERE, "lib")
LIB = os.path.join(LIBDIR, "librbffd_sm100.so")
OBJDIR = os.path.join(HERE, "_build")

NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
COMMON = ["-O3", "-std=c++17", "-lineinfo", "-Xcompiler", "-fPIC,-ffp-contract=off", "-I" + os.path.join(ROOT, "include")]


def sources():
    out = []
    for f in sorted(os.listdir(CSRC)):
        if f.endswith((".cu", ".cpp")):
            out.append(os.path.join(CSRC, f))
    return out


def headers():
    hs = [os.path.join(ROOT, "include", f) for f in os.listdir(os.path.join(ROOT, "include")) if f.endswith(".h")]
    hs += [os.path.join(CSRC, f) for f in os.listdir(CSRC) if f.endswith((".h", ".cuh"))]
    return hs


def _mtime(p):
    return os.path.getmtime(p) if os.path.exists(p) else -1.0


def _run(cmd):
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        sys.stderr.write(r.stdout + r.stderr)
        raise RuntimeError("build failed: " + " ".join(cmd))
    return r.stdout + r.stderr


def build(force=False, verbose=False, ptxas_v=False):
    os.makedirs(LIBDIR, exist_ok=True)
    os.makedirs(OBJDIR, exist_ok=True)
    hdr_t = max([_mtime(h) for h in headers()] + [_mtime(__file__)])
    objs = []
    for src in sources():
        obj = os.path.join(OBJDIR, os.path.basename(src) + ".o")
        objs.append(obj)
        if force or _mtime(obj) < max(_mtime(src), hdr_t):
            cmd = [NVCC] + ARCH + COMMON + ["-c", src, "-o", obj]
            if src.endswith(".cpp"):
                cmd = [NVCC] + COMMON + ["-x", "cu"] + ARCH + ["-c", src, "-o", obj]
            if ptxas_v and src.endswith(".cu"):
                cmd += ["-Xptxas", "-v"]
            out = _run(cmd)
            if verbose and out:
                sys.stdout.write(out)
    if force or _mtime(LIB) < max(_mtime(o) for o in objs):
        _run([NVCC] + ARCH + ["-shared", "-o", LIB] + objs + ["-lpthread"])
    build_drivers(force)
    return LIB


CPP = os.path.join(HERE, "cpp")
# C++ drivers on the C++ API (cpp/rbffd_cuda.hpp), linked against the library
DRIVERS = {"cosine_bell_cuda": "cosine_bell_main.cpp", "vortex_rollup_cuda": "vortex_rollup_main.cpp"}


def build_drivers(force=False):
    hdr = max(_mtime(os.path.join(CPP, "rbffd_cuda.hpp")), _mtime(os.path.join(ROOT, "include", "rbffd_sm100.h")))
    for exe, src in DRIVERS.items():
        out = os.path.join(LIBDIR, exe)
        srcp = os.path.join(CPP, src)
        if force or _mtime(out) < max(_mtime(srcp), hdr, _mtime(LIB)):
            _run(["g++", "-O2", "-std=c++17", "-Wall", "-I" + os.path.join(ROOT, "include"), "-I" + CPP, srcp,
                  "-L" + LIBDIR, "-lrbffd_sm100", "-Wl,-rpath,$ORIGIN", "-o", out])


if __name__ == "__main__":
    print(build(force="--force" in sys.argv, verbose=True, ptxas_v="--ptxas-v" in sys.argv))
