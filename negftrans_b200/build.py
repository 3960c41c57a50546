"""Build libnegfgpu.so in-tree with nvcc for sm_100a.

The library is a plain C-ABI shared object (include/negf_gpu.h); the CUDA
runtime is linked statically so that the .so loads on any box with a driver.
"""
from __future__ import annotations

import os
import subprocess

PKG = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(PKG)
CSRC = os.path.join(PKG, "csrc")
LIB = os.path.join(PKG, "libnegfgpu.so")
DRIVER = os.path.join(PKG, "negftrans")   # the main.f90-style executable
SOURCES = ["negf_engine.cu", "negf_host.cpp", "mlp.cu", "negf_mixed.cu"]
HEADERS = ["rgf_device.cuh", "tc_umma.cuh", "mixed_device.cuh"]
# private headers each source includes
DEPS = {"negf_engine.cu": ("rgf_device.cuh",),
        "negf_mixed.cu": ("rgf_device.cuh", "tc_umma.cuh", "mixed_device.cuh")}
PUBLIC_HEADERS = ["negf_gpu.h", "negf_mlp.h"]
OBJDIR = os.path.join(PKG, "_build")
NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]


def _stale() -> bool:
    if not os.path.exists(LIB):
        return True
    t = os.path.getmtime(LIB)
    deps = [os.path.join(CSRC, f) for f in SOURCES + HEADERS]
    deps += [os.path.join(ROOT, "include", h) for h in PUBLIC_HEADERS]
    return any(os.path.getmtime(d) > t for d in deps)


def build_driver(force: bool = False) -> str:
    src = os.path.join(CSRC, "negftrans_main.cpp")
    if (not force and os.path.exists(DRIVER)
            and os.path.getmtime(DRIVER) >= max(os.path.getmtime(src), os.path.getmtime(LIB))):
        return DRIVER
    cmd = ["g++", "-O2", "-std=c++17", "-I", os.path.join(ROOT, "include"), src, "-L", PKG, "-lnegfgpu",
           "-Wl,-rpath,$ORIGIN", "-o", DRIVER]
    subprocess.run(cmd, check=True)
    return DRIVER


def build(force: bool = False, verbose: bool = False) -> str:
    if not force and not _stale():
        build_driver()
        return LIB
    # one object per source, compiled in parallel, then one link
    os.makedirs(OBJDIR, exist_ok=True)
    base = [NVCC, *ARCH, "-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC",
            "-I", os.path.join(ROOT, "include"), "-I", CSRC]
    if verbose:
        base += ["-Xptxas", "-v"]
    procs, objs = [], []
    pub_t = max(os.path.getmtime(os.path.join(ROOT, "include", h)) for h in PUBLIC_HEADERS)
    for f in SOURCES:
        obj = os.path.join(OBJDIR, os.path.splitext(f)[0] + ".o")
        objs.append(obj)
        src = os.path.join(CSRC, f)
        dep_t = max([os.path.getmtime(src), pub_t] + [os.path.getmtime(os.path.join(CSRC, h))
                                                      for h in DEPS.get(f, ())])
        # an object newer than its source and the headers it includes is reused
        if not force and os.path.exists(obj) and os.path.getmtime(obj) >= dep_t:
            continue
        procs.append((f, subprocess.Popen(base + ["-c", src, "-o", obj])))
    bad = [f for f, p in procs if p.wait() != 0]
    if bad:
        raise RuntimeError("nvcc failed on " + ", ".join(bad))
    subprocess.run([NVCC, *ARCH, "-shared", "-cudart", "static", *objs, "-o", LIB], check=True)
    build_driver(force=True)
    return LIB


if __name__ == "__main__":
    import sys
    print(build(force=True, verbose="-v" in sys.argv))
