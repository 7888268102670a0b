"""Builds libcam.so (the C-ABI library in csrc/) in-tree for sm_100a.

    python -m cosmicatlas_b200.build [--verbose]

Each .cu is compiled separately (in parallel) and linked into
cosmicatlas_b200/libcam.so with the CUDA runtime linked statically, so the
library does not depend on which libcudart the host process already loaded.
"""
from __future__ import annotations

import concurrent.futures as cf
import os
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
BUILD = os.path.join(HERE, "_build")
LIB = os.path.join(HERE, "libcam.so")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVCC_FLAGS = ["-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC,-O2", "--expt-relaxed-constexpr",
              "-Xptxas", "-warn-spills"]


def nvcc() -> str:
    for c in (os.environ.get("NVCC"), "/usr/local/cuda/bin/nvcc", shutil.which("nvcc")):
        if c and os.path.exists(c):
            return c
    raise RuntimeError("nvcc not found")


def _host_compiler_args():
    # nvcc needs a host g++; prefer the system one (the image may put a
    # toolchain without libstdc++ headers first on PATH).
    for c in ("/usr/bin/g++",):
        if os.path.exists(c):
            return ["-ccbin", c]
    return []


def sources():
    return sorted(os.path.join(CSRC, f) for f in os.listdir(CSRC) if f.endswith(".cu"))


def _compile(src: str, verbose: bool) -> str:
    obj = os.path.join(BUILD, os.path.basename(src)[:-3] + ".o")
    headers = [os.path.join(CSRC, f) for f in os.listdir(CSRC) if f.endswith((".h", ".cuh"))]
    headers.append(os.path.join(HERE, "..", "include", "cam.h"))
    newest = max([os.path.getmtime(src)] + [os.path.getmtime(h) for h in headers if os.path.exists(h)])
    if os.path.exists(obj) and os.path.getmtime(obj) >= newest:
        return obj
    cmd = [nvcc()] + _host_compiler_args() + ARCH + NVCC_FLAGS + ["-c", src, "-o", obj]
    if verbose:
        cmd += ["-Xptxas", "-v"]
        print(" ".join(cmd), flush=True)
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"nvcc failed on {src}:\n{r.stdout}\n{r.stderr}")
    if verbose and r.stderr:
        print(r.stderr, file=sys.stderr)
    return obj


def build(verbose: bool = False) -> str:
    os.makedirs(BUILD, exist_ok=True)
    srcs = sources()
    with cf.ThreadPoolExecutor(max_workers=min(8, os.cpu_count() or 4)) as ex:
        objs = list(ex.map(lambda s: _compile(s, verbose), srcs))
    if not os.path.exists(LIB) or os.path.getmtime(LIB) < max(os.path.getmtime(o) for o in objs):
        cmd = [nvcc()] + _host_compiler_args() + ARCH + ["-shared", "-cudart", "static", "-o", LIB] + objs
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError(f"link failed:\n{r.stdout}\n{r.stderr}")
    return LIB


SHIM_SRC = os.path.join(HERE, "shim", "cam_reference_api.cpp")
SHIM_LIB = os.path.join(HERE, "libcam_refapi.so")


def build_shim() -> str:
    """libcam_refapi.so: the reference's C++ signatures over libcam.so."""
    lib = build()
    deps = [SHIM_SRC, lib, os.path.join(HERE, "..", "include", "cam_reference_api.h")]
    if os.path.exists(SHIM_LIB) and os.path.getmtime(SHIM_LIB) >= max(os.path.getmtime(d) for d in deps):
        return SHIM_LIB
    gxx = "/usr/bin/g++" if os.path.exists("/usr/bin/g++") else "g++"
    cmd = [gxx, "-O2", "-std=c++17", "-fPIC", "-shared", "-o", SHIM_LIB, SHIM_SRC, "-L" + HERE, "-lcam",
           "-Wl,-rpath,$ORIGIN"]
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"shim build failed:\n{r.stdout}\n{r.stderr}")
    return SHIM_LIB


if __name__ == "__main__":
    print(build(verbose="--verbose" in sys.argv))
    print(build_shim())
