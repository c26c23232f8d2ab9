"""Builds libsunset_b200.so in-tree with nvcc for sm_100a (no JIT, no torch extension).

The setup, weight and step sources are compiled with -fmad=false so every product and
sum rounds separately, as in the reference (the mixed-precision step shares those kernels).
"""
from __future__ import annotations

import os
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
LIBDIR = os.path.join(HERE, "lib")
LIB = os.path.join(LIBDIR, "libsunset_b200.so")
HOSTCHECK = os.path.join(LIBDIR, "libsunset_hostcheck.so")  # host build of the pointwise adjoint (tests)
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
SOURCES = {  # file -> extra flags
    "setup.cu": ["-fmad=false"],
    "weights.cu": ["-fmad=false"],
    "step.cu": ["-fmad=false"],
    "step3d.cu": ["-fmad=false"],
    "stream.cu": [],
    "bank_deal.cu": [],
    "noalloc.cu": [],
    "abi.cu": [],
}


def nvcc() -> str:
    for c in [os.environ.get("NVCC"), "/usr/local/cuda/bin/nvcc", shutil.which("nvcc")]:
        if c and os.path.exists(c):
            return c
    raise RuntimeError("nvcc not found")


def _stale(out: str, deps) -> bool:
    if not os.path.exists(out):
        return True
    t = os.path.getmtime(out)
    return any(os.path.getmtime(d) > t for d in deps)


def build(verbose: bool = False, force: bool = False) -> str:
    os.makedirs(os.path.join(LIBDIR, "obj"), exist_ok=True)
    headers = [os.path.join(CSRC, f) for f in os.listdir(CSRC) if f.endswith((".cuh", ".h"))]
    headers.append(os.path.join(HERE, "..", "include", "sunset_gpu.h"))
    objs = []
    for src, extra in SOURCES.items():
        s = os.path.join(CSRC, src)
        o = os.path.join(LIBDIR, "obj", src.replace(".cu", ".o"))
        objs.append(o)
        if force or _stale(o, [s, __file__] + headers):
            cmd = [nvcc(), *ARCH, "-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC", "-c", s, "-o", o,
                   "-Xptxas", "-v" if verbose else "-O3", *extra]
            r = subprocess.run(cmd, capture_output=True, text=True)
            if r.returncode != 0:
                raise RuntimeError(f"nvcc failed for {src}:\n{r.stdout}\n{r.stderr}")
            if verbose:
                sys.stderr.write(r.stderr)
    if force or _stale(LIB, objs):
        cmd = [nvcc(), *ARCH, "-shared", "-o", LIB, *objs, "-lcudart"]
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError(f"link failed:\n{r.stdout}\n{r.stderr}")
    src = [os.path.join(CSRC, "hostcheck.cu"), os.path.join(CSRC, "bank_deal.cu")]
    if force or _stale(HOSTCHECK, src + [__file__] + headers):
        cmd = [nvcc(), "-O2", "-std=c++17", "-Xcompiler", "-fPIC", "-shared", "-fmad=false", *src, "-o", HOSTCHECK]
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError(f"nvcc failed for hostcheck.cu:\n{r.stdout}\n{r.stderr}")
    return LIB


if __name__ == "__main__":
    print(build(verbose="-v" in sys.argv, force="-f" in sys.argv))
