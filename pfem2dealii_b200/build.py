"""Builds libpfem2gpu.so in-tree (pfem2dealii_b200/_build/) for sm_100a.

kernels_f64.cu, window_f64.cu, noalloc.cu and fem.cu are compiled with --fmad=false: the FP64 form
rounds every product and sum separately, as the CPU build of the reference
arithmetic does.
The other sources use the default contraction.  Run ``python -m
pfem2dealii_b200.build`` or call ``build()``.
"""
from __future__ import annotations

import hashlib
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
SRC = os.path.join(HERE, "csrc")
OUT = os.path.join(HERE, "_build")
LIB = os.path.join(OUT, "libpfem2gpu.so")
INCLUDE = os.path.join(os.path.dirname(HERE), "include")

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
COMMON = ["-std=c++17", "-O3", "-lineinfo", "-Xcompiler", "-fPIC", "-Xptxas", "-v", "-I", INCLUDE]
SOURCES = {
    "kernels_f64.cu": ["--fmad=false"],
    "kernels_f32.cu": [],
    "misc.cu": [],
    "api.cu": [],
    "noalloc.cu": ["--fmad=false"],
    "window_f64.cu": ["--fmad=false"],
    "window_f32.cu": [],
    "mesh_io.cu": [],
    "fem.cu": ["--fmad=false"],
}


def _nvcc():
    for c in (os.environ.get("NVCC"), "/usr/local/cuda/bin/nvcc", "nvcc"):
        if c and (os.path.isabs(c) and os.path.exists(c) or not os.path.isabs(c)):
            return c
    return "nvcc"


def _fingerprint():
    h = hashlib.sha256()
    for name in sorted(os.listdir(SRC)):
        with open(os.path.join(SRC, name), "rb") as f:
            h.update(name.encode() + f.read())
    with open(os.path.join(INCLUDE, "pfem2gpu.h"), "rb") as f:
        h.update(f.read())
    h.update(repr((ARCH, COMMON, SOURCES)).encode())
    return h.hexdigest()


def build(force: bool = False, verbose: bool = False) -> str:
    os.makedirs(OUT, exist_ok=True)
    stamp = os.path.join(OUT, "stamp")
    fp = _fingerprint()
    if not force and os.path.exists(LIB) and os.path.exists(stamp) and open(stamp).read() == fp:
        return LIB
    nvcc = _nvcc()
    objs = []
    log = []
    for name, extra in SOURCES.items():
        obj = os.path.join(OUT, name + ".o")
        cmd = [nvcc, *ARCH, *COMMON, *extra, "-c", os.path.join(SRC, name), "-o", obj]
        r = subprocess.run(cmd, capture_output=True, text=True)
        log.append(" ".join(cmd) + "\n" + r.stdout + r.stderr)
        if r.returncode != 0:
            sys.stderr.write(r.stdout + r.stderr)
            raise RuntimeError(f"nvcc failed on {name}")
        objs.append(obj)
    cmd = [nvcc, *ARCH, "-shared", "-o", LIB, *objs]
    r = subprocess.run(cmd, capture_output=True, text=True)
    log.append(" ".join(cmd) + "\n" + r.stdout + r.stderr)
    if r.returncode != 0:
        sys.stderr.write(r.stdout + r.stderr)
        raise RuntimeError("nvcc link failed")
    with open(os.path.join(OUT, "build.log"), "w") as f:
        f.write("\n".join(log))
    with open(stamp, "w") as f:
        f.write(fp)
    if verbose:
        print("\n".join(log))
    return LIB


if __name__ == "__main__":
    print(build(force="--force" in sys.argv, verbose="-v" in sys.argv))
