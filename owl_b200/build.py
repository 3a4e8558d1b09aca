"""In-tree build of the sm_100a shared library (nvcc, no JIT cache): every
translation unit compiled in parallel, then linked into one .so."""
from __future__ import annotations

import os
import subprocess
from concurrent.futures import ThreadPoolExecutor

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
LIB = os.path.join(HERE, "lib", "libowl_ssg.so")
OBJ = os.path.join(HERE, "lib", "obj")
SOURCES = ["shared.cu", "ssg_base.cu", "ac2d.cu", "ac3d.cu", "el2d.cu", "el3d.cu", "adjsrc.cu", "dtw.cu", "su.cu",
           "optim.cu", "capi.cu", "noalloc.cu", "mpml.cu"]
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVCC_FLAGS = ["-O3", "-std=c++17"] + ARCH + ["-lineinfo", "-Xcompiler", "-fPIC"]


def nvcc() -> str:
    for p in (os.environ.get("NVCC"), "/usr/local/cuda/bin/nvcc", "nvcc"):
        if p and (os.path.sep not in p or os.path.exists(p)):
            return p
    return "nvcc"


def stale() -> bool:
    if not os.path.exists(LIB):
        return True
    t = os.path.getmtime(LIB)
    deps = [os.path.join(CSRC, f) for f in os.listdir(CSRC)] + [os.path.join(HERE, "..", "include", "owl_ssg.h")]
    return any(os.path.getmtime(d) > t for d in deps if os.path.exists(d))


def build_library(force: bool = False, verbose: bool = False) -> str:
    if not force and not stale():
        return LIB
    os.makedirs(OBJ, exist_ok=True)
    jobs = []
    for src in SOURCES:
        obj = os.path.join(OBJ, src.replace(".cu", ".o"))
        jobs.append(([nvcc()] + NVCC_FLAGS + ["-c", os.path.join(CSRC, src), "-o", obj], obj))

    def run(cmd):
        if verbose:
            print(" ".join(cmd))
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError(f"nvcc failed: {' '.join(cmd)}\n{r.stdout}\n{r.stderr}")
        return r

    with ThreadPoolExecutor(max_workers=max(1, min(len(jobs), os.cpu_count() or 1))) as ex:
        list(ex.map(run, [c for c, _ in jobs]))
    run([nvcc()] + ARCH + ["-shared", "-cudart", "static", "-o", LIB] + [o for _, o in jobs])
    return LIB


if __name__ == "__main__":
    print(build_library(force=True, verbose=True))
