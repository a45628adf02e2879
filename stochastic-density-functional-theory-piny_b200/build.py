"""Build the sm_100a library lib/libsdft_b200.so with nvcc (in tree).

Each translation unit compiles in parallel to an object in _build/, then
they link into one shared library (cudart linked statically, so the
library loads on hosts without a GPU for ABI checks)."""
from __future__ import annotations

import concurrent.futures as cf
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
OUT = os.path.join(HERE, "lib", "libsdft_b200.so")
BUILD = os.path.join(HERE, "_build")
SOURCES = ["sdft_host.cpp", "sdft_api.cu", "sdft_kernels.cu", "sdft_kernels2.cu", "sdft_kb.cu", "sdft_gemm_oz.cu",
           "sdft_noalloc.cu", "sdft_noise.cu", "sdft_lanczos.cu",
           "sdft_mixer.cu", "sdft_xc.cu", "sdft_vks.cu"]
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
FLAGS = ["-O3", "-std=c++17", "-lineinfo", "-Xcompiler", "-fPIC,-ffp-contract=off", "-Xptxas", "-O3"]


def _nvcc():
    for c in (os.environ.get("NVCC"), "/usr/local/cuda/bin/nvcc", "nvcc"):
        if c and (os.path.sep not in c or os.path.exists(c)):
            return c
    raise RuntimeError("nvcc not found")


def _stale(obj, deps):
    if not os.path.exists(obj):
        return True
    t = os.path.getmtime(obj)
    return any(os.path.getmtime(d) > t for d in deps)


def build(verbose=False, force=False):
    os.makedirs(BUILD, exist_ok=True)
    os.makedirs(os.path.dirname(OUT), exist_ok=True)
    nvcc = _nvcc()
    headers = [os.path.join(CSRC, f) for f in os.listdir(CSRC) if f.endswith((".h", ".cuh"))]
    headers.append(os.path.join(HERE, "..", "include", "sdft_b200.h"))
    srcs = [s for s in SOURCES if os.path.exists(os.path.join(CSRC, s))]
    jobs = []
    for s in srcs:
        src = os.path.join(CSRC, s)
        obj = os.path.join(BUILD, s + ".o")
        if force or _stale(obj, [src] + headers):
            jobs.append([nvcc, *ARCH, *FLAGS, "-c", src, "-o", obj])
    def run(cmd):
        r = subprocess.run(cmd, capture_output=True, text=True)
        return cmd, r
    with cf.ThreadPoolExecutor(max_workers=max(1, min(len(jobs), os.cpu_count() or 4))) as ex:
        for cmd, r in ex.map(run, jobs):
            if verbose or r.returncode:
                sys.stderr.write(" ".join(cmd) + "\n" + r.stdout + r.stderr)
            if r.returncode:
                raise RuntimeError(f"nvcc failed: {cmd[-3]}")
    objs = [os.path.join(BUILD, s + ".o") for s in srcs]
    if force or jobs or _stale(OUT, objs):
        cmd = [nvcc, *ARCH, "-shared", "-o", OUT, *objs]
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode:
            sys.stderr.write(r.stdout + r.stderr)
            raise RuntimeError("link failed")
    return OUT


if __name__ == "__main__":
    print(build(verbose="-v" in sys.argv, force="-f" in sys.argv))
