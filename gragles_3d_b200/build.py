"""Build the CUDA library ``libgg_b200.so`` in-tree for sm_100a.

Every kernel is compiled with ``-fmad=false`` so that no multiply-add is fused
unless the source asks for it with ``fma()``: the FP64 path relies on that to
reproduce the reference's arithmetic bit for bit.  Host code is compiled without
floating-point contraction for the same reason (the DFT twiddle and Gaussian
tables are built on the host).

    python -m gragles_3d_b200.build      (or call build())
"""
from __future__ import annotations

import concurrent.futures as cf
import os
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
OBJ = os.path.join(HERE, "_build")
LIB = os.path.join(HERE, "libgg_b200.so")
RUNNER = os.path.join(HERE, "gg_run")
SOURCES = ["gg_api.cu", "gg_plan.cu", "gg_conv_f64.cu", "gg_conv_tc.cu", "gg_conv_umma.cu", "gg_lists.cu", "gg_compare.cu",
           "gg_mc.cu", "gg_redist.cu", "gg_init.cu", "gg_noalloc.cu", "gg_hull.cu", "gg_coarsen.cu", "gg_rtree.cu"]
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]


def nvcc() -> str:
    for cand in (os.environ.get("NVCC"), "/usr/local/cuda/bin/nvcc", shutil.which("nvcc")):
        if cand and os.path.exists(cand):
            return cand
    raise RuntimeError("nvcc not found")


def flags() -> list[str]:
    return ARCH + ["-O3", "-lineinfo", "-std=c++17", "-fmad=false", "-ccbin", "g++",
                   "-Xcompiler", "-fPIC,-ffp-contract=off,-O2", "-Xptxas", "-O3"]


def _stale(src: str, obj: str) -> bool:
    if not os.path.exists(obj):
        return True
    t = os.path.getmtime(obj)
    deps = [src] + [os.path.join(CSRC, f) for f in os.listdir(CSRC) if f.endswith((".cuh", ".inc"))]
    deps.append(os.path.join(os.path.dirname(HERE), "include", "gg_b200.h"))
    return any(os.path.getmtime(d) > t for d in deps)


def build(verbose: bool = False) -> str:
    os.makedirs(OBJ, exist_ok=True)
    cc = nvcc()
    jobs = []
    for s in SOURCES:
        src = os.path.join(CSRC, s)
        obj = os.path.join(OBJ, s.replace(".cu", ".o"))
        if _stale(src, obj):
            jobs.append([cc] + flags() + ["-c", src, "-o", obj])

    def run(cmd):
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError(f"nvcc failed:\n{' '.join(cmd)}\n{r.stdout}\n{r.stderr}")
        if verbose and (r.stdout or r.stderr):
            print(r.stdout + r.stderr)
        return r

    with cf.ThreadPoolExecutor(max_workers=min(8, os.cpu_count() or 1)) as ex:
        list(ex.map(run, jobs))
    objs = [os.path.join(OBJ, s.replace(".cu", ".o")) for s in SOURCES]
    if jobs or not os.path.exists(LIB):
        run([cc] + ARCH + ["-shared", "-o", LIB] + objs + ["-lcudart"])
    # the C++ host driver (gg_run): the reference's mode-4 run through the C ABI
    host_src = os.path.join(HERE, "host", "gg_run.cpp")
    if not os.path.exists(RUNNER) or os.path.getmtime(RUNNER) < max(os.path.getmtime(host_src), os.path.getmtime(LIB)):
        run(["g++", "-O2", "-std=c++17", "-ffp-contract=off", host_src, "-I",
             os.path.join(os.path.dirname(HERE), "include"), "-L", HERE, "-lgg_b200", "-Wl,-rpath,$ORIGIN",
             "-o", RUNNER])
    return LIB


if __name__ == "__main__":
    print(build(verbose="-v" in sys.argv))
