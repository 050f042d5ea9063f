"""Build libbqb_gpu.so (the C-ABI library) in-tree with nvcc for sm_100a.

``python -m parallel_biqbin_maxcut_b200.build`` compiles every ``csrc/*.cu``
and ``csrc/*.cpp`` into ``parallel_biqbin_maxcut_b200/lib/libbqb_gpu.so``.
Objects are rebuilt when a source or any header is newer than them.
"""
from __future__ import annotations

import concurrent.futures as cf
import glob
import os
import shutil
import subprocess
import sys

PKG = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(PKG)
CSRC = os.path.join(PKG, "csrc")
OBJ = os.path.join(PKG, "_build")
LIBDIR = os.path.join(PKG, "lib")
LIB = os.path.join(LIBDIR, "libbqb_gpu.so")

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
# -fmad=false: no multiply and add is contracted into an FMA behind the
# source's back.  The device bodies shared by the bounding kernels (IPM,
# bundle, cut operators, annealing) are inlined into several kernels, and the
# compiler's contraction choices could differ between those contexts; with
# contraction off, every FMA is one the source writes (fma()), so every
# kernel that runs a body computes the same bits.  The hot loops already
# write their FMAs explicitly.
NVCC_FLAGS = ARCH + [
    "-O3", "-lineinfo", "-std=c++17", "--extended-lambda", "-fmad=false", "-Xcompiler", "-fPIC,-fvisibility=hidden",
    "-I" + os.path.join(ROOT, "include"),
]


CUDA_HOME = os.environ.get("CUDA_HOME", "/usr/local/cuda")
# Host-only C++ sources are compiled with g++.  host_sep.cpp restates the
# reference's simulated annealing and takes the reference's floating-point
# flags (-O3 -ffast-math, reference Makefile:17) so its accept/reject
# decisions match the reference build.
CXX_FLAGS = ["-O3", "-fPIC", "-fvisibility=hidden", "-std=c++17", "-I" + os.path.join(ROOT, "include"),
             "-I" + os.path.join(CUDA_HOME, "include")]
PER_FILE_FLAGS = {"host_sep.cpp": ["-ffast-math"]}


def nvcc() -> str:
    for cand in (os.environ.get("NVCC"), shutil.which("nvcc"), "/usr/local/cuda/bin/nvcc"):
        if cand and os.path.exists(cand):
            return cand
    raise RuntimeError("nvcc not found")


def _headers_mtime() -> float:
    hs = glob.glob(os.path.join(CSRC, "*.h")) + glob.glob(os.path.join(CSRC, "*.cuh")) + \
        glob.glob(os.path.join(ROOT, "include", "*.h"))
    return max((os.path.getmtime(h) for h in hs), default=0.0)


def _compile(src: str, hdr_mtime: float, extra: list[str]) -> str:
    obj = os.path.join(OBJ, os.path.basename(src) + ".o")
    if os.path.exists(obj) and os.path.getmtime(obj) >= max(os.path.getmtime(src), hdr_mtime):
        return obj
    if src.endswith(".cpp"):
        cmd = ["g++"] + CXX_FLAGS + PER_FILE_FLAGS.get(os.path.basename(src), []) + ["-c", src, "-o", obj]
    else:
        cmd = [nvcc()] + NVCC_FLAGS + extra + ["-c", src, "-o", obj]
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"nvcc failed on {src}:\n{r.stdout}\n{r.stderr}")
    return obj


def build(verbose: bool = False, extra: list[str] | None = None) -> str:
    os.makedirs(OBJ, exist_ok=True)
    os.makedirs(LIBDIR, exist_ok=True)
    # objects built with other flags are rebuilt
    stamp = os.path.join(OBJ, "flags.txt")
    flags = " ".join(NVCC_FLAGS + CXX_FLAGS + (extra or []))
    if not os.path.exists(stamp) or open(stamp).read() != flags:
        for o in glob.glob(os.path.join(OBJ, "*.o")):
            os.remove(o)
        with open(stamp, "w") as fh:
            fh.write(flags)
    srcs = sorted(glob.glob(os.path.join(CSRC, "*.cu")) + glob.glob(os.path.join(CSRC, "*.cpp")))
    hm = _headers_mtime()
    with cf.ThreadPoolExecutor(max_workers=min(8, os.cpu_count() or 2)) as ex:
        objs = list(ex.map(lambda s: _compile(s, hm, extra or []), srcs))
    newest = max(os.path.getmtime(o) for o in objs)
    if not os.path.exists(LIB) or os.path.getmtime(LIB) < newest:
        cmd = [nvcc()] + ARCH + ["-shared", "-o", LIB] + objs + [
            "-Xlinker", "-Bsymbolic-functions", "-lcudart", "-lpthread"]
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError(f"link failed:\n{r.stdout}\n{r.stderr}")
    if verbose:
        print(LIB)
    return LIB


def ptxas_report() -> str:
    """Registers / spills / smem per kernel (-Xptxas -v), for profiling notes."""
    out = []
    for src in sorted(glob.glob(os.path.join(CSRC, "*.cu"))):
        cmd = [nvcc()] + NVCC_FLAGS + ["-Xptxas", "-v", "-c", src, "-o", os.devnull]
        r = subprocess.run(cmd, capture_output=True, text=True)
        out.append(f"== {os.path.basename(src)}\n{r.stderr}")
    return "\n".join(out)


if __name__ == "__main__":
    if len(sys.argv) > 1 and sys.argv[1] == "--ptxas":
        print(ptxas_report())
    else:
        build(verbose=True)
