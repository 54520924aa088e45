"""Build libdimgpu.so (the CUDA kernels + C-ABI) in-tree for sm_100a.

    python -m diffuse_vs_gfm_mms_b200.build

Each translation unit is compiled by nvcc in parallel; the shared library is
written next to this file so it travels with the source tree.  FP64 rounding
parity with the reference requires -fmad=false (the reference is compiled
without FMA contraction).
"""
from __future__ import annotations

import os
import subprocess
import sys
from concurrent.futures import ThreadPoolExecutor

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
OBJ = os.path.join(HERE, "_build")
LIB = os.path.join(HERE, "libdimgpu.so")
# bench.py's FP64 throughput probe, kept out of the C-ABI library
PROBE_LIB = os.path.join(HERE, "libdimprobe.so")
PROBE_SRC = os.path.join(CSRC, "fp64_peak.cu")

NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
FLAGS = ["-O3", "-std=c++17", "-lineinfo", "-fmad=false", "-Xcompiler", "-fPIC",
         "-ccbin", "g++", f"-I{os.path.join(ROOT, 'include')}", f"-I{CSRC}"]
SOURCES = ["inst_nm1.cu", "inst_nm2.cu", "inst_nm3.cu", "inst_nm4.cu", "inst_euler.cu", "dimgpu_api.cu",
           "dimgpu_noalloc.cu", "dimgpu_batch.cu", "dimgpu_io.cu", "dimgpu_server.cu", "dimgpu_slabs.cu"]
HEADERS = ["dim_physics.h", "dim_line.h", "dim_kernels.cuh", "dim_launch.h", "dim_batch.cuh", "dim_mixed.h",
           "dimgpu_validate.h", "dimgpu_session.h", "dim_io.cuh", "range_alloc.h", "pdl.cuh", "fastdiv.h",
           "euler_physics.h", "euler_kernels.cuh"]


def _mtime(p):
    return os.path.getmtime(p) if os.path.exists(p) else 0.0


def _compile(src: str, verbose: bool, extra) -> str:
    obj = os.path.join(OBJ, src.replace(".cu", ".o"))
    deps = [os.path.join(CSRC, src)] + [os.path.join(CSRC, h) for h in HEADERS] + \
        [os.path.join(ROOT, "include", "dimgpu.h")]
    if _mtime(obj) >= max(_mtime(d) for d in deps) and not extra:
        return obj
    cmd = [NVCC, *ARCH, *FLAGS, *extra, "-c", os.path.join(CSRC, src), "-o", obj]
    if verbose:
        print(" ".join(cmd), flush=True)
    out = subprocess.run(cmd, capture_output=True, text=True)
    if out.returncode != 0:
        raise RuntimeError(f"nvcc failed on {src}:\n{out.stdout}\n{out.stderr}")
    if verbose and out.stderr.strip():
        print(out.stderr, flush=True)
    return obj


def build(verbose: bool = False, ptxas_verbose: bool = False) -> str:
    os.makedirs(OBJ, exist_ok=True)
    extra = ["-Xptxas", "-v"] if ptxas_verbose else []
    with ThreadPoolExecutor(max_workers=len(SOURCES)) as ex:
        objs = list(ex.map(lambda s: _compile(s, verbose or ptxas_verbose, extra), SOURCES))
    if _mtime(LIB) < max(_mtime(o) for o in objs) or extra:
        cmd = [NVCC, *ARCH, "-shared", "-o", LIB, *objs, "-lcudart_static", "-ldl", "-lrt", "-lpthread"]
        out = subprocess.run(cmd, capture_output=True, text=True)
        if out.returncode != 0:
            raise RuntimeError(f"link failed:\n{out.stdout}\n{out.stderr}")
    if _mtime(PROBE_LIB) < _mtime(PROBE_SRC):
        cmd = [NVCC, *ARCH, "-O3", "-std=c++17", "-Xcompiler", "-fPIC", "-shared", PROBE_SRC, "-o", PROBE_LIB,
               "-lcudart_static", "-ldl", "-lrt", "-lpthread"]
        out = subprocess.run(cmd, capture_output=True, text=True)
        if out.returncode != 0:
            raise RuntimeError(f"nvcc failed on fp64_peak.cu:\n{out.stdout}\n{out.stderr}")
    return LIB


if __name__ == "__main__":
    build(verbose=True, ptxas_verbose="-v" in sys.argv)
    print(LIB)
