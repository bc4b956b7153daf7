"""Build the engine's shared library for sm_100a (in-tree).

    python -m xatu_b200.build        ->  xatu_b200/_lib/libxatu_bse.so

nvcc compiles every CUDA source with ``-gencode arch=compute_100a,code=sm_100a``
(objects in parallel), then links one shared object against cuBLAS and cuSOLVER.
"""
from __future__ import annotations

import concurrent.futures as cf
import os
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
OUT_DIR = os.path.join(HERE, "_lib")
OBJ_DIR = os.path.join(OUT_DIR, "obj")
LIB = os.path.join(OUT_DIR, "libxatu_bse.so")

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
COMMON = ["-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC", "-Xcompiler", "-O3",
          "--expt-relaxed-constexpr", "-I" + os.path.join(HERE, "..", "include")]
SOURCES = ["api.cu", "geometry.cpp", "lattice_kernels.cu", "bands.cu", "bands_select.cu", "assembly.cu", "assembly_f32.cu", "assembly_f64.cu", "assembly_batch.cu", "dense.cu", "hx.cu",
           "hx_tc.cu", "hx_noalloc.cu", "davidson.cu", "oscillator.cu", "postproc.cu", "adjoint.cu", "batch.cu", "osc_grad.cu"]


def _nvcc() -> str:
    for cand in (shutil.which("nvcc"), "/usr/local/cuda/bin/nvcc"):
        if cand and os.path.exists(cand):
            return cand
    raise RuntimeError("nvcc not found")


def _compile(src: str, verbose_ptxas: bool) -> str:
    obj = os.path.join(OBJ_DIR, os.path.splitext(src)[0] + ".o")
    path = os.path.join(CSRC, src)
    deps = [os.path.join(CSRC, f) for f in os.listdir(CSRC)]
    if os.path.exists(obj) and os.path.getmtime(obj) >= max(os.path.getmtime(d) for d in deps) and not verbose_ptxas:
        return obj
    cmd = [_nvcc(), "-c", path, "-o", obj] + ARCH + COMMON
    if src.endswith(".cpp"):
        cmd = [_nvcc(), "-x", "cu", "-c", path, "-o", obj] + ARCH + COMMON
    if verbose_ptxas:
        cmd += ["-Xptxas", "-v"]
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"nvcc failed for {src}:\n{r.stdout}\n{r.stderr}")
    if verbose_ptxas:
        sys.stderr.write(r.stderr)
    return obj


def build(force: bool = False, verbose_ptxas: bool = False) -> str:
    os.makedirs(OBJ_DIR, exist_ok=True)
    if force:
        for f in os.listdir(OBJ_DIR):
            os.remove(os.path.join(OBJ_DIR, f))
    with cf.ThreadPoolExecutor(max_workers=min(8, os.cpu_count() or 4)) as ex:
        objs = list(ex.map(lambda s: _compile(s, verbose_ptxas), SOURCES))
    newest = max(os.path.getmtime(o) for o in objs)
    if force or not os.path.exists(LIB) or os.path.getmtime(LIB) < newest:
        # cuBLAS / cuSOLVER of the CUDA toolkit the kernels are built with (explicit run path)
        cudalib = os.path.join(os.path.dirname(os.path.dirname(os.path.realpath(_nvcc()))), "lib64")
        cmd = [_nvcc(), "-shared", "-o", LIB] + objs + ARCH + ["-lcublas", "-lcusolver", "-Xlinker", "-rpath",
                                                               "-Xlinker", cudalib]
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError(f"link failed:\n{r.stdout}\n{r.stderr}")
    return LIB


if __name__ == "__main__":
    print(build(force="--force" in sys.argv, verbose_ptxas="-v" in sys.argv))
