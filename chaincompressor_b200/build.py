"""Builds the native parts of chaincompressor_b200 in-tree (sm_100a only).

* ``libchain_b200.so``           CUDA kernels + host orchestration + the C ABI
                                 (include/chain_b200.h)
* ``lcps_gpu_cpp.so``            pybind11 module, same surface as the reference's
                                 lcps_gpu_cpp (cu/chain/lcps_gpu_cpp.cu:1095-1102)
* ``lcps_gpu_decompress_ans.so`` pybind11 module, same surface as the reference's
                                 lcps_gpu_decompress_ans (.../lcps_gpu_decompress_ans.cu:2898-2921)

FP64 exactness: no fast-math, ``--fmad=false`` (no contraction of a*b+c), IEEE
division and square root; the only fused multiply-add is the explicit ``fma()`` of
the reconstruction rule.

Run ``python -m chaincompressor_b200.build`` (or ``__graft_entry__.build()``).
"""
from __future__ import annotations

import os
import subprocess
import sys
import sysconfig
from concurrent.futures import ThreadPoolExecutor
from pathlib import Path

PKG = Path(__file__).resolve().parent
ROOT = PKG.parent
CSRC = PKG / "csrc"
OBJ = PKG / "_build"
CUDA_HOME = Path(os.environ.get("CUDA_HOME", "/usr/local/cuda"))
NVCC = str(CUDA_HOME / "bin" / "nvcc")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVCC_FLAGS = ARCH + ["-O3", "-lineinfo", "-std=c++17", "--fmad=false", "-prec-div=true", "-prec-sqrt=true",
                     "-ftz=false", "-Xcompiler", "-fPIC", "-Xcompiler", "-fvisibility=hidden",
                     "--expt-relaxed-constexpr", "-Xptxas", "-warn-spills"]
LIB_SOURCES = ["capi.cu", "encode.cu", "decode.cu", "noalloc.cu", "batch.cu", "server.cu", "transcode.cu"]
HEADERS = ["chain_common.cuh", "chain_format.h", "ctx.h", "radix_sort.cuh", "rans.cuh", "scan.cuh"]
LIB = PKG / "libchain_b200.so"
PYMODS = {"lcps_gpu_cpp": "pymod_compress.cpp", "lcps_gpu_decompress_ans": "pymod_decompress.cpp"}


def _newer(target: Path, deps) -> bool:
    if not target.exists():
        return True
    t = target.stat().st_mtime
    return any(Path(d).stat().st_mtime > t for d in deps)


def _run(cmd):
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError("build failed:\n" + " ".join(cmd) + "\n" + r.stdout + r.stderr)
    return r.stdout + r.stderr


def build(verbose: bool = False, force: bool = False) -> Path:
    OBJ.mkdir(exist_ok=True)
    headers = [CSRC / h for h in HEADERS] + [ROOT / "include" / "chain_b200.h"]
    jobs = []
    objs = []
    for src in LIB_SOURCES:
        obj = OBJ / (Path(src).stem + ".o")
        objs.append(obj)
        if force or _newer(obj, [CSRC / src] + headers + [Path(__file__)]):
            jobs.append([NVCC, *NVCC_FLAGS, "-I", str(ROOT / "include"), "-c", str(CSRC / src), "-o", str(obj)])
    with ThreadPoolExecutor(max_workers=len(jobs) or 1) as ex:
        for out in ex.map(_run, jobs):
            if verbose and out.strip():
                print(out)
    if force or _newer(LIB, objs):
        _run([NVCC, *ARCH, "-shared", "-o", str(LIB), *map(str, objs), "-lcudart"])
    py_inc = sysconfig.get_paths()["include"]
    import pybind11

    ext = ".so"
    for mod, src in PYMODS.items():
        target = PKG / f"{mod}{ext}"
        if force or _newer(target, [CSRC / src, LIB, ROOT / "include" / "chain_b200.h"]):
            _run(["g++", "-O2", "-std=c++17", "-shared", "-fPIC", "-fvisibility=hidden",
                  "-I", py_inc, "-I", pybind11.get_include(), "-I", str(ROOT / "include"),
                  "-I", str(CUDA_HOME / "include"), str(CSRC / src), "-o", str(target),
                  "-L", str(PKG), "-lchain_b200", "-Wl,-rpath,$ORIGIN",
                  "-L", str(CUDA_HOME / "lib64"), "-lcudart"])
    return LIB


if __name__ == "__main__":
    build(verbose="-v" in sys.argv, force="-f" in sys.argv)
    print("built", LIB)
