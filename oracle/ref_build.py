"""Builds oracle/_ref/libykref.so: the reference YKCBCT CUDA implementation of
the FDK and Joseph paths, compiled for sm_100a from its own source files where
they lie (never copied), plus oracle/ref_driver.cu.  TEST INFRASTRUCTURE ONLY:
the parity tests and the reference timing use it; the product never does.

The recipe follows the reference's CMake settings for its library target
(CMakeLists.txt:106-160): CUDA flags ``-O3 -use_fast_math --extended-lambda``,
``NDEBUG``, ``YKCBCT_HAS_HELICAL=0``, include dirs ``include``, ``src``,
``src/util`` and the vendored header-only spdlog, linked against cudart and
cuFFT.  Only the translation units on the FDK / flat FP-BP path are compiled.

One shim header is generated into oracle/_ref/shim.  It is needed because
src/FlatFpBp/BP/kernels/YkFlatJosephBpLaunch.cuh:4 includes
``FlatFpBp/BP/YkBpCommon.cuh``, while the file is ``YkBPCommon.cuh``; the
reference was developed on a case-insensitive file system.

Usage: python oracle/ref_build.py [--reference DIR] [-j N]
The reference tree is DIR, else $YKB_REFERENCE_DIR, else /root/reference.
Exits 0 without building when the reference tree is absent.
"""
from __future__ import annotations

import argparse
import concurrent.futures as cf
import hashlib
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
OUT = os.path.join(HERE, "_ref")
DEFAULT_REFERENCE = os.environ.get("YKB_REFERENCE_DIR", "/root/reference")


def reference_present(reference: str = DEFAULT_REFERENCE) -> bool:
    return os.path.isdir(os.path.join(reference, "src"))


# translation units of the FDK pipeline, the flat FP/BP operators and the
# iterative vector kernels their CGLS uses
SOURCES = [
    "src/Reconstruction/Analytic/Circular/Flat/FDK/kernels/YkFDKBpKernels.cu",
    "src/Reconstruction/Analytic/Circular/Flat/FDK/kernels/YkFDKBpPrecompute.cu",
    "src/Reconstruction/Analytic/Circular/Flat/FDK/kernels/YkFDKPreWeightKernels.cu",
    "src/Reconstruction/Analytic/Circular/Flat/FDK/kernels/YkFDKFilterKernels.cu",
    "src/Reconstruction/Analytic/Circular/Flat/FDK/kernels/YkFDKParkerKernels.cu",
    "src/Filter/YkCreateFilterKernelKernels.cu",
    "src/Filter/YkConvKernels.cu",
    "src/FlatFpBp/FP/kernels/YkFPKernels.cu",
    "src/FlatFpBp/FP/kernels/YkFlatFootprintKernels.cu",
    "src/FlatFpBp/FP/kernels/YkFPSiddonKernel.cu",
    "src/FlatFpBp/BP/kernels/YkBpFdkKernel.cu",
    "src/FlatFpBp/BP/kernels/YkBPJosephKernel.cu",
    "src/FlatFpBp/BP/kernels/YkBPSiddonKernel.cu",
    "src/Reconstruction/Iterative/Common/kernels/YkIterKernels.cu",
    "src/global/YkLog.cpp",
]

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
DEFINES = ["-DNDEBUG", "-DYKCBCT_EXPORTS", "-DYKCBCT_HAS_HELICAL=0"]
CUDA_FLAGS = ["-O3", "-use_fast_math", "--extended-lambda", "-std=c++17", "-Xcompiler", "-fPIC",
              "-w"]


def _shim() -> str:
    d = os.path.join(OUT, "shim", "FlatFpBp", "BP")
    os.makedirs(d, exist_ok=True)
    with open(os.path.join(d, "YkBpCommon.cuh"), "w") as f:
        f.write('#pragma once\n#include "FlatFpBp/BP/YkBPCommon.cuh"\n')
    return os.path.join(OUT, "shim")


def _includes(ref: str) -> list[str]:
    return ["-I", _shim(), "-I", os.path.join(ref, "src"), "-I", os.path.join(ref, "src", "util"),
            "-I", os.path.join(ref, "include"),
            "-isystem", os.path.join(ref, "thirdparty", "spdlog", "include"),
            "-I", os.path.join(ROOT, "include")]


def _compile(src: str, obj: str, inc: list[str]) -> tuple[str, int, str]:
    cmd = ["nvcc", *ARCH, *CUDA_FLAGS, *DEFINES, *inc, "-c", src, "-o", obj]
    if src.endswith(".cpp"):
        cmd = ["nvcc", "-x", "cu", *cmd[1:]]
    r = subprocess.run(cmd, capture_output=True, text=True)
    return src, r.returncode, r.stderr


def build(reference: str = DEFAULT_REFERENCE, jobs: int = 8) -> str | None:
    if not reference_present(reference):
        print(f"reference tree not found at {reference}; oracle/_ref not built")
        return None
    objdir = os.path.join(OUT, "obj")
    os.makedirs(objdir, exist_ok=True)
    inc = _includes(reference)
    todo = []
    objs = []
    for rel in SOURCES + [os.path.join(HERE, "ref_driver.cu")]:
        src = rel if os.path.isabs(rel) else os.path.join(reference, rel)
        obj = os.path.join(objdir, os.path.basename(src).rsplit(".", 1)[0] + ".o")
        objs.append(obj)
        stamp = obj + ".sha1"
        with open(src, "rb") as f:
            key = hashlib.sha1(f.read() + " ".join(ARCH + CUDA_FLAGS + DEFINES).encode()).hexdigest()
        if os.path.exists(obj) and os.path.exists(stamp) and open(stamp).read() == key:
            continue
        todo.append((src, obj, stamp, key))
    with cf.ThreadPoolExecutor(max_workers=jobs) as ex:
        futs = {ex.submit(_compile, s, o, inc): (s, o, st, k) for s, o, st, k in todo}
        for fut in cf.as_completed(futs):
            s, o, st, k = futs[fut]
            _, rc, err = fut.result()
            if rc != 0:
                raise RuntimeError(f"nvcc failed on {s}:\n{err[-4000:]}")
            with open(st, "w") as f:
                f.write(k)
    lib = os.path.join(OUT, "libykref.so")
    cmd = ["nvcc", *ARCH, "-shared", "-o", lib, *objs, "-lcufft", "-Xcompiler", "-fopenmp"]
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"link failed:\n{r.stderr[-4000:]}")
    return lib


def main() -> int:
    ap = argparse.ArgumentParser()
    ap.add_argument("--reference", default=DEFAULT_REFERENCE)
    ap.add_argument("-j", type=int, default=8)
    a = ap.parse_args()
    lib = build(a.reference, a.j)
    if lib:
        print(lib)
    return 0


if __name__ == "__main__":
    sys.exit(main())
