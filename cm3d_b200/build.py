"""Build libcm3d_nb.so (the CUDA engine + C ABI) in-tree for sm_100a.

    python -m cm3d_b200.build        # or cm3d_b200.build.build()

Sources that must reproduce CM3D's FP64 rounding (the list builder and the
plain FP64 pair kernels) are compiled with -fmad=false; the mixed-precision
kernels keep FMA contraction.  Host code is compiled without FP contraction
so the table builders round exactly as CM3D's C code does.
"""
from __future__ import annotations

import concurrent.futures as cf
import os
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
BUILD = os.path.join(HERE, "_build")
LIB = os.path.join(HERE, "libcm3d_nb.so")

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
COMMON = ["-O3", "-std=c++17", "-lineinfo", "--extended-lambda", "-Xptxas", "-v",
          "-Xcompiler", "-fPIC,-ffp-contract=off,-O2", "-I" + os.path.join(HERE, "..", "include")]
# (source, extra flags)
SOURCES = [
    ("nb_list.cu", ["-fmad=false"]),
    ("nb_plain.cu", ["-fmad=false"]),
    ("nb_pair.cu", []),
    ("nb_cwin.cu", []),
    ("nb_kspace.cu", []),
    ("nb_step.cu", []),
    ("nb_capi.cu", []),
]


def nvcc() -> str:
    for cand in (os.environ.get("NVCC"), shutil.which("nvcc"), "/usr/local/cuda/bin/nvcc"):
        if cand and os.path.exists(cand):
            return cand
    raise RuntimeError("nvcc not found")


def _compile(src: str, extra: list[str], verbose: bool) -> tuple[str, str]:
    obj = os.path.join(BUILD, src.replace(".cu", ".o"))
    cmd = [nvcc(), *ARCH, *COMMON, *extra, "-c", os.path.join(CSRC, src), "-o", obj]
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"nvcc failed for {src}:\n{r.stdout}\n{r.stderr}")
    return obj, r.stderr


def _stale() -> bool:
    if not os.path.exists(LIB):
        return True
    t = os.path.getmtime(LIB)
    deps = [os.path.join(CSRC, f) for f in os.listdir(CSRC)]
    deps.append(os.path.join(HERE, "..", "include", "cm3d_nb.h"))
    deps.append(os.path.abspath(__file__))
    return any(os.path.getmtime(d) > t for d in deps)


def build(force: bool = False, verbose: bool = False) -> str:
    if not force and not _stale():
        return LIB
    os.makedirs(BUILD, exist_ok=True)
    with cf.ThreadPoolExecutor(max_workers=len(SOURCES)) as ex:
        futs = [ex.submit(_compile, s, e, verbose) for s, e in SOURCES]
        results = [f.result() for f in futs]
    objs = [o for o, _ in results]
    if verbose:
        for _, log in results:
            sys.stdout.write(log)
    tmp = LIB + ".tmp"
    cmd = [nvcc(), *ARCH, "-shared", "-o", tmp, *objs, "-lcudart_static", "-lrt", "-ldl", "-lpthread"]
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"link failed:\n{r.stdout}\n{r.stderr}")
    os.replace(tmp, LIB)
    with open(os.path.join(BUILD, "ptxas.log"), "w") as fh:
        for _, log in results:
            fh.write(log)
    return LIB


if __name__ == "__main__":
    print(build(force="--force" in sys.argv, verbose="-v" in sys.argv))
