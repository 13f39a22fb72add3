"""Build the sm_100a library libopenpfc_b200.so in place (next to this file).

usage: python -m openpfc_b200.build [--force] [--jobs N]

Each .cu under csrc/ is compiled by nvcc for `-gencode
arch=compute_100a,code=sm_100a` with -lineinfo and linked into one shared
library with a C ABI (include/openpfc_b200.h).  The CUDA runtime is linked
statically, so the library needs only the driver at run time.
"""
from __future__ import annotations

import argparse
import concurrent.futures as cf
import os
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
BUILD = os.path.join(HERE, "_build")
LIB = os.path.join(HERE, "libopenpfc_b200.so")
SOURCES = ["kernels_f32.cu", "kernels_f64.cu", "ensemble_f32.cu", "ensemble_f64.cu", "opfc.cu", "noalloc.cu",
           "ensemble.cu", "io.cu", "wait_check.cu"]
HEADERS = ["fft_core.cuh", "kernels.cuh", "launch.h", "col_tma.cuh", "x_tma.cuh", "x_sq.cuh", "twiddle.h",
           "ensemble.cuh", "autotune.h", "io.h"]

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVCC_FLAGS = ARCH + ["-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC",
                     "--expt-relaxed-constexpr", "-ccbin", "g++",
                     "-I" + os.path.join(ROOT, "include"), "-I" + CSRC]


def nvcc() -> str:
    for cand in (shutil.which("nvcc"), "/usr/local/cuda/bin/nvcc"):
        if cand and os.path.exists(cand):
            return cand
    raise RuntimeError("nvcc not found; the CUDA toolkit is required to build openpfc_b200")


def _stale(target: str, deps) -> bool:
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(d) > t for d in deps)


def _deps(obj: str, src: str):
    """Headers the object was built from (nvcc -MD file), else every header."""
    dfile = obj[:-2] + ".d"
    if os.path.exists(dfile):
        with open(dfile) as f:
            text = f.read().replace("\\\n", " ")
        files = [t for t in text.split(":", 1)[-1].split() if t.startswith(ROOT)]
        if files and all(os.path.exists(t) for t in files):
            return files
    return [os.path.join(CSRC, src)] + [os.path.join(CSRC, h) for h in HEADERS] + \
        [os.path.join(ROOT, "include", "openpfc_b200.h")]


def _compile(src: str, extra) -> str:
    obj = os.path.join(BUILD, os.path.splitext(src)[0] + ".o")
    if _stale(obj, _deps(obj, src)):
        cmd = [nvcc()] + NVCC_FLAGS + list(extra) + ["-MD", "-MF", obj[:-2] + ".d",
                                                     "-c", os.path.join(CSRC, src), "-o", obj]
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError(f"nvcc failed for {src}:\n{r.stdout}\n{r.stderr}")
    return obj


def build(force: bool = False, jobs: int = 3, extra=()) -> str:
    os.makedirs(BUILD, exist_ok=True)
    if force:
        for f in os.listdir(BUILD):
            os.remove(os.path.join(BUILD, f))
    with cf.ThreadPoolExecutor(max_workers=jobs) as ex:
        objs = list(ex.map(lambda s: _compile(s, extra), SOURCES))
    if force or _stale(LIB, objs):
        cmd = [nvcc()] + ARCH + ["-shared", "-o", LIB] + objs + ["-lpthread"]
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError(f"link failed:\n{r.stdout}\n{r.stderr}")
    return LIB


def main(argv=None) -> int:
    ap = argparse.ArgumentParser()
    ap.add_argument("--force", action="store_true")
    ap.add_argument("--jobs", type=int, default=3)
    ap.add_argument("--verbose-ptxas", action="store_true")
    a = ap.parse_args(argv)
    extra = ["-Xptxas", "-v"] if a.verbose_ptxas else []
    print(build(force=a.force, jobs=a.jobs, extra=extra))
    return 0


if __name__ == "__main__":
    sys.exit(main())
