"""Builds ``libmsb200.so`` in-tree for sm_100a, and its checked twin
``libmsb200_checked.so`` (``MSB_DEVICE_CHECKS=1``: the hot gathers check
their indices and report MSB_ERR_DEVICE_CHECK instead of reading out of
range; for debugging and its own tests, not for timing).

CUDA sources are compiled by nvcc with ``--fmad=false`` (no contracted
multiply-adds, so FP32 results round like the reference's) and IEEE division
and square root; the host engine is C++23 compiled by g++.  The CUDA runtime is
linked statically so the library loads without a toolkit on the path.
"""

from __future__ import annotations

import os
import shutil
import subprocess
import sys
from concurrent.futures import ThreadPoolExecutor
from pathlib import Path

PACKAGE = Path(__file__).resolve().parent
CSRC = PACKAGE / "csrc"
BUILD = PACKAGE / "_build"
OUTPUT = PACKAGE / "libmsb200.so"
CHECKED_OUTPUT = PACKAGE / "libmsb200_checked.so"
INCLUDE = PACKAGE.parent / "include"

CUDA_HOME = Path(os.environ.get("CUDA_HOME", "/usr/local/cuda"))
NVCC = str(CUDA_HOME / "bin" / "nvcc")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVCC_FLAGS = [
    *ARCH,
    "-O3",
    "-lineinfo",
    "--fmad=false",
    "-prec-div=true",
    "-prec-sqrt=true",
    "-std=c++20",
    "-Xcompiler",
    "-fPIC",
    "-Xptxas",
    "-v",
]
CXX_FLAGS = ["-std=gnu++23", "-O2", "-fPIC", "-Wall", f"-I{CUDA_HOME / 'include'}"]


def _sources():
    cu = sorted(CSRC.glob("*.cu"))
    cpp = sorted(CSRC.glob("*.cpp"))
    return cu, cpp


def _stale(target: Path, deps) -> bool:
    if not target.exists():
        return True
    mtime = target.stat().st_mtime
    return any(d.stat().st_mtime > mtime for d in deps)


def build(verbose: bool = False, force: bool = False, checked: bool = False) -> Path:
    """Compiles every CUDA and C++ source and links the shared library (the
    checked twin with ``checked``)."""
    if shutil.which(NVCC) is None and not Path(NVCC).exists():
        raise RuntimeError(f"nvcc not found at {NVCC}")
    build_dir = BUILD / "checked" if checked else BUILD
    output = CHECKED_OUTPUT if checked else OUTPUT
    nvcc_flags = [*NVCC_FLAGS, "-DMSB_DEVICE_CHECKS=1"] if checked else NVCC_FLAGS
    build_dir.mkdir(parents=True, exist_ok=True)
    cu, cpp = _sources()
    headers = list(CSRC.glob("*.h")) + list(CSRC.glob("*.cuh")) + list(INCLUDE.glob("*.h"))
    jobs = []
    objects = []
    for src in cu:
        obj = build_dir / (src.stem + ".cu.o")
        objects.append(obj)
        if force or _stale(obj, [src, *headers]):
            jobs.append([NVCC, *nvcc_flags, "-c", str(src), "-o", str(obj)])
    for src in cpp:
        obj = build_dir / (src.stem + ".o")
        objects.append(obj)
        if force or _stale(obj, [src, *headers]):
            jobs.append(["g++", *CXX_FLAGS, "-c", str(src), "-o", str(obj)])

    def run(cmd):
        result = subprocess.run(cmd, capture_output=True, text=True)
        if result.returncode != 0:
            raise RuntimeError(f"compile failed: {' '.join(cmd)}\n{result.stdout}\n{result.stderr}")
        return cmd, result.stderr

    with ThreadPoolExecutor(max_workers=min(8, os.cpu_count() or 1)) as pool:
        for cmd, log in pool.map(run, jobs):
            if verbose:
                print(" ".join(cmd[-3:]), file=sys.stderr)
                print(log, file=sys.stderr)
    if force or jobs or _stale(output, objects):
        link = [
            NVCC,
            *ARCH,
            "-shared",
            "-o",
            str(output),
            *map(str, objects),
            "-cudart=static",
            "-Xcompiler",
            "-fPIC",
            "-Xlinker",
            "--no-undefined",
        ]
        result = subprocess.run(link, capture_output=True, text=True)
        if result.returncode != 0:
            raise RuntimeError(f"link failed: {' '.join(link)}\n{result.stdout}\n{result.stderr}")
    return output


if __name__ == "__main__":
    print(build(verbose="-v" in sys.argv, force="-f" in sys.argv))
