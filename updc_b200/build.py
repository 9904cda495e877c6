"""Build the sm_100a engine library and the drop-in executable in-tree.

    python -m updc_b200.build [--force]

Produces ``updc_b200/libupdc_b200.so`` (the C ABI of include/updc_b200.h) and
``updc_b200/bin/updc_jwst_c`` (the 18-argument drop-in for the frozen core).
nvcc cross-compiles for sm_100a, so this also runs on machines without a GPU.
"""
from __future__ import annotations

import concurrent.futures
import os
import shutil
import subprocess
import sys
from pathlib import Path

PKG = Path(__file__).resolve().parent
ROOT = PKG.parent
CSRC = PKG / "csrc"
BUILD = PKG / "_build"
LIB = PKG / "libupdc_b200.so"
EXE = PKG / "bin" / "updc_jwst_c"
PROJECTOR = PKG / "bin" / "updc_psf_projector"

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVCC_FLAGS = ["-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC", "--expt-relaxed-constexpr",
              "-Xcompiler", "-Wall", "-I", str(ROOT / "include")]
# geometry must not contract multiply-adds (bit-exact LinkMaps)
PER_FILE = {"linkmap.cu": ["-fmad=false"], "projector.cu": ["-fmad=false"]}
SOURCES = ["linkmap.cu", "engine.cu", "capi.cu", "noalloc.cu", "batch.cu", "projector.cu", "preprocess.cu"]
HEADERS = ["common.cuh", "fft.cuh", "fft_ct.cuh", "kernels.cuh", "kernels_ct.cuh", "pointwise.cuh", "engine.cuh", "geometry.cuh", "linkmap.cuh",
           "tma.cuh", "nll.cuh", "preprocess.cuh"]


def nvcc() -> str:
    for cand in (os.environ.get("NVCC"), shutil.which("nvcc"), "/usr/local/cuda/bin/nvcc"):
        if cand and Path(cand).exists():
            return cand
    raise RuntimeError("nvcc not found")


def _stale(target: Path, deps) -> bool:
    if not target.exists():
        return True
    t = target.stat().st_mtime
    return any(Path(d).stat().st_mtime > t for d in deps)


def build(force: bool = False, verbose: bool = False) -> Path:
    BUILD.mkdir(exist_ok=True)
    (PKG / "bin").mkdir(exist_ok=True)
    headers = [CSRC / h for h in HEADERS] + [ROOT / "include" / "updc_b200.h"]
    objs = []
    jobs = []
    for src in SOURCES:
        obj = BUILD / (src + ".o")
        objs.append(obj)
        if force or _stale(obj, [CSRC / src, *headers, Path(__file__)]):
            cmd = [nvcc(), *ARCH, *NVCC_FLAGS, *PER_FILE.get(src, []), "-c", str(CSRC / src), "-o", str(obj)]
            jobs.append(cmd)
    if jobs:
        with concurrent.futures.ThreadPoolExecutor(max_workers=len(jobs)) as ex:
            results = list(ex.map(lambda c: subprocess.run(c, capture_output=True, text=True), jobs))
        for cmd, r in zip(jobs, results):
            if verbose or r.returncode:
                sys.stderr.write(" ".join(cmd) + "\n" + r.stdout + r.stderr)
            if r.returncode:
                raise RuntimeError(f"nvcc failed for {cmd[-3]}")
    if force or jobs or _stale(LIB, objs):
        cmd = [nvcc(), *ARCH, "-shared", "-o", str(LIB), *map(str, objs), "-lcudart_static", "-lrt", "-lpthread", "-ldl"]
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode:
            raise RuntimeError("link failed:\n" + r.stdout + r.stderr)
    for exe, main_src in ((EXE, CSRC / "updc_jwst_c.c"), (PROJECTOR, CSRC / "updc_psf_projector.c")):
        if force or _stale(exe, [LIB, main_src]):
            cmd = ["gcc", "-O2", "-std=gnu11", "-Wall", "-o", str(exe), str(main_src), f"-L{PKG}", "-lupdc_b200",
                   f"-Wl,-rpath,$ORIGIN/.."]
            r = subprocess.run(cmd, capture_output=True, text=True)
            if r.returncode:
                raise RuntimeError("executable link failed:\n" + r.stdout + r.stderr)
    return LIB


if __name__ == "__main__":
    build(force="--force" in sys.argv, verbose="-v" in sys.argv)
    print(LIB)
