"""Build recipe for libmvs_b200.so (sm_100a) and the test oracles.

    python plane-sweep-cuda_b200/build.py          # library + oracle (+ reference-on-CPU when available)

The library is compiled in-tree into ``mvs_b200/libmvs_b200.so`` with nvcc for
``sm_100a`` only.  Every translation unit uses ``-fmad=false`` so plain
``a*b+c`` keeps two roundings (the reference's arithmetic); kernels that want
fused multiply-adds ask for them explicitly.
"""
from __future__ import annotations

import concurrent.futures as cf
import os
import pathlib
import shutil
import subprocess
import sys

PKG = pathlib.Path(__file__).resolve().parent
ROOT = PKG.parent
CSRC = PKG / "csrc"
OUT = PKG / "mvs_b200" / "libmvs_b200.so"
BUILD = PKG / "_build"
ORACLE = ROOT / "oracle"
# The reference's source tree (its src/ folder), used only to build the test
# oracles; set MVS_REFERENCE_SRC to point elsewhere.  Absent -> only the C oracle.
REFERENCE_SRC = pathlib.Path(os.environ.get("MVS_REFERENCE_SRC", "/root/reference/src"))

NVCC_FLAGS = [
    "-gencode", "arch=compute_100a,code=sm_100a",
    "-O3", "-lineinfo", "-std=c++17", "-fmad=false",
    "-Xcompiler", "-fPIC", "-Xcompiler", "-O2",
    "-I" + str(ROOT / "include"),
]


def _nvcc():
    cand = shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc"
    if not pathlib.Path(cand).exists():
        raise RuntimeError("nvcc not found")
    return cand


def _stale(target: pathlib.Path, deps) -> bool:
    if not target.exists():
        return True
    t = target.stat().st_mtime
    return any(pathlib.Path(d).stat().st_mtime > t for d in deps)


def build_library(force: bool = False, verbose: bool = False) -> pathlib.Path:
    sources = sorted(CSRC.glob("*.cu"))
    headers = sorted(CSRC.glob("*.cuh")) + sorted((ROOT / "include").glob("*.h*"))
    BUILD.mkdir(exist_ok=True)
    nvcc = _nvcc()
    objs = []
    jobs = []
    for src in sources:
        obj = BUILD / (src.stem + ".o")
        objs.append(obj)
        if force or _stale(obj, [src] + headers + [pathlib.Path(__file__)]):
            jobs.append([nvcc, *NVCC_FLAGS, "-c", str(src), "-o", str(obj)])

    def run(cmd):
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError(f"nvcc failed:\n{' '.join(cmd)}\n{r.stdout}\n{r.stderr}")
        if verbose and (r.stdout or r.stderr):
            print(r.stdout, r.stderr, file=sys.stderr)

    if jobs:
        with cf.ThreadPoolExecutor(max_workers=min(len(jobs), os.cpu_count() or 4)) as ex:
            list(ex.map(run, jobs))
    if force or jobs or _stale(OUT, objs):
        run([nvcc, "-gencode", "arch=compute_100a,code=sm_100a", "-shared", "-o", str(OUT),
             *map(str, objs), "-lcudart", "-Xlinker", "-rpath,/usr/local/cuda/lib64"])
    return OUT


def build_oracle(verbose: bool = False) -> None:
    """The C oracle always; the reference compiled for the CPU when its tree is present."""
    targets = ["oracle"]
    if (REFERENCE_SRC / "kernels.cu").exists():
        targets += ["ref", "ref_gpu"]
    r = subprocess.run(["make", "-C", str(ORACLE), f"REF={REFERENCE_SRC}", *targets], capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"oracle build failed:\n{r.stdout}\n{r.stderr}")
    if verbose:
        print(r.stdout, file=sys.stderr)


def build(force: bool = False, verbose: bool = False) -> pathlib.Path:
    lib = build_library(force=force, verbose=verbose)
    build_oracle(verbose=verbose)
    return lib


if __name__ == "__main__":
    print(build(force="--force" in sys.argv, verbose=True))
