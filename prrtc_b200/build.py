"""Build libprrtc_b200.so (sm_100a) in-tree with nvcc, and the host packer
module ``_hostpack`` with g++.

Each ``csrc/*.cu`` is compiled to an object in ``prrtc_b200/_build/`` (in
parallel), then linked into ``prrtc_b200/libprrtc_b200.so``;
``csrc/hostpack.cc`` (CPython C API, no CUDA) becomes
``prrtc_b200/_hostpack<EXT_SUFFIX>``.  Each rebuilds only when a source or
header is newer than its output.
"""
from __future__ import annotations

import concurrent.futures as cf
import os
import shutil
import subprocess
import sys
import sysconfig
from pathlib import Path

HERE = Path(__file__).resolve().parent
CSRC = HERE / "csrc"
BUILD = HERE / "_build"
LIB = HERE / "libprrtc_b200.so"
INCLUDE = HERE.parent / "include"
HOSTPACK_SRC = CSRC / "hostpack.cc"
HOSTPACK = HERE / ("_hostpack" + (sysconfig.get_config_var("EXT_SUFFIX") or ".so"))

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVCC_FLAGS = ["-O3", "-std=c++17", "-lineinfo", "-Xcompiler", "-fPIC", "--expt-relaxed-constexpr",
              "-Xptxas", "-warn-spills", "-diag-suppress", "550"]


def nvcc() -> str:
    for cand in (os.environ.get("NVCC"), shutil.which("nvcc"), "/usr/local/cuda/bin/nvcc"):
        if cand and Path(cand).exists():
            return cand
    raise RuntimeError("nvcc not found")


def _sources():
    return sorted(CSRC.glob("*.cu"))


def _deps():
    return _sources() + sorted(CSRC.glob("*.cuh")) + sorted(CSRC.glob("*.h")) + sorted(INCLUDE.glob("*.h")) + [
        Path(__file__)]


def up_to_date() -> bool:
    if not LIB.exists():
        return False
    t = LIB.stat().st_mtime
    return all(p.stat().st_mtime <= t for p in _deps())


def build_hostpack(force: bool = False) -> Path:
    """g++ -O2 -shared of the CPython host packer (CPython and numpy C APIs)."""
    if not force and HOSTPACK.exists() and all(
            p.stat().st_mtime <= HOSTPACK.stat().st_mtime for p in (HOSTPACK_SRC, Path(__file__))):
        return HOSTPACK
    cxx = os.environ.get("CXX") or shutil.which("g++") or "g++"
    tmp = HOSTPACK.with_name(HOSTPACK.name + ".tmp")
    import numpy

    cmd = [cxx, "-O2", "-std=c++17", "-shared", "-fPIC", "-fno-strict-aliasing", "-Wall",
           "-I", sysconfig.get_paths()["include"], "-I", numpy.get_include(), str(HOSTPACK_SRC), "-o", str(tmp)]
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"g++ failed for {HOSTPACK_SRC.name}:\n{r.stdout}\n{r.stderr}")
    os.replace(tmp, HOSTPACK)
    return HOSTPACK


def build(force: bool = False, verbose: bool = False, extra_flags: list[str] | None = None) -> Path:
    build_hostpack(force)
    if not force and up_to_date():
        return LIB
    BUILD.mkdir(exist_ok=True)
    flags = ARCH + NVCC_FLAGS + (extra_flags or [])
    exe = nvcc()

    def compile_one(src: Path) -> Path:
        obj = BUILD / (src.stem + ".o")
        cmd = [exe, *flags, "-I", str(INCLUDE), "-c", str(src), "-o", str(obj)]
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError(f"nvcc failed for {src.name}:\n{r.stdout}\n{r.stderr}")
        if verbose and (r.stdout or r.stderr):
            print(r.stdout + r.stderr, file=sys.stderr)
        return obj

    with cf.ThreadPoolExecutor(max_workers=min(8, os.cpu_count() or 1)) as ex:
        objs = list(ex.map(compile_one, _sources()))
    tmp = LIB.with_suffix(".so.tmp")
    cmd = [exe, *ARCH, "-shared", "-o", str(tmp), *map(str, objs), "-lcudart"]
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"link failed:\n{r.stdout}\n{r.stderr}")
    os.replace(tmp, LIB)
    return LIB


if __name__ == "__main__":
    build(force="--force" in sys.argv, verbose=True,
          extra_flags=["-Xptxas", "-v"] if "--ptxas-v" in sys.argv else None)
    print(LIB)
