"""Builds the engine's shared library libneonufft_b200.so in-tree, for sm_100a only.

Every CUDA source is compiled by nvcc with
``-gencode arch=compute_100a,code=sm_100a -lineinfo -O3`` into ``neonufft_b200/_build/`` (in
parallel), then linked with the CUDA runtime (static) and cuFFT (shared). Rebuilds only when a
source, a header or this script is newer than the library.

``--checked`` builds the checked variant libneonufft_b200_checked.so (objects in
``_build_checked/``) with ``-DNNB_CHECKED``: device bounds checks on every grid, record and
output index of the hot kernels, which record the first failure instead of accessing out of
bounds, and a device synchronisation plus check after every C ABI call that reports a failure
as InternalError (a debugging build; load it with NEONUFFT_B200_LIB).

Usage: ``python -m neonufft_b200.build [--force] [--verbose] [--checked]``.
"""
from __future__ import annotations

import argparse
import concurrent.futures as cf
import os
import shutil
import subprocess
import sys
from pathlib import Path

PKG = Path(__file__).resolve().parent
ROOT = PKG.parent
CSRC = PKG / "csrc"
BUILD = PKG / "_build"
LIB = PKG / "libneonufft_b200.so"
BUILD_CHECKED = PKG / "_build_checked"
LIB_CHECKED = PKG / "libneonufft_b200_checked.so"
INCLUDE = ROOT / "include"

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVCC_FLAGS = [
    "-std=c++17", "-O3", "-lineinfo", "-Xcompiler", "-fPIC", "-Xcompiler", "-fvisibility=hidden",
    "--expt-relaxed-constexpr", "-I", str(INCLUDE), "-I", str(CSRC),
]


def _nvcc() -> str:
    for cand in (os.environ.get("NVCC"), shutil.which("nvcc"), "/usr/local/cuda/bin/nvcc"):
        if cand and Path(cand).exists():
            return cand
    raise RuntimeError("nvcc not found")


def _cuda_lib_dir() -> Path:
    nvcc = Path(_nvcc()).resolve()
    for cand in (nvcc.parent.parent / "lib64", Path("/usr/local/cuda/lib64")):
        if (cand / "libcufft.so").exists():
            return cand
    raise RuntimeError("libcufft.so not found")


def sources() -> list[Path]:
    return sorted(list(CSRC.glob("*.cu")) + list(CSRC.glob("*.cpp")))


def _headers() -> list[Path]:
    hs = list(CSRC.glob("*.hpp")) + list(CSRC.glob("*.cuh")) + list(INCLUDE.rglob("*.h"))
    hs += list(INCLUDE.rglob("*.hpp"))
    return hs


def _stale(lib: Path, extra: list[Path]) -> bool:
    if not lib.exists():
        return True
    t = lib.stat().st_mtime
    return any(p.stat().st_mtime > t for p in sources() + _headers() + extra)


def _compile(src: Path, verbose: bool, checked: bool = False) -> Path:
    obj = (BUILD_CHECKED if checked else BUILD) / (src.name + ".o")
    extra = ["-DNNB_CHECKED"] if checked else []
    cmd = [_nvcc(), *ARCH, *NVCC_FLAGS, *extra, "-x", "cu", "-c", str(src), "-o", str(obj)]
    if verbose:
        print(" ".join(cmd), flush=True)
    res = subprocess.run(cmd, capture_output=True, text=True)
    if res.returncode != 0:
        raise RuntimeError(f"nvcc failed for {src.name}:\n{res.stdout}\n{res.stderr}")
    if verbose and res.stderr.strip():
        print(res.stderr, flush=True)
    return obj


def build(force: bool = False, verbose: bool = False, checked: bool = False) -> Path:
    """Compiles and links the library (the checked variant with checked=True); returns its
    path."""
    lib = LIB_CHECKED if checked else LIB
    if not force and not _stale(lib, [Path(__file__)]):
        return lib
    (BUILD_CHECKED if checked else BUILD).mkdir(exist_ok=True)
    srcs = sources()
    workers = max(1, min(len(srcs), os.cpu_count() or 4))
    with cf.ThreadPoolExecutor(workers) as ex:
        objs = list(ex.map(lambda s: _compile(s, verbose, checked), srcs))
    tmp = lib.with_suffix(".so.tmp")
    cmd = [_nvcc(), *ARCH, "-shared", "-o", str(tmp), *map(str, objs),
           "-cudart", "static", "-L", str(_cuda_lib_dir()), "-lcufft",
           "-Xlinker", "-rpath," + str(_cuda_lib_dir())]
    if verbose:
        print(" ".join(cmd), flush=True)
    res = subprocess.run(cmd, capture_output=True, text=True)
    if res.returncode != 0:
        raise RuntimeError(f"link failed:\n{res.stdout}\n{res.stderr}")
    os.replace(tmp, lib)
    return lib


def main() -> int:
    ap = argparse.ArgumentParser()
    ap.add_argument("--force", action="store_true")
    ap.add_argument("--verbose", action="store_true")
    ap.add_argument("--checked", action="store_true")
    a = ap.parse_args()
    print(build(force=a.force, verbose=a.verbose, checked=a.checked))
    return 0


if __name__ == "__main__":
    sys.exit(main())
