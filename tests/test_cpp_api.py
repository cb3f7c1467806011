"""C++ callers: tests/cpp/plan_api.cpp is user code written against the reference's GPU plan
headers (include/neonufft/gpu/plan.hpp, device_allocator.hpp, exceptions.hpp), compiled here with
g++ against the engine's headers and linked to libneonufft_b200.so.

- `cpu` mode (no device): argument errors raise the reference's exception types.
- `gpu` mode: Plan<T, DIM> type 1 / type 2 / set_points and PlanT3<T, DIM> (points and bounds
  constructors, add_input accumulation, reset, batch) against FP64 direct sums, on a caller's
  stream; device memory through a caller's Allocator, all of it returned; an allocator that
  fails at each allocation point raises MemoryAllocError and leaks nothing.
"""
import os
import shutil
import subprocess
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parent.parent
SRC = ROOT / "tests" / "cpp" / "plan_api.cpp"
OUT = ROOT / "tests" / "cpp" / "_build" / "plan_api"
CUDA = Path(os.environ.get("CUDA_HOME", "/usr/local/cuda"))


@pytest.fixture(scope="module")
def plan_api(engine):
    if shutil.which("g++") is None:
        pytest.skip("g++ not available")
    lib_dir = ROOT / "neonufft_b200"
    assert (lib_dir / "libneonufft_b200.so").exists()
    OUT.parent.mkdir(parents=True, exist_ok=True)
    cmd = ["g++", "-std=c++17", "-O2", "-Wall", "-Werror", "-I", str(ROOT / "include"),
           "-I", str(CUDA / "include"), str(SRC), "-o", str(OUT),
           "-L", str(lib_dir), "-lneonufft_b200", f"-Wl,-rpath,{lib_dir}",
           "-L", str(CUDA / "lib64"), "-lcudart", f"-Wl,-rpath,{CUDA / 'lib64'}"]
    r = subprocess.run(cmd, capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    return OUT


def _run(binary, mode, timeout):
    r = subprocess.run([str(binary), mode], capture_output=True, text=True, timeout=timeout)
    print(r.stdout)
    assert r.returncode == 0, r.stdout + r.stderr
    assert "checks passed" in r.stdout
    return r.stdout


def test_cpp_argument_errors(plan_api):
    out = _run(plan_api, "cpu", 60)
    assert out.count("Input error") == 6


@pytest.mark.gpu
def test_cpp_plans_on_device(plan_api, cuda):
    out = _run(plan_api, "gpu", 600)
    assert "FAIL" not in out
    assert "MemoryAllocError at each of" in out
