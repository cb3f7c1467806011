"""The bounds-checked debugging build (libneonufft_b200_checked.so, -DNNB_CHECKED).

In that build every grid, record and output index of the spreading, interpolation,
deconvolution and binning kernels is checked on the device; a failed check records its line,
index and bound and skips the access (no trap), and after every C ABI call the library
synchronises and reports a recorded failure as NEONUFFT_INTERNAL_ERROR -- the counterpart of the
reference's debug-build sync-and-check after each launch (src/neonufft/gpu/util/runtime.hpp:27-30).

The GPU test runs the small-case parity suites (the reference's type-1/2 and type-3 matrices,
every spreading method and tile including the tensor-core spreading, the edge cases and the
batches) and the large-set binning suite (whose records the checked build also checks for being
a permutation of the points) in a child process that loads
the checked library, so that any out-of-range index in those kernels fails the run.
"""
import os
import subprocess
import sys
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parent.parent
CHECKED = ROOT / "neonufft_b200" / "libneonufft_b200_checked.so"
NORMAL = ROOT / "neonufft_b200" / "libneonufft_b200.so"


def _flag(lib_path):
    code = ("from neonufft_b200 import _lib as L; lib = L.load(); "
            "print(lib.nnb_is_checked_build(), L.LIB_PATH)")
    env = dict(os.environ, NEONUFFT_B200_LIB=str(lib_path), CUDA_VISIBLE_DEVICES="")
    res = subprocess.run([sys.executable, "-c", code], cwd=str(ROOT), env=env,
                         capture_output=True, text=True, timeout=120)
    assert res.returncode == 0, res.stdout + res.stderr
    return res.stdout.split()


def test_checked_and_normal_builds_report_their_flag():
    if not CHECKED.exists():
        pytest.skip("checked build not present (python -m neonufft_b200.build --checked)")
    assert _flag(NORMAL)[0] == "0"
    out = _flag(CHECKED)
    assert out[0] == "1" and out[1].endswith("libneonufft_b200_checked.so")


@pytest.mark.gpu
def test_parity_suites_under_the_checked_build(cuda):
    if not CHECKED.exists():
        pytest.fail("the checked build is missing: python -m neonufft_b200.build --checked")
    suites = ["tests/test_gpu_type12.py", "tests/test_gpu_type3.py", "tests/test_gpu_methods.py",
              "tests/test_gpu_tcgen05.py", "tests/test_gpu_edges.py", "tests/test_gpu_batch.py",
              "tests/test_gpu_binning.py"]
    env = dict(os.environ, NEONUFFT_B200_LIB=str(CHECKED))
    res = subprocess.run([sys.executable, "-m", "pytest", "-m", "gpu", "-x", "-q",
                          "-p", "no:cacheprovider", *suites],
                         cwd=str(ROOT), env=env, capture_output=True, text=True, timeout=1800)
    tail = "\n".join((res.stdout + res.stderr).splitlines()[-15:])
    assert res.returncode == 0, tail
    assert " passed" in res.stdout, tail
