"""The host copy pool behind page-locked staging (nmslib_b200/csrc/host_stage.cc), without a GPU:
tests/host_copy_check.cc links that source with g++ and checks random piece layouts, sizes around
the pool's block limits, zero-length pieces, more pieces than one job carries, concurrent callers
and workers woken from sleep. The CUDA calls of the same file (page-locked buffers and their
copies) run in the GPU tests, where every host-buffer search goes through them."""
import os
import shutil
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
CSRC = os.path.join(ROOT, "nmslib_b200", "csrc")


def _cuda_home():
    for cand in (os.environ.get("CUDA_HOME"), "/usr/local/cuda"):
        if cand and os.path.exists(os.path.join(cand, "include", "cuda_runtime.h")):
            return cand
    return None


def test_host_copy_pool(tmp_path):
    cuda = _cuda_home()
    if shutil.which("g++") is None or cuda is None:
        pytest.skip("g++ and the CUDA toolkit headers are needed to build the check")
    exe = str(tmp_path / "host_copy_check")
    libdir = os.path.join(cuda, "lib64")
    subprocess.run(["g++", "-O2", "-std=c++17", "-pthread", "-I", CSRC, "-I", os.path.join(cuda, "include"),
                    os.path.join(ROOT, "tests", "host_copy_check.cc"), os.path.join(CSRC, "host_stage.cc"),
                    "-L", libdir, "-Wl,-rpath," + libdir, "-lcudart", "-o", exe], check=True)
    out = subprocess.run([exe], capture_output=True, text=True, timeout=300)
    assert out.returncode == 0, out.stdout + out.stderr
    assert out.stdout.startswith("ok "), out.stdout
