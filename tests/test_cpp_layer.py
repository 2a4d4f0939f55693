"""C++ drop-in layer: the reference's C++ entry points (algorithms library,
sycl::reduction in parallel_for, group algorithms, atomic_ref, stdpar
overloads) compiled with nvcc against include/hipSYCL_b2p/ and libb2p.

The CPU test builds the test program (cross-compiling for sm_100a needs no
GPU); the GPU test runs it.  The program checks the cases of the
reference's own tests (tests/pstl/*.cpp, tests/sycl/reduction.cpp,
tests/sycl/group_functions/*, tests/sycl/atomic.cpp) against expected values
it computes on the host, and prints ALL PASSED when every check holds.
"""
import glob
import os
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
SRC = os.path.join(ROOT, "tests", "cpp", "test_cpp_layer.cu")
BIN = os.path.join(ROOT, "tests", "cpp", "_build", "test_cpp_layer")
LIBDIR = os.path.join(ROOT, "opensycl_b200", "_lib")
NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")


def build_program() -> str:
    deps = [SRC] + glob.glob(os.path.join(ROOT, "include", "hipSYCL_b2p", "*.hpp")) + \
        glob.glob(os.path.join(ROOT, "include", "b2p_device", "*.cuh")) + \
        [os.path.join(ROOT, "include", "b2p.h")]
    if not os.path.exists(os.path.join(LIBDIR, "libb2p.so")):
        from opensycl_b200 import build
        build.build()
    lib = os.path.join(LIBDIR, "libb2p.so")
    if os.path.exists(BIN) and os.path.getmtime(BIN) >= max(os.path.getmtime(p) for p in deps + [lib]):
        return BIN
    os.makedirs(os.path.dirname(BIN), exist_ok=True)
    cmd = [NVCC, "-gencode", "arch=compute_100a,code=sm_100a", "-O2", "-std=c++17", "--extended-lambda",
           "--expt-relaxed-constexpr", "-I" + os.path.join(ROOT, "include"), "-o", BIN, SRC,
           "-L" + LIBDIR, "-lb2p", "-Xlinker", "-rpath," + LIBDIR]
    r = subprocess.run(cmd, capture_output=True, text=True)
    assert r.returncode == 0, r.stdout + r.stderr
    return BIN


def test_cpp_layer_builds():
    assert os.path.exists(build_program())


@pytest.mark.gpu
def test_cpp_layer_runs_on_gpu(dev):
    exe = build_program()
    r = subprocess.run([exe], capture_output=True, text=True, timeout=600)
    for line in r.stdout.splitlines():
        if line.startswith("TIMING"):
            print(line)
    assert r.returncode == 0 and "ALL PASSED" in r.stdout, r.stdout[-4000:] + r.stderr[-2000:]
