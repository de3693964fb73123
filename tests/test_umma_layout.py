"""Tensor-core operand layout of the closure network, checked on the CPU:
umma_index is the K-major no-swizzle canonical layout with the shared-memory
descriptors' strides for every operand shape the inference kernel uses, the
shared-memory regions are aligned and disjoint, and the instruction
descriptor has the documented value (kind::f16, FP32 accumulator, M = 128,
N = 32).  The host code of tests/cuda/umma_layout_check.cu runs
without a GPU."""
import ctypes
import os
import shutil
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


@pytest.fixture(scope="module")
def checker(tmp_path_factory):
    nvcc = shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc"
    if not os.path.exists(nvcc):
        pytest.skip("nvcc not available")
    out = str(tmp_path_factory.mktemp("umma") / "libummacheck.so")
    subprocess.run([nvcc, "-std=c++17", "-gencode", "arch=compute_100a,code=sm_100a", "-Xcompiler", "-fPIC", "-shared",
                    "-I" + os.path.join(ROOT, "cudalbm_b200", "csrc"), "-I" + os.path.join(ROOT, "include"),
                    os.path.join(ROOT, "tests", "cuda", "umma_layout_check.cu"), "-o", out], check=True)
    L = ctypes.CDLL(out)
    L.umma_layout_check.argtypes = [ctypes.POINTER(ctypes.c_uint32)]
    return L


def test_operand_layouts_and_descriptors(checker):
    n32 = ctypes.c_uint32()
    assert checker.umma_layout_check(ctypes.byref(n32)) == 0
    # D = FP32 (bit 4), N >> 3 at bit 17, M >> 4 at bit 24
    assert n32.value == 0x08080010
