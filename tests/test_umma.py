"""tcgen05 building blocks (periodsearch_b200/csrc/ps_umma.cuh) on the device:
a 128 x 64 x K split-BF16 GEMM against an FP64 product.  Split BF16
(hi*hi + hi*lo + lo*hi) keeps ~16 mantissa bits per product, so the result
must agree to ~1e-5 relative (normwise)."""
import ctypes
import os
import subprocess

import numpy as np
import pytest

from conftest import REPO

pytestmark = pytest.mark.gpu

SRC = os.path.join(REPO, "tests", "umma_selftest.cu")
LIB = os.path.join(REPO, "tests", "_build", "libumma_selftest.so")


def build_selftest():
    if os.path.exists(LIB) and os.path.getmtime(LIB) >= max(
            os.path.getmtime(SRC), os.path.getmtime(os.path.join(REPO, "periodsearch_b200", "csrc", "ps_umma.cuh"))):
        return LIB
    os.makedirs(os.path.dirname(LIB), exist_ok=True)
    subprocess.run(["nvcc", "-shared", "-Xcompiler", "-fPIC", "-O3", "-gencode", "arch=compute_100a,code=sm_100a",
                    "-o", LIB, SRC], check=True)
    return LIB


@pytest.mark.parametrize("K", [64, 192, 832])
def test_split_bf16_gemm(K):
    lib = ctypes.CDLL(build_selftest())
    fp = ctypes.POINTER(ctypes.c_float)
    lib.umma_selftest.argtypes = [fp, fp, ctypes.c_int, fp]
    rng = np.random.default_rng(K)
    A = rng.normal(size=(128, K)).astype(np.float32)
    B = rng.normal(size=(64, K)).astype(np.float32)
    A[:, -7:] = 0  # padded facets are zero in the fit kernel
    D = np.zeros((128, 64), np.float32)
    rc = lib.umma_selftest(A.ctypes.data_as(fp), B.ctypes.data_as(fp), K, D.ctypes.data_as(fp))
    assert rc == 0
    ref = A.astype(np.float64) @ B.astype(np.float64).T
    err = np.linalg.norm(D - ref) / np.linalg.norm(ref)
    assert err < 2e-5, err
    # element-wise: every row and column landed where it belongs
    assert np.max(np.abs(D - ref)) < 1e-3 * np.max(np.abs(ref))


@pytest.mark.parametrize("K", [32, 96, 800])
def test_split_tf32_gemm(K):
    """The same GEMM on kind::tf32 with split-TF32 operands (hi*hi + hi*lo +
    lo*hi; ~22 mantissa bits per product): ~1e-6 relative, normwise."""
    lib = ctypes.CDLL(build_selftest())
    fp = ctypes.POINTER(ctypes.c_float)
    lib.umma_selftest_tf32.argtypes = [fp, fp, ctypes.c_int, fp]
    rng = np.random.default_rng(K + 1)
    A = rng.normal(size=(128, K)).astype(np.float32)
    B = rng.normal(size=(64, K)).astype(np.float32)
    A[90:, :] = 0  # rows past the free parameters are zero in the mixed fit kernel
    D = np.zeros((128, 64), np.float32)
    rc = lib.umma_selftest_tf32(A.ctypes.data_as(fp), B.ctypes.data_as(fp), K, D.ctypes.data_as(fp))
    assert rc == 0
    ref = A.astype(np.float64) @ B.astype(np.float64).T
    err = np.linalg.norm(D - ref) / np.linalg.norm(ref)
    assert err < 1e-5, err  # FP32 accumulation over K terms dominates at large K
    assert np.max(np.abs(D - ref)) < 1e-4 * np.max(np.abs(ref))
