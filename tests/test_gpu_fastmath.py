"""The kernels' Newton-Raphson reciprocal and reciprocal square root against IEEE
division and square root, over the range of exponent sums, rho and Boys values."""

import ctypes
import os
import subprocess

import numpy as np
import pytest

HERE = os.path.dirname(os.path.abspath(__file__))


@pytest.mark.gpu
def test_newton_reciprocal_and_rsqrt(cuda_ok, tmp_path):
    from tonto_b200 import build
    so = str(tmp_path / "fast_math_check.so")
    subprocess.run([build.nvcc()] + build.flags() + ["-I", build.CSRC, "-o", so,
                    os.path.join(HERE, "fast_math_check.cu")], check=True)
    L = ctypes.CDLL(so)
    dp = ctypes.POINTER(ctypes.c_double)
    L.fast_math_check.argtypes = [dp, ctypes.c_int, dp, dp]
    rng = np.random.default_rng(5)
    x = 10.0 ** rng.uniform(-8, 8, size=1 << 20)
    x[:4] = [1.0, 0.5, 2.0, 3.0]
    er, eq = np.empty_like(x), np.empty_like(x)
    p = lambda a: a.ctypes.data_as(dp)  # noqa: E731
    assert L.fast_math_check(p(x), len(x), p(er), p(eq)) == 0
    ulp = np.finfo(np.float64).eps
    assert er.max() <= 3 * ulp and eq.max() <= 4 * ulp       # the reference 1/sqrt rounds twice
