"""The 3xTF32 tensor-core GEMM (tcgen05 + TMA) against a float64 product.

3xTF32 keeps the hi*hi, hi*lo and lo*hi products of the tf32 splits, so
its error is that of an FP32 GEMM: a random-walk accumulation error of
about sqrt(k) * 6e-8 of the row-norm x column-norm scale of each entry,
bounded here by 1e-7 * (sqrt(k) + 1).
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def acc():
    import nec_accel

    return nec_accel


@pytest.mark.parametrize("m,n,k", [(128, 128, 32), (300, 200, 100), (512, 384, 1000), (1, 1, 1), (129, 257, 33)])
def test_tf32x3_gemm_matches_float64(acc, m, n, k):
    rng = np.random.default_rng(m * 7 + n * 3 + k)
    a = rng.standard_normal((m, k)).astype(np.float32)
    b = rng.standard_normal((n, k)).astype(np.float32)
    c = acc.selftest_tf32x3_gemm(a, b)
    ref = a.astype(np.float64) @ b.astype(np.float64).T
    scale = np.outer(np.linalg.norm(a, axis=1), np.linalg.norm(b, axis=1))
    err = np.abs(c - ref) / scale
    assert err.max() <= 1e-7 * (np.sqrt(k) + 1), err.max()


def test_tf32x3_beats_plain_tf32(acc):
    """Values with bits below tf32's 10-bit mantissa: 1xTF32 would lose them
    (error ~5e-4 of the result for these 64-term sums); 3xTF32 keeps them to
    FP32 accumulation error (~1e-6)."""
    rng = np.random.default_rng(5)
    a = (1.0 + rng.random((128, 64)) * 1e-3).astype(np.float32)
    b = (1.0 + rng.random((128, 64)) * 1e-3).astype(np.float32)
    c = acc.selftest_tf32x3_gemm(a, b)
    ref = a.astype(np.float64) @ b.astype(np.float64).T
    assert np.abs(c - ref).max() / np.abs(ref).max() <= 2e-6
