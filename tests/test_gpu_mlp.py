"""Tensor-core (tcgen05) building blocks of the learned flux: a BF16 x BF16
-> FP32 tile product against numpy."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def to_bf16_bits(x):
    """Round-to-nearest-even FP32 -> BF16 bit patterns (uint16)."""
    u = np.ascontiguousarray(x, dtype=np.float32).view(np.uint32)
    r = ((u >> 16) & 1) + 0x7FFF
    return ((u + r) >> 16).astype(np.uint16)


def from_bf16_bits(b):
    return (b.astype(np.uint32) << 16).view(np.float32)


@pytest.mark.parametrize("N,K", [(64, 16), (64, 64), (16, 128), (256, 32), (128, 256)])
def test_umma_tile_product(lib, N, K):
    rng = np.random.default_rng(N * 1000 + K)
    A = to_bf16_bits(rng.standard_normal((128, K)))
    B = to_bf16_bits(rng.standard_normal((N, K)))
    D = np.zeros((128, N), dtype=np.float32)
    assert lib.tracer_selftest_umma(N, K, A.ctypes.data, B.ctypes.data, D.ctypes.data) == 0
    ref = from_bf16_bits(A).astype(np.float64) @ from_bf16_bits(B).astype(np.float64).T
    assert np.allclose(D, ref, rtol=1e-5, atol=1e-5 * np.abs(ref).max()), np.abs(D - ref).max()
