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


def _mlp_case(S, seed):
    import mlp_oracle as mo
    rng = np.random.default_rng(seed)
    X = mo.bf16_bits(rng.standard_normal((S, mo.F)) * 1.5)
    p = mo.init_params(seed)
    p[mo.OFF["b1"]:mo.OFF["W2"]] = rng.standard_normal(mo.H) * 0.1
    p[mo.OFF["b2"]:mo.OFF["w3"]] = rng.standard_normal(mo.H) * 0.1
    p[mo.OFF["b3"]] = 0.3
    return X, p


@pytest.mark.parametrize("S", [1, 128, 1000, 50000])
def test_mlp_forward_matches_cpu(lib, S):
    import mlp_oracle as mo
    X, p = _mlp_case(S, S)
    y = np.zeros(S, dtype=np.float32)
    assert lib.tracer_mlp_forward(X.ctypes.data, S, p.ctypes.data, y.ctypes.data) == 0
    ref, _ = mo.forward(from_bf16_bits(X), p)
    # error relative to the output's scale: the first hidden layer's GELU runs
    # in FP16 pairs (FP16 rounding 2^-11, tanh.approx.f16x2) and the second's
    # in FP32 (tanh.approx.f32, about 2^-11); the BF16 rounding of the first
    # hidden activation can flip on the resulting differences.  Measured: 1.5e-2
    # at the 99.9 % quantile (below 1e-2 with both layers in FP32), 1.8e-2 at most.
    err = np.abs(y - ref) / max(np.sqrt(np.mean(ref ** 2)), 1e-30)
    assert np.quantile(err, 0.999) < 2.5e-2 and err.max() < 5e-2, (np.quantile(err, 0.999), err.max())


@pytest.mark.parametrize("S", [128, 777, 20000])
def test_mlp_gradients_match_cpu(lib, S):
    """Tensor-core backward pass (weight gradients accumulated in TMEM over
    every tile of a CTA, then across CTAs) against the CPU restatement."""
    import mlp_oracle as mo
    X, p = _mlp_case(S, S + 7)
    dy = np.random.default_rng(S).standard_normal(S).astype(np.float32) / S
    g = np.zeros(mo.NPARAMS, dtype=np.float32)
    assert lib.tracer_mlp_grads(X.ctypes.data, dy.ctypes.data, S, p.ctypes.data, g.ctypes.data) == 0
    ref = mo.grads(from_bf16_bits(X), dy, p)
    for name, (a, b) in {"W1": (0, 1024), "b1": (1024, 1088), "W2": (1088, 5184), "b2": (5184, 5248),
                         "w3": (5248, 5312), "b3": (5312, 5313)}.items():
        rel = np.linalg.norm(g[a:b] - ref[a:b]) / (np.linalg.norm(ref[a:b]) + 1e-30)
        assert rel < 5e-3, (name, rel)
