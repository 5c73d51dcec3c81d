"""CPU restatement of the learned-flux MLP (16 -> 64 -> 64 -> 1, GELU).

TEST INFRASTRUCTURE ONLY: the checker of the tensor-core kernels in
fesom2_tracer_dwarf_b200/csrc/mlp.cu (tests/ only).  The network has no
counterpart in the reference; its operands are quantised to BF16 exactly
where the kernels quantise them (features, W1, W2, the hidden activation
fed to the second layer, and the back-propagated pre-activation gradients
fed to the weight-gradient products); everything else is FP64 here.
"""
from __future__ import annotations

import math

import numpy as np

F, H = 16, 64
OFF = {"W1": 0, "b1": H * F, "W2": H * F + H, "b2": H * F + H + H * H, "w3": H * F + 2 * H + H * H,
       "b3": H * F + 3 * H + H * H}
NPARAMS = H * F + 3 * H + H * H + 1

def bf16(x):
    """Round-to-nearest-even to BF16, returned as float64."""
    u = np.ascontiguousarray(np.asarray(x, dtype=np.float32)).view(np.uint32)
    r = ((u >> 16) & 1) + 0x7FFF
    return (((u + r) >> 16) << 16).astype(np.uint32).view(np.float32).astype(np.float64)


def bf16_bits(x):
    u = np.ascontiguousarray(np.asarray(x, dtype=np.float32)).view(np.uint32)
    r = ((u >> 16) & 1) + 0x7FFF
    return ((u + r) >> 16).astype(np.uint16)


C_GELU, A_GELU = math.sqrt(2.0 / math.pi), 0.044715


def gelu(z):
    """GELU, tanh form (Hendrycks & Gimpel 2016), as the kernels evaluate it."""
    return 0.5 * z * (1.0 + np.tanh(C_GELU * (z + A_GELU * z ** 3)))


def gelu_grad(z):
    t = np.tanh(C_GELU * (z + A_GELU * z ** 3))
    return 0.5 * (1.0 + t) + 0.5 * z * (1.0 - t * t) * C_GELU * (1.0 + 3.0 * A_GELU * z * z)


def unpack(p):
    p = np.asarray(p, dtype=np.float64)
    return (p[OFF["W1"]:OFF["b1"]].reshape(H, F), p[OFF["b1"]:OFF["W2"]], p[OFF["W2"]:OFF["b2"]].reshape(H, H),
            p[OFF["b2"]:OFF["w3"]], p[OFF["w3"]:OFF["b3"]], p[OFF["b3"]])


def init_params(seed=0):
    rng = np.random.default_rng(seed)
    p = np.zeros(NPARAMS, dtype=np.float32)
    p[OFF["W1"]:OFF["b1"]] = rng.standard_normal(H * F) * math.sqrt(2.0 / F)
    p[OFF["W2"]:OFF["b2"]] = rng.standard_normal(H * H) * math.sqrt(2.0 / H)
    p[OFF["w3"]:OFF["b3"]] = rng.standard_normal(H) * math.sqrt(1.0 / H)
    return p


def forward(X, p, quantize=True):
    """X (S, 16) float (already BF16-representable when quantize).  Returns y and
    the activations the backward pass needs."""
    W1, b1, W2, b2, w3, b3 = unpack(p)
    q = bf16 if quantize else (lambda a: np.asarray(a, dtype=np.float64))
    x = q(X)
    z1 = x @ q(W1).T + b1
    h1 = gelu(z1)
    h1q = q(h1)
    z2 = h1q @ q(W2).T + b2
    h2 = gelu(z2)
    y = h2 @ w3 + b3
    return y, (x, z1, h1q, z2, h2)


def grads(X, dy, p, quantize=True):
    """d/dparams of sum_s dy[s] y(X[s]), packed like the parameters."""
    W1, b1, W2, b2, w3, b3 = unpack(p)
    q = bf16 if quantize else (lambda a: np.asarray(a, dtype=np.float64))
    y, (x, z1, h1q, z2, h2) = forward(X, p, quantize)
    dy = np.asarray(dy, dtype=np.float64)
    dz2 = dy[:, None] * w3[None, :] * gelu_grad(z2)
    dz2q = q(dz2)
    g = np.zeros(NPARAMS)
    g[OFF["W2"]:OFF["b2"]] = (dz2q.T @ h1q).ravel()
    g[OFF["b2"]:OFF["w3"]] = dz2.sum(0)
    g[OFF["w3"]:OFF["b3"]] = (dy[:, None] * h2).sum(0)
    g[OFF["b3"]] = dy.sum()
    dh1 = dz2q @ q(W2)
    dz1 = dh1 * gelu_grad(z1)
    dz1q = q(dz1)
    g[OFF["W1"]:OFF["b1"]] = (dz1q.T @ x).ravel()
    g[OFF["b1"]:OFF["W2"]] = dz1.sum(0)
    return g
