"""TEST INFRASTRUCTURE ONLY: FP64 CPU reference of the warm-start network's
forward pass, BCE loss and gradients, used to check the GPU kernels of
mrtrix3_b200/csrc/mlp.cu.

Layout (matching csd_mlp_get_params): a flat FP32 vector [W1 b1 W2 b2 W3 b3]
with W1 [H][ld_in], W2 [H][H], W3 [ld_out][H].  With ``bf16=True`` the values
are rounded to BF16 wherever the GPU path stores BF16 (inputs, weights used
by the GEMMs, pre-activations, activations and back-propagated gradients),
so the comparison isolates accumulation-order differences.
"""
from __future__ import annotations

import math

import numpy as np
from scipy.special import erf


def to_bf16(a: np.ndarray) -> np.ndarray:
    """Round to the nearest BF16 value (ties to even), returned as float64."""
    f = np.ascontiguousarray(a, np.float32)
    u = f.view(np.uint32).astype(np.uint64)
    r = ((u + 0x7FFF + ((u >> 16) & 1)) >> 16) << 16
    return r.astype(np.uint32).view(np.float32).astype(np.float64)


def gelu(x):
    return 0.5 * x * (1.0 + erf(x / math.sqrt(2.0)))


def gelu_grad(x):
    return 0.5 * (1.0 + erf(x / math.sqrt(2.0))) + x * np.exp(-0.5 * x * x) / math.sqrt(2.0 * math.pi)


def unpack(p, n_in, H, n_out):
    ld_in = (n_in + 15) // 16 * 16
    ld_out = (n_out + 7) // 8 * 8
    o = 0
    out = {}
    for name, shape in (("W1", (H, ld_in)), ("b1", (H,)), ("W2", (H, H)), ("b2", (H,)), ("W3", (ld_out, H)),
                        ("b3", (ld_out,))):
        size = int(np.prod(shape))
        out[name] = np.asarray(p[o:o + size], np.float64).reshape(shape)
        o += size
    return out, ld_in, ld_out


def forward_backward(p, x, y_bits, n_in, H, n_out, bf16=True):
    """x [n][ld_in] inputs, y_bits [n][nw] uint32 targets -> (logits, loss, grad flat fp64)."""
    P, ld_in, ld_out = unpack(p, n_in, H, n_out)
    r = to_bf16 if bf16 else (lambda a: np.asarray(a, np.float64))
    n = x.shape[0]
    X = r(x)
    W1, W2, W3 = r(P["W1"]), r(P["W2"]), r(P["W3"])
    A1 = r(X @ W1.T + P["b1"])
    H1 = r(gelu(A1))
    A2 = r(H1 @ W2.T + P["b2"])
    H2 = r(gelu(A2))
    Z = H2 @ W3.T + P["b3"]
    Y = np.unpackbits(np.ascontiguousarray(y_bits).view(np.uint8), axis=1, bitorder="little")[:, :ld_out]
    Y = Y.astype(np.float64)
    Y[:, n_out:] = 0.0
    scale = 1.0 / (n * n_out)
    Zo = Z[:, :n_out]
    loss = np.sum(np.maximum(Zo, 0) - Zo * Y[:, :n_out] + np.log1p(np.exp(-np.abs(Zo)))) * scale
    dZ = (1.0 / (1.0 + np.exp(-Z)) - Y) * scale
    dZ[:, n_out:] = 0.0
    dZ = r(dZ)
    g = {}
    g["W3"] = dZ.T @ H2
    g["b3"] = dZ.sum(axis=0)
    dA2 = r((dZ @ W3) * gelu_grad(A2))
    g["W2"] = dA2.T @ H1
    g["b2"] = dA2.sum(axis=0)
    dA1 = r((dA2 @ W2) * gelu_grad(A1))
    g["W1"] = dA1.T @ X
    g["b1"] = dA1.sum(axis=0)
    flat = np.concatenate([g[k].ravel() for k in ("W1", "b1", "W2", "b2", "W3", "b3")])
    return Z, loss, flat
