"""CPU oracle of the learned VR warm-start network -- TEST INFRASTRUCTURE ONLY.

Only tests/, the smoke check and the bench's CPU legs import this file, and
only to check the GPU kernels of dnds_b200/csrc/dndsg_mlp.cuh.  The network
has no counterpart in the reference (DNDS has no learned component), so there
is nothing of the reference to pin it to; it is pinned instead by a central
finite-difference check of its own backward pass (tests/test_mlp.py).

Network: 64 -> 64 -> 64 -> 64 -> 20, SiLU on the hidden layers, linear output;
loss = mean over rows and the 20 outputs of (y - t)^2.  Parameters are one
flat FP32 vector with the kernels' padded layout:
W1[64][64] b1[64] W2[64][64] b2[64] W3[64][64] b3[64] W4[32][64] b4[32]
(W[n][k]: output unit n, input k; padded rows/columns are zero).

With bf16=True the arithmetic is rounded to bfloat16 (round to nearest even)
at exactly the points where the GPU kernels round: features, weights and
hidden activations before each product, and the back-propagated dz before
each product; accumulation, biases and the bias gradients stay in wide
precision.  With bf16=False everything is FP64.
"""
from __future__ import annotations

import numpy as np

N_IN, N_INP, N_HID, N_OUT, N_OUTP = 64, 64, 64, 20, 32
OFF_W1 = 0
OFF_B1 = OFF_W1 + N_HID * N_INP
OFF_W2 = OFF_B1 + N_HID
OFF_B2 = OFF_W2 + N_HID * N_HID
OFF_W3 = OFF_B2 + N_HID
OFF_B3 = OFF_W3 + N_HID * N_HID
OFF_W4 = OFF_B3 + N_HID
OFF_B4 = OFF_W4 + N_OUTP * N_HID
N_PARAM = OFF_B4 + N_OUTP


def bf16(a: np.ndarray) -> np.ndarray:
    """Round float values to bfloat16 (nearest, ties to even), returned as float64."""
    f = np.ascontiguousarray(a, dtype=np.float32)
    b = f.view(np.uint32).astype(np.uint64)
    b = (b + 0x7FFF + ((b >> 16) & 1)) & 0xFFFF0000
    return b.astype(np.uint32).view(np.float32).astype(np.float64)


def unpack(p: np.ndarray):
    p = np.asarray(p, dtype=np.float64)
    W1 = p[OFF_W1:OFF_B1].reshape(N_HID, N_INP)
    W2 = p[OFF_W2:OFF_B2].reshape(N_HID, N_HID)
    W3 = p[OFF_W3:OFF_B3].reshape(N_HID, N_HID)
    W4 = p[OFF_W4:OFF_B4].reshape(N_OUTP, N_HID)
    return (W1, p[OFF_B1:OFF_W2], W2, p[OFF_B2:OFF_W3], W3, p[OFF_B3:OFF_W4], W4, p[OFF_B4:N_PARAM])


def _sig(z):
    return 1.0 / (1.0 + np.exp(-z))


def _silu(z):
    return z * _sig(z)


def _silu_grad(z):
    s = _sig(z)
    return s * (1.0 + z * (1.0 - s))


def forward(p: np.ndarray, X: np.ndarray, bf: bool = False, keep: bool = False):
    """Y [n][20] for X [n][64]."""
    r = bf16 if bf else (lambda a: np.asarray(a, dtype=np.float64))
    W1, b1, W2, b2, W3, b3, W4, b4 = unpack(p)
    n = X.shape[0]
    x = np.zeros((n, N_INP))
    x[:, :N_IN] = X
    x = r(x)
    z1 = x @ r(W1).T + b1
    h1 = r(_silu(z1))
    z2 = h1 @ r(W2).T + b2
    h2 = r(_silu(z2))
    z3 = h2 @ r(W3).T + b3
    h3 = r(_silu(z3))
    y = (h3 @ r(W4).T + b4)[:, :N_OUT]
    if keep:
        return y, (x, z1, h1, z2, h2, z3, h3)
    return y


def loss_and_grad(p: np.ndarray, X: np.ndarray, T: np.ndarray, bf: bool = False):
    """(mean-square loss, gradient [N_PARAM]) as the training kernel computes them."""
    r = bf16 if bf else (lambda a: np.asarray(a, dtype=np.float64))
    W1, b1, W2, b2, W3, b3, W4, b4 = unpack(p)
    n = X.shape[0]
    cnt = n * N_OUT
    y, (x, z1, h1, z2, h2, z3, h3) = forward(p, X, bf, keep=True)
    d = y - T
    loss = float(np.sum(d * d)) / cnt
    dy = np.zeros((n, N_OUTP))
    dy[:, :N_OUT] = 2.0 * d * (np.float32(1.0) / np.float32(cnt) if bf else 1.0 / cnt)
    g = np.zeros(N_PARAM)
    dz4 = r(dy)
    g[OFF_W4:OFF_B4] = (dz4.T @ h3).ravel()
    g[OFF_B4:N_PARAM] = dy.sum(0)
    dz3 = (dz4 @ r(W4)) * _silu_grad(z3)
    g[OFF_B3:OFF_W4] = dz3.sum(0)
    dz3r = r(dz3)
    g[OFF_W3:OFF_B3] = (dz3r.T @ h2).ravel()
    dz2 = (dz3r @ r(W3)) * _silu_grad(z2)
    g[OFF_B2:OFF_W3] = dz2.sum(0)
    dz2r = r(dz2)
    g[OFF_W2:OFF_B2] = (dz2r.T @ h1).ravel()
    dz1 = (dz2r @ r(W2)) * _silu_grad(z1)
    g[OFF_B1:OFF_W2] = dz1.sum(0)
    dz1r = r(dz1)
    g[OFF_W1:OFF_B1] = (dz1r.T @ x).ravel()
    # padded entries carry no gradient
    g[OFF_W1:OFF_B1].reshape(N_HID, N_INP)[:, N_IN:] = 0.0
    g[OFF_W4:OFF_B4].reshape(N_OUTP, N_HID)[N_OUT:, :] = 0.0
    g[OFF_B4 + N_OUT:N_PARAM] = 0.0
    return loss, g


def random_params(seed: int, scale: float = 1.0) -> np.ndarray:
    """Glorot-uniform weights, small random biases, zero padding (float32)."""
    rng = np.random.default_rng(seed)
    p = np.zeros(N_PARAM)
    W1, b1, W2, b2, W3, b3, W4, b4 = unpack(p)  # views into p
    for W, nin, nout in ((W1, N_IN, N_HID), (W2, N_HID, N_HID), (W3, N_HID, N_HID), (W4, N_HID, N_OUT)):
        a = scale * np.sqrt(6.0 / (nin + nout))
        W[:nout, :nin] = rng.uniform(-a, a, (nout, nin))
    for b, nout in ((b1, N_HID), (b2, N_HID), (b3, N_HID), (b4, N_OUT)):
        b[:nout] = rng.uniform(-0.1, 0.1, nout)
    return p.astype(np.float32)
