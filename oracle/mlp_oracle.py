"""CPU float64 restatement of the flow-map surrogate network (test infrastructure only).

The surrogate has no counterpart in the reference, so this oracle is the
definition its CUDA kernels are checked against: ``tests/`` compare the GPU
forward pass, loss, every weight/bias gradient and the Jacobian tangents with
these functions on the same BF16 weights and inputs.  Only tests import it.

Network (row-major, one sample per row):
    feat   = [sin(phase) | cos(phase)],  phase_f = kx_f x + ky_f y + kt_f t + c_f
    Z_l    = H_{l-1} W_l^T + b_l         (H_{-1} = feat)
    H_l    = silu(Z_l)                   for the hidden layers
    Y      = H_last W_out^T + b_out
    loss   = sum_rows sum_{c < outs} (Y - target)^2 / n
The GPU rounds to BF16 at fixed points: the features, the weights, every H_l,
the output gradient dY and every back-propagated dZ_l.  ``bf16_points=True``
rounds at the same points (round-to-nearest-even on the FP32 value), so the
only remaining difference is FP32 vs FP64 accumulation.
"""

from __future__ import annotations

from typing import Dict, List, Sequence

import numpy as np


def bf16(x: np.ndarray) -> np.ndarray:
    """Round to the nearest BF16 (ties to even) via FP32, returned as float64."""
    f = np.ascontiguousarray(np.asarray(x, dtype=np.float32))
    u = f.view(np.uint32).astype(np.uint64)
    u = (u + 0x7FFF + ((u >> 16) & 1)) & 0xFFFF0000
    return u.astype(np.uint32).view(np.float32).astype(np.float64)


def _id(x):
    return np.asarray(x, dtype=np.float64)


def sigmoid(z):
    return 1.0 / (1.0 + np.exp(-z))


def silu(z):
    return z * sigmoid(z)


def dsilu(z):
    s = sigmoid(z)
    return s * (1.0 + z * (1.0 - s))


def features(points: np.ndarray, freq: np.ndarray, tangents: bool = False):
    """2D: points (n, 3) = (x, y, t), freq (F, 4) = (kx, ky, kt, phase);
    3D: points (n, 4) = (x, y, z, t), freq (F, 8) = (kx, ky, kz, kt, phase, 0, 0, 0).
    Returns the features, and with ``tangents`` their derivatives along each
    spatial axis (tx, ty(, tz))."""
    p = np.asarray(points, dtype=np.float64)
    k = np.asarray(freq, dtype=np.float32).astype(np.float64)
    d = p.shape[1] - 1
    ph = p @ k[:, :d + 1].T + k[:, d + 1]
    s, c = np.sin(ph), np.cos(ph)
    feat = np.concatenate([s, c], axis=1)
    if not tangents:
        return feat
    return (feat,) + tuple(np.concatenate([k[:, a] * c, -k[:, a] * s], axis=1)
                           for a in range(d))


def forward(feat: np.ndarray, weights: Sequence[np.ndarray], biases: Sequence[np.ndarray],
            bf16_points: bool = True) -> Dict[str, List[np.ndarray]]:
    r = bf16 if bf16_points else _id
    h = r(feat)
    Z, H = [], [h]
    for l, (W, b) in enumerate(zip(weights, biases)):
        z = h @ r(W).T + b
        if l < len(weights) - 1:
            Z.append(z)
            h = r(silu(z))
            H.append(h)
        else:
            return {"Z": Z, "H": H, "Y": z}
    raise ValueError("empty network")


def loss_and_grads(feat, weights, biases, target, outs: int, bf16_points: bool = True):
    """Loss and gradients (dW_l, db_l) of the MSE over the first `outs` columns."""
    r = bf16 if bf16_points else _id
    fw = forward(feat, weights, biases, bf16_points)
    Y, Z, H = fw["Y"], fw["Z"], fw["H"]
    n = Y.shape[0]
    d = Y[:, :outs] - target
    loss = float(np.sum(d * d) / n)
    dY = np.zeros_like(Y)
    dY[:, :outs] = 2.0 * d / n
    g = r(dY)
    gW = [None] * len(weights)
    gb = [None] * len(weights)
    for l in range(len(weights) - 1, -1, -1):
        gW[l] = g.T @ H[l]
        gb[l] = g.sum(axis=0)
        if l > 0:
            g = r((g @ r(weights[l])) * dsilu(Z[l - 1]))
    return loss, gW, gb, Y


def jacobian_n(feat, tangents, weights, biases, bf16_points: bool = True):
    """Forward-mode tangents dY/dx_a through the network, one per seed tangent."""
    r = bf16 if bf16_points else _id
    fw = forward(feat, weights, biases, bf16_points)
    out = []
    for t in tangents:
        t = r(t)
        for l, W in enumerate(weights):
            t = t @ r(W).T
            if l < len(weights) - 1:
                t = r(t * dsilu(fw["Z"][l]))
        out.append(t)
    return fw["Y"], out


def jacobian(feat, tx, ty, weights, biases, bf16_points: bool = True):
    """2D form of jacobian_n: (Y, dY/dx, dY/dy)."""
    y, (jx, jy) = jacobian_n(feat, (tx, ty), weights, biases, bf16_points)
    return y, jx, jy


def ftle_from_tangents(J, scale: float, T: float) -> np.ndarray:
    """FTLE of x -> x + scale * y(x) from the tangents J[a] = dY/dx_a (n, >= dim):
    F = I + scale * [dY_r/dx_a], C = F^T F, largest eigenvalue in float64."""
    d = len(J)
    n = J[0].shape[0]
    F = np.empty((n, d, d))
    for a in range(d):
        F[:, :, a] = scale * J[a][:, :d]
    F += np.eye(d)
    C = np.einsum("nra,nrb->nab", F, F)
    lam = np.linalg.eigvalsh(C)[:, -1]
    return np.log(np.sqrt(lam)) / abs(T)
