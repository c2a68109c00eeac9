"""CPU restatement of the learned k-proposal network -- TEST INFRASTRUCTURE ONLY.

The proposal network has no counterpart in the reference (RBMD samples k only from the Gaussian,
rbmd/framework/model/RBEPSample.h:63-175); this file is the checker for the library's tcgen05
kernel (copy_gpu_b200/csrc/kernels_mlp.cuh): the same 16 -> 64 -> 64 -> 1 tanh network and the
same group loss l = log sum_b W_b e^{h_b} + log sum_b C_b e^{-h_b}, evaluated in FP64 with the
operands rounded to BF16 where the kernel rounds them (X, W1, W2, A1, dZ2) so that the kernel's
gradients can be compared to 1e-3.  With bf16=False everything stays FP64; the finite-difference
test pins that version.
"""
from __future__ import annotations

import numpy as np

N_IN, N_HID, ROWS = 16, 64, 256
OW1, OB1, OW2, OB2, OW3, OB3 = 0, 1024, 1088, 5184, 5248, 5312
N_PARAM = 5313


def bf16(a):
    """Round FP32 values to BF16 (round to nearest even), returned as float64."""
    a = np.asarray(a, dtype=np.float32)
    u = a.view(np.uint32).astype(np.uint64)
    r = ((u + 0x7FFF + ((u >> 16) & 1)) >> 16) << 16
    return r.astype(np.uint32).view(np.float32).astype(np.float64)


def unpack(p):
    p = np.asarray(p, dtype=np.float64)
    return (p[OW1:OB1].reshape(N_HID, N_IN), p[OB1:OW2], p[OW2:OB2].reshape(N_HID, N_HID), p[OB2:OW3],
            p[OW3:OB3], p[OB3])


def init_params(seed=0, scale=1.0):
    rng = np.random.default_rng(seed)
    p = np.zeros(N_PARAM, np.float32)
    p[OW1:OB1] = rng.normal(0, scale / np.sqrt(N_IN), N_HID * N_IN)
    p[OW2:OB2] = rng.normal(0, scale / np.sqrt(N_HID), N_HID * N_HID)
    p[OW3:OB3] = rng.normal(0, scale / np.sqrt(N_HID), N_HID)
    p[OB1:OW2] = rng.normal(0, 0.1, N_HID)
    p[OB2:OW3] = rng.normal(0, 0.1, N_HID)
    return p


def forward(p, x, bf=True):
    W1, b1, W2, b2, w3, b3 = unpack(p)
    r = bf16 if bf else (lambda a: np.asarray(a, np.float64))
    xb = r(x)
    z1 = xb @ r(W1).T + b1
    a1 = np.tanh(z1)
    a1b = r(a1)
    z2 = a1b @ r(W2).T + b2
    a2 = np.tanh(z2)
    h = a2 @ w3 + b3
    return h, dict(xb=xb, a1b=a1b, a2=a2)


def loss_and_grad(p, x, wbin, cbin, bf=True):
    """x: [G*256, 16]; returns (mean group loss, per-group losses, gradient [N_PARAM], h)."""
    W1, b1, W2, b2, w3, b3 = unpack(p)
    r = bf16 if bf else (lambda a: np.asarray(a, np.float64))
    h, c = forward(p, x, bf)
    G = len(h) // ROWS
    hg = h.reshape(G, ROWS)
    wg = np.asarray(wbin, np.float64).reshape(G, ROWS)
    cg = np.asarray(cbin, np.float64).reshape(G, ROWS)
    hmax = hg.max(1, keepdims=True)
    hmin = hg.min(1, keepdims=True)
    ep = wg * np.exp(hg - hmax)
    em = cg * np.exp(hmin - hg)
    Z, V = ep.sum(1, keepdims=True), em.sum(1, keepdims=True)
    losses = (hmax + np.log(Z) - hmin + np.log(V)).ravel()
    dh = ((ep / Z - em / V) / G).ravel()
    a2, a1b, xb = c["a2"], c["a1b"], c["xb"]
    g = np.zeros(N_PARAM)
    g[OB3] = dh.sum()
    g[OW3:OB3] = dh @ a2
    dz2 = dh[:, None] * w3[None, :] * (1 - a2 * a2)
    g[OB2:OW3] = dz2.sum(0)
    dz2b = r(dz2)
    g[OW2:OB2] = (dz2b.T @ a1b).ravel()
    da1 = dz2b @ r(W2)
    dz1 = da1 * (1 - a1b * a1b) if bf else da1 * (1 - a1b * a1b)
    g[OB1:OW2] = dz1.sum(0)
    g[OW1:OB1] = (dz1.T @ xb).ravel()
    return losses.mean(), losses, g, h
