"""NumPy oracle of the recurrent surrogate's forward and backward pass -- test infrastructure.

float64 restatement of one truncated-BPTT window of the surrogate in
concrete_impact_b200/rno.py: per step x = [strain, rate, z] -> 3 GELU layers -> linear
output (stress 6, latent rate 6); z' = z + c * zdot (the forward-Euler latent step of the
reference, src/concrete_impact/nn/models/rve_rno.py:383-387); loss = mean squared stress
error over the window.  Weights use the padded shapes of the device model
(W1 (h, 32), W4 (16, h)).  Optional bf16 rounding reproduces the device's rounding points.
"""

from __future__ import annotations

import numpy as np
from scipy.special import erf

IN_REAL, IN_PAD, OUT_PAD = 18, 32, 16


def bf16_round(x: np.ndarray) -> np.ndarray:
    """Round float values to bf16 (round to nearest even on the float32 bit pattern)."""
    f = np.asarray(x, dtype=np.float32)
    bits = f.view(np.uint32).astype(np.uint64)
    lsb = (bits >> 16) & 1
    bits = (bits + 0x7FFF + lsb) & 0xFFFF0000
    return bits.astype(np.uint32).view(np.float32).astype(np.float64)


def gelu(x):
    return 0.5 * x * (1.0 + erf(x / np.sqrt(2.0)))


def gelu_grad(x):
    return 0.5 * (1.0 + erf(x / np.sqrt(2.0))) + x * np.exp(-0.5 * x * x) / np.sqrt(2.0 * np.pi)


def window_forward_backward(params, strain, rate, target, coef, z0, bf16: bool = False, skip=None):
    """Loss and gradients of one window.

    params: list of (W (out, in_pad), b (out,)) for the 4 layers; strain/rate/target
    (T, B, 6); coef (T, B); z0 (B, 6); skip: optional 6x6 K adding K (strain - z) to the
    stress output.  Returns (loss, grads [(dW, db)], z_T, Y (T, B, 16)); Y[:, :, :6] is
    the stress including the skip term.
    """
    rnd = bf16_round if bf16 else (lambda a: np.asarray(a, dtype=np.float64))
    T, B = strain.shape[0], strain.shape[1]
    Ws = [rnd(W) for W, _ in params]
    bs = [np.asarray(b, dtype=np.float64) for _, b in params]
    z = np.zeros((T + 1, B, 6))
    z[0] = z0
    X, Zs, Hs, Y = [], [], [], []
    for t in range(T):
        x = np.zeros((B, IN_PAD))
        x[:, 0:6], x[:, 6:12], x[:, 12:18] = strain[t], rate[t], z[t]
        x = rnd(x)
        X.append(x)
        a = x
        zl, hl = [], []
        for i in range(3):
            pre = a @ Ws[i].T + bs[i]
            h = rnd(gelu(pre))
            zl.append(pre)
            hl.append(h)
            a = h
        y = a @ Ws[3].T + bs[3]
        if skip is not None:
            y = y.copy()
            y[:, :6] += (strain[t] - z[t]) @ np.asarray(skip, dtype=np.float64).T
        Zs.append(zl)
        Hs.append(hl)
        Y.append(y)
        z[t + 1] = z[t] + coef[t][:, None] * y[:, 6:12]
    Y = np.asarray(Y)
    diff = Y[:, :, :6] - target
    loss = float(np.mean(diff**2))
    gY = 2.0 * diff / diff.size
    grads = [(np.zeros_like(Ws[i]), np.zeros_like(bs[i])) for i in range(4)]
    dz_next = np.zeros((B, 6))
    for t in range(T - 1, -1, -1):
        dy = np.zeros((B, OUT_PAD))
        dy[:, :6] = gY[t]
        dy[:, 6:12] = coef[t][:, None] * dz_next
        dy = rnd(dy)
        grads[3][0][...] += dy.T @ Hs[t][2]
        grads[3][1][...] += dy.sum(0)
        g = dy
        for i in (2, 1, 0):
            dh = g @ Ws[i + 1]
            dzl = rnd(dh * gelu_grad(Zs[t][i]))
            inp = X[t] if i == 0 else Hs[t][i - 1]
            grads[i][0][...] += dzl.T @ inp
            grads[i][1][...] += dzl.sum(0)
            g = dzl
        dx = g @ Ws[0]
        dz_next = dz_next + dx[:, 12:18]
        if skip is not None:
            dz_next = dz_next - gY[t] @ np.asarray(skip, dtype=np.float64)
    return loss, grads, z[T], Y
