"""mlp_oracle.py -- TEST INFRASTRUCTURE. Not part of the product.

CPU (numpy) restatement of the warm-start network of libsolfec_b200.so
(b2_mlp.cuh): BF16 MLP 32 -> 128 -> 128 -> 16, GELU (tanh form), FP32
accumulation, mean-squared loss over the first 3 outputs. The forward and
backward passes round to BF16 exactly where the device kernels store BF16
operands (inputs, weights, activations, output gradient, pre-activation
gradients), so the device gradients can be checked against these. The
network has no counterpart in the reference solver; its parity bar is the
gradient check against this restatement, which is itself checked against
finite differences in float64 (tests/test_learn_cpu.py).

Parameter vector layout (float32): W1[128][32] (column 25 is the bias of
layer 1, fed by a constant input 1), W2[128][128], b2[128], W3[16][128],
b3[16].
"""
from __future__ import annotations

import numpy as np

IN, HID, OUT, USED_OUT, BIAS_COL = 32, 128, 16, 3, 25
PW1 = 0
PW2 = PW1 + HID * IN
PB2 = PW2 + HID * HID
PW3 = PB2 + HID
PB3 = PW3 + OUT * HID
NPARAMS = PB3 + OUT
C_GELU, A_GELU = 0.7978845608028654, 0.044715


def bf16(x):
    """Round float32 values to the nearest BF16 (ties to even), as float32."""
    x = np.ascontiguousarray(x, dtype=np.float32)
    u = x.view(np.uint32).astype(np.uint64)
    r = (u + 0x7FFF + ((u >> 16) & 1)) & 0xFFFF0000
    return r.astype(np.uint32).view(np.float32).reshape(x.shape)


def unpack(P):
    P = np.asarray(P)
    W1 = P[PW1:PW2].reshape(HID, IN)
    W2 = P[PW2:PB2].reshape(HID, HID)
    b2 = P[PB2:PW3]
    W3 = P[PW3:PB3].reshape(OUT, HID)
    b3 = P[PB3:NPARAMS]
    return W1, W2, b2, W3, b3


def gelu(x, xp=np):
    u = C_GELU * (x + A_GELU * x * x * x)
    return 0.5 * x * (1.0 + xp.tanh(u))


def gelu_grad(x, xp=np):
    u = C_GELU * (x + A_GELU * x * x * x)
    t = xp.tanh(u)
    return 0.5 * (1.0 + t) + 0.5 * x * (1.0 - t * t) * C_GELU * (1.0 + 3.0 * A_GELU * x * x)


def forward(P, X, rounding=True):
    """Outputs [n, 3] and the intermediates of the backward pass."""
    dt = np.float32 if rounding else np.float64
    q = bf16 if rounding else (lambda a: np.asarray(a, dtype=np.float64))
    W1, W2, b2, W3, b3 = (np.asarray(a, dtype=dt) for a in unpack(P))
    Xb = q(np.asarray(X, dtype=dt))
    W1b, W2b, W3b = q(W1), q(W2), q(W3)
    Z1 = Xb @ W1b.T
    H1 = q(gelu(Z1))
    Z2 = H1 @ W2b.T + b2
    H2 = q(gelu(Z2))
    Y = H2 @ W3b.T + b3
    cache = dict(Xb=Xb, W2b=W2b, W3b=W3b, Z1=Z1, H1=H1, Z2=Z2, H2=H2)
    return Y[:, :USED_OUT], cache


def loss_and_grad(P, X, T, rounding=True):
    """Mean-squared loss (mean over samples, sum over the 3 outputs) and its
    gradient with respect to the parameter vector."""
    dt = np.float32 if rounding else np.float64
    q = bf16 if rounding else (lambda a: np.asarray(a, dtype=np.float64))
    n = X.shape[0]
    y, c = forward(P, X, rounding)
    T = np.asarray(T, dtype=dt)
    e = y - T
    loss = float(np.sum(e.astype(np.float64) ** 2) / n)
    dy = np.zeros((n, OUT), dtype=dt)
    dy[:, :USED_OUT] = (2.0 * e) * (dt(1.0) / dt(n))
    dyb = q(dy)
    g = np.zeros(NPARAMS, dtype=np.float64)
    g[PB3:NPARAMS] = dy.sum(axis=0)
    g[PW3:PB3] = (dyb.T @ c['H2']).ravel()
    dH2 = dyb @ c['W3b']
    dZ2 = dH2 * gelu_grad(c['Z2'])
    g[PB2:PW3] = dZ2.sum(axis=0)
    dZ2b = q(dZ2)
    g[PW2:PB2] = (dZ2b.T @ c['H1']).ravel()
    dH1 = dZ2b @ c['W2b']
    dZ1b = q(dH1 * gelu_grad(c['Z1']))
    g[PW1:PW2] = (dZ1b.T @ c['Xb']).ravel()
    return loss, g


def init_params(seed=0):
    """The initialisation the package uses (solfec_b200.learn.init_params)."""
    rng = np.random.default_rng(seed)
    P = np.zeros(NPARAMS, dtype=np.float32)
    W1 = rng.normal(0.0, 1.0 / np.sqrt(BIAS_COL + 1), size=(HID, IN)).astype(np.float32)
    W1[:, BIAS_COL:] = 0.0
    P[PW1:PW2] = W1.ravel()
    P[PW2:PB2] = rng.normal(0.0, 1.0 / np.sqrt(HID), size=HID * HID).astype(np.float32)
    return P
