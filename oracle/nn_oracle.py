"""CPU restatement of the coolingh surrogate's network (TEST INFRASTRUCTURE ONLY).

Used by tests/ to check the device training kernel's loss and gradients and
the forward pass.  The library never imports this module.

The network is 4 -> 64 -> 64 -> 2; hidden layer 1 uses the cubic saturating
activation g(x) = y (1 - y^2/12), y = clamp(x, -2, 2), hidden layer 2
uses tanh; parameters are a
flat vector (W1 [64][4], b1, W2 [64][64], b2, W3 [2][64], b3).  The device
computes its matrix products on BF16 operands with FP32 accumulation; with
``bf16=True`` this restatement rounds the same operands to BF16 (round to
nearest even) at the same points and accumulates in float64, so that the
two agree to accumulation-order and one-ulp-of-bf16 effects.  With
``bf16=False`` it is the plain float64 network, whose gradient is checked
against finite differences.
"""
from __future__ import annotations

import numpy as np

H, NIN, NOUT = 64, 4, 2
LOSS_W1 = 4.0     # weight of output 1 (temperature rate) in the loss
P_W1 = 0
P_B1 = P_W1 + H * NIN
P_W2 = P_B1 + H
P_B2 = P_W2 + H * H
P_W3 = P_B2 + H
P_B3 = P_W3 + NOUT * H
NPARAM = P_B3 + NOUT


def bf16(x: np.ndarray) -> np.ndarray:
    """Round to bfloat16 (nearest even) and return as float64."""
    f = np.asarray(x, np.float32)
    u = f.view(np.uint32).astype(np.uint64)
    r = ((u + 0x7FFF + ((u >> 16) & 1)) >> 16) << 16
    return r.astype(np.uint32).view(np.float32).astype(np.float64)


def unpack(p: np.ndarray):
    p = np.asarray(p, np.float64)
    W1 = p[P_W1:P_B1].reshape(H, NIN)
    b1 = p[P_B1:P_W2]
    W2 = p[P_W2:P_B2].reshape(H, H)
    b2 = p[P_B2:P_W3]
    W3 = p[P_W3:P_B3].reshape(NOUT, H)
    b3 = p[P_B3:NPARAM]
    return W1, b1, W2, b2, W3, b3


def forward(p, X, bf: bool = True):
    """X: (n, 4) features -> (n, 2) outputs, plus the hidden activations."""
    r = bf16 if bf else (lambda a: np.asarray(a, np.float64))
    W1, b1, W2, b2, W3, b3 = unpack(p)
    Xb = r(X)
    Y1 = np.clip(Xb @ r(W1).T + b1, -2.0, 2.0)
    H1 = Y1 * (1.0 - Y1 * Y1 / 12.0)
    H1b = r(H1)
    H2 = np.tanh(H1b @ r(W2).T + b2)
    H2b = r(H2)
    O = H2b @ r(W3).T + b3
    return O, (Xb, Y1, H1b, H2, H2b)


def loss_grad(p, X, Y, bf: bool = True):
    """Mean over samples of the weighted summed squared output error (output
    1 weighted LOSS_W1), and its gradient."""
    r = bf16 if bf else (lambda a: np.asarray(a, np.float64))
    _, b1, W2, b2, W3, b3 = unpack(p)
    n = X.shape[0]
    O, (Xb, Y1, H1b, H2, H2b) = forward(p, X, bf)
    E = O - Y
    wt = np.array([1.0, LOSS_W1])
    loss = float((E * E * wt).sum() / n)
    dO = 2.0 * E * wt / n
    dOb = r(dO)
    dZ2 = (dOb @ r(W3)) * (1.0 - H2 * H2)
    dZ2b = r(dZ2)
    dZ1 = (dZ2b @ r(W2)) * (1.0 - Y1 * Y1 / 4.0)
    dZ1b = r(dZ1)
    g = np.zeros(NPARAM)
    g[P_W1:P_B1] = (dZ1b.T @ Xb).ravel()
    g[P_B1:P_W2] = dZ1.sum(0)
    g[P_W2:P_B2] = (dZ2b.T @ H1b).ravel()
    g[P_B2:P_W3] = dZ2.sum(0)
    g[P_W3:P_B3] = (dOb.T @ H2b).ravel()
    g[P_B3:NPARAM] = dO.sum(0)
    return loss, g


def groups():
    """Parameter groups (name, slice) for per-group comparisons."""
    return [("W1", slice(P_W1, P_B1)), ("b1", slice(P_B1, P_W2)), ("W2", slice(P_W2, P_B2)),
            ("b2", slice(P_B2, P_W3)), ("W3", slice(P_W3, P_B3)), ("b3", slice(P_B3, NPARAM))]
