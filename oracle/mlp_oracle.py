"""Numpy float64 restatement of the learned tuner's MLP (TEST INFRASTRUCTURE ONLY).

The device implementation lives in deleglise-rivat_b200/csrc/dr_mlp.cu; this is
the CPU oracle its forward pass and gradients are checked against.  Same
parameter layout (W1[64][4] b1[64] W2[64][64] b2[64] W3[4][64] b3[4]), same
loss (mean over the B x 4 outputs of the squared error), same feature and
target normalisation.  Pinned by finite differences in tests/test_mlp_oracle.py.
"""
import math

import numpy as np

K_IN, K_HID, K_OUT = 4, 64, 4
O_W1 = 0
O_B1 = O_W1 + K_HID * K_IN
O_W2 = O_B1 + K_HID
O_B2 = O_W2 + K_HID * K_HID
O_W3 = O_B2 + K_HID
O_B3 = O_W3 + K_OUT * K_HID
N_PARAMS = O_B3 + K_OUT  # 4740

IN_MEAN = np.array([13.0, 35.0, 148.0, 0.0])
IN_SCALE = np.array([3.0, 3.0, 64.0, 8.0])
OUT_MEAN = np.array([1.2, 0.0, 34.0, 16.0])
OUT_SCALE = np.array([0.5, 1.5, 4.0, 1.5])


def unpack(P):
    P = np.asarray(P, dtype=np.float64)
    W1 = P[O_W1:O_B1].reshape(K_HID, K_IN)
    b1 = P[O_B1:O_W2]
    W2 = P[O_W2:O_B2].reshape(K_HID, K_HID)
    b2 = P[O_B2:O_W3]
    W3 = P[O_W3:O_B3].reshape(K_OUT, K_HID)
    b3 = P[O_B3:N_PARAMS]
    return W1, b1, W2, b2, W3, b3


def forward(P, x):
    W1, b1, W2, b2, W3, b3 = unpack(P)
    x = np.asarray(x, dtype=np.float64)
    z1 = x @ W1.T + b1
    h1 = np.maximum(z1, 0.0)
    z2 = h1 @ W2.T + b2
    h2 = np.maximum(z2, 0.0)
    y = h2 @ W3.T + b3
    return y, (x, z1, h1, z2, h2)


def loss(P, x, t):
    y, _ = forward(P, x)
    return float(np.mean((y - np.asarray(t, dtype=np.float64)) ** 2))


def grad(P, x, t):
    """d loss / d P by back-propagation, in the flat parameter layout."""
    W1, b1, W2, b2, W3, b3 = unpack(P)
    y, (x, z1, h1, z2, h2) = forward(P, x)
    B = x.shape[0]
    dy = 2.0 * (y - np.asarray(t, dtype=np.float64)) / (B * K_OUT)
    g = np.zeros(N_PARAMS)
    g[O_W3:O_B3] = (dy.T @ h2).ravel()
    g[O_B3:N_PARAMS] = dy.sum(0)
    d2 = (dy @ W3) * (z2 > 0)
    g[O_W2:O_B2] = (d2.T @ h1).ravel()
    g[O_B2:O_W3] = d2.sum(0)
    d1 = (d2 @ W2) * (z1 > 0)
    g[O_W1:O_B1] = (d1.T @ x).ravel()
    g[O_B1:O_W2] = d1.sum(0)
    return g


def features(X, budget_bytes, sms, batch):
    lx = min(16.0, max(10.0, math.log10(max(X, 2))))  # clamped to the training domain
    lb = min(37.33, max(33.0, math.log2(max(budget_bytes, 1))))
    raw = np.array([lx, lb, float(sms), math.log2(max(batch, 1))])
    return (raw - IN_MEAN) / IN_SCALE
