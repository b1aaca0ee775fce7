"""CPU restatement of the learned Davidson preconditioner.  TEST INFRASTRUCTURE
ONLY: the tests check the GPU training (forward and backward) and inference
kernels against it; the product never imports it.

The preconditioner has no counterpart in the reference, whose Davidson uses
the diagonal correction t_i = r_i / (E0 - H_ii) (chemistry/tpb/davidson.h:853-862).
Here a small network shifts that denominator per determinant:

    features x_i  (see ``features``)
    h1 = relu(W1 x + b1), h2 = relu(W2 h1 + b2)     (128 units each, BF16 weights)
    z  = w3 . h2 + b3,    s = S tanh(z)
    t_i = r_i / (E0 - H_ii - s_i)                   (regularised like the diagonal)

Training minimises, for one harvested (u, r, t) triple, the scale-invariant
loss 1 - cos^2(P t_hat, t) over weighted samples, P the projection
orthogonal to the Ritz vector u (Davidson removes that component anyway).

Everything here is float64 on the effective (BF16-rounded) weights, with
straight-through gradients, as the GPU kernels compute them in FP32.
"""
from __future__ import annotations

import numpy as np

HID = 128
WINDOW = 8  # orbitals either side of the Fermi level per spin


def feature_width() -> int:
    """Raw features (2 + 2 spins x (2 x WINDOW + 1)) padded to a multiple of 16."""
    raw = 2 + 2 * (2 * WINDOW + 1)
    return (raw + 15) // 16 * 16


def bf16(x):
    """Round to the nearest bfloat16 (ties to even), returned as float64."""
    a = np.asarray(x, dtype=np.float32).copy()
    u = a.view(np.uint32).astype(np.uint64)
    lsb = (u >> np.uint64(16)) & np.uint64(1)
    u = (u + np.uint64(0x7FFF) + lsb) & np.uint64(0xFFFF0000)
    return u.astype(np.uint32).view(np.float32).astype(np.float64)


def n_params(F: int) -> int:
    return HID * F + HID + HID * HID + HID + HID + 1


def unpack(w, F: int):
    w = np.asarray(w, dtype=np.float64)
    o = 0
    W1 = w[o:o + HID * F].reshape(HID, F); o += HID * F
    b1 = w[o:o + HID]; o += HID
    W2 = w[o:o + HID * HID].reshape(HID, HID); o += HID * HID
    b2 = w[o:o + HID]; o += HID
    w3 = w[o:o + HID]; o += HID
    b3 = w[o]
    return W1, b1, W2, b2, w3, b3


def pack(W1, b1, W2, b2, w3, b3) -> np.ndarray:
    return np.concatenate([np.ravel(W1), b1, np.ravel(W2), b2, w3, [b3]])


def effective(w, F: int, rounding: bool = True) -> np.ndarray:
    """The weights the kernels use: every parameter rounded to BF16
    (rounding=False only for finite-difference checks of this file)."""
    w = np.asarray(w, dtype=np.float64)
    return bf16(w) if rounding else w


def _string_features(s: np.ndarray, ne: int) -> np.ndarray:
    """Holes in the WINDOW orbitals below the Fermi level, particles in the
    WINDOW orbitals above it, and the excitation rank / ne."""
    s = np.asarray(s, dtype=np.uint64)
    out = np.zeros((len(s), 2 * WINDOW + 1))
    for j in range(WINDOW):
        p = ne - 1 - j
        if p >= 0:
            out[:, j] = 1.0 - ((s >> np.uint64(p)) & np.uint64(1)).astype(np.float64)
        p = ne + j
        if p < 64:
            out[:, WINDOW + j] = ((s >> np.uint64(p)) & np.uint64(1)).astype(np.float64)
    aufbau = np.uint64((1 << ne) - 1)
    rank = np.array([bin(int(x) & ~int(aufbau)).count("1") for x in s], dtype=np.float64)
    out[:, 2 * WINDOW] = rank / max(ne, 1)
    return out


def features(astr, bstr, ia, ib, hii, theta, r, n_total):
    """Features of determinants (ia, ib): asinh(H_ii - theta),
    asinh(|r_i| sqrt(N)) / 4 (the magnitude only, so the correction
    r_i / (den - s) flips sign with r_i whatever the sign convention of the
    vectors), then each spin's window bits and rank."""
    astr = np.asarray(astr, dtype=np.uint64)
    bstr = np.asarray(bstr, dtype=np.uint64)
    ne_a = bin(int(astr[0])).count("1")
    ne_b = bin(int(bstr[0])).count("1")
    F = feature_width()
    X = np.zeros((len(ia), F))
    X[:, 0] = np.arcsinh(np.asarray(hii) - theta)
    X[:, 1] = np.arcsinh(np.abs(np.asarray(r)) * np.sqrt(n_total)) / 4.0
    k = 2 * WINDOW + 1
    X[:, 2:2 + k] = _string_features(astr[np.asarray(ia)], ne_a)
    X[:, 2 + k:2 + 2 * k] = _string_features(bstr[np.asarray(ib)], ne_b)
    return X


def forward(w, F, X, S, bf16_acts=False, rounding=True):
    """(z, s, h1, h2, a1, a2) for features X [n, F]; bf16_acts rounds X and
    h1 to BF16 as the tensor-core inference kernel's operands are."""
    W1, b1, W2, b2, w3, b3 = unpack(effective(w, F, rounding), F)
    Xe = bf16(X) if bf16_acts else np.asarray(X, dtype=np.float64)
    a1 = Xe @ W1.T + b1
    h1 = np.maximum(a1, 0.0)
    if bf16_acts:
        h1 = bf16(h1)
    a2 = h1 @ W2.T + b2
    h2 = np.maximum(a2, 0.0)
    z = h2 @ w3 + b3
    return z, S * np.tanh(z), h1, h2, a1, a2


def correction(r, den, s, eps_reg):
    dd = den - s
    dd = np.where(np.abs(dd) > eps_reg, dd, dd - eps_reg)
    return r / dd, dd


def loss_and_grad(w, F, X, r, den, u, t, wt, S, eps_reg, rounding=True):
    """Loss 1 - cos^2(P t_hat, t) with weights wt, and its gradient with
    respect to the (master) parameters, straight through the BF16 rounding."""
    W1, b1, W2, b2, w3, b3 = unpack(effective(w, F, rounding), F)
    z, s, h1, h2, a1, a2 = forward(w, F, X, S, rounding=rounding)
    th, dd = correction(r, den, s, eps_reg)
    p = np.sum(wt * u * th)
    uu = np.sum(wt * u * u)
    c = np.sum(wt * th * t) - (p / uu) * np.sum(wt * u * t)
    a = np.sum(wt * th * th) - p * p / uu
    b = np.sum(wt * t * t)
    q = np.sum(wt * u * t)
    loss = 1.0 - c * c / (a * b)
    tp = th - (p / uu) * u
    g_th = wt * (2.0 * c / (a * b)) * (c * tp / a - t) + (wt * u / uu) * (2.0 * c * q / (a * b))
    g_s = g_th * th / dd
    g_z = g_s * S * (1.0 - np.tanh(z) ** 2)
    dw3 = h2.T @ g_z
    db3 = np.sum(g_z)
    g_h2 = np.outer(g_z, w3) * (a2 > 0)
    dW2 = g_h2.T @ h1
    db2 = g_h2.sum(0)
    g_h1 = (g_h2 @ W2) * (a1 > 0)
    dW1 = g_h1.T @ np.asarray(X, dtype=np.float64)
    db1 = g_h1.sum(0)
    return loss, pack(dW1, db1, dW2, db2, dw3, db3)


def init_weights(F: int, seed: int) -> np.ndarray:
    """He-initialised hidden layers, a small output layer (the network starts
    close to the diagonal preconditioner, s ~ 0)."""
    rng = np.random.default_rng(seed)
    W1 = rng.normal(0.0, np.sqrt(2.0 / F), size=(HID, F))
    W2 = rng.normal(0.0, np.sqrt(2.0 / HID), size=(HID, HID))
    w3 = rng.normal(0.0, 0.01, size=HID)
    return pack(W1, np.zeros(HID), W2, np.zeros(HID), w3, 0.0)
