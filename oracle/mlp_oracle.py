"""CPU restatement of the learned preconditioner's network (test infrastructure).

This file is the oracle for the hand-written MLP kernels of libftsp
(ftspolysol_b200/csrc/learned.cuh): the same parameter layout, the same tanh
network and the same loss, written with numpy in float64 so that the GPU's
FP32 forward pass, back-propagation and Adam step can be checked against it.
The network has no counterpart in the reference (the reference has no
semi-implicit scheme); the oracle's own gradient is pinned by central finite
differences in tests/test_mlp_oracle.py.

Layout (floats): W1[H][NIN] b1[H] W2[H][H] b2[H] W3[nout][H] b3[nout].
Loss: L = sum_s sum_f m_sf (z_sf - t_sf)^2 / sum_sf m_sf.
"""
from __future__ import annotations

import numpy as np

NIN = 6
H = 64


def n_params(nout: int) -> int:
    return H * NIN + H + H * H + H + nout * H + nout


def unpack(w: np.ndarray, nout: int):
    w = np.asarray(w, dtype=np.float64)
    o = 0
    W1 = w[o:o + H * NIN].reshape(H, NIN); o += H * NIN
    b1 = w[o:o + H]; o += H
    W2 = w[o:o + H * H].reshape(H, H); o += H * H
    b2 = w[o:o + H]; o += H
    W3 = w[o:o + nout * H].reshape(nout, H); o += nout * H
    b3 = w[o:o + nout]; o += nout
    assert o == len(w)
    return W1, b1, W2, b2, W3, b3


def forward(w, x, nout):
    """x [n, NIN] -> z [n, nout] (and the hidden activations)."""
    W1, b1, W2, b2, W3, b3 = unpack(w, nout)
    h1 = np.tanh(x @ W1.T + b1)
    h2 = np.tanh(h1 @ W2.T + b2)
    z = h2 @ W3.T + b3
    return z, h1, h2


def loss_and_grad(w, x, t, m, nout):
    """Loss and its gradient with respect to w (flat, same layout)."""
    x = np.asarray(x, dtype=np.float64)
    t = np.asarray(t, dtype=np.float64)
    m = np.asarray(m, dtype=np.float64)
    W1, b1, W2, b2, W3, b3 = unpack(w, nout)
    z, h1, h2 = forward(w, x, nout)
    ms = m.sum()
    norm = 1.0 / ms if ms > 0 else 0.0
    e = z - t
    loss = float((m * e * e).sum() * norm)
    dz = 2.0 * m * e * norm                      # [n, nout]
    gW3 = dz.T @ h2
    gb3 = dz.sum(0)
    d2 = (dz @ W3) * (1.0 - h2 * h2)             # [n, H]
    gW2 = d2.T @ h1
    gb2 = d2.sum(0)
    d1 = (d2 @ W2) * (1.0 - h1 * h1)
    gW1 = d1.T @ x
    gb1 = d1.sum(0)
    g = np.concatenate([gW1.ravel(), gb1, gW2.ravel(), gb2, gW3.ravel(), gb3])
    return loss, g


def adam_step(w, g, m1, m2, t, lr, beta1=0.9, beta2=0.999, eps=1e-8):
    """One Adam step (Kingma & Ba, 2015) with bias correction at step t."""
    m1 = beta1 * m1 + (1 - beta1) * g
    m2 = beta2 * m2 + (1 - beta2) * g * g
    mh = m1 / (1 - beta1 ** t)
    vh = m2 / (1 - beta2 ** t)
    return w - lr * mh / (np.sqrt(vh) + eps), m1, m2


def features(k2, Pw, Pp, N, lB, salt):
    """Network inputs of wave vectors with |k|^2 = k2 and spectral powers Pw, Pp."""
    k2 = np.asarray(k2, dtype=np.float64)
    n = k2.size
    return np.stack([np.log1p(k2), np.log1p(np.maximum(Pw, 0)), np.log1p(np.maximum(Pp, 0)),
                     np.full(n, N / 50.0), np.full(n, lB), np.full(n, 10.0 * salt)], axis=1)
