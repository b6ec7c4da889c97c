"""CPU oracle of the learned-proposal network (test infrastructure only).

Float64 restatement of the forward and backward passes of
gaffa_b200/csrc/proposal.cu, used to check the CUDA kernels' outputs and
gradients.  Like the kernels, it takes bf16 weights and inputs and rounds each
layer's post-ReLU output to bf16 before the next layer.  There is no
reference counterpart: gaffa has no learned component.
"""
from __future__ import annotations

import numpy as np


def bf16_round(x: np.ndarray) -> np.ndarray:
    """Round-to-nearest-even to bfloat16, returned as float64."""
    f = np.ascontiguousarray(x, np.float32)
    u = f.view(np.uint32).astype(np.uint64)
    u = (u + 0x7FFF + ((u >> 16) & 1)) & 0xFFFF0000
    return u.astype(np.uint32).view(np.float32).astype(np.float64)


def conv1d(x: np.ndarray, w: np.ndarray, b: np.ndarray | None) -> np.ndarray:
    """y[n][co][t] = b[co] + sum_{ci,k} w[co][ci][k] x[n][ci][t + k - K//2] (zero padding)."""
    n, cin, L = x.shape
    cout, _, K = w.shape
    P = K // 2
    xp = np.zeros((n, cin, L + 2 * P))
    xp[:, :, P:P + L] = x
    y = np.zeros((n, cout, L))
    for k in range(K):
        y += np.einsum("oc,ncl->nol", w[:, :, k], xp[:, :, k:k + L])
    if b is not None:
        y += b[None, :, None]
    return y


def forward(feat, ws, bs, wh, bh, octaves: int, rounding: bool = True):
    """(logits [n][octaves], activations, per-octave softmax) with bf16
    rounding of weights and activations (rounding=False: exact float64, for
    finite-difference checks of the oracle itself)."""
    rnd = bf16_round if rounding else (lambda a: np.asarray(a, np.float64))
    acts = [rnd(feat)]
    x = acts[0]
    for w, b in zip(ws, bs):
        x = rnd(np.maximum(conv1d(x, rnd(w), b), 0.0))
        acts.append(x)
    s = np.einsum("c,ncl->nl", wh, x) + bh[0]
    n, L = s.shape
    bins = L // octaves
    s = s.reshape(n, octaves, bins)
    m = s.max(axis=2, keepdims=True)
    e = np.exp(s - m)
    logits = m[..., 0] + np.log(e.sum(axis=2)) - np.log(bins)
    return logits, acts, e / e.sum(axis=2, keepdims=True)


def softplus(z):
    return np.maximum(z, 0.0) + np.log1p(np.exp(-np.abs(z)))


def loss_and_grads(feat, ws, bs, wh, bh, labels, pos_weight: float, octaves: int, rounding: bool = True):
    """Mean positive-weighted BCE over n x octaves and its gradients
    (d ws, d bs, d wh, d bh); weights of the conv layers as the kernels see
    them (bf16) for the forward pass, gradients w.r.t. the fp32 masters."""
    logits, acts, soft = forward(feat, ws, bs, wh, bh, octaves, rounding)
    rnd = bf16_round if rounding else (lambda a: np.asarray(a, np.float64))
    y = labels
    loss = (pos_weight * y * softplus(-logits) + (1 - y) * softplus(logits)).sum()
    sig = 1.0 / (1.0 + np.exp(-logits))
    dlogit = sig * (1 - y + pos_weight * y) - pos_weight * y
    n, _, L = acts[-1].shape
    ds = (dlogit[..., None] * soft).reshape(n, L)
    dwh = np.einsum("nl,ncl->c", ds, acts[-1])
    dbh = np.array([ds.sum()])
    dy = wh[None, :, None] * ds[:, None, :]
    dws, dbs = [None] * len(ws), [None] * len(ws)
    for i in range(len(ws) - 1, -1, -1):
        w = rnd(ws[i])
        dz = dy * (acts[i + 1] > 0)
        x = acts[i]
        K = w.shape[2]
        P = K // 2
        xp = np.zeros((n, x.shape[1], L + 2 * P))
        xp[:, :, P:P + L] = x
        dws[i] = np.stack([np.einsum("nol,ncl->oc", dz, xp[:, :, k:k + L]) for k in range(K)], axis=2)
        dbs[i] = dz.sum(axis=(0, 2))
        dzp = np.zeros((n, dz.shape[1], L + 2 * P))
        dzp[:, :, P:P + L] = dz
        dy = np.zeros_like(x)
        for k in range(K):
            dy += np.einsum("oc,nol->ncl", w[:, :, k], dzp[:, :, 2 * P - k:2 * P - k + L])
    scale = 1.0 / (n * octaves)
    return loss * scale, [g * scale for g in dws], [g * scale for g in dbs], dwh * scale, dbh * scale, logits
