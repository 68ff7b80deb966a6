"""CPU restatement of the learned QMC spawning proposal (test infrastructure only).

The learned proposal has no counterpart in noci-rs (whose generators are uniform, heat-bath and
overlap-weighted, src/input/qmc.rs:10; the uniform one is src/stochastic/state.rs:707-726).
This file states, in numpy FP64, what the GPU kernels compute, so they can be checked:

* bins: child reference x (rank_a, rank_b) class, bin = parent * 25 + rank_a * 5 + rank_b;
* descriptor of a determinant: one-hot parent, one-hot rank_a, one-hot rank_b, and per spin
  the indicator of the orbitals whose occupation its excitation changes (zero-padded to din);
* network din -> 128 -> 128 -> nbin with ReLU, weights rounded to BF16 (round to nearest even)
  in every product, biases in FP32;
* p(bin | parent) = softmax over the bins that hold a child of the parent;
* loss -sum_r w_r log p(bin_r | parent_r) / sum_r w_r and its gradient by backpropagation;
* pgen(child | parent) = mix / (N - 1) + (1 - mix) p(bin(child) | parent) / |bin without parent|.
"""
from __future__ import annotations

import numpy as np

WIDTH = 128
RANK_BINS = 25


def bf16(x: np.ndarray) -> np.ndarray:
    """Round float32 values to the nearest BF16 value (ties to even), returned as float64."""
    b = np.asarray(x, np.float32).view(np.uint32).astype(np.uint64)
    b = (b + 0x7FFF + ((b >> 16) & 1)) & 0xFFFF0000
    return b.astype(np.uint32).view(np.float32).astype(np.float64)


def bins(basis: np.ndarray, nref: int):
    """det_bin, bin sizes."""
    db = basis["parent"].astype(np.int64) * RANK_BINS + basis["rank_a"].astype(np.int64) * 5 + \
        basis["rank_b"].astype(np.int64)
    return db, np.bincount(db, minlength=nref * RANK_BINS)


def features(basis: np.ndarray, rows, nref: int, nmo: int, din: int) -> np.ndarray:
    x = np.zeros((len(rows), din))
    for i, g in enumerate(rows):
        d = basis[g]
        x[i, int(d["parent"])] = 1.0
        x[i, nref + int(d["rank_a"])] = 1.0
        x[i, nref + 5 + int(d["rank_b"])] = 1.0
        for k in range(int(d["rank_a"])):
            x[i, nref + 10 + int(d["idx_a"][k])] = 1.0
            x[i, nref + 10 + int(d["idx_a"][4 + k])] = 1.0
        for k in range(int(d["rank_b"])):
            x[i, nref + 10 + nmo + int(d["idx_b"][k])] = 1.0
            x[i, nref + 10 + nmo + int(d["idx_b"][4 + k])] = 1.0
    return x


def unpack(params: np.ndarray, din: int, nout: int, round_bf16: bool = True):
    p = np.asarray(params, np.float32 if round_bf16 else np.float64)
    o = 0
    out = []
    for shape in ((WIDTH, din), (WIDTH,), (WIDTH, WIDTH), (WIDTH,), (nout, WIDTH), (nout,)):
        n = int(np.prod(shape))
        out.append(p[o:o + n].reshape(shape))
        o += n
    w1, b1, w2, b2, w3, b3 = out
    r = bf16 if round_bf16 else (lambda a: np.asarray(a, np.float64))
    return r(w1), b1.astype(np.float64), r(w2), b2.astype(np.float64), r(w3), b3.astype(np.float64)


def valid_mask(det_bin, sizes, rows):
    m = np.repeat(sizes[None, :], len(rows), axis=0)
    m[np.arange(len(rows)), det_bin[np.asarray(rows)]] -= 1
    return m > 0


def forward(params, x, din, nout, round_bf16=True):
    w1, b1, w2, b2, w3, b3 = unpack(params, din, nout, round_bf16)
    h1 = np.maximum(x @ w1.T + b1, 0.0)
    h2 = np.maximum(h1 @ w2.T + b2, 0.0)
    return h1, h2, h2 @ w3.T + b3


def probs(z, mask):
    zm = np.where(mask, z, -np.inf)
    zm = zm - zm.max(axis=1, keepdims=True)
    e = np.where(mask, np.exp(zm), 0.0)
    return e / e.sum(axis=1, keepdims=True)


def loss_grad(params, x, mask, tbin, w, din, nout, round_bf16=True):
    """Loss and the gradient with respect to the float parameter vector (the BF16 rounding is
    treated as the identity in the backward pass, as the kernels do)."""
    w1, b1, w2, b2, w3, b3 = unpack(params, din, nout, round_bf16)
    h1, h2, z = forward(params, x, din, nout, round_bf16)
    p = probs(z, mask)
    wn = w / w.sum()
    r = np.arange(len(tbin))
    loss = -(wn * np.log(p[r, tbin])).sum()
    dz = p.copy()
    dz[r, tbin] -= 1.0
    dz *= wn[:, None]
    dz[~mask] = 0.0
    gw3, gb3 = dz.T @ h2, dz.sum(0)
    d2 = (dz @ w3) * (h2 > 0)
    gw2, gb2 = d2.T @ h1, d2.sum(0)
    d1 = (d2 @ w2) * (h1 > 0)
    gw1, gb1 = d1.T @ x, d1.sum(0)
    return loss, np.concatenate([gw1.ravel(), gb1, gw2.ravel(), gb2, gw3.ravel(), gb3])


def pgen(cdf_row, det_bin, sizes, g, lam, n, mix):
    b = det_bin[lam]
    pb = cdf_row[b] - (cdf_row[b - 1] if b > 0 else 0.0)
    size = sizes[b] - (1 if det_bin[g] == b else 0)
    return mix / (n - 1) + (1 - mix) * pb / size
