"""Test infrastructure: the CPU oracle of the learned block proposal (no
counterpart in the reference).  Only tests and the bench's checks import it.

* ``block_features``: the incoherent power-sum features of every block of a
  band, per decimation level and harmonic count, as cs_block_features
  defines them (FP64 here).
* ``mlp_forward`` / ``mlp_backward``: the proposal network
  din -> dh -> dh -> 1 with ReLU, weights rounded to BF16 as the device uses
  them, FP64 arithmetic; the weighted binary cross-entropy with logits and
  the gradients of every parameter, against which the device's FP32 kernels
  are checked.
"""
import math

import numpy as np


def bf16_round(x):
    """FP32 values rounded to BF16 (nearest, ties to even), as FP32."""
    u = np.ascontiguousarray(x, np.float32).view(np.uint32).astype(np.uint64)
    u = (u + 0x7FFF + ((u >> 16) & 1)) & 0xFFFF0000
    return u.astype(np.uint32).view(np.float32)


def block_features(amps, r_lo, lodr, Nprof, total, levels):
    """[nblocks, sum of Hk]: per block and decimation level (k, Hk) in `levels`
    order, for H = 1..Hk, z = (S - H)/sqrt(H) with S(r) = sum_{i<=H}
    |X[rint(i*k*r)]|^2 at every trial r of the block (bins outside
    [1, len(amps)) count 1); the feature is asinh(max over the block of z)."""
    namps = len(amps)
    pw = np.abs(amps.astype(np.complex128)) ** 2
    nb = -(-total // Nprof)
    out = np.zeros((nb, sum(H for _, H in levels)))
    for b in range(nb):
        n = min(Nprof, total - b * Nprof)
        r = r_lo + (b * Nprof + np.arange(n)) * lodr
        col = 0
        for k, Hk in levels:
            i = np.arange(1, Hk + 1)
            bins = np.rint((i[None, :] * k) * r[:, None]).astype(np.int64)
            ok = (bins >= 1) & (bins < namps)
            p = np.where(ok, pw[np.clip(bins, 0, namps - 1)], 1.0)
            z = (np.cumsum(p, axis=1) - i[None, :]) / np.sqrt(i)[None, :]
            out[b, col:col + Hk] = np.arcsinh(z.max(axis=0))
            col += Hk
    return out


def levels_of(nharms, decimations):
    """(k, Hk) of the search's levels: k = 1, then every decimation above 1."""
    return [(1, nharms)] + [(k, nharms // k) for k in decimations if k > 1]


def _w(params, k, round_weights):
    w = np.asarray(params[k])
    return (bf16_round(w) if round_weights else w).astype(np.float64)


def mlp_forward(params, x, round_weights=True):
    """params: dict of FP32 masters w1 [dh,din], b1, w2 [dh,dh], b2, w3 [dh], b3 [1].
    Returns (h1, h2, z) with BF16-rounded weights (as the device uses them;
    round_weights=False: the masters themselves), FP64 arithmetic."""
    w1, w2, w3 = (_w(params, k, round_weights) for k in ("w1", "w2", "w3"))
    x = np.asarray(x, np.float64)
    h1 = np.maximum(x @ w1.T + params["b1"].astype(np.float64), 0.0)
    h2 = np.maximum(h1 @ w2.T + params["b2"].astype(np.float64), 0.0)
    z = h2 @ w3 + float(params["b3"][0])
    return h1, h2, z


def bce_loss(z, y, pos_weight):
    w = np.where(y > 0.5, pos_weight, 1.0)
    sp = np.where(z > 0, z + np.log1p(np.exp(-np.abs(z))), np.log1p(np.exp(-np.abs(z))))
    return float(np.mean(w * (sp - y * z)))


def mlp_backward(params, x, y, pos_weight, round_weights=True):
    """(loss, grads) of the weighted BCE with logits, mean over rows; the
    backward pass uses the same (BF16-rounded) weights as the forward."""
    w2, w3 = (_w(params, k, round_weights) for k in ("w2", "w3"))
    x = np.asarray(x, np.float64)
    y = np.asarray(y, np.float64)
    h1, h2, z = mlp_forward(params, x, round_weights)
    n = len(x)
    w = np.where(y > 0.5, pos_weight, 1.0)
    dz = w * (1.0 / (1.0 + np.exp(-z)) - y) / n
    g = {"w3": h2.T @ dz, "b3": np.array([dz.sum()])}
    dh2 = dz[:, None] * w3[None, :] * (h2 > 0)
    g["w2"] = dh2.T @ h1
    g["b2"] = dh2.sum(axis=0)
    dh1 = (dh2 @ w2) * (h1 > 0)
    g["w1"] = dh1.T @ x
    g["b1"] = dh1.sum(axis=0)
    return bce_loss(z, y, pos_weight), g
