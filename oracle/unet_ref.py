"""CPU restatement of the learned preconditioner's network (``vr_unet``).
TEST INFRASTRUCTURE ONLY: the tests use it to check the GPU forward pass and
the GPU gradients; the product package never imports it.

The network has no counterpart in the reference.  This module restates the
same map in numpy FP64: the same layer order and weight layout ([cout][tap][cin]
per 3x3 layer, tap = 3 dr + dz for the neighbour (j + dr - 1, k + dz - 1),
zero padding), the same BF16 rounding points (weights; the input; every
stored activation: conv outputs, pooled and concatenated tensors), and
exact (FP64) sums where the GPU accumulates in FP32.  Gradients are the
hand-written reverse pass of the same graph (gradient tensors are not
rounded, as on the GPU).

Activations are (H, W, C) arrays over the level's (nr_l, nz_l) grid.
"""
from __future__ import annotations

import numpy as np


def bf16(a) -> np.ndarray:
    """Round to the nearest BF16 value, ties to even (as __float2bfloat16_rn)."""
    f = np.asarray(a, dtype=np.float32)
    u = f.view(np.uint32).astype(np.uint64)
    u = (u + 0x7FFF + ((u >> 16) & 1)) & 0xFFFF0000
    return u.astype(np.uint32).view(np.float32).astype(np.float64)


def layers(ch):
    """(cin, cout, level) of the 14 3x3 layers, then the head (c0, 1, 0)."""
    c0, c1, c2, c3 = ch
    L = [(1, c0, 0), (c0, c0, 0), (c0, c1, 1), (c1, c1, 1), (c1, c2, 2), (c2, c2, 2), (c2, c3, 3), (c3, c3, 3),
         (c3 + c2, c2, 2), (c2, c2, 2), (c2 + c1, c1, 1), (c1, c1, 1), (c1 + c0, c0, 0), (c0, c0, 0)]
    return L


def split_params(w, ch):
    out, off = [], 0
    for cin, cout, _ in layers(ch):
        n = cout * 9 * cin
        out.append(np.asarray(w[off:off + n], dtype=np.float64).reshape(cout, 9, cin))
        off += n
    out.append(np.asarray(w[off:off + ch[0]], dtype=np.float64))
    return out


def _shift(a, dr, dz):
    """b[j, k] = a[j + dr - 1, k + dz - 1] with zeros outside."""
    H, W = a.shape[:2]
    b = np.zeros_like(a)
    j0, j1 = max(0, 1 - dr), min(H, H + 1 - dr)
    k0, k1 = max(0, 1 - dz), min(W, W + 1 - dz)
    b[j0:j1, k0:k1] = a[j0 + dr - 1:j1 + dr - 1, k0 + dz - 1:k1 + dz - 1]
    return b


def _unshift(a, dr, dz):
    """Adjoint of _shift: b[j + dr - 1, k + dz - 1] += a[j, k]."""
    return _shift(a, 2 - dr, 2 - dz)


def conv3(x, w):
    y = np.zeros(x.shape[:2] + (w.shape[0],))
    for t in range(9):
        y += _shift(x, t // 3, t % 3) @ w[:, t, :].T
    return y


def conv3_bwd(x, w, gy):
    gw = np.zeros_like(w)
    gx = np.zeros_like(x)
    for t in range(9):
        xs = _shift(x, t // 3, t % 3)
        gw[:, t, :] = np.einsum("hwo,hwi->oi", gy, xs)
        gx += _unshift(gy @ w[:, t, :], t // 3, t % 3)
    return gw, gx


def pool(x, F=2):
    """F x F average: children summed r fastest (dz outer, dr inner), then / F^2."""
    s = np.zeros((x.shape[0] // F, x.shape[1] // F) + x.shape[2:])
    for dz in range(F):
        for dr in range(F):
            s = s + x[dr::F, dz::F]
    return s / (F * F)


def pool_bwd(g, F=2):
    return np.repeat(np.repeat(g, F, axis=0), F, axis=1) / (F * F)


def upcat(coarse, skip, F=2):
    up = np.repeat(np.repeat(coarse, F, axis=0), F, axis=1)
    return np.concatenate([up, skip], axis=2)


def forward(w, ch, x, keep=False, rnd=None, F=2):
    """N(x) for x (nr, nz); BF16 rounding where the GPU stores BF16 (rnd
    replaces the rounding, e.g. the identity for a finite-difference check)."""
    bf16 = rnd if rnd is not None else globals()["bf16"]
    W = split_params(w, ch)
    Wr = [bf16(a) for a in W]
    a = {}
    a["x0"] = bf16(x)[:, :, None]
    a["e0a"] = bf16(conv3(a["x0"], Wr[0]))
    a["e0"] = bf16(conv3(a["e0a"], Wr[1]))
    a["p1"] = bf16(pool(a["e0"], F))
    a["e1a"] = bf16(conv3(a["p1"], Wr[2]))
    a["e1"] = bf16(conv3(a["e1a"], Wr[3]))
    a["p2"] = bf16(pool(a["e1"], F))
    a["e2a"] = bf16(conv3(a["p2"], Wr[4]))
    a["e2"] = bf16(conv3(a["e2a"], Wr[5]))
    a["p3"] = bf16(pool(a["e2"], F))
    a["b3a"] = bf16(conv3(a["p3"], Wr[6]))
    a["b3"] = bf16(conv3(a["b3a"], Wr[7]))
    a["u2"] = upcat(a["b3"], a["e2"], F)
    a["d2a"] = bf16(conv3(a["u2"], Wr[8]))
    a["d2"] = bf16(conv3(a["d2a"], Wr[9]))
    a["u1"] = upcat(a["d2"], a["e1"], F)
    a["d1a"] = bf16(conv3(a["u1"], Wr[10]))
    a["d1"] = bf16(conv3(a["d1a"], Wr[11]))
    a["u0"] = upcat(a["d1"], a["e0"], F)
    a["d0a"] = bf16(conv3(a["u0"], Wr[12]))
    a["d0"] = bf16(conv3(a["d0a"], Wr[13]))
    y = a["d0"] @ Wr[14]
    return (y, a, Wr) if keep else y


def backward(w, ch, x, g, rnd=None, F=2):
    """(dL/dw, dL/dx) of L = sum(g * N(x)) through the same graph."""
    y, a, Wr = forward(w, ch, x, keep=True, rnd=rnd, F=F)
    gw = [None] * 15
    gw[14] = np.einsum("hw,hwc->c", g, a["d0"])
    gd0 = g[:, :, None] * Wr[14][None, None, :]
    gw[13], gd0a = conv3_bwd(a["d0a"], Wr[13], gd0)
    gw[12], gu0 = conv3_bwd(a["u0"], Wr[12], gd0a)
    c1 = ch[1]
    gd1 = pool(gu0[:, :, :c1], F) * (F * F)
    ge0 = gu0[:, :, c1:].copy()
    gw[11], gd1a = conv3_bwd(a["d1a"], Wr[11], gd1)
    gw[10], gu1 = conv3_bwd(a["u1"], Wr[10], gd1a)
    c2 = ch[2]
    gd2 = pool(gu1[:, :, :c2], F) * (F * F)
    ge1 = gu1[:, :, c2:].copy()
    gw[9], gd2a = conv3_bwd(a["d2a"], Wr[9], gd2)
    gw[8], gu2 = conv3_bwd(a["u2"], Wr[8], gd2a)
    c3 = ch[3]
    gb3 = pool(gu2[:, :, :c3], F) * (F * F)
    ge2 = gu2[:, :, c3:].copy()
    gw[7], gb3a = conv3_bwd(a["b3a"], Wr[7], gb3)
    gw[6], gp3 = conv3_bwd(a["p3"], Wr[6], gb3a)
    ge2 += pool_bwd(gp3, F)
    gw[5], ge2a = conv3_bwd(a["e2a"], Wr[5], ge2)
    gw[4], gp2 = conv3_bwd(a["p2"], Wr[4], ge2a)
    ge1 += pool_bwd(gp2, F)
    gw[3], ge1a = conv3_bwd(a["e1a"], Wr[3], ge1)
    gw[2], gp1 = conv3_bwd(a["p1"], Wr[2], ge1a)
    ge0 += pool_bwd(gp1, F)
    gw[1], ge0a = conv3_bwd(a["e0a"], Wr[1], ge0)
    gw[0], gx0 = conv3_bwd(a["x0"], Wr[0], ge0a)
    flat = np.concatenate([gw[i].ravel() for i in range(15)])
    return flat, gx0[:, :, 0]


def nparams(ch) -> int:
    return sum(ci * co * 9 for ci, co, _ in layers(ch)) + ch[0]
