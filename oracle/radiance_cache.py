"""TEST INFRASTRUCTURE: numpy restatement of the GPU library's learned radiance cache.

The reference renderer has no radiance cache, so there is no reference code to pin this
against: "parity unpinned" as far as the reference goes. What pins it instead:
  * the encoding is restated in float32 operation for operation (the GPU result must be
    bit-identical);
  * the network's forward and backward passes are restated in float64 with the GPU's BF16
    rounding points (inputs, activations, back-propagated errors), and checked against
    central finite differences of an unrounded float64 copy of the same network
    (tests/test_cache_oracle.py);
  * Adam is restated in float32 operation for operation.

Methods restated (published descriptions, no code from any implementation): multiresolution
hash encoding (Mueller, Evans, Schied, Keller, "Instant Neural Graphics Primitives",
SIGGRAPH 2022) with the spatial hash of primes 1, 2654435761, 805459861; the relative L2 loss
of neural radiance caching (Mueller, Rousselle, Novak, Keller, SIGGRAPH 2021); Adam (Kingma &
Ba, ICLR 2015).

Only tests/ (and bench.py's CPU arms) import this module.
"""
from __future__ import annotations

import math

import numpy as np

LEVELS = 16
INPUTS = 64
HIDDEN = 64
OUTPUTS = 16
WEIGHTS = 4 * 64 * 64 + 16 * 64
F32 = np.float32


# ---------------------------------------------------------------------------------------------
# number formats
# ---------------------------------------------------------------------------------------------
def bf16_bits(x) -> np.ndarray:
    """float32 -> BF16 bit patterns, round to nearest even."""
    u = np.ascontiguousarray(x, np.float32).view(np.uint32).astype(np.uint64)
    u = (u + 0x7FFF + ((u >> 16) & 1)) >> 16
    return u.astype(np.uint16)


def bf16_value(bits) -> np.ndarray:
    return (np.asarray(bits, np.uint16).astype(np.uint32) << 16).view(np.float32)


def bf16_round(x) -> np.ndarray:
    """Round to BF16 (through float32, as the GPU rounds its FP32 values)."""
    return bf16_value(bf16_bits(np.asarray(x, np.float64).astype(np.float32)))


def f16_value(bits) -> np.ndarray:
    return np.asarray(bits, np.uint16).view(np.float16).astype(np.float32)


# ---------------------------------------------------------------------------------------------
# configuration
# ---------------------------------------------------------------------------------------------
def resolutions(min_res: int, max_res: int, levels: int = LEVELS):
    """Geometric series of grid resolutions: floor(min * 2^(l * log2(max/min) / (L-1)))."""
    r = math.log2(max_res / min_res)
    return [int(math.floor(min_res * 2.0 ** (l * r / (levels - 1)))) for l in range(levels)]


def dense_mask(res, table_size: int) -> int:
    m = 0
    for l, n in enumerate(res):
        if (n + 1) ** 3 <= table_size:
            m |= 1 << l
    return m


class Cache:
    """Parameters of one cache, in the values the GPU computes with."""

    def __init__(self, res, log2_table, lo, hi, grid_f16_bits, mlp_bf16_bits):
        self.res = [int(r) for r in res]
        self.log2_table = int(log2_table)
        self.table = 1 << self.log2_table
        self.dense = dense_mask(self.res, self.table)
        self.lo = np.asarray(lo, F32)
        self.inv_ext = (F32(1.0) / (np.asarray(hi, F32) - self.lo)).astype(F32)
        self.grid_bits = np.asarray(grid_f16_bits, np.uint16).reshape(LEVELS, self.table, 2)
        self.grid = f16_value(self.grid_bits)                      # float32 [L, T, 2]
        self.mlp_bits = np.asarray(mlp_bf16_bits, np.uint16).reshape(WEIGHTS)
        self.W = split_weights(bf16_value(self.mlp_bits).astype(np.float64))


def split_weights(flat):
    flat = np.asarray(flat)
    Ws = [flat[l * 4096:(l + 1) * 4096].reshape(64, 64) for l in range(4)]
    Ws.append(flat[4 * 4096:].reshape(16, 64))
    return Ws


def join_weights(Ws):
    return np.concatenate([w.reshape(-1) for w in Ws])


# ---------------------------------------------------------------------------------------------
# encoding (float32, operation for operation)
# ---------------------------------------------------------------------------------------------
def unit_position(c: Cache, pos):
    p = (np.asarray(pos, F32) - c.lo).astype(F32)
    p = (p * c.inv_ext).astype(F32)
    return np.minimum(np.maximum(p, F32(0.0)), F32(1.0))


def level_cell(c: Cache, l: int, p):
    n = c.res[l]
    x = (p * F32(n)).astype(F32)
    i = np.floor(x).astype(np.uint32)
    i = np.minimum(i, np.uint32(n - 1))
    w = (x - i.astype(F32)).astype(F32)
    return i, w


def corner_index(c: Cache, l: int, i, k: int):
    x = i[:, 0] + np.uint32(k & 1)
    y = i[:, 1] + np.uint32((k >> 1) & 1)
    z = i[:, 2] + np.uint32(k >> 2)
    if (c.dense >> l) & 1:
        n1 = np.uint32(c.res[l] + 1)
        return x + n1 * (y + n1 * z)
    h = x ^ (y * np.uint32(2654435761)) ^ (z * np.uint32(805459861))
    return h & np.uint32(c.table - 1)


def corner_weight(w, k: int):
    one = F32(1.0)
    wx = w[:, 0] if k & 1 else (one - w[:, 0]).astype(F32)
    wy = w[:, 1] if (k >> 1) & 1 else (one - w[:, 1]).astype(F32)
    wz = w[:, 2] if k >> 2 else (one - w[:, 2]).astype(F32)
    return ((wx * wy).astype(F32) * wz).astype(F32)


def encode(c: Cache, records) -> np.ndarray:
    """The 64 float32 network inputs of each record (before BF16 rounding)."""
    r = np.asarray(records, F32).reshape(-1, 16)
    n = len(r)
    out = np.zeros((n, INPUTS), F32)
    with np.errstate(over="ignore"):
        p = unit_position(c, r[:, 0:3])
        for l in range(LEVELS):
            i, w = level_cell(c, l, p)
            f0 = np.zeros(n, F32)
            f1 = np.zeros(n, F32)
            for k in range(8):
                wt = corner_weight(w, k)
                v = c.grid[l, corner_index(c, l, i, k)]
                f0 = (f0 + (wt * v[:, 0]).astype(F32)).astype(F32)
                f1 = (f1 + (wt * v[:, 1]).astype(F32)).astype(F32)
            out[:, 2 * l] = f0
            out[:, 2 * l + 1] = f1
    d = r[:, 3:6]
    for a in range(3):
        s = ((d[:, a] + F32(1.0)).astype(F32) * F32(2.0)).astype(F32)
        for k in range(5):
            out[:, 32 + 5 * a + k] = np.maximum(F32(0.0), (F32(1.0) - np.abs((s - F32(k)).astype(F32))).astype(F32))
    out[:, 47:50] = r[:, 6:9]
    out[:, 50] = r[:, 9]
    out[:, 51:54] = r[:, 10:13]
    out[:, 54:57] = r[:, 13:16]
    out[:, 57] = 1.0
    return out


def corners(c: Cache, records):
    """Per level: corner indices [n, 8] and float32 trilinear weights [n, 8]."""
    r = np.asarray(records, F32).reshape(-1, 16)
    p = unit_position(c, r[:, 0:3])
    res = []
    for l in range(LEVELS):
        i, w = level_cell(c, l, p)
        res.append((np.stack([corner_index(c, l, i, k) for k in range(8)], 1),
                    np.stack([corner_weight(w, k) for k in range(8)], 1)))
    return res


# ---------------------------------------------------------------------------------------------
# network (float64 with the GPU's BF16 rounding points, or unrounded)
# ---------------------------------------------------------------------------------------------
def forward(Ws, x, rounded: bool = True):
    """Activations a0..a4 and the 16 outputs. rounded: a_l rounded to BF16 like the GPU."""
    rnd = bf16_round if rounded else (lambda v: np.asarray(v, np.float64))
    a = [rnd(x).astype(np.float64)]
    for l in range(4):
        z = a[-1] @ Ws[l].T
        a.append(rnd(np.maximum(z, 0.0)).astype(np.float64))
    y = a[-1] @ Ws[4].T
    return a, y


def loss_and_grad(y, t, mask=None, rounded: bool = True, den=None):
    """Mean relative L2 loss over samples and channels and its gradient w.r.t. y[:, :3]
    (the prediction held constant in the denominator; `den` fixes that denominator, for
    finite differences of the surrogate whose exact gradient this is)."""
    y3 = np.asarray(y, np.float64)[:, :3]
    t = np.asarray(t, np.float64)
    m = np.ones_like(y3, bool) if mask is None else np.asarray(mask, bool)
    n = len(y3)
    if rounded:  # float32 as the GPU computes it
        yf = y3.astype(F32)
        tf = t.astype(F32)
        scale = F32(1.0) / (F32(3.0) * F32(n))
        d = (yf - tf).astype(F32)
        den = ((yf * yf).astype(F32) + F32(0.01)).astype(F32)
        g = (((F32(2.0) * d).astype(F32) / den).astype(F32) * scale).astype(F32)
        lt = ((d * d).astype(F32) / den).astype(F32)
        g = np.where(m, g, F32(0.0))
        loss = float(np.sum(np.where(m, lt, 0.0), dtype=np.float64) * float(scale))
        return loss, g.astype(np.float64)
    scale = 1.0 / (3.0 * n)
    d = y3 - t
    if den is None:
        den = y3 * y3 + 0.01
    g = np.where(m, 2.0 * d / den * scale, 0.0)
    loss = float(np.sum(np.where(m, d * d / den, 0.0)) * scale)
    return loss, g


def backward(Ws, a, gy, rounded: bool = True):
    """Weight gradients [dW0..dW4] (row = output) and the gradient of the 32 hash inputs."""
    rnd = bf16_round if rounded else (lambda v: np.asarray(v, np.float64))
    n = len(gy)
    d = [None] * 6
    dy = np.zeros((n, OUTPUTS))
    dy[:, :3] = gy
    d[5] = rnd(dy).astype(np.float64)
    for l in range(4, 0, -1):
        d[l] = rnd((d[l + 1] @ Ws[l]) * (a[l] > 0)).astype(np.float64)
    g_in = d[1] @ Ws[0][:, :32]
    dW = [d[l + 1].T @ a[l] for l in range(5)]
    return dW, g_in


def loss_unrounded_full(c: Cache, Ws, grid, records, targets, den):
    """The loss with a fixed denominator as a function of float64 weights and grid features
    (finite differences of this equal the gradient the GPU computes, up to rounding)."""
    saved = c.grid
    c.grid = grid
    try:
        x = encode64(c, records)
        a, y = forward(Ws, x, rounded=False)
        loss, _ = loss_and_grad(y, targets, rounded=False, den=den)
        return loss
    finally:
        c.grid = saved


def encode64(c: Cache, records):
    """encode() in float64 (features interpolated from float64 grid values)."""
    r = np.asarray(records, F32).reshape(-1, 16)
    x = encode(c, r).astype(np.float64)
    for l, (idx, wt) in enumerate(corners(c, r)):
        g = np.asarray(c.grid[l], np.float64)[idx]          # [n, 8, 2]
        x[:, 2 * l:2 * l + 2] = np.einsum("nk,nkf->nf", wt.astype(np.float64), g)
    return x


def grid_grad(c: Cache, records, g_in):
    """Scatter of the hash-input gradients to a dense [L, T, 2] float64 gradient."""
    out = np.zeros((LEVELS, c.table, 2))
    for l, (idx, wt) in enumerate(corners(c, records)):
        for k in range(8):
            w = wt[:, k].astype(np.float64)
            np.add.at(out[l, :, 0], idx[:, k], w * g_in[:, 2 * l])
            np.add.at(out[l, :, 1], idx[:, k], w * g_in[:, 2 * l + 1])
    return out


def gradients(c: Cache, records, targets, mask=None):
    """Loss, weight gradients and dense grid gradient as the GPU computes them."""
    x = encode(c, records)
    a, y = forward(c.W, x)
    loss, gy = loss_and_grad(y, targets, mask)
    dW, g_in = backward(c.W, a, gy)
    return loss, dW, grid_grad(c, records, g_in)


def infer(c: Cache, records):
    x = encode(c, records)
    _, y = forward(c.W, x)
    return np.maximum(y[:, :3], 0.0)


# ---------------------------------------------------------------------------------------------
# Adam (float32, operation for operation)
# ---------------------------------------------------------------------------------------------
def adam(p, m, v, g, lr, b1, b2, eps, t, active=None):
    """One Adam step; `active` (bool, same shape) limits the update to those parameters."""
    p, m, v, g = (np.asarray(a, F32).copy() for a in (p, m, v, g))
    lr, b1, b2, eps = F32(lr), F32(b1), F32(b2), F32(eps)
    c1 = F32(1.0 - float(b1) ** t)
    c2 = F32(1.0 - float(b2) ** t)
    m2 = ((b1 * m).astype(F32) + ((F32(1.0) - b1) * g).astype(F32)).astype(F32)
    v2 = ((b2 * v).astype(F32) + (((F32(1.0) - b2) * g).astype(F32) * g).astype(F32)).astype(F32)
    mh = (m2 / c1).astype(F32)
    vh = (v2 / c2).astype(F32)
    p2 = (p - ((lr * mh).astype(F32) / (np.sqrt(vh).astype(F32) + eps).astype(F32)).astype(F32)).astype(F32)
    if active is None:
        return p2, m2, v2
    return np.where(active, p2, p), np.where(active, m2, m), np.where(active, v2, v)
