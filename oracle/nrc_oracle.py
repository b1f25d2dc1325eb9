"""TEST ORACLE for the neural radiance cache (numpy, CPU).

The reference renderer has no radiance cache; this module restates, for the
tests only, the cache that libyrcuda implements on the GPU so that its
forward pass, gradients and optimiser step can be checked value by value:

* encoding (64 inputs): a 16-level hash grid over the position normalised to
  the scene box (2 features per level, 2^19 entries per level, resolutions
  from 16 to 2048; a level whose (ceil(scale) + 2)^3 grid fits in 2^19
  entries is indexed densely, the others by the spatial hash
  x ^ y * 2654435761 ^ z * 805459861 mod 2^19; trilinear weights), the 16
  real spherical harmonics of degrees 0-3 of the view direction, the normal
  mapped to [0, 1], roughness, diffuse and specular albedo, a constant 1 and
  zero padding;
* network: 5 hidden layers of width 64 with ReLU and a 3-wide output layer
  (stored as 16 rows, the last 13 zero), exp activation (argument clamped at
  15); weights and activations rounded to bf16 at the points where the GPU
  stores them, products accumulated in fp32;
* loss: relative L2, mean over samples and channels of
  (rgb - target)^2 / (stop_grad(rgb)^2 + 0.01);
* optimiser: Adam (lr 1e-2, betas 0.9 / 0.99, eps 1e-15) on fp32 master
  copies of the weights and of the grid, with bias correction; on the grid
  lazily (the sparse-Adam variant, e.g. PyTorch's SparseAdam): only the
  entries a step's samples touched update, as does their moving average.

Only tests import this module.
"""
from __future__ import annotations

import math

import numpy as np

LEVELS = 16
FEATURES = 2
LOG2_TABLE = 19
TABLE = 1 << LOG2_TABLE
BASE_RES = 16.0
FINEST_RES = 2048.0
WIDTH = 64
HIDDEN = 5
OUT_ROWS = 16
LR, BETA1, BETA2, EPS = 1.0e-2, 0.9, 0.99, 1.0e-15
LOSS_EPS = 0.01
O_CLAMP = 15.0
PRIME_Y, PRIME_Z = 2654435761, 805459861


def level_scales() -> np.ndarray:
    """Per-level float32 scale (grid cells per unit of normalised position)."""
    b = math.exp(math.log(FINEST_RES / BASE_RES) / (LEVELS - 1))
    return np.array([BASE_RES * b ** l for l in range(LEVELS)], np.float32)


def level_dense_side(scale: np.float32) -> int:
    """Side of the dense grid of a level, or 0 when the level is hashed."""
    n = int(math.ceil(float(scale))) + 2
    return n if n ** 3 <= TABLE else 0


def bf16(x: np.ndarray) -> np.ndarray:
    """Round float32 to the nearest bf16 (ties to even), kept in float32."""
    u = np.ascontiguousarray(x, np.float32).view(np.uint32).astype(np.uint64)
    r = ((u + 0x7FFF + ((u >> 16) & 1)) >> 16) << 16
    out = r.astype(np.uint32).view(np.float32)
    nan = np.isnan(x)
    return np.where(nan, np.float32(np.nan), out).astype(np.float32)


def sh4(d: np.ndarray) -> np.ndarray:
    """Real spherical harmonics of degrees 0-3 (16 values) of unit vectors d."""
    x, y, z = (d[:, k].astype(np.float32) for k in range(3))
    xx, yy, zz = x * x, y * y, z * z
    out = np.empty((d.shape[0], 16), np.float32)
    out[:, 0] = 0.28209479177387814
    out[:, 1] = -0.48860251190291987 * y
    out[:, 2] = 0.48860251190291987 * z
    out[:, 3] = -0.48860251190291987 * x
    out[:, 4] = 1.0925484305920792 * x * y
    out[:, 5] = -1.0925484305920792 * y * z
    out[:, 6] = 0.94617469575755997 * zz - 0.31539156525251999
    out[:, 7] = -1.0925484305920792 * x * z
    out[:, 8] = 0.54627421529603959 * (xx - yy)
    out[:, 9] = 0.59004358992664352 * y * (-3.0 * xx + yy)
    out[:, 10] = 2.8906114426405538 * x * y * z
    out[:, 11] = 0.45704579946446572 * y * (1.0 - 5.0 * zz)
    out[:, 12] = 0.3731763325901154 * z * (5.0 * zz - 3.0)
    out[:, 13] = 0.45704579946446572 * x * (1.0 - 5.0 * zz)
    out[:, 14] = 1.4453057213202769 * z * (xx - yy)
    out[:, 15] = 0.59004358992664352 * x * (-xx + 3.0 * yy)
    return out


def grid_corners(pos01: np.ndarray):
    """For each level: (indices (N, 8) int64, weights (N, 8) float32)."""
    scales = level_scales()
    out = []
    n = pos01.shape[0]
    for l in range(LEVELS):
        g = (pos01.astype(np.float32) * scales[l]).astype(np.float32)
        base = np.floor(g).astype(np.int64)
        f = (g - base.astype(np.float32)).astype(np.float32)
        side = level_dense_side(scales[l])
        idx = np.empty((n, 8), np.int64)
        w = np.empty((n, 8), np.float32)
        for c in range(8):
            cx, cy, cz = c & 1, (c >> 1) & 1, (c >> 2) & 1
            x, y, z = base[:, 0] + cx, base[:, 1] + cy, base[:, 2] + cz
            if side:
                idx[:, c] = x + y * side + z * side * side
            else:
                h = (x.astype(np.uint64) ^ ((y.astype(np.uint64) * PRIME_Y) & 0xFFFFFFFF)
                     ^ ((z.astype(np.uint64) * PRIME_Z) & 0xFFFFFFFF)) & (TABLE - 1)
                idx[:, c] = h.astype(np.int64)
            wx = f[:, 0] if cx else np.float32(1) - f[:, 0]
            wy = f[:, 1] if cy else np.float32(1) - f[:, 1]
            wz = f[:, 2] if cz else np.float32(1) - f[:, 2]
            w[:, c] = (wx * wy).astype(np.float32) * wz
        out.append((idx, w))
    return out


def encode(q: dict, table: np.ndarray, box_lo, box_inv):
    """Inputs (N, 64) float32 (not yet rounded) and the grid corners.
    q: pos (N,3), dir (N,3), normal (N,3), roughness (N,), diffuse (N,3),
    specular (N,3). table: (LEVELS, TABLE, 2) float32 (fp16-valued).
    The position is normalised as clamp((pos - box_lo) * box_inv, 0, 1) with
    box_lo a 3-vector (or scalar) and box_inv one scalar (1 / box extent)."""
    n = q["pos"].shape[0]
    lo = np.asarray(box_lo, np.float32)
    p01 = np.clip((q["pos"].astype(np.float32) - lo) * np.float32(box_inv), 0.0, 1.0)
    p01 = p01.astype(np.float32)
    corners = grid_corners(p01)
    x = np.zeros((n, WIDTH), np.float32)
    for l, (idx, w) in enumerate(corners):
        feats = table[l][idx]  # (N, 8, 2)
        x[:, 2 * l:2 * l + 2] = (feats * w[:, :, None]).sum(axis=1, dtype=np.float32)
    x[:, 32:48] = sh4(q["dir"])
    x[:, 48:51] = q["normal"] * 0.5 + 0.5
    x[:, 51] = q["roughness"]
    x[:, 52:55] = q["diffuse"]
    x[:, 55:58] = q["specular"]
    x[:, 58] = 1.0
    return x, corners


def _round(x, rnd: bool):
    return bf16(x) if rnd else x


def forward(x: np.ndarray, weights: list[np.ndarray], rnd: bool = True):
    """weights: 5 arrays (64, 64) and one (16, 64), bf16-valued float32.
    Returns (activations a_0..a_5 (bf16-valued), o (N, 3), rgb (N, 3)).
    rnd=False skips the bf16 rounding (float64 inputs give a float64 model
    for finite-difference checks)."""
    acts = [_round(x, rnd)]
    for l in range(HIDDEN):
        h = acts[-1] @ weights[l].T
        acts.append(_round(np.maximum(h, 0.0), rnd))
    o = (acts[-1] @ weights[HIDDEN].T)[:, :3]
    rgb = np.exp(np.minimum(o, O_CLAMP))
    return acts, o, rgb


def loss_and_grad(o: np.ndarray, rgb: np.ndarray, target: np.ndarray):
    """Relative L2 loss and its gradient with respect to o (the denominator
    is treated as a constant)."""
    n = o.shape[0]
    denom = rgb * rgb + LOSS_EPS
    diff = rgb - target
    loss = float(np.mean(diff * diff / denom, dtype=np.float64))
    drgb = (2.0 * diff / denom) / (3 * n)
    do = np.where(o < O_CLAMP, drgb * rgb, 0.0).astype(o.dtype)
    return loss, do


def backward(acts, weights, do, rnd: bool = True):
    """Gradients of the 6 weight matrices and of the 64 inputs."""
    n = do.shape[0]
    g = np.zeros((n, OUT_ROWS), do.dtype)
    g[:, :3] = do
    g = _round(g, rnd)
    grads = [None] * (HIDDEN + 1)
    for l in range(HIDDEN, -1, -1):
        grads[l] = g.T @ acts[l]
        dx = g @ weights[l]
        if l > 0:
            g = _round(np.where(acts[l] > 0, dx, 0.0), rnd)
        else:
            return grads, dx
    raise AssertionError


def grid_backward(dx: np.ndarray, corners) -> np.ndarray:
    """Scatter of the grid-feature gradients: (LEVELS, TABLE, 2) float32."""
    grad = np.zeros((LEVELS, TABLE, FEATURES), np.float64)
    for l, (idx, w) in enumerate(corners):
        for j in range(FEATURES):
            contrib = (w * dx[:, 2 * l + j][:, None]).astype(np.float64)
            np.add.at(grad[l, :, j], idx.reshape(-1), contrib.reshape(-1))
    return grad.astype(np.float32)


def touched(corners) -> np.ndarray:
    """(LEVELS, TABLE) bool: the grid entries a batch's samples read (all
    eight corners on every level, whatever their trilinear weight)."""
    mask = np.zeros((LEVELS, TABLE), bool)
    for l, (idx, _) in enumerate(corners):
        mask[l, idx.reshape(-1)] = True
    return mask


def adam(param: np.ndarray, grad: np.ndarray, m: np.ndarray, v: np.ndarray, step: int, mask=None):
    """One Adam step in place (fp32); step counts from 1. With `mask` (the
    shape of the parameters' leading axes, e.g. touched()), lazy Adam: only
    the masked entries update their moments and parameters; the others keep
    theirs (the bias corrections still use the global step)."""
    if mask is not None:
        sub = [a[mask] for a in (param, grad, m, v)]
        adam(*sub, step)
        for a, b in zip((param, m, v), (sub[0], sub[2], sub[3])):
            a[mask] = b
        return
    m *= np.float32(BETA1)
    m += np.float32(1 - BETA1) * grad
    v *= np.float32(BETA2)
    v += np.float32(1 - BETA2) * grad * grad
    mhat = m / np.float32(1 - BETA1 ** step)
    vhat = v / np.float32(1 - BETA2 ** step)
    param -= np.float32(LR) * mhat / (np.sqrt(vhat) + np.float32(EPS))


def average(avg: np.ndarray, param: np.ndarray, step: int, decay_max: float = 0.99, mask=None):
    """Moving average of the parameters after optimiser step `step` (counted
    from 1), in place: decay = min(decay_max, (1 + t) / (10 + t)) rounded to
    fp32, avg = decay * avg + (1 - decay) * param in fp32; with `mask`, only
    the masked entries (the lazy optimiser's updated ones)."""
    decay = np.float32(min(float(np.float32(decay_max)), (1.0 + step) / (10.0 + step)))
    keep = np.float32(1.0 - float(decay))
    if mask is not None:
        avg[mask] = (decay * avg[mask]).astype(np.float32) + (keep * param[mask]).astype(np.float32)
        return
    avg[...] = (decay * avg).astype(np.float32) + (keep * param).astype(np.float32)


def init_weights(seed: int) -> list[np.ndarray]:
    """Xavier-uniform weights rounded to bf16; output rows 3..15 zero."""
    rng = np.random.default_rng(seed)
    ws = []
    for l in range(HIDDEN):
        a = math.sqrt(6.0 / (WIDTH + WIDTH))
        ws.append(bf16(rng.uniform(-a, a, (WIDTH, WIDTH)).astype(np.float32)))
    a = math.sqrt(6.0 / (WIDTH + 3))
    w = np.zeros((OUT_ROWS, WIDTH), np.float32)
    w[:3] = rng.uniform(-a, a, (3, WIDTH))
    ws.append(bf16(w))
    return ws
