"""TEST INFRASTRUCTURE, not product code: the FP64 numpy oracle of the learned tile proposal.

The reference has no counterpart (it runs CAMBI's c-values on every pixel, src/kernels.cu:224-278); this file states
the network the CUDA kernels implement, so their forward pass, gradients and optimizer step can be checked:

* features of scale 0 (the words value | mask << 15 that CAMBI's c-values read), per 4 x 4 pixel block: the mean value
  as (mean - 512) / 256 and the share of masked pixels; pixels outside the picture count as absent (a block with none
  has features 0, as the zero padding outside the picture);
* a 4-layer network of valid 3 x 3 convolutions, 2 -> 16 -> 16 -> 16 -> 1 channels, ReLU after the first three, with
  weights rounded to bfloat16 (round to nearest even) and the output of each ReLU rounded to bfloat16 in the fused
  inference kernel (``round_acts``);
* the tile prediction: the mean of the last layer over each 16 x 16 block of its output (one 64 x 64 CAMBI tile of
  scale 0), and the loss: the mean squared difference to the label log1p(mean positive c-value of the tile's pixels);
* Adam (Kingma and Ba 2015, bias-corrected) on FP32 master weights.

Only tests and the training script import this module.
"""

from __future__ import annotations

import math

import numpy as np

CHANNELS = (2, 16, 16, 16, 1)
HALO = 4          # valid 3 x 3 convolutions shrink each side by 1 per layer
TILE = 16         # output pixels per side of one CAMBI tile (64 x 64 pixels at scale 0, 4 x downscaled)
MASK_BIT = 0x8000
N_PARAMS = 5089   # per layer w (co, ci, 3, 3) then b (co,), flattened in order


def bf16(x: np.ndarray) -> np.ndarray:
    """Round float32 values to the nearest bfloat16 (ties to even), returned as float64."""
    a = np.ascontiguousarray(np.asarray(x, np.float32))
    u = a.view(np.uint32).astype(np.uint64)
    r = ((u + 0x7FFF + ((u >> 16) & 1)) >> 16) << 16
    return r.astype(np.uint32).view(np.float32).astype(np.float64)


def features(words: np.ndarray, x0: int, y0: int, fw: int, fh: int) -> np.ndarray:
    """The 2 x fh x fw feature map whose pixel (u, v) covers scale-0 pixels (x0 + 4u .. + 3, y0 + 4v .. + 3) of the
    picture `words` (h x w uint16, value | mask << 15); x0, y0 may be negative."""
    h, w = words.shape
    out = np.zeros((2, fh, fw), np.float64)
    for v in range(fh):
        for u in range(fw):
            xa, ya = x0 + 4 * u, y0 + 4 * v
            xs, xe, ys, ye = max(xa, 0), min(xa + 4, w), max(ya, 0), min(ya + 4, h)
            if xs >= xe or ys >= ye:
                continue
            blk = words[ys:ye, xs:xe].astype(np.int64)
            n = blk.size
            out[0, v, u] = ((blk & 0x7FFF).sum() / n - 512.0) / 256.0
            out[1, v, u] = ((blk & MASK_BIT) != 0).sum() / 16.0
    return out


def features_fast(words: np.ndarray, x0: int, y0: int, fw: int, fh: int) -> np.ndarray:
    """features() vectorised: the same values in the same float64 arithmetic for sums, counts and the division."""
    h, w = words.shape
    H, W = 4 * fh, 4 * fw
    vals = np.zeros((H, W), np.int64)
    cnt = np.zeros((H, W), np.int64)
    msk = np.zeros((H, W), np.int64)
    xs, ys = max(x0, 0), max(y0, 0)
    xe, ye = min(x0 + W, w), min(y0 + H, h)
    if xs < xe and ys < ye:
        blk = words[ys:ye, xs:xe].astype(np.int64)
        vals[ys - y0:ye - y0, xs - x0:xe - x0] = blk & 0x7FFF
        cnt[ys - y0:ye - y0, xs - x0:xe - x0] = 1
        msk[ys - y0:ye - y0, xs - x0:xe - x0] = (blk & MASK_BIT) != 0
    s = vals.reshape(fh, 4, fw, 4).sum(axis=(1, 3))
    n = cnt.reshape(fh, 4, fw, 4).sum(axis=(1, 3))
    m = msk.reshape(fh, 4, fw, 4).sum(axis=(1, 3))
    out = np.zeros((2, fh, fw), np.float64)
    on = n > 0
    out[0][on] = (s[on] / n[on] - 512.0) / 256.0
    out[1] = m / 16.0
    return out


def init_params(seed: int = 0) -> list:
    """He-initialised FP32 master weights: [(w (co, ci, 3, 3), b (co,)) per layer]."""
    rng = np.random.default_rng(seed)
    params = []
    for ci, co in zip(CHANNELS[:-1], CHANNELS[1:]):
        w = rng.normal(0.0, np.sqrt(2.0 / (9 * ci)), (co, ci, 3, 3)).astype(np.float32)
        b = np.zeros(co, np.float32)
        params.append((w, b))
    return params


def flatten(params: list) -> np.ndarray:
    """The flat float32 parameter array the CUDA kernels take."""
    return np.concatenate([np.concatenate([np.asarray(w, np.float32).ravel(), np.asarray(b, np.float32).ravel()]) for w, b in params])


def unflatten(flat: np.ndarray) -> list:
    out, at = [], 0
    for ci, co in zip(CHANNELS[:-1], CHANNELS[1:]):
        w = np.asarray(flat[at:at + co * ci * 9], np.float32).reshape(co, ci, 3, 3)
        at += co * ci * 9
        b = np.asarray(flat[at:at + co], np.float32)
        at += co
        out.append((w, b))
    return out


def conv(x: np.ndarray, w: np.ndarray, b: np.ndarray) -> np.ndarray:
    """Valid 3 x 3 cross-correlation: x (n, ci, h, w), w (co, ci, 3, 3) -> (n, co, h - 2, w - 2)."""
    n, ci, h, wd = x.shape
    out = np.zeros((n, w.shape[0], h - 2, wd - 2), np.float64)
    for ky in range(3):
        for kx in range(3):
            patch = x[:, :, ky:ky + h - 2, kx:kx + wd - 2]
            out += np.einsum("nchw,oc->nohw", patch, w[:, :, ky, kx].astype(np.float64))
    return out + b.astype(np.float64)[None, :, None, None]


def forward(x: np.ndarray, params: list, round_acts: bool = False, round_weights: bool = True) -> list:
    """Activations [x, a1, a2, a3, z] of the network on x (n, 2, h, w); weights are used rounded to bfloat16 (unless
    round_weights is false, for finite-difference checks)."""
    rw = bf16 if round_weights else (lambda a: np.asarray(a, np.float64))
    acts = [np.asarray(x, np.float64)]
    for i, (w, b) in enumerate(params):
        y = conv(acts[-1], rw(w), rw(b))
        if i < len(params) - 1:
            y = np.maximum(y, 0.0)
            if round_acts:
                y = bf16(y)
        acts.append(y)
    return acts


def tile_means(z: np.ndarray) -> np.ndarray:
    """(n, 1, 16 a, 16 b) -> (n, a, b): the mean of each 16 x 16 block."""
    n, _, h, w = z.shape
    return z[:, 0].reshape(n, h // TILE, TILE, w // TILE, TILE).mean(axis=(2, 4))


def loss_and_grads(x: np.ndarray, labels: np.ndarray, params: list, round_weights: bool = True) -> tuple:
    """Loss mean((tile_means - labels)^2) and its gradients with respect to each layer's (w, b), taken at the
    bfloat16-rounded weights (the straight-through gradient of the FP32 master weights)."""
    rw = bf16 if round_weights else (lambda a: np.asarray(a, np.float64))
    acts = forward(x, params, round_weights=round_weights)
    pred = tile_means(acts[-1])
    diff = pred - labels
    loss = float(np.mean(diff * diff))
    g = (2.0 / diff.size) * diff / (TILE * TILE)                      # d loss / d z, per block
    gz = np.repeat(np.repeat(g, TILE, axis=1), TILE, axis=2)[:, None]  # (n, 1, h, w)
    grads = [None] * len(params)
    for i in range(len(params) - 1, -1, -1):
        w = rw(params[i][0])
        inp = acts[i]
        gw = np.zeros(w.shape, np.float64)
        for ky in range(3):
            for kx in range(3):
                patch = inp[:, :, ky:ky + gz.shape[2], kx:kx + gz.shape[3]]
                gw[:, :, ky, kx] = np.einsum("nohw,nchw->oc", gz, patch)
        gb = gz.sum(axis=(0, 2, 3))
        grads[i] = (gw, gb)
        if i == 0:
            break
        # gradient of the input: full correlation with the flipped kernel, then the ReLU of layer i - 1
        gin = np.zeros(inp.shape, np.float64)
        for ky in range(3):
            for kx in range(3):
                gin[:, :, ky:ky + gz.shape[2], kx:kx + gz.shape[3]] += np.einsum("nohw,oc->nchw", gz, w[:, :, ky, kx])
        gz = gin * (acts[i] > 0)
    return loss, grads


class Adam:
    """Adam with bias correction on FP32 master weights (the arithmetic of the CUDA step, in float64)."""

    def __init__(self, params: list, lr: float = 1e-3, b1: float = 0.9, b2: float = 0.999, eps: float = 1e-8):
        self.lr, self.b1, self.b2, self.eps = lr, b1, b2, eps
        self.m = [[np.zeros_like(w, np.float64), np.zeros_like(b, np.float64)] for w, b in params]
        self.v = [[np.zeros_like(w, np.float64), np.zeros_like(b, np.float64)] for w, b in params]
        self.t = 0

    def step(self, params: list, grads: list) -> list:
        self.t += 1
        c1, c2 = 1.0 - self.b1 ** self.t, 1.0 - self.b2 ** self.t
        out = []
        for i, ((w, b), (gw, gb)) in enumerate(zip(params, grads)):
            new = []
            for j, (p, g) in enumerate(((w, gw), (b, gb))):
                m = self.m[i][j] = self.b1 * self.m[i][j] + (1 - self.b1) * g
                v = self.v[i][j] = self.b2 * self.v[i][j] + (1 - self.b2) * g * g
                new.append((p.astype(np.float64) - self.lr * (m / c1) / (np.sqrt(v / c2) + self.eps)).astype(np.float32))
            out.append(tuple(new))
        return out


def label_of(mass_fx: np.ndarray, pixels: np.ndarray) -> np.ndarray:
    """Tile label log1p(sum of the tile's positive c-values / its pixel count), from the exact sum in 2^-24 units."""
    return np.log1p(mass_fx.astype(np.float64) / 16777216.0 / np.maximum(pixels, 1))


def budget_threshold(pred: np.ndarray, w: int, h: int, k0: int, window: int, threshold: float, budget: float,
                     tile: int = 64, bins: int = 1024, per_unit: float = 128.0) -> float:
    """The budget mode's skip threshold of one picture (test restatement of the device's): scale-0 tile t of predicted
    label p_t (row-major over ceil(w / tile) x ceil(h / tile) tiles, -inf where nothing needs a c-value) is predicted to
    add scale * expm1(max(p_t, 0)) * pixels_t to the score, scale = 16 / (k0 window^2); contributions are binned by
    prediction (per_unit bins per unit from 0, the last bin open above) in 2^-40 fixed point, and the threshold is the
    lower edge of the first bin whose inclusion would exceed the budget (infinity when none does), at least
    `threshold`."""
    tx = (w + tile - 1) // tile
    ty = (h + tile - 1) // tile
    scale = 16.0 / (k0 * window * window)
    acc = [0] * bins
    p = np.asarray(pred, np.float32).reshape(ty, tx)
    for y in range(ty):
        for x in range(tx):
            v = float(p[y, x])
            if v == -np.inf:
                continue
            px = min(tile, w - x * tile) * min(tile, h - y * tile)
            c = scale * math.expm1(max(v, 0.0)) * px
            fx = int(min(c * 2.0 ** 40, 2.0e15))
            b = min(bins - 1, max(0, int(np.float32(v) * np.float32(per_unit))))
            acc[b] += fx
    limit = int(min(budget * 2.0 ** 40, 1.8e19))
    n, incl = 0, 0
    for b in range(bins):
        incl += acc[b]
        if incl <= limit:
            n += 1
    t = np.inf if n >= bins else n / per_unit
    return float(max(np.float32(t), np.float32(threshold)))
