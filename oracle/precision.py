"""TEST INFRASTRUCTURE, not product code: the FP64 oracle of the texture window energies on windows of 16 k pixels.

Definitions of src/kernels.cu:346-428 and reference/encode_score/compare.py:77-108 (fine = y - box3, mid = box3 - box9,
box-3 gradients by central differences, 0 on the border columns / rows; edge pixels repeated for the boxes), evaluated
exactly in int64 numerators (fine and gradients x 9, mid x 81) and rounded once per figure to float64, in the
operation order of the CUDA exact mode. Only tests and the precision report import this module.
"""

from __future__ import annotations

import numpy as np


def _box(y: np.ndarray, r: int) -> np.ndarray:
    p = np.pad(y.astype(np.int64), r, mode="edge")
    c = np.cumsum(np.cumsum(p, axis=0), axis=1)
    c = np.pad(c, ((1, 0), (1, 0)))
    n = 2 * r + 1
    h, w = y.shape
    return c[n:n + h, n:n + w] - c[0:h, n:n + w] - c[n:n + h, 0:w] + c[0:h, 0:w]


def terms(y: np.ndarray, up: int):
    """Exact numerators (fine x 9, mid x 81, gx x 9, gy x 9) of every pixel of y (values << up)."""
    v = y.astype(np.int64) << up
    s3, s9 = _box(v, 1), _box(v, 4)
    f = 9 * v - s3
    m = 9 * s3 - s9
    gx = np.zeros_like(v)
    gy = np.zeros_like(v)
    gx[:, 1:-1] = s3[:, 2:] - s3[:, :-2]
    gy[1:-1, :] = s3[2:, :] - s3[:-2, :]
    return f, m, gx, gy


def window_figures(yr: np.ndarray, yd: np.ndarray, up: int, window: int) -> np.ndarray:
    """(windows, 8) float64: [src fine^2, src mid^2, enc fine^2, enc mid^2, fine x, mid x, src oriented, enc oriented],
    windows row by row, only whole windows of the 16 x 16 block grid."""
    fr, mr, gxr, gyr = terms(yr, up)
    fd, md, gxd, gyd = terms(yd, up)
    h, w = yr.shape
    k = window // 16
    bw, bh = w // 16, h // 16
    ww, wh = bw // k, bh // k
    H, W = wh * window, ww * window
    q = [fr * fr, mr * mr, fd * fd, md * md, fr * fd, mr * md, gxr * gxr, gyr * gyr, gxr * gyr, gxd * gxd, gyd * gyd, gxd * gyd]
    s = [a[:H, :W].reshape(wh, window, ww, window).sum(axis=(1, 3)).reshape(-1) for a in q]
    out = np.zeros((ww * wh, 8), np.float64)
    out[:, 0] = s[0].astype(np.float64) / 81.0
    out[:, 1] = s[1].astype(np.float64) / 6561.0
    out[:, 2] = s[2].astype(np.float64) / 81.0
    out[:, 3] = s[3].astype(np.float64) / 6561.0
    out[:, 4] = s[4].astype(np.float64) / 81.0
    out[:, 5] = s[5].astype(np.float64) / 6561.0
    dr, xr = (s[6] - s[7]).astype(np.float64), s[8].astype(np.float64)
    dd, xd = (s[9] - s[10]).astype(np.float64), s[11].astype(np.float64)
    out[:, 6] = np.sqrt(dr * dr + 4.0 * xr * xr) / 81.0
    out[:, 7] = np.sqrt(dd * dd + 4.0 * xd * xd) / 81.0
    return out
