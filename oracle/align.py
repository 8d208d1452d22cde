"""TEST INFRASTRUCTURE, not product code: the CPU oracle of the offset search between a source and its encodes.

* thumbnail(): src/kernels.cu:502-520 (tiny_luma): the 64 x 36 box means of the cropped luma on a 10-bit scale. The
  reference adds the samples in float; every partial sum is an integer below 2^24 for cells of up to 16,400 pixels, so
  it is exact there, and this restatement adds in int64 and divides once in float32.
* find_offset(): src/main.cpp:336-353, in its order of operations: per lag, the differences in float32 added in double
  frame by frame and pixel by pixel, the early stop once a lag's partial total reaches the best total, the first lag of
  least mean, and the refusal of a mean above 16.

Only tests import this module.
"""

from __future__ import annotations

import numpy as np

TW, TH = 64, 36
PIXELS = TW * TH


class NoMatch(Exception):
    def __init__(self, best: float):
        super().__init__(f"no lag matches (closest mean difference {best})")
        self.best = best


def thumbnail(y: np.ndarray, depth: int, x0: int, y0: int, w: int, h: int) -> np.ndarray:
    """The thumbnail of luma plane y (integer samples at `depth` bits) cropped to w x h at (x0, y0): float32 [36][64]."""
    v = y.astype(np.int64) << (10 - depth)
    out = np.empty((TH, TW), np.float32)
    for ty in range(TH):
        ya, yb = y0 + ty * h // TH, y0 + (ty + 1) * h // TH
        for tx in range(TW):
            xa, xb = x0 + tx * w // TW, x0 + (tx + 1) * w // TW
            n = (xb - xa) * (yb - ya)
            with np.errstate(invalid="ignore", divide="ignore"):
                out[ty, tx] = np.float32(v[ya:yb, xa:xb].sum()) / np.float32(n)
    return out


def _sequential(start: float, terms: np.ndarray) -> float:
    """start + terms[0] + terms[1] + ... in double, left to right (np.cumsum adds in order)."""
    return float(np.cumsum(np.concatenate(([start], terms.astype(np.float64))))[-1])


def lag_totals(ref: np.ndarray, probe: np.ndarray) -> np.ndarray:
    """Per lag, the full double total of |ref[l + i][p] - probe[i][p]| in frame-then-pixel order (no early stop)."""
    ref = ref.reshape(-1, PIXELS).astype(np.float32)
    probe = probe.reshape(-1, PIXELS).astype(np.float32)
    n = len(probe)
    return np.array([_sequential(0.0, np.abs(ref[l:l + n] - probe).ravel()) for l in range(len(ref) - n + 1)])


def find_offset(ref: np.ndarray, ref_times, probe: np.ndarray, probe_times) -> tuple[float, int, float]:
    """(offset, lag, best mean) as src/main.cpp:336-353 finds them; raises ValueError for too few frames and NoMatch
    when the best mean exceeds 16."""
    ref = ref.reshape(-1, PIXELS).astype(np.float32)
    probe = probe.reshape(-1, PIXELS).astype(np.float32)
    n = len(probe)
    if n < 24 or len(ref) < n:
        raise ValueError("too few frames to find the offset")
    best, lag = 1e30, 0
    for l in range(len(ref) - n + 1):
        total = 0.0
        for i in range(n):
            if not total < best * n * 2304:
                break
            total = _sequential(total, np.abs(ref[l + i] - probe[i]))
        mean = total / (n * 2304.0)
        if mean < best:
            best, lag = mean, l
    if best > 16.0:
        raise NoMatch(best)
    return ref_times[lag] - probe_times[0], lag, best
