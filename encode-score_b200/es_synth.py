"""Seeded synthetic frames for the measurement workloads (no video files are available here or on the GPU hosts).

Each workload is a source and its encodes as 4:2:0 planes (uint16 arrays holding 8- or 10-bit codes):

* ``c1``  1920x1080 8-bit: 3 random linear/radial gradients spanning codes 16-235 plus Gaussian grain (sigma 2.5),
  one encode = 5x5 Gaussian blur (sigma 1.2) with the left half requantised to multiples of 4 codes.
* ``c2``  3840x2160 10-bit dark content: low-frequency gradients over codes 64-300 plus grain (sigma 8); three encodes
  blurred with sigma 0.8 / 1.5 / 2.5, the third also de-grained by a 7x7 box, each requantised to steps of 8 / 16 / 32
  codes on random rectangles covering 30% of the picture.
* ``c3``  16 sources of uneven sizes scored together (6 x 1280x720 8-bit, 6 x 1920x800 10-bit cropped from
  1920x1080 frames with black bars, 4 x 3840x1600 10-bit), each made like ``c1`` with its own grain sigma (uniform in
  1-12 codes) and banding step (one of 4, 8, 16, 32 codes).
* ``c4``  bright 10-bit gradient (codes 600-940) with heavy grain (sigma 20), for the precision checks.

Chroma is the luma halved and downsampled 2x2. Frame i of source s draws from numpy's PCG64 seeded with
``seed + 1000 * s + i``; the gradient field of a source drifts slowly from frame to frame while grain is fresh.
Any size can be asked for, so tests use the same generators at small sizes.
"""

from __future__ import annotations

from dataclasses import dataclass, field

import numpy as np
from scipy import ndimage


@dataclass
class Picture:
    y: np.ndarray
    u: np.ndarray
    v: np.ndarray
    depth: int


@dataclass
class Step:
    source: Picture
    encodes: list = field(default_factory=list)


def _field(rng_src: np.random.Generator, w: int, h: int, frame: int, count: int = 3, low_freq: bool = False) -> np.ndarray:
    """Sum of `count` linear or radial gradients in [0, 1], drifting with `frame`."""
    yy, xx = np.mgrid[0:h, 0:w].astype(np.float32)
    xx /= max(w - 1, 1)
    yy /= max(h - 1, 1)
    out = np.zeros((h, w), np.float32)
    for _ in range(count):
        drift = 0.002 * frame
        if rng_src.random() < 0.5:
            a = rng_src.uniform(0, 2 * np.pi)
            g = np.cos(a) * xx + np.sin(a) * yy + drift
        else:
            cx, cy = rng_src.uniform(0, 1, 2)
            g = np.sqrt((xx - cx - drift) ** 2 + (yy - cy) ** 2)
        if low_freq:
            g = 0.5 + 0.5 * np.sin(np.pi * rng_src.uniform(0.5, 1.5) * g + rng_src.uniform(0, np.pi))
        out += g.astype(np.float32)
    out -= out.min()
    out /= max(float(out.max()), 1e-6)
    return out


def _chroma(y: np.ndarray) -> np.ndarray:
    h, w = y.shape
    c = y[: h // 2 * 2, : w // 2 * 2].astype(np.float32).reshape(h // 2, 2, w // 2, 2).mean(axis=(1, 3)) / 2
    return np.rint(c).astype(np.uint16)


def _picture(y: np.ndarray, depth: int) -> Picture:
    y = y.astype(np.uint16)
    c = _chroma(y)
    return Picture(y, c, c.copy(), depth)


def _rects(rng: np.random.Generator, w: int, h: int, share: float) -> np.ndarray:
    mask = np.zeros((h, w), bool)
    while mask.mean() < share:
        rw, rh = int(rng.uniform(0.1, 0.35) * w), int(rng.uniform(0.1, 0.35) * h)
        x, y = int(rng.uniform(0, w - rw)), int(rng.uniform(0, h - rh))
        mask[y:y + rh, x:x + rw] = True
    return mask


def c1_step(frame: int, w: int = 1920, h: int = 1080, seed: int = 1, source: int = 0) -> Step:
    base = np.random.Generator(np.random.PCG64(seed + 1000 * source))
    rng = np.random.Generator(np.random.PCG64(seed + 1000 * source + frame + 500))
    luma = 16 + 219 * _field(base, w, h, frame)
    src = np.clip(np.rint(luma + rng.normal(0, 2.5, (h, w))), 16, 235)
    blur = ndimage.gaussian_filter(src.astype(np.float32), 1.2, truncate=2.0 / 1.2, mode="nearest")
    enc = np.clip(np.rint(blur), 16, 235)
    enc[:, : w // 2] = np.clip(np.rint(enc[:, : w // 2] / 4) * 4, 16, 235)
    return Step(_picture(src, 8), [_picture(enc, 8)])


def c2_step(frame: int, w: int = 3840, h: int = 2160, seed: int = 2, source: int = 0, n_encodes: int = 3) -> Step:
    base = np.random.Generator(np.random.PCG64(seed + 1000 * source))
    rng = np.random.Generator(np.random.PCG64(seed + 1000 * source + frame + 500))
    luma = 64 + 236 * _field(base, w, h, frame, low_freq=True)
    src = np.clip(np.rint(luma + rng.normal(0, 8, (h, w))), 64, 300).astype(np.float32)
    encodes = []
    for e, (sigma, step) in enumerate(zip((0.8, 1.5, 2.5), (8, 16, 32))):
        if e >= n_encodes:
            break
        enc = ndimage.gaussian_filter(src, sigma, mode="nearest")
        if e == 2:
            enc = ndimage.uniform_filter(enc, 7, mode="nearest")
        region = _rects(rng, w, h, 0.30)
        enc = np.where(region, np.rint(enc / step) * step, np.rint(enc))
        encodes.append(_picture(np.clip(enc, 64, 300), 10))
    return Step(_picture(src, 10), encodes)


C3_SOURCES = [(1280, 720, 8)] * 6 + [(1920, 800, 10)] * 6 + [(3840, 1600, 10)] * 4
C3_BARS = {(1920, 800): (1920, 1080)}  # decoded frame size of a cropped source: the picture sits centred in black bars


def c3_step(frame: int, source: int, w: int, h: int, depth: int, seed: int = 3) -> Step:
    """One source of the uneven batch and its encode: c1's recipe at (w, h, depth) with this source's grain sigma and
    banding step."""
    base = np.random.Generator(np.random.PCG64(seed + 1000 * source))
    rng = np.random.Generator(np.random.PCG64(seed + 1000 * source + frame + 500))
    sigma = float(base.uniform(1, 12))
    step = int(base.choice([4, 8, 16, 32]))
    lo, hi = (16, 235) if depth == 8 else (64, 940)
    luma = lo + (hi - lo) * _field(base, w, h, frame)
    src = np.clip(np.rint(luma + rng.normal(0, sigma, (h, w))), lo, hi)
    blur = ndimage.gaussian_filter(src.astype(np.float32), 1.2, truncate=2.0 / 1.2, mode="nearest")
    enc = np.clip(np.rint(blur), lo, hi)
    enc[:, : w // 2] = np.clip(np.rint(enc[:, : w // 2] / step) * step, lo, hi)
    return Step(_picture(src, depth), [_picture(enc, depth)])


def c4_step(frame: int, w: int = 3840, h: int = 2160, seed: int = 4, source: int = 0) -> Step:
    base = np.random.Generator(np.random.PCG64(seed + 1000 * source))
    rng = np.random.Generator(np.random.PCG64(seed + 1000 * source + frame + 500))
    luma = 600 + 340 * _field(base, w, h, frame)
    src = np.clip(np.rint(luma + rng.normal(0, 20, (h, w))), 0, 1023)
    enc = np.clip(np.rint(ndimage.gaussian_filter(src.astype(np.float32), 1.0, mode="nearest")), 0, 1023)
    return Step(_picture(src, 10), [_picture(enc, 10)])


def texture_step(frame: int, w: int = 640, h: int = 360, seed: int = 7, source: int = 0) -> Step:
    """Persistent texture for the lasting-texture measure: a static sum of 4 oriented sinusoids (periods 6-24 pixels)
    around code 512 of a 10-bit picture plus fresh grain (sigma 6) every frame; the encode blurs it (sigma 0.9) and
    requantises its left half to even codes."""
    base = np.random.Generator(np.random.PCG64(seed + 1000 * source))
    rng = np.random.Generator(np.random.PCG64(seed + 1000 * source + frame + 500))
    yy, xx = np.mgrid[0:h, 0:w].astype(np.float32)
    tex = np.zeros((h, w), np.float32)
    for _ in range(4):
        a, period, phase = base.uniform(0, np.pi), base.uniform(6, 24), base.uniform(0, 2 * np.pi)
        tex += np.sin(2 * np.pi * (xx * np.cos(a) + yy * np.sin(a)) / period + phase).astype(np.float32)
    src = np.clip(np.rint(512 + 30 * tex + rng.normal(0, 6, (h, w))), 0, 1023)
    enc = np.rint(ndimage.gaussian_filter(src.astype(np.float32), 0.9, mode="nearest"))
    enc[:, : w // 2] = np.rint(enc[:, : w // 2] / 2) * 2
    return Step(_picture(src, 10), [_picture(np.clip(enc, 0, 1023), 10)])


WORKLOADS = {"c1": c1_step, "c2": c2_step, "c4": c4_step, "texture": texture_step}
