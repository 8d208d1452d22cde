"""TEST INFRASTRUCTURE, not product code: the CPU oracle of encode-score's per-frame measurement path.

Two parts:

* ctypes bindings of ``liboracle.so`` (``es_oracle.c``), the plain-C restatement of the per-pixel work: frame
  unpacking, CAMBI, the exact detail / texture window figures, PSNR squared errors and color sums;
* a numpy restatement of the reference's host logic: the per-frame reduction of window figures into per-segment
  accumulators (``src/main.cpp:577-643``), ``Histogram`` / ``Accum`` / ``score`` (``src/stats.hpp:10-83``), PSNR
  (``src/main.cpp:272-277``) and the JSON ``parts`` of a segment (``src/main.cpp:738-757``).

Only tests, ``__graft_entry__.smoke()`` and bench.py's CPU-baseline leg import this module.
"""

from __future__ import annotations

import ctypes
import math
import os
import subprocess
from dataclasses import dataclass, field

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "liboracle.so")
SCALES = 5
SCALE_WEIGHTS = (16, 8, 4, 2, 1)


def build() -> str:
    """Compile liboracle.so next to this file (gcc, no contraction of floating-point operations)."""
    src = os.path.join(HERE, "es_oracle.c")
    if not os.path.exists(LIB_PATH) or os.path.getmtime(LIB_PATH) < max(os.path.getmtime(src), os.path.getmtime(os.path.join(HERE, "es_oracle.h"))):
        subprocess.run(["gcc", "-O2", "-std=c11", "-Wall", "-ffp-contract=off", "-fPIC", "-shared", src, "-o", LIB_PATH, "-lm"], check=True)
    return LIB_PATH


class FrameView(ctypes.Structure):
    """``src/kernels.cu:284-287`` Frame / ``src/main.cpp:99-102`` FrameView."""
    _fields_ = [("y", ctypes.c_void_p), ("u", ctypes.c_void_p), ("v", ctypes.c_void_p), ("ypitch", ctypes.c_int), ("cpitch", ctypes.c_int),
                ("semi", ctypes.c_int), ("bytes", ctypes.c_int), ("shift", ctypes.c_int), ("depth", ctypes.c_int)]


class CambiParams(ctypes.Structure):
    """``src/cambi.cpp:39-53`` derived parameters (``src/kernels.cu:65-69`` CambiParams, plus window/mask index/topk)."""
    _fields_ = [("w", ctypes.c_int), ("h", ctypes.c_int), ("window", ctypes.c_int), ("pad", ctypes.c_int), ("mask_index", ctypes.c_int),
                ("band_base", ctypes.c_int), ("band_size", ctypes.c_int), ("vlt", ctypes.c_int), ("tvi", ctypes.c_int * 4),
                ("weight", ctypes.c_int * 4), ("topk", ctypes.c_double)]

    def as_dict(self) -> dict:
        return {"w": self.w, "h": self.h, "window": self.window, "pad": self.pad, "mask_index": self.mask_index, "band_base": self.band_base,
                "band_size": self.band_size, "vlt": self.vlt, "tvi": list(self.tvi), "weight": list(self.weight), "topk": self.topk}


_lib = None


def lib():
    global _lib
    if _lib is None:
        _lib = ctypes.CDLL(build())
        P = ctypes.c_void_p
        _lib.eso_cambi_score.restype = ctypes.c_double
        _lib.eso_cambi_pool.restype = ctypes.c_double
        _lib.eso_cambi_pool.argtypes = [P, ctypes.c_size_t, ctypes.c_double]
        _lib.eso_topk_count.restype = ctypes.c_size_t
        _lib.eso_topk_count.argtypes = [ctypes.c_size_t, ctypes.c_double]
        _lib.eso_plane_sse.restype = ctypes.c_uint64
        _lib.eso_plane_sse.argtypes = [P, P, ctypes.c_size_t]
        _lib.eso_color_sums.argtypes = [P, P, ctypes.c_size_t, ctypes.c_int, P]
        _lib.eso_tvi_for_diff.argtypes = [ctypes.c_int, ctypes.c_double]
        _lib.eso_vlt_luma.argtypes = [ctypes.c_double]
        _lib.eso_find_offset_lag.restype = ctypes.c_double
        _lib.eso_find_offset_lag.argtypes = [P, ctypes.c_int, P, ctypes.c_int, ctypes.POINTER(ctypes.c_int)]
    return _lib


def _ptr(a: np.ndarray) -> ctypes.c_void_p:
    assert a.flags["C_CONTIGUOUS"]
    return ctypes.c_void_p(a.ctypes.data)


def scale_sizes(w: int, h: int) -> list[tuple[int, int]]:
    """Width and height of each CAMBI scale (``src/cambi.cpp:57-58``)."""
    out = [(w, h)]
    for _ in range(1, SCALES):
        w, h = (w + 1) >> 1, (h + 1) >> 1
        out.append((w, h))
    return out


# ------------------------------------------------------------------------------------------------------------------
# Per-pixel work (C)
# ------------------------------------------------------------------------------------------------------------------

def frame_planes(y: np.ndarray, u: np.ndarray, v: np.ndarray | None, semi: int, shift: int, depth: int, x0: int, y0: int, pd: int,
                 w: int, h: int) -> tuple[np.ndarray, np.ndarray, np.ndarray]:
    """``src/kernels.cu:297-310``: planes of (h', w') uint8/uint16 arrays (pitch = row bytes) to uint16 planes at depth pd."""
    f = FrameView(y.ctypes.data, u.ctypes.data, v.ctypes.data if v is not None else None, y.strides[0], u.strides[0], semi, y.itemsize, shift, depth)
    Y = np.zeros((h, w), np.uint16)
    U = np.zeros((h // 2, w // 2), np.uint16)
    V = np.zeros((h // 2, w // 2), np.uint16)
    lib().eso_frame_planes(ctypes.byref(f), x0, y0, pd, w, h, _ptr(Y), _ptr(U), _ptr(V))
    return Y, U, V


def cambi_params(w: int, h: int) -> CambiParams:
    p = CambiParams()
    lib().eso_cambi_params_derive(w, h, ctypes.byref(p))
    return p


def cambi_mask(img: np.ndarray, index: int) -> np.ndarray:
    h, w = img.shape
    img = np.ascontiguousarray(img, np.uint16)
    out = np.zeros((h, w), np.uint8)
    lib().eso_cambi_mask(_ptr(img), w, h, index, _ptr(out))
    return out


def cambi_mode(img: np.ndarray) -> np.ndarray:
    h, w = img.shape
    img = np.ascontiguousarray(img, np.uint16)
    out = np.zeros((h, w), np.uint16)
    lib().eso_cambi_mode(_ptr(img), w, h, _ptr(out))
    return out


def cambi_preprocess(img: np.ndarray, depth: int) -> np.ndarray:
    h, w = img.shape
    img = np.ascontiguousarray(img, np.uint16)
    out = np.zeros((h, w), np.uint16)
    lib().eso_cambi_preprocess(_ptr(img), w, w, h, depth, _ptr(out))
    return out


def cambi_cvalues(img: np.ndarray, mask: np.ndarray, p: CambiParams) -> tuple[np.ndarray, int, int]:
    h, w = img.shape
    img = np.ascontiguousarray(img, np.uint16)
    mask = np.ascontiguousarray(mask, np.uint8)
    out = np.zeros((h, w), np.float32)
    s, c = ctypes.c_uint64(), ctypes.c_uint64()
    q = CambiParams.from_buffer_copy(p)
    q.w, q.h = w, h
    lib().eso_cambi_cvalues(_ptr(img), _ptr(mask), w, h, ctypes.byref(q), _ptr(out), ctypes.byref(s), ctypes.byref(c))
    return out, s.value, c.value


def cambi_pool(c: np.ndarray, topk: float = 0.6) -> float:
    c = np.ascontiguousarray(c, np.float32).ravel()
    return lib().eso_cambi_pool(_ptr(c), c.size, topk)


@dataclass
class CambiResult:
    score: float
    pooled: list
    sums_fx: list
    counts: list
    images: list | None = None
    masks: list | None = None
    cvalues: list | None = None


def cambi(img: np.ndarray, depth: int, params: CambiParams | None = None, keep: bool = False) -> CambiResult:
    """``src/cambi.cpp:88-184``: the CAMBI score of one plane (uint16 values at `depth` bits), optionally with every
    scale's image, mask and c-values."""
    h, w = img.shape
    img = np.ascontiguousarray(img, np.uint16)
    p = params or cambi_params(w, h)
    sizes = scale_sizes(w, h)
    images = [np.zeros((sh, sw), np.uint16) for sw, sh in sizes] if keep else None
    masks = [np.zeros((sh, sw), np.uint8) for sw, sh in sizes] if keep else None
    cvals = [np.zeros((sh, sw), np.float32) for sw, sh in sizes] if keep else None

    def arr(lst, ctype):
        if lst is None:
            return None
        return (ctypes.c_void_p * SCALES)(*[a.ctypes.data for a in lst])

    pooled = (ctypes.c_double * SCALES)()
    sums = (ctypes.c_uint64 * SCALES)()
    counts = (ctypes.c_uint64 * SCALES)()
    score = lib().eso_cambi_score(_ptr(img), w, w, h, depth, ctypes.byref(p), arr(images, None), arr(masks, None), arr(cvals, None), pooled, sums, counts)
    return CambiResult(score, list(pooled), list(sums), list(counts), images, masks, cvals)


def window_stats(yr: np.ndarray, yd: np.ndarray, up: int) -> tuple[np.ndarray, np.ndarray]:
    """Exact ``window_stats`` (``src/kernels.cu:346-428``): (windows, 8) in float64 and rounded to float32."""
    h, w = yr.shape
    ww, wh = w // 16, h // 16
    o64 = np.zeros((wh * ww, 8), np.float64)
    o32 = np.zeros((wh * ww, 8), np.float32)
    lib().eso_window_stats(_ptr(np.ascontiguousarray(yr, np.uint16)), _ptr(np.ascontiguousarray(yd, np.uint16)), up, w, h, _ptr(o64), _ptr(o32))
    return o64, o32


def mid81(y: np.ndarray, up: int) -> np.ndarray:
    h, w = y.shape
    out = np.zeros((h, w), np.int32)
    lib().eso_mid81(_ptr(np.ascontiguousarray(y, np.uint16)), up, w, h, _ptr(out))
    return out


def persist_stats(ring: list, yd: np.ndarray, up: int) -> tuple[np.ndarray, np.ndarray]:
    """Exact ``persist_stats`` (``src/kernels.cu:435-451``): `ring` = source luma of frames centre-6 .. centre+6."""
    assert len(ring) == 13
    h, w = yd.shape
    ww, wh = w // 16, h // 16
    ring = [np.ascontiguousarray(r, np.uint16) for r in ring]
    ptrs = (ctypes.c_void_p * 13)(*[r.ctypes.data for r in ring])
    o64 = np.zeros((wh * ww, 5), np.float64)
    o32 = np.zeros((wh * ww, 5), np.float32)
    lib().eso_persist_stats(ptrs, _ptr(np.ascontiguousarray(yd, np.uint16)), up, w, h, _ptr(o64), _ptr(o32))
    return o64, o32


def plane_sse(a: np.ndarray, b: np.ndarray) -> int:
    a = np.ascontiguousarray(a, np.uint16)
    b = np.ascontiguousarray(b, np.uint16)
    return int(lib().eso_plane_sse(_ptr(a), _ptr(b), a.size))


def color_sums(u: np.ndarray, v: np.ndarray, up: int) -> np.ndarray:
    out = np.zeros(3, np.float64)
    u = np.ascontiguousarray(u, np.uint16)
    v = np.ascontiguousarray(v, np.uint16)
    lib().eso_color_sums(_ptr(u), _ptr(v), u.size, up, _ptr(out))
    return out


# ------------------------------------------------------------------------------------------------------------------
# Host logic (numpy): src/stats.hpp and src/main.cpp collect
# ------------------------------------------------------------------------------------------------------------------

HIST_BINS = 20001
HIST_LO, HIST_STEP = -500.0, 0.05
KSTATS, KPERSIST, RADIUS = 8, 5, 6


def lround_nonneg(x: np.ndarray) -> np.ndarray:
    """``std::lround`` for non-negative doubles: halves go up."""
    t = np.trunc(x)
    return (t + ((x - t) >= 0.5)).astype(np.int64)


def hist_bins(pct: np.ndarray) -> np.ndarray:
    """``Histogram::add``'s bin of each percentage (``src/stats.hpp:14-19``)."""
    pct = np.asarray(pct, np.float64)
    return lround_nonneg((np.clip(pct, HIST_LO, -HIST_LO) - HIST_LO) / HIST_STEP)


@dataclass
class Histogram:
    """``src/stats.hpp:10-32``."""
    bins: np.ndarray = field(default_factory=lambda: np.zeros(HIST_BINS, np.uint64))
    n: int = 0

    def add(self, pcts) -> None:
        b = hist_bins(np.atleast_1d(pcts))
        np.add.at(self.bins, b, 1)
        self.n += int(b.size)

    def quantile(self, q: float) -> float:
        if not self.n:
            return float("nan")
        target = q * float(self.n - 1)
        seen = np.cumsum(self.bins.astype(np.float64))
        idx = np.nonzero(seen > target)[0]
        return HIST_LO + float(idx[0]) * HIST_STEP if idx.size else -HIST_LO

    def merge(self, o: "Histogram") -> None:
        self.bins += o.bins
        self.n += o.n


WEIGHTS = {"fidelity": 0.30, "texture": 0.30, "banding": 0.25, "grain": 0.15}


@dataclass
class Accum:
    """``src/stats.hpp:36-83``."""
    frames: int = 0
    vmaf: float = 0.0
    vmaf_min: float = 1e9
    psnr: np.ndarray = field(default_factory=lambda: np.zeros(3))
    cambi: float = 0.0
    cambi_source: float = 0.0
    color_r: np.ndarray = field(default_factory=lambda: np.zeros(3))
    color_d: np.ndarray = field(default_factory=lambda: np.zeros(3))
    all_r: np.ndarray = field(default_factory=lambda: np.zeros(3))
    all_d: np.ndarray = field(default_factory=lambda: np.zeros(3))
    st_r: np.ndarray = field(default_factory=lambda: np.zeros(3))
    st_d: np.ndarray = field(default_factory=lambda: np.zeros(3))
    amount: list = field(default_factory=lambda: [Histogram() for _ in range(3)])
    sh_all_r: np.ndarray = field(default_factory=lambda: np.zeros(2))
    sh_all_x: np.ndarray = field(default_factory=lambda: np.zeros(2))
    sh_st_r: np.ndarray = field(default_factory=lambda: np.zeros(2))
    sh_st_x: np.ndarray = field(default_factory=lambda: np.zeros(2))
    matching: list = field(default_factory=lambda: [Histogram() for _ in range(2)])
    own: float = 0.0
    mine: float = 0.0
    lasting: Histogram = field(default_factory=Histogram)

    def merge(self, o: "Accum") -> None:
        self.frames += o.frames
        self.vmaf += o.vmaf
        self.vmaf_min = min(self.vmaf_min, o.vmaf_min)
        self.cambi += o.cambi
        self.cambi_source += o.cambi_source
        self.own += o.own
        self.mine += o.mine
        for name in ("psnr", "color_r", "color_d", "all_r", "all_d", "st_r", "st_d", "sh_all_r", "sh_all_x", "sh_st_r", "sh_st_x"):
            getattr(self, name)[:] += getattr(o, name)
        for a, b in zip(self.amount, o.amount):
            a.merge(b)
        for a, b in zip(self.matching, o.matching):
            a.merge(b)
        self.lasting.merge(o.lasting)

    @staticmethod
    def kept(d: float, r: float) -> float:
        return 100.0 * math.sqrt(d / r) if r > 0 else float("nan")

    def score(self, weights: dict | None = None) -> dict:
        w = weights or WEIGHTS
        clamp = lambda v: min(max(v, 0.0), 100.0)  # noqa: E731
        fidelity = clamp(self.vmaf / self.frames) if self.frames else float("nan")
        texture = clamp(self.lasting.quantile(0.5)) / 2 + clamp(self.lasting.quantile(0.1)) / 2 if self.lasting.n >= 100 else float("nan")
        banding = clamp(100.0 * (1 - (self.cambi - self.cambi_source) / self.frames / 5.0)) if self.frames else float("nan")
        grain = clamp(100.0 - abs(self.kept(self.all_d[0], self.all_r[0]) - 100.0))
        parts = {"fidelity": fidelity, "texture": texture, "banding": banding, "grain": grain}
        total = weight = 0.0
        for k in ("fidelity", "texture", "banding", "grain"):
            if not math.isnan(parts[k]):
                total += parts[k] * w[k]
                weight += w[k]
        parts["score"] = total / weight if weight else float("nan")
        return parts


def psnr(sse: int, n: int, depth: int) -> float:
    """``src/main.cpp:272-277``."""
    mse = float(sse) / float(n)
    peak = float((1 << depth) - 1)
    return min(10.0 * math.log10(peak * peak / max(mse, 1e-16)), 6.0 * depth + 12)


def quantile_like_reference(v: np.ndarray, q: float) -> np.float32:
    """``src/main.cpp:280-289``: numpy's linear quantile from exact order statistics, float arithmetic as the C++."""
    v = np.asarray(v, np.float32)
    pos = q * float(v.size - 1)
    lo = int(pos)
    s = np.sort(v)
    a = s[lo]
    if lo + 1 >= v.size:
        return a
    b = s[lo + 1]
    diff = np.float32(b - a)  # float subtraction, then double arithmetic
    return np.float32(float(a) + float(diff) * (pos - float(lo)))


def collect_frame(acc: Accum, stats: np.ndarray) -> np.ndarray:
    """The per-window part of ``src/main.cpp:606-629``: adds one frame's window figures to `acc` and returns the
    structure mask (oriented >= its 0.8 quantile and > 0)."""
    st = np.asarray(stats, np.float32).reshape(-1, KSTATS)
    q = quantile_like_reference(st[:, 6], 0.8)
    m = (st[:, 6] >= q) & (st[:, 6] > 0)
    er = st[:, [0, 1, 6]].astype(np.float64)
    ed = st[:, [2, 3, 7]].astype(np.float64)
    for key in range(3):
        acc.all_r[key] += er[:, key].sum()
        acc.all_d[key] += ed[:, key].sum()
        acc.st_r[key] += er[m, key].sum()
        acc.st_d[key] += ed[m, key].sum()
        acc.amount[key].add(100.0 * np.sqrt(ed[m, key] / np.maximum(er[m, key], 1e-9)))
    for key in range(2):
        x = st[:, 4 + key].astype(np.float64)
        acc.sh_all_r[key] += er[:, key].sum()
        acc.sh_all_x[key] += x.sum()
        acc.sh_st_r[key] += er[m, key].sum()
        acc.sh_st_x[key] += x[m].sum()
        acc.matching[key].add(100.0 * x[m] / np.maximum(er[m, key], 1e-9))
    return m


def collect_lasting(acc: Accum, persist: np.ndarray, centre_mask: np.ndarray) -> None:
    """``src/main.cpp:630-641``: lasting texture of the centre frame into its segment's accumulator."""
    s = np.asarray(persist, np.float32).reshape(-1, KPERSIST)
    agree = s[:, 2].astype(np.float64) / np.sqrt(np.maximum(s[:, 3].astype(np.float64) * s[:, 4].astype(np.float64), 1e-9))
    keep = centre_mask.astype(bool) & (agree > 0.5) & (s[:, 0] > 0)
    acc.own += s[keep, 0].astype(np.float64).sum()
    acc.mine += s[keep, 1].astype(np.float64).sum()
    acc.lasting.add(100.0 * s[keep, 1].astype(np.float64) / s[keep, 0].astype(np.float64))


def parts_json(a: Accum) -> dict:
    """The JSON object of one segment (``src/main.cpp:738-757``), with NaN for null."""
    p = a.score()
    f = float(a.frames)
    k = Accum.kept
    return {"frames": a.frames, "score": p["score"], "fidelity": p["fidelity"], "texture": p["texture"], "banding": p["banding"], "grain": p["grain"],
            "vmaf": a.vmaf / f, "vmaf_min": a.vmaf_min, "psnr_y": a.psnr[0] / f, "psnr_cb": a.psnr[1] / f, "psnr_cr": a.psnr[2] / f,
            "cambi": a.cambi / f, "cambi_source": a.cambi_source / f,
            "lasting": {"windows": a.lasting.n, "median": a.lasting.quantile(0.5), "worst_tenth": a.lasting.quantile(0.1),
                        "total": 100.0 * a.mine / a.own if a.own > 0 else float("nan")},
            "amount": {"all": [k(a.all_d[i], a.all_r[i]) for i in range(3)], "structure": [k(a.st_d[i], a.st_r[i]) for i in range(3)],
                       "median": [a.amount[i].quantile(0.5) for i in range(3)], "worst_tenth": [a.amount[i].quantile(0.1) for i in range(3)]},
            "matching": {"all": [100.0 * a.sh_all_x[i] / a.sh_all_r[i] if a.sh_all_r[i] else float("nan") for i in range(2)],
                         "structure": [100.0 * a.sh_st_x[i] / a.sh_st_r[i] if a.sh_st_r[i] else float("nan") for i in range(2)],
                         "median": [a.matching[i].quantile(0.5) for i in range(2)], "worst_tenth": [a.matching[i].quantile(0.1) for i in range(2)]},
            "color_source": [a.color_r[i] / f for i in range(3)], "color_encode": [a.color_d[i] / f for i in range(3)]}


def find_offset_lag(ref: np.ndarray, probe: np.ndarray) -> tuple[int, float]:
    """``src/main.cpp:339-348`` in C (eso_find_offset_lag): (lag, least mean difference) of the probe's thumbnails."""
    ref = np.ascontiguousarray(ref, np.float32)
    probe = np.ascontiguousarray(probe, np.float32)
    lag = ctypes.c_int()
    best = lib().eso_find_offset_lag(_ptr(ref), ref.size // 2304, _ptr(probe), probe.size // 2304, ctypes.byref(lag))
    return lag.value, best
