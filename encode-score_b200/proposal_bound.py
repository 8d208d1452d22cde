#!/usr/bin/env python3
"""The bound on any tile proposal for CAMBI on given content: how many c-value tiles a perfect predictor could skip.

CAMBI pools, per scale, the mean of the top 60 % of a picture's c-values over all its pixels (src/cambi.cpp:28-29,
172-184): while fewer than k values are positive, every positive c-value adds to the score; above k, only those above
the k-th. A proposal skips whole 64 x 64 tiles of scales 0 and 1 (scale-1 tiles of 64 x 64 cover 2 x 2 scale-0 tiles).
An oracle that knows every tile's exact c-values skips, per picture, the tiles of least mass first while the score
stays within the tolerance (|delta CAMBI| <= 0.05 by default), recomputing the exact pooled score each time; no real
network can skip more. The script reports, per encode of the c2 workload (4K 10-bit), the tiles that need a c-value,
those with any positive one, the share an oracle could skip, and the CDF of tile masses, from the CPU oracle's c-value
planes (no GPU needed).

Usage: python proposal_bound.py [--frames N] [--tolerance T] [--out FILE]
"""

from __future__ import annotations

import argparse
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, HERE)
sys.path.insert(0, os.path.join(os.path.dirname(HERE), "oracle"))

TILE = 64
WEIGHTS = (16.0, 8.0, 4.0, 2.0, 1.0)


def pooled(values: np.ndarray, n: int, topk: float = 0.6) -> float:
    """Mean of the top k of n c-values (values: the positive ones), k = clip(int(topk n), 1, n)."""
    k = min(max(int(topk * n), 1), n)
    if values.size <= k:
        return float(values.astype(np.float64).sum()) / k
    top = np.partition(values, values.size - k)[values.size - k:]
    return float(top.astype(np.float64).sum()) / k


def score_of(cvals: list, window: int) -> float:
    total = sum(WEIGHTS[s] * pooled(c[c > 0], c.size) for s, c in enumerate(cvals))
    return min(total / (window * window), 1000.0)


def tile_masks(shape, tile):
    h, w = shape
    return [(slice(y, min(y + tile, h)), slice(x, min(x + tile, w))) for y in range(0, h, tile) for x in range(0, w, tile)]


def oracle_skip(cvals: list, window: int, tolerance: float) -> dict:
    """Greedy: skip scale-0 and scale-1 tiles in ascending mass while the exact score stays within tolerance."""
    base = score_of(cvals, window)
    tiles = []
    for s in (0, 1):
        for sl in tile_masks(cvals[s].shape, TILE):
            tiles.append((float(cvals[s][sl].astype(np.float64).sum()), s, sl))
    need = len(tiles)
    tiles.sort(key=lambda t: t[0])
    work = [c.copy() for c in cvals]
    skipped = 0
    # skip in growing steps, backing off on the first step that breaks the tolerance
    lo, step = 0, 64
    while lo < len(tiles):
        hi = min(len(tiles), lo + step)
        trial = [c.copy() for c in work]
        for _, s, sl in tiles[lo:hi]:
            trial[s][sl] = 0
        if abs(score_of(trial, window) - base) <= tolerance:
            work, skipped, lo = trial, hi, hi
            step *= 2
        elif step > 1:
            step //= 2
        else:
            break
    return {"tiles": need, "zero_mass": sum(1 for m, _, _ in tiles if m == 0.0), "skippable": skipped, "score": base}


def main() -> None:
    ap = argparse.ArgumentParser()
    ap.add_argument("--frames", type=int, default=3)
    ap.add_argument("--tolerance", type=float, default=0.05)
    ap.add_argument("--out", default=None)
    args = ap.parse_args()

    import es_synth
    import oracle

    p = oracle.cambi_params(3840, 2160)
    rows = []
    masses = {0: [], 1: [], 2: []}
    for f in range(args.frames):
        step = es_synth.c2_step(f)
        for e, enc in enumerate(step.encodes):
            r = oracle.cambi(enc.y, 10, p, keep=True)
            res = oracle_skip(r.cvalues, p.window, args.tolerance)
            rows.append((f, e, res))
            for sl in tile_masks(r.cvalues[0].shape, TILE):
                masses[e].append(float(r.cvalues[0][sl].astype(np.float64).sum()))
            print(f"frame {f} encode {e}: CAMBI {res['score']:.4f}, scale 0-1 tiles {res['tiles']}, zero mass {res['zero_mass']}, "
                  f"oracle-skippable {res['skippable']} ({100.0 * res['skippable'] / res['tiles']:.1f} %)", flush=True)
    lines = ["# Bound on the learned tile proposal: what a perfect predictor could skip (4K10 c2 encodes)", "",
             f"`python encode-score_b200/proposal_bound.py --frames {args.frames} --tolerance {args.tolerance}` (CPU oracle, "
             "exact c-value planes; no GPU).", "",
             "A perfect predictor skips, per picture, the 64 x 64 tiles of scales 0 and 1 of least exact mass first while the "
             f"exact score stays within {args.tolerance} of the full score.", "",
             "| frame | encode | CAMBI | scale 0-1 tiles | tiles of zero mass | skippable by an oracle | share |",
             "|---|---|---|---|---|---|---|"]
    for f, e, res in rows:
        lines.append(f"| {f} | {e} | {res['score']:.4f} | {res['tiles']} | {res['zero_mass']} | {res['skippable']} | "
                     f"{100.0 * res['skippable'] / res['tiles']:.1f} % |")
    lines += ["", "Scale-0 tile mass CDF (exact sum of a tile's positive c-values), per encode:", "",
              "| encode | p10 | p25 | p50 | p75 | p90 | share of tiles with mass 0 |", "|---|---|---|---|---|---|---|"]
    for e, m in masses.items():
        a = np.array(m)
        q = np.percentile(a, [10, 25, 50, 75, 90])
        lines.append(f"| {e} | " + " | ".join(f"{v:.3g}" for v in q) + f" | {100.0 * np.mean(a == 0):.1f} % |")
    text = "\n".join(lines) + "\n"
    if args.out:
        with open(args.out, "w") as fh:
            fh.write(text)
    print(text)


if __name__ == "__main__":
    main()
