#!/usr/bin/env python3
"""TEST INFRASTRUCTURE: times the reference's own CPU path for the detail / texture / color measures,
reference/encode_score/compare.py:129-194 (compare_frames), imported unmodified from the reference checkout, on the
4K10 c2 frame pairs (seeded es_synth frames) with the steady halves built as tests/test_native.py:110-111 builds them.

It runs only where the reference checkout exists (REFERENCE_ROOT, default the container's checkout); the GPU hosts do
not have it, so bench.py cannot time it there. One process, one core (BLAS threads 1). Prints seconds per frame pair.

Usage: python oracle/time_compare_frames.py [--pairs N] [--w 3840 --h 2160]
"""

from __future__ import annotations

import argparse
import os
import sys
import time

os.environ.setdefault("OMP_NUM_THREADS", "1")
os.environ.setdefault("OPENBLAS_NUM_THREADS", "1")
os.environ.setdefault("MKL_NUM_THREADS", "1")

import numpy as np  # noqa: E402

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(os.path.dirname(HERE), "encode-score_b200"))


def main() -> None:
    ap = argparse.ArgumentParser()
    ap.add_argument("--pairs", type=int, default=3)
    ap.add_argument("--w", type=int, default=3840)
    ap.add_argument("--h", type=int, default=2160)
    args = ap.parse_args()
    ref_root = os.environ.get("REFERENCE_ROOT", "/root/reference")
    sys.path.insert(0, os.path.join(ref_root, "reference"))
    from encode_score import compare as reference  # the unmodified module

    import es_synth

    n = args.pairs + 12  # the lasting texture of a centre frame reads 6 frames either side
    steps = [es_synth.c2_step(f, w=args.w, h=args.h, n_encodes=1) for f in range(n)]
    ref = [{"y": s.source.y, "u": s.source.u, "v": s.source.v} for s in steps]
    dist = [{"y": s.encodes[0].y, "u": s.encodes[0].u, "v": s.encodes[0].v} for s in steps]
    centres = range(6, n - 6)
    t0 = time.perf_counter()
    steady = [(np.mean([ref[c + o]["y"].astype(np.float64) for o in (-6, -4, -2, 2, 4, 6)], axis=0),
               np.mean([ref[c + o]["y"].astype(np.float64) for o in (-5, -3, -1, 1, 3, 5)], axis=0)) for c in centres]
    reference.compare_frames([ref[c] for c in centres], [dist[c] for c in centres], steady)
    secs = time.perf_counter() - t0
    pairs = len(centres)
    print(f"compare_frames with steady halves: {pairs} pairs of {args.w}x{args.h} in {secs:.2f} s, "
          f"{secs / pairs:.3f} s per pair, {pairs / secs:.3f} frame pairs/s on 1 core")


if __name__ == "__main__":
    main()
