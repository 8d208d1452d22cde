#!/usr/bin/env python3
"""The c-value tile autotuner: picks, per picture size, the rows of the c-value kernel's tiles at each of CAMBI's five
scales (64, 32 or 16; tiles are 64 pixels wide), and writes the table es_b200.Batch reads (autotune.json).

Taller tiles stage proportionally less window margin (rows + 2 pad region rows per tile), shorter tiles balance the
few tiles of the small scales over more blocks; which wins depends on the picture size and window. For each size the
tuner scores a source and an encode of synthetic content (es_synth: the c2 recipe at 10 bits, c3's at 8), timing the
c-value launch alone with CUDA events (es_kernel_timing) over a few steps, and runs a coordinate descent: starting
from 64 rows everywhere, each scale in turn tries 32 and 16 and keeps the fastest when it gains more than 2%.
"""

from __future__ import annotations

import argparse
import json
import os
import sys
import time

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, HERE)

CLASSES = [(1920, 1080, 8), (3840, 2160, 10), (1280, 720, 8), (1920, 800, 10), (3840, 1600, 10)]


def main() -> None:
    ap = argparse.ArgumentParser()
    ap.add_argument("--steps", type=int, default=4)
    ap.add_argument("--out", default=os.path.join(HERE, "autotune.json"))
    ap.add_argument("--classes", default=None, help="WxHxD,... (default: the workloads' sizes)")
    args = ap.parse_args()

    import numpy as np
    import torch

    import es_b200
    import es_synth

    torch.cuda.set_device(0)
    module = es_b200.Module()
    classes = CLASSES if not args.classes else [tuple(int(v) for v in c.split("x")) for c in args.classes.split(",")]
    table = {"device": torch.cuda.get_device_name(0), "method": "coordinate descent over scales, 2% gain to switch",
             "classes": {}}
    stream = torch.cuda.current_stream().cuda_stream
    for (w, h, depth) in classes:
        steps = []
        for f in range(2):
            st = es_synth.c2_step(f, w=w, h=h, n_encodes=1) if depth == 10 else es_synth.c3_step(f, 0, w, h, depth)
            steps.append(st)
        dev = [es_b200.device_step(torch, st) for st in steps]

        def time_rows(rows):
            b = es_b200.Batch(module, [(w, h, depth, 1)], use_graphs=False, tuning={(w, h): rows})
            acc = [es_b200.new_accum()]
            f = 0
            for _ in range(2):
                keep, views = dev[f % 2]
                b.queue(f, views, stream)
                b.collect(f, acc, acc)
                f += 1
            es_b200.kernel_timing(True, serial=True)
            for _ in range(args.steps):
                keep, views = dev[f % 2]
                b.queue(f, views, stream)
                b.collect(f, acc, acc)
                f += 1
            times = es_b200.kernel_times()
            es_b200.kernel_timing(False)
            b.close()
            return times["cambi_cvalues"][0] / args.steps

        t0 = time.time()
        best = [64] * 5
        best_ms = time_rows(best)
        base_ms = best_ms
        tried = [[list(best), best_ms]]
        for s in range(5):
            for r in (32, 16):
                cand = list(best)
                cand[s] = r
                ms = time_rows(cand)
                tried.append([cand, ms])
                if ms < best_ms * 0.98:
                    best, best_ms = cand, ms
        table["classes"][f"{w}x{h}"] = {"depth": depth, "cv_tile_rows": best, "cvalues_ms": best_ms, "cvalues_ms_all_64": base_ms,
                                        "tried": tried, "seconds": time.time() - t0}
        print(f"{w}x{h}@{depth}: {best} {best_ms:.3f} ms (all 64: {base_ms:.3f} ms)", flush=True)
    with open(args.out, "w") as fh:
        json.dump(table, fh, indent=1)
    module.close()


if __name__ == "__main__":
    main()
