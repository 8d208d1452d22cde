#!/usr/bin/env python3
"""The c-value tile autotuner: picks, per picture size, the shape of the c-value kernel's tiles at each of CAMBI's five
scales -- 64 or 128 columns (blocks of 256 or 512 threads) by 64, 32 or 16 rows -- and writes the table es_b200.Batch
reads (autotune.json).

Wider and taller tiles stage proportionally less window margin ((columns + 2 pad) x (rows + 2 pad) region pixels per
tile), smaller tiles balance the few tiles of the small scales over more blocks; which wins depends on the picture size
and window. For each size the tuner scores a source and an encode of synthetic content (es_synth: the c2 recipe at 10
bits, c3's at 8), timing the c-value launches alone with CUDA events (es_kernel_timing) over a few steps, and runs a
coordinate descent: starting from the library's default shapes, each scale in turn tries every shape and keeps the
fastest when it gains more than 2%.
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
    table = {"device": torch.cuda.get_device_name(0), "method": "coordinate descent over scales and tile shapes, 2% gain to switch",
             "classes": {}}
    stream = torch.cuda.current_stream().cuda_stream
    for (w, h, depth) in classes:
        steps = []
        for f in range(2):
            st = es_synth.c2_step(f, w=w, h=h, n_encodes=1) if depth == 10 else es_synth.c3_step(f, 0, w, h, depth)
            steps.append(st)
        dev = [es_b200.device_step(torch, st) for st in steps]

        def time_shape(rows, cols):
            b = es_b200.Batch(module, [(w, h, depth, 1)], use_graphs=False, tuning={(w, h): {"rows": rows, "cols": cols}})
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
        rows, cols = [64] * 5, [64] * 5  # the library's defaults
        best_ms = time_shape(rows, cols)
        base_ms = best_ms
        tried = [[list(rows), list(cols), best_ms]]
        for s in range(5):
            for c in (128, 64):
                for r in (64, 32, 16):
                    if (r, c) == (rows[s], cols[s]):
                        continue
                    cr, cc = list(rows), list(cols)
                    cr[s], cc[s] = r, c
                    ms = time_shape(cr, cc)
                    tried.append([cr, cc, ms])
                    if ms < best_ms * 0.98:
                        rows, cols, best_ms = cr, cc, ms
        table["classes"][f"{w}x{h}"] = {"depth": depth, "cv_tile_rows": rows, "cv_tile_cols": cols, "cvalues_ms": best_ms,
                                        "cvalues_ms_defaults": base_ms, "tried": tried, "seconds": time.time() - t0}
        print(f"{w}x{h}@{depth}: rows {rows} cols {cols} {best_ms:.3f} ms (defaults: {base_ms:.3f} ms)", flush=True)
    with open(args.out, "w") as fh:
        json.dump(table, fh, indent=1)
    module.close()


if __name__ == "__main__":
    main()
