#!/usr/bin/env python3
"""The precision study of the texture window energies on the GPU: --frames seeded 3840x2160 10-bit pairs of the
precision workload (es_synth_gpu.c4_pair: bright gradient 600-940 with grain sigma 20, encode blurred sigma 1.0),
windows of 32 and 128 pixels, figures from integer summed-area tables (exact, the FP64 reference), compensated FP32 and
plain FP32 (es_windows_*).

Reports per arithmetic and window: the max, median and 99.9th-percentile relative error per window figure (max over all
windows and frames, percentiles over every 10th frame; relative to the exact figure; figures of 0 excluded) and the relative error of the per-segment accumulations (each
figure summed in FP64 over all windows of all frames, as the segment sums of src/main.cpp:614-629 are).
"""

from __future__ import annotations

import argparse
import json
import os
import sys
import time

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, HERE)

W, H = 3840, 2160
FIGURES = ["src_fine2", "src_mid2", "enc_fine2", "enc_mid2", "fine_x", "mid_x", "src_oriented", "enc_oriented"]


def main() -> None:
    ap = argparse.ArgumentParser()
    ap.add_argument("--frames", type=int, default=1000)
    ap.add_argument("--windows", default="32,128")
    ap.add_argument("--out", default=None)
    args = ap.parse_args()

    import numpy as np
    import torch

    import es_b200
    import es_synth_gpu

    torch.cuda.set_device(0)
    module = es_b200.Module()
    win = es_b200.Windows(W, H)
    sizes = [int(s) for s in args.windows.split(",")]
    outs = {(s, m): torch.zeros(((W // s) * (H // s), 8), dtype=torch.float64, device="cuda") for s in sizes for m in range(3)}
    # per window figure: running max and a sample for the median; per segment: FP64 sums
    rel_max = {(s, m): np.zeros(8) for s in sizes for m in (1, 2)}
    rel_samples = {(s, m): [] for s in sizes for m in (1, 2)}
    seg = {(s, m): np.zeros(8) for s in sizes for m in range(3)}
    t0 = time.time()
    ms_compute = 0.0
    ev = [torch.cuda.Event(enable_timing=True) for _ in range(2)]
    for f in range(args.frames):
        src, enc = es_synth_gpu.c4_pair(torch, f)
        ev[0].record()
        win.compute(src.data_ptr(), enc.data_ptr(), 0, torch.cuda.current_stream().cuda_stream)
        for s in sizes:
            for m in range(3):
                win.figures(s, m, outs[(s, m)].data_ptr(), torch.cuda.current_stream().cuda_stream)
        ev[1].record()
        torch.cuda.synchronize()
        ms_compute += ev[0].elapsed_time(ev[1])
        for s in sizes:
            exact = outs[(s, 0)]
            seg[(s, 0)] += exact.sum(dim=0).cpu().numpy()
            nz = exact != 0
            for m in (1, 2):
                approx = outs[(s, m)]
                rel = torch.where(nz, (approx - exact).abs() / exact.abs().clamp_min(1e-300), torch.zeros_like(exact))
                rel_max[(s, m)] = np.maximum(rel_max[(s, m)], rel.max(dim=0).values.cpu().numpy())
                if f % 10 == 0:
                    rel_samples[(s, m)].append(rel.cpu().numpy())
                seg[(s, m)] += approx.sum(dim=0).cpu().numpy()
    report = {"frames": args.frames, "workload": "3840x2160 10-bit, bright gradient 600-940 + grain sigma 20; encode blur sigma 1.0",
              "gpu_ms_per_frame_all_modes": ms_compute / args.frames, "seconds": time.time() - t0, "windows": {}}
    names = {1: "compensated_fp32", 2: "fp32"}
    for s in sizes:
        entry = {}
        for m in (1, 2):
            sample = np.concatenate(rel_samples[(s, m)], axis=0)
            seg_rel = np.abs(seg[(s, m)] - seg[(s, 0)]) / np.abs(seg[(s, 0)])
            entry[names[m]] = {
                "per_window_max_rel": dict(zip(FIGURES, rel_max[(s, m)].tolist())),
                "per_window_median_rel": dict(zip(FIGURES, np.median(sample, axis=0).tolist())),
                "per_window_p999_rel": dict(zip(FIGURES, np.percentile(sample, 99.9, axis=0).tolist())),
                "per_segment_rel": dict(zip(FIGURES, seg_rel.tolist())),
            }
        entry["integer"] = "exact: the reference for the other two (int64 numerators, one rounding per figure)"
        report["windows"][str(s)] = entry
    text = json.dumps(report, indent=1)
    print(text)
    if args.out:
        with open(args.out, "w") as fh:
            fh.write(text)
    win.close()
    module.close()


if __name__ == "__main__":
    main()
