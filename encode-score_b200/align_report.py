#!/usr/bin/env python3
"""Throughput of the offset search on one B200 (one JSON line).

* thumbnails: es_thumbnails of 64 seeded 3840x2160 10-bit frames in one launch, timed with CUDA events after warm-up;
  frames/s and the luma bytes read per second against the measured HBM copy bandwidth (MEASURED_PEAKS.json);
* offset search: es_find_offset of 8 s of an encode (192 thumbnails at 24 fps) against 28 s of the source (674
  thumbnails), as src/main.cpp:412-419 sizes it: the lag totals kernel timed with CUDA events, and the whole call
  (kernel, copy of the totals, the choice on the host) with a host clock.
"""

from __future__ import annotations

import json
import os
import sys
import time

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, HERE)

import numpy as np
import torch

import es_b200


def main() -> None:
    w, h, n = 3840, 2160, 64
    rng = np.random.default_rng(11)
    planes = torch.from_numpy(rng.integers(64, 941, (n, h, w), dtype=np.int16)).cuda()
    views = [es_b200.FrameView(planes[i].data_ptr(), planes[i].data_ptr(), planes[i].data_ptr(), w * 2, w, 0, 2, 0, 10) for i in range(n)]
    out = torch.zeros(n * 2304, dtype=torch.float32, device="cuda")
    stream = torch.cuda.current_stream().cuda_stream
    for _ in range(3):
        es_b200.thumbnails(views, 0, 0, w, h, out.data_ptr(), stream)
    reps = 10
    s, e = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    s.record()
    for _ in range(reps):
        es_b200.thumbnails(views, 0, 0, w, h, out.data_ptr(), stream)
    e.record()
    e.synchronize()
    ms = s.elapsed_time(e) / reps
    gbs = n * w * h * 2 / (ms / 1000.0) / 1e9
    peak = None
    peaks = os.path.join(os.path.dirname(HERE), "MEASURED_PEAKS.json")
    if os.path.exists(peaks):
        peak = json.load(open(peaks)).get("hbm_gbs")
    del planes

    n_ref, n_probe = (2 * 10 + 8) * 24 + 2, 8 * 24
    yy, xx = np.mgrid[0:36, 0:64].astype(np.float32)
    ref = np.array([512 + 200 * np.sin(0.2 * xx + 0.35 * t) * np.cos(0.15 * yy - 0.25 * t) for t in range(n_ref)], np.float32)
    probe = ref[240:240 + n_probe] + rng.normal(0, 2, (n_probe, 36, 64)).astype(np.float32)
    d_ref, d_probe = torch.from_numpy(ref.ravel()).cuda(), torch.from_numpy(probe.ravel().copy()).cuda()
    totals = torch.zeros(n_ref - n_probe + 1, dtype=torch.float64, device="cuda")
    es_b200.offset_totals(d_ref.data_ptr(), n_ref, d_probe.data_ptr(), n_probe, totals.data_ptr(), stream)
    s.record()
    es_b200.offset_totals(d_ref.data_ptr(), n_ref, d_probe.data_ptr(), n_probe, totals.data_ptr(), stream)
    e.record()
    e.synchronize()
    totals_ms = s.elapsed_time(e)
    t_ref = [k / 24.0 for k in range(n_ref)]
    es_b200.find_offset(d_ref.data_ptr(), t_ref, d_probe.data_ptr(), [0.0] * n_probe, stream)  # warm-up
    t0 = time.perf_counter()
    off, best = es_b200.find_offset(d_ref.data_ptr(), t_ref, d_probe.data_ptr(), [0.0] * n_probe, stream)
    call_ms = 1000.0 * (time.perf_counter() - t0)
    print(json.dumps({
        "thumbnails": {"frames": n, "size": f"{w}x{h} 10-bit", "ms_per_launch": ms, "frames_per_s": n / (ms / 1000.0),
                       "luma_gb_per_s": gbs, "hbm_peak_gb_per_s": peak, "frac": gbs / peak if peak else None},
        "offset_search": {"probe_frames": n_probe, "reference_frames": n_ref, "lags": n_ref - n_probe + 1,
                          "abs_differences": (n_ref - n_probe + 1) * n_probe * 2304, "totals_kernel_ms": totals_ms,
                          "find_offset_call_ms": call_ms, "lag_found": round(off * 24), "best_mean": best},
    }))


if __name__ == "__main__":
    main()
