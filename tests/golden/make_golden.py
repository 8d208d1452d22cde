"""Writes tests/golden/compare_golden.npz: outputs of the reference's numpy specification
(reference/encode_score/compare.py, imported unmodified from the reference checkout) on seeded synthetic frames.

It runs only where the reference checkout exists (default /root/reference, or REFERENCE_ROOT); the tests read the
committed fixture. Contents:

* frames: 14 frames of a 160 x 96 10-bit source and one encode (es_synth's persistent-texture recipe), y / u / v;
* per-window energies (fine, mid, oriented) of the source and the encode of frame 0 and the cross sums of fine and
  mid detail, from the stock module (float32 box means) and from the same module with `box` patched only to skip its
  final float32 cast (so its arithmetic runs in float64);
* compare_frames over all 14 frames, and over the centres 6 .. 7 with the steady halves built in float64 as the
  reference's tests/test_native.py:110-111 builds them (the persistent-texture figures), flattened to key -> value.

Usage: python tests/golden/make_golden.py [REFERENCE_ROOT]
"""

import json
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, os.path.join(ROOT, "encode-score_b200"))
import es_synth  # noqa: E402

REF = sys.argv[1] if len(sys.argv) > 1 else os.environ.get("REFERENCE_ROOT", "/root/reference")
sys.path.insert(0, os.path.join(REF, "reference"))
from encode_score import compare  # noqa: E402

W, H, N = 160, 96, 14


def flatten(d, prefix=""):
    out = {}
    for k, v in d.items():
        key = f"{prefix}{k}"
        if isinstance(v, dict):
            out.update(flatten(v, key + "."))
        elif isinstance(v, (int, float, np.floating, np.integer)):
            out[key] = float(v)
    return out


def energies(box):
    saved = compare.box
    compare.box = box
    try:
        frames = FRAMES
        r = frames[0][0]["y"].astype(np.float64 if box is not saved else np.float32)
        d = frames[0][1]["y"].astype(np.float64 if box is not saved else np.float32)
        br, bd = compare.bands(r), compare.bands(d)
        er, ed = compare.window_energies(br["smooth"], br), compare.window_energies(bd["smooth"], bd)
        cross = {k: compare.window_sums(br[k] * bd[k]) for k in ("fine", "mid")}
        return er, ed, cross
    finally:
        compare.box = saved


def box64(a, k):
    """compare.box without its final float32 cast."""
    r = k // 2
    c = np.pad(a, r, mode="edge").cumsum(0, dtype=np.float64).cumsum(1, dtype=np.float64)
    c = np.pad(c, ((1, 0), (1, 0)))
    return (c[k:, k:] - c[:-k, k:] - c[k:, :-k] + c[:-k, :-k]) / (k * k)


steps = [es_synth.texture_step(f, w=W, h=H) for f in range(N)]
FRAMES = [({"y": s.source.y, "u": s.source.u, "v": s.source.v}, {"y": s.encodes[0].y, "u": s.encodes[0].u, "v": s.encodes[0].v}) for s in steps]

out = {}
for p in ("y", "u", "v"):
    out[f"src_{p}"] = np.stack([f[0][p] for f in FRAMES]).astype(np.uint16)
    out[f"enc_{p}"] = np.stack([f[1][p] for f in FRAMES]).astype(np.uint16)
for tag, box in (("f32", compare.box), ("f64", box64)):
    er, ed, cross = energies(box)
    for k in ("fine", "mid", "oriented"):
        out[f"{tag}_src_{k}"] = er[k].astype(np.float64)
        out[f"{tag}_enc_{k}"] = ed[k].astype(np.float64)
    for k in ("fine", "mid"):
        out[f"{tag}_cross_{k}"] = cross[k].astype(np.float64)

ref = [f[0] for f in FRAMES]
dist = [f[1] for f in FRAMES]
whole = compare.compare_frames(ref, dist)
centres = range(6, N - 6)
steady = [(np.mean([ref[c + o]["y"].astype(np.float64) for o in (-6, -4, -2, 2, 4, 6)], axis=0),
           np.mean([ref[c + o]["y"].astype(np.float64) for o in (-5, -3, -1, 1, 3, 5)], axis=0)) for c in centres]
lasting = compare.compare_frames([ref[c] for c in centres], [dist[c] for c in centres], steady)
figures = {"whole": flatten({k: v for k, v in whole.items() if k != "worst"}), "lasting": flatten(lasting["persistent"])}
out["figures_json"] = np.frombuffer(json.dumps(figures, sort_keys=True).encode(), dtype=np.uint8)
np.savez_compressed(os.path.join(HERE, "compare_golden.npz"), **out)
print("wrote", os.path.join(HERE, "compare_golden.npz"), {k: v.shape for k, v in out.items()})
