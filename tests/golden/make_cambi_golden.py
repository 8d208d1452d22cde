"""Writes cambi_ref_golden.npz: CAMBI outputs of the reference's own GPU implementation (its src/kernels.cu,
src/cambi.cpp and src/gpu.cpp compiled unmodified into oracle/_ref/libref.so by `make -C oracle ref`) on small seeded
pictures, for the CPU test that pins the oracle to them (tests/test_golden_cpu.py).

Per case: the input plane, the parameters, every scale's mode-filtered picture, mask and c-values from the reference's
kernels run with its own launch shapes (src/cambi.cpp:88-135), its per-scale sums and counts of positive c-values, and
the score of its Cambi class (src/cambi.cpp:172-184).

Needs an sm_100 GPU and oracle/_ref/libref.so. Usage: python tests/golden/make_cambi_golden.py OUT.npz
"""

import json
import os
import sys

import numpy as np
import torch

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path[:0] = [os.path.join(ROOT, "oracle"), os.path.join(ROOT, "encode-score_b200")]
import es_b200  # noqa: E402
import refgpu  # noqa: E402


def banded(w, h, seed, lo, hi, step, grain=0.0, top=1023):
    rng = np.random.default_rng(seed)
    yy, xx = np.mgrid[0:h, 0:w]
    a = rng.uniform(0, 2 * np.pi)
    g = np.cos(a) * xx / w + np.sin(a) * yy / h
    g = (g - g.min()) / max(np.ptp(g), 1e-9)
    v = lo + (hi - lo) * g + (rng.normal(0, grain, (h, w)) if grain else 0)
    return np.clip(np.round(v / step) * step, 0, top).astype(np.uint16)


def blocks(w, h, seed, lo, hi, size):
    rng = np.random.default_rng(seed)
    b = rng.integers(lo, hi, ((h + size - 1) // size, (w + size - 1) // size))
    return np.kron(b, np.ones((size, size), np.int64))[:h, :w].astype(np.uint16)


CASES = [
    ("banded10", banded(176, 100, 41, 80, 200, 2), 10, 17),
    ("banded8", banded(160, 90, 42, 20, 60, 1, top=255), 8, 15),
    ("blocks10", blocks(192, 112, 43, 90, 170, 5), 10, 21),
    ("grainy10", banded(144, 80, 44, 100, 180, 1, grain=0.4), 10, 13),
]


def main(out_path):
    torch.cuda.init()
    ref = refgpu.load()
    assert ref is not None, "oracle/_ref/libref.so is missing"
    out, meta = {}, {}
    for name, img, depth, window in CASES:
        h, w = img.shape
        p = es_b200.derive_params(w, h)
        p.window, p.pad = window, window // 2
        sizes = []
        sw, sh = w, h
        for _ in range(5):
            sizes.append((sw, sh))
            sw, sh = (sw + 1) >> 1, (sh + 1) >> 1
        dev = lambda shape, dt: torch.zeros(shape, dtype=dt, device="cuda")  # noqa: E731
        images = [dev((b, a), torch.int16) for a, b in sizes]
        masks = [dev((b, a), torch.uint8) for a, b in sizes]
        cvals = [dev((b, a), torch.float32) for a, b in sizes]
        scratch = dev((h, w), torch.int16)
        sums = dev((10,), torch.float64)
        dimg = torch.from_numpy(img.view(np.int16)).cuda()
        ref.cambi_steps(dimg.data_ptr(), w, w, h, depth, p.as_dict(), [t.data_ptr() for t in images], [t.data_ptr() for t in masks],
                        [t.data_ptr() for t in cvals], scratch.data_ptr(), sums.data_ptr())
        torch.cuda.synchronize()
        out[f"{name}_input"] = img
        for s in range(5):
            out[f"{name}_image{s}"] = images[s].cpu().numpy().view(np.uint16)
            out[f"{name}_mask{s}"] = masks[s].cpu().numpy()
            out[f"{name}_cvalues{s}"] = cvals[s].cpu().numpy()
        sv = sums.cpu().numpy()
        out[f"{name}_sums"] = sv[:5].copy()
        out[f"{name}_counts"] = sv[5:].view(np.uint64).copy()
        # the reference's Cambi class derives its own window from the picture size
        meta[name] = {"depth": depth, "params": p.as_dict(), "class_score": ref.cambi_score(dimg.data_ptr(), w, h, depth),
                      "class_params": es_b200.derive_params(w, h).as_dict()}
    out["meta_json"] = np.frombuffer(json.dumps(meta, sort_keys=True).encode(), dtype=np.uint8)
    np.savez_compressed(out_path, **out)
    print("wrote", out_path, json.dumps({k: v["class_score"] for k, v in meta.items()}))


if __name__ == "__main__":
    main(sys.argv[1] if len(sys.argv) > 1 else os.path.join(HERE, "cambi_ref_golden.npz"))
