#!/usr/bin/env python3
"""Trains the tile-proposal network on the GPU with the library's own training kernels (es_proposal_net_train_step).

Data: frame pairs from es_synth_gpu (3840x2160 10-bit, seeds from --seed on), each picture scored by the plain GPU
CAMBI (es_cambi) with per-tile c-value sums; the label of a 64 x 64 scale-0 tile is log1p(sum of its positive
c-values / its pixels). Each step takes --batch crops of 4 x 4 tiles (72 x 72 feature pixels with the network's 4-pixel
margin) from the step's pictures, crops with no tile that needs a c-value left out, and one Adam step (lr --lr).

Writes the FP32 parameters (ES_PROPOSAL_PARAMS floats, .npy) and a JSON record of the run (loss curve, validation
figures and the threshold chosen on validation frames: the largest threshold that keeps the skipped tiles' share of the
score -- before any audit -- under --budget on at least --coverage of the validation pictures).
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
TILE = 64
CROP_TILES = 4
FEAT = 8 + 16 * CROP_TILES  # 72


def scale_tiles(w, h):
    out = []
    for _ in range(5):
        out.append(((w + TILE - 1) // TILE, (h + TILE - 1) // TILE, w, h))
        w, h = (w + 1) >> 1, (h + 1) >> 1
    return out


class Labeller:
    """es_cambi of 3840x2160 10-bit pictures with per-tile c-value sums; one instance per picture slot, so a picture's
    scale-0 words stay valid until its slot is run again."""

    def __init__(self, torch, es_b200, module, slots: int = 2):
        self.torch, self.es = torch, es_b200
        self.ntiles = es_b200.cambi_tile_count(W, H)
        self.mass = torch.zeros(self.ntiles, dtype=torch.int64, device="cuda")
        self.cambis = [es_b200.Cambi(module, W, H, 10) for _ in range(slots)]
        for c in self.cambis:
            c.set_tile_mass(self.mass.data_ptr())
        self.grid = scale_tiles(W, H)
        p = es_b200.derive_params(W, H)
        self.window = p.window
        self.k = [max(1, min(int(0.6 * w * h), w * h)) for _, _, w, h in self.grid]
        # pixels of each scale-0 / scale-1 tile (edge tiles are partial)
        self.pixels = []
        for tx, ty, w, h in self.grid[:2]:
            xs = torch.clamp(w - TILE * torch.arange(tx, device="cuda"), max=TILE)
            ys = torch.clamp(h - TILE * torch.arange(ty, device="cuda"), max=TILE)
            self.pixels.append((ys.view(-1, 1) * xs.view(1, -1)).double())

    def run(self, plane, slot: int = 0):
        """CAMBI of one int16 plane; returns (score, scale-0 masses (ty, tx) float64, scale-1 masses, words address)."""
        c = self.cambis[slot]
        c.launch(plane.data_ptr(), W, self.torch.cuda.current_stream().cuda_stream)
        score = c.finish()
        m = self.mass.double()
        tx0, ty0 = self.grid[0][:2]
        tx1, ty1 = self.grid[1][:2]
        m0 = m[:tx0 * ty0].view(ty0, tx0)
        m1 = m[tx0 * ty0:tx0 * ty0 + tx1 * ty1].view(ty1, tx1)
        return score, m0, m1, c.scale_words(0)

    def labels(self, m0):
        return self.torch.log1p(m0 / 16777216.0 / self.pixels[0]).float()

    def delta_if_skipped(self, m0, m1, keep0, keep1):
        """The score the skipped tiles would add (the sum / k case of the pooling): 16 M0 / k0 + 8 M1 / k1 over
        window^2, M the skipped tiles' c-value sums (numpy arrays)."""
        s0 = float((m0 * (~keep0)).sum()) / 16777216.0
        s1 = float((m1 * (~keep1)).sum()) / 16777216.0
        return (16.0 * s0 / self.k[0] + 8.0 * s1 / self.k[1]) / (self.window * self.window)

    def close(self):
        for c in self.cambis:
            c.close()


def keep_masks(np, pred, threshold):
    """Tiles of scales 0 and 1 that run (numpy): scale 0 where pred >= threshold; scale 1 where a covered scale-0 tile
    runs."""
    k0 = pred >= threshold
    ty, tx = k0.shape
    pad = np.zeros(((ty + 1) // 2 * 2, (tx + 1) // 2 * 2), bool)
    pad[:ty, :tx] = k0
    k1 = pad.reshape(pad.shape[0] // 2, 2, pad.shape[1] // 2, 2).any(axis=(1, 3))
    return k0, k1


def main() -> None:
    ap = argparse.ArgumentParser()
    ap.add_argument("--steps", type=int, default=20000)
    ap.add_argument("--batch", type=int, default=32)
    ap.add_argument("--lr", type=float, default=1e-3)
    ap.add_argument("--seed", type=int, default=50000)
    ap.add_argument("--pictures-per-frame", type=int, default=2, help="1: the encode only; 2: source and encode")
    ap.add_argument("--frame-every", type=int, default=1, help="steps per new frame pair")
    ap.add_argument("--val-frames", type=int, default=100)
    ap.add_argument("--budget", type=float, default=0.025)
    ap.add_argument("--coverage", type=float, default=0.995)
    ap.add_argument("--out", default=os.path.join(HERE, "proposal_net.npy"))
    ap.add_argument("--time-limit", type=float, default=1e9, help="seconds of training before stopping early")
    args = ap.parse_args()

    import numpy as np
    import torch

    import es_b200
    import es_synth_gpu

    torch.cuda.set_device(0)
    module = es_b200.Module()
    lab = Labeller(torch, es_b200, module)
    net = es_b200.ProposalNet(seed=args.seed)
    rng = np.random.default_rng(args.seed)
    tx0, ty0 = lab.grid[0][:2]
    x = torch.zeros(args.batch, 2, FEAT, FEAT, device="cuda")
    y = torch.zeros(args.batch, CROP_TILES, CROP_TILES, device="cuda")
    xy = torch.zeros(args.batch, 2, dtype=torch.int32, device="cuda")
    curve = []
    t0 = time.time()
    pics = []
    step = 0
    frame = 0
    while step < args.steps and time.time() - t0 < args.time_limit:
        if step % args.frame_every == 0 or not pics:
            src, enc, _ = es_synth_gpu.frame_pair(torch, frame, seed=args.seed)
            frame += 1
            pics = []
            for slot, plane in enumerate([enc] if args.pictures_per_frame == 1 else [src, enc]):
                _, m0, _, words = lab.run(plane, slot)
                pics.append((words, lab.labels(m0), m0.cpu().numpy()))
        # crops: tile positions of 4 x 4 blocks, preferring blocks with some c-value mass
        origins = []
        labels = []
        for i in range(args.batch):
            wcopy, lbl, m0 = pics[i % len(pics)]
            for _ in range(8):
                cx, cy = int(rng.integers(0, tx0 - CROP_TILES + 1)), int(rng.integers(0, ty0 - CROP_TILES + 1))
                if m0[cy:cy + CROP_TILES, cx:cx + CROP_TILES].sum() > 0 or rng.random() < 0.25:
                    break
            origins.append((i % len(pics), TILE * cx - 16, TILE * cy - 16))
            labels.append(lbl[cy:cy + CROP_TILES, cx:cx + CROP_TILES])
        y.copy_(torch.stack(labels))
        for pi in range(len(pics)):
            idx = [i for i, o in enumerate(origins) if o[0] == pi]
            if not idx:
                continue
            xy_cpu = torch.tensor([[origins[i][1], origins[i][2]] for i in idx], dtype=torch.int32)
            xy_dev = xy_cpu.cuda()
            out = torch.empty(len(idx), 2, FEAT, FEAT, device="cuda")
            es_b200.proposal_features(pics[pi][0], W, H, xy_dev.data_ptr(), len(idx), FEAT, FEAT, out.data_ptr())
            x[idx] = out
        want = step % 100 == 0 or step == args.steps - 1
        loss, _ = net.train_step(x.data_ptr(), y.data_ptr(), args.batch, FEAT, FEAT, args.lr,
                                 stream=torch.cuda.current_stream().cuda_stream, want_loss=want)
        if want:
            curve.append((step, loss))
            print(f"step {step} loss {loss:.4f} frames {frame} {time.time() - t0:.0f}s", flush=True)
        step += 1
    train_s = time.time() - t0

    # validation: predictions on fresh frames, and the threshold
    pred = torch.zeros(ty0, tx0, device="cuda")
    results = []
    for v in range(args.val_frames):
        src, enc, prm = es_synth_gpu.frame_pair(torch, v, seed=args.seed + 10_000_000)
        for plane in (src, enc):
            score, m0, m1, words = lab.run(plane)
            net.predict(words, W, H, pred.data_ptr())
            results.append((score, m0.cpu().numpy(), m1.cpu().numpy(), pred.cpu().numpy(), lab.labels(m0).cpu().numpy()))
    thresholds = [-10.0] + [float(t) for t in np.linspace(-1.0, 8.0, 181)]
    table = []
    for thr in thresholds:
        deltas, kept, nonempty_n = [], 0, 0
        for score, m0, m1, p, _ in results:
            nonempty = p > -np.inf
            k0, k1 = keep_masks(np, p, thr)
            deltas.append(lab.delta_if_skipped(m0, m1, k0 | ~nonempty, k1))
            kept += int((k0 & nonempty).sum())
            nonempty_n += int(nonempty.sum())
        deltas = np.array(deltas)
        table.append({"threshold": thr, "share_within_budget": float(np.mean(deltas <= args.budget)),
                      "max_delta": float(deltas.max()), "kept_share": kept / max(1, nonempty_n)})
    ok = [t for t in table if t["share_within_budget"] >= args.coverage]
    chosen = max(ok, key=lambda t: t["threshold"]) if ok else table[0]
    params = net.params()
    np.save(args.out, params)
    # label / prediction agreement on the non-empty tiles
    pl = np.concatenate([p[p > -np.inf] for _, _, _, p, _ in results])
    ll = np.concatenate([l[p > -np.inf] for _, _, _, p, l in results])
    r2 = 1.0 - float(np.mean((pl - ll) ** 2) / max(np.var(ll), 1e-12))
    record = {"steps": step, "batch": args.batch, "lr": args.lr, "seed": args.seed, "frames": frame, "train_seconds": train_s,
              "loss_curve": curve, "val_pictures": len(results), "val_r2_nonempty_tiles": r2, "budget": args.budget,
              "coverage": args.coverage, "threshold": chosen["threshold"], "chosen": chosen, "thresholds": table}
    with open(os.path.splitext(args.out)[0] + ".json", "w") as f:
        json.dump(record, f, indent=1)
    print(json.dumps({k: record[k] for k in ("steps", "frames", "train_seconds", "val_r2_nonempty_tiles", "threshold", "chosen")}))
    net.close()
    lab.close()
    module.close()


if __name__ == "__main__":
    main()
