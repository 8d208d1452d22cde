#!/usr/bin/env python3
"""A run of 4K10 frame steps for profilers: one source and three encodes (es_synth c2, two distinct steps
alternating), scored by es_batch with or without the learned proposal and without CUDA graphs, so each kernel is its
own launch. Usage: profile_step.py [frames] [--plain] (default 14 frames, learned proposal on)."""

import os
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, HERE)


def main() -> None:
    import torch

    import es_b200
    import es_synth
    import eval_proposal

    frames = int(sys.argv[1]) if len(sys.argv) > 1 and sys.argv[1].isdigit() else 14
    torch.cuda.set_device(0)
    m = es_b200.Module()
    devs = [es_b200.device_step(torch, es_synth.c2_step(f)) for f in range(2)]
    b = es_b200.Batch(m, [(3840, 2160, 10, 3)], use_graphs=False)
    net = None
    if "--plain" not in sys.argv:
        net, meta = eval_proposal.load_net(es_b200)
        b.set_proposal(net, threshold=meta["threshold"])
    acc = [es_b200.new_accum() for _ in range(3)]
    s = torch.cuda.current_stream().cuda_stream
    res = []
    for f in range(frames):
        b.queue(f, devs[f % 2][1], s)
        res = b.collect(f, acc, acc)
    print("CAMBI of the last step's encodes:", [round(r.cambi, 6) for r in res])
    b.close()
    if net:
        net.close()
    m.close()


if __name__ == "__main__":
    main()
