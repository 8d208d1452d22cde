"""The trained tile-proposal network (encode-score_b200/proposal_net.npy) on fresh seeded 3840x2160 10-bit frame pairs,
against the exact batched step on the same inputs: |delta CAMBI| <= 0.05 on every picture here (at least 99% is the
bar), fewer tiles computed than the exact step, and -- the ablation -- a He-initialised network at the same
threshold, whose proposals the audit rejects (fallback to every tile) far more often."""

import os

import numpy as np
import pytest

import es_b200

pytestmark = pytest.mark.gpu

HERE = os.path.dirname(os.path.abspath(__file__))
NET = os.path.join(HERE, "..", "encode-score_b200", "proposal_net.npy")


@pytest.mark.skipif(not os.path.exists(NET), reason="no trained network committed")
def test_trained_proposal_keeps_cambi_and_computes_fewer_tiles(cuda, module):
    import eval_proposal

    net, meta = eval_proposal.load_net(es_b200)
    frames = 24
    rows, timing = eval_proposal.run(cuda, es_b200, module, frames, 77_000_000, net, meta["threshold"])
    trained = eval_proposal.summarize(rows, timing)
    raw = es_b200.ProposalNet(seed=12345)
    rows_u, timing_u = eval_proposal.run(cuda, es_b200, module, frames, 77_000_000, raw, meta["threshold"])
    untrained = eval_proposal.summarize(rows_u, timing_u)
    net.close()
    raw.close()
    # accuracy: the audit and fallback keep every picture within the tolerance
    assert trained["share_within_0.05"] == 1.0, trained
    assert untrained["share_within_0.05"] >= 0.99, untrained
    # gain: the trained network runs a smaller share of the tiles than the exact step (1.0)
    assert trained["tiles_run_share"] < 1.0, trained
    # ablation: without training the audit finds the skipped tiles matter and falls back far more often
    assert untrained["fallback_rate"] > 0.1 and trained["fallback_rate"] < 0.5 * untrained["fallback_rate"], (trained, untrained)
