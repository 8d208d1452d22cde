"""The batched step with the learned tile proposal in its limiting settings, where the exact outcome is known: with
every tile proposed, or every tile audited, or the fallback taken, the scores equal the exact batched step's bit for
bit; with no tile proposed or audited, scales 0 and 1 pool nothing while scales 2-4 stay exact. Graph replay (from
frame 14) is covered by running 16 frames."""

import numpy as np
import pytest

import es_b200
import es_synth
from gpu_util import step_to_dev, to_dev

pytestmark = pytest.mark.gpu

SOURCES = [(320, 192, 10, 2), (256, 160, 8, 1)]
FRAMES = 16


def make_step(f, s, w, h, pd, n):
    return es_synth.c2_step(f, w=w, h=h, source=s, n_encodes=n) if pd == 10 else es_synth.c3_step(f, s, w, h, pd)


@pytest.fixture(scope="module")
def steps():
    return [[make_step(f, s, *src) for s, src in enumerate(SOURCES)] for f in range(FRAMES)]


def run(cuda, module, steps, net=None, **opt):
    stream = cuda.cuda.current_stream().cuda_stream
    b = es_b200.Batch(module, SOURCES)
    if net is not None:
        b.set_proposal(net, **opt)
    out = []
    for f in range(FRAMES):
        keep, views = [], []
        for s in range(len(SOURCES)):
            k, sv, ev = step_to_dev(cuda, es_b200, steps[f][s])
            keep.append(k)
            views += [sv] + ev
        b.queue(f, views, stream)
        res = b.collect(f)
        pooled = [b.scale_pooled(p) for p in range(b.n_pictures)]
        stats = [b.proposal_stats(p) for p in range(b.n_pictures)] if net is not None else None
        out.append(([(r.cambi, r.cambi_source) for r in res], pooled, stats))
    assert b.graph_launches() == FRAMES - 14
    b.close()
    return out


@pytest.fixture(scope="module")
def exact(cuda, module, steps):
    return run(cuda, module, steps)


@pytest.fixture(scope="module")
def net(cuda):
    n = es_b200.ProposalNet(seed=2)
    yield n
    n.close()


def test_everything_proposed_is_exact(cuda, module, steps, exact, net):
    got = run(cuda, module, steps, net, threshold=-1e30, audit=(0, 0), tolerance=0.0)
    for (r, p, st), (re, pe, _) in zip(got, exact):
        assert r == re and p == pe
        assert all(s["skipped"] == [0, 0] and s["audited"] == [0, 0] and s["fallback"] == 0 for s in st)


def test_everything_audited_is_exact(cuda, module, steps, exact, net):
    got = run(cuda, module, steps, net, threshold=1e30, audit=(1000, 1000), tolerance=0.0)
    for (r, p, st), (re, pe, _) in zip(got, exact):
        assert r == re and p == pe
        assert all(s["run"] == [0, 0] and s["skipped"] == [0, 0] for s in st)


def test_nothing_proposed_or_audited_pools_only_the_coarse_scales(cuda, module, steps, exact, net):
    got = run(cuda, module, steps, net, threshold=1e30, audit=(0, 0), tolerance=0.0)
    for (r, p, st), (re, pe, _) in zip(got, exact):
        for pic, pic_e in zip(p, pe):
            assert pic[0] == 0.0 and pic[1] == 0.0
            assert pic[2:] == pic_e[2:]
        assert all(s["fallback"] == 0 and s["estimate"] == 0.0 for s in st)


def test_fallback_restores_the_exact_scores(cuda, module, steps, exact, net):
    got = run(cuda, module, steps, net, threshold=1e30, audit=(300, 300), tolerance=0.0)
    fell = 0
    for (r, p, st), (re, pe, _) in zip(got, exact):
        for i, s in enumerate(st):
            if s["fallback"]:
                fell += 1
                assert p[i] == pe[i]
            if s["audited"][0] + s["audited"][1] and s["estimate"] > 0:
                assert s["fallback"] == 1
    assert fell > 0


def test_budget_skips_the_tiles_the_oracle_picks(cuda, module, steps, exact, net):
    """Budget mode with every skip candidate audited: per picture, the scale-0 tiles audited are exactly those whose
    prediction (es_proposal_predict on the same picture's scale-0 words) lies below the oracle's budget threshold, the
    others run, and the scores stay exact (audited tiles run too); the candidates grow with the budget."""
    import proposal as op

    torch = cuda
    stream = torch.cuda.current_stream().cuda_stream
    frames = (0, FRAMES - 1)
    preds = {}
    for f in frames:
        pic = 0
        for s, (w, h, pd, n) in enumerate(SOURCES):
            for plane in [steps[f][s].source] + list(steps[f][s].encodes):
                cam = es_b200.Cambi(module, w, h, pd)
                y = to_dev(torch, plane.y)
                cam.launch(y.data_ptr(), w, stream)
                cam.finish()
                p = torch.empty(((w + 63) // 64) * ((h + 63) // 64), dtype=torch.float32, device="cuda")
                net.predict(cam.scale_words(0), w, h, p.data_ptr(), stream)
                torch.cuda.synchronize()
                window = es_b200.derive_params(w, h).window
                k0 = max(1, min(w * h, int(0.6 * w * h)))
                preds[(f, pic)] = (p.cpu().numpy(), w, h, k0, window)
                cam.close()
                pic += 1
    last = None
    for budget in (1e-9, 1e-6, 1e-4, 1e30):
        got = run(cuda, module, steps, net, threshold=-1e30, audit=(1000, 1000), tolerance=1e30, budget=budget)
        audited = []
        for f in frames:
            (r, p, st), (re, pe, _) = got[f], exact[f]
            assert r == re and p == pe
            for pic, s in enumerate(st):
                pr, w, h, k0, window = preds[(f, pic)]
                t = op.budget_threshold(pr, w, h, k0, window, -1e30, budget)
                finite = pr[pr != -np.inf]
                assert s["audited"][0] == int((finite < t).sum()), (budget, f, pic, s, t)
                assert s["run"][0] == int((finite >= t).sum()), (budget, f, pic, s, t)
                audited.append(s["audited"][0])
        if last is not None:
            assert all(a >= b for a, b in zip(audited, last))
        last = audited
    assert all(s["run"][0] == 0 for s in got[frames[-1]][2])
