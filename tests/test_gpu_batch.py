"""The batched frame step (es_batch_*) against one plain es_frame per source: sources of uneven sizes and depths,
scored together with one launch per stage and, from frame 14 on, replayed from CUDA graphs, must give the same
per-frame results, window and lasting-texture figures and segment accumulators as scoring each source alone (which
the frame tests pin to the CPU oracle)."""

import ctypes

import numpy as np
import pytest

import es_b200
import es_synth
from gpu_util import step_to_dev

pytestmark = pytest.mark.gpu

SOURCES = [(160, 96, 8, 1), (192, 128, 10, 2), (128, 80, 10, 1)]
FRAMES = 17


def make_step(f, s, w, h, pd, n):
    if n == 1:
        return es_synth.c3_step(f, s, w, h, pd)
    return es_synth.c2_step(f, w=w, h=h, source=s, n_encodes=n)


def accum_bytes(a):
    return bytes(memoryview(ctypes.string_at(ctypes.addressof(a), ctypes.sizeof(a))))


def run_plain(cuda, module, steps, source_cambi=None):
    stream = cuda.cuda.current_stream().cuda_stream
    out = []
    accs = []
    for s, (w, h, pd, n) in enumerate(SOURCES):
        fr = es_b200.Frame(module, w, h, pd, n)
        acc = [es_b200.new_accum() for _ in range(n)]
        res, wins = [], []
        cached = None
        for f in range(FRAMES):
            keep, sv, ev = step_to_dev(cuda, es_b200, steps[f][s])
            run = source_cambi is None or source_cambi[f][s]
            fr.queue(f, sv, ev, stream, source_cambi=run)
            r = fr.collect(f, acc, acc, cached_source_cambi=None if run else 1.25)
            res.append([(x.cambi, x.cambi_source, tuple(x.psnr), tuple(x.color_source), tuple(x.color_encode), x.texture,
                         x.structure_windows, x.lasting_windows) for x in r])
            wins.append([fr.read_windows(e, persist=f >= 12) for e in range(n)])
        fr.close()
        out.append((res, wins))
        accs.append(acc)
    return out, accs


def run_batch(cuda, module, steps, use_graphs=True, source_cambi=None, tuning=None):
    stream = cuda.cuda.current_stream().cuda_stream
    b = es_b200.Batch(module, SOURCES, use_graphs=use_graphs, tuning=tuning)
    accs = [es_b200.new_accum() for _ in range(b.n_encodes)]
    per_source = [([], []) for _ in SOURCES]
    for f in range(FRAMES):
        keep, views = [], []
        for s in range(len(SOURCES)):
            k, sv, ev = step_to_dev(cuda, es_b200, steps[f][s])
            keep.append(k)
            views += [sv] + ev
        flags = source_cambi[f] if source_cambi is not None else None
        b.queue(f, views, stream, source_cambi=flags)
        r = b.collect(f, accs, accs, cached_source_cambi=[1.25] * len(SOURCES))
        k = 0
        for s, (w, h, pd, n) in enumerate(SOURCES):
            per_source[s][0].append([(x.cambi, x.cambi_source, tuple(x.psnr), tuple(x.color_source), tuple(x.color_encode),
                                      x.texture, x.structure_windows, x.lasting_windows) for x in r[k:k + n]])
            per_source[s][1].append([b.read_windows(s, e, persist=f >= 12) for e in range(n)])
            k += n
    graphs = b.graph_launches()
    b.close()
    return per_source, accs, graphs


@pytest.fixture(scope="module")
def steps():
    return [[make_step(f, s, *src) for s, src in enumerate(SOURCES)] for f in range(FRAMES)]


def compare(plain, plain_acc, batch, batch_acc):
    k = 0
    for s, (w, h, pd, n) in enumerate(SOURCES):
        (pres, pwin), (bres, bwin) = plain[s], batch[s]
        for f in range(FRAMES):
            assert bres[f] == pres[f], (s, f, bres[f], pres[f])
            for e in range(n):
                assert np.array_equal(bwin[f][e][0].view(np.uint32), pwin[f][e][0].view(np.uint32)), (s, f, e)
                if f >= 12:
                    assert np.array_equal(bwin[f][e][1].view(np.uint32), pwin[f][e][1].view(np.uint32)), (s, f, e)
        for e in range(n):
            assert accum_bytes(batch_acc[k + e]) == accum_bytes(plain_acc[s][e]), (s, e)
        k += n


def test_batch_equals_one_frame_per_source(cuda, module, steps):
    plain, pacc = run_plain(cuda, module, steps)
    batch, bacc, graphs = run_batch(cuda, module, steps)
    assert graphs == FRAMES - 14
    compare(plain, pacc, batch, bacc)
    # banding is exercised: some encode has a positive CAMBI
    assert max(r[0] for res, _ in plain for fr in res for r in fr) > 0


def test_batch_without_graphs_equals_with(cuda, module, steps):
    l0 = es_b200.launch_count()
    a, aacc, ga = run_batch(cuda, module, steps, use_graphs=False)
    l1 = es_b200.launch_count()
    b, bacc, gb = run_batch(cuda, module, steps, use_graphs=True)
    l2 = es_b200.launch_count()
    assert ga == 0 and gb == FRAMES - 14
    # a replayed step counts its graph's kernel nodes: the same launches as the step launched one by one
    assert l2 - l1 == l1 - l0 > 0
    for s in range(len(SOURCES)):
        assert a[s][0] == b[s][0]
    assert [accum_bytes(x) for x in aacc] == [accum_bytes(x) for x in bacc]


def test_short_cvalue_tiles_equal_the_plain_step(cuda, module, steps):
    """The autotuner's shorter c-value tiles (16 or 32 rows at some scales) give the same results as the plain step."""
    plain, pacc = run_plain(cuda, module, steps)
    tuning = {(w, h): rows for (w, h, _, _), rows in zip(SOURCES, ([16, 32, 16, 32, 16], [32, 16, 64, 16, 32], [16, 16, 32, 64, 16]))}
    batch, bacc, _ = run_batch(cuda, module, steps, tuning=tuning)
    compare(plain, pacc, batch, bacc)


@pytest.mark.parametrize("cols", [[64] * 5, [128] * 5, [64, 128, 64, 128, 128]])
def test_cvalue_tile_widths_equal_the_plain_step(cuda, module, steps, cols):
    """c-value tiles 64 or 128 columns wide, at any scale and with any rows, give the same results as the plain step
    (whose CAMBI uses the library's default widths)."""
    plain, pacc = run_plain(cuda, module, steps)
    rows = ([64, 32, 16, 64, 32], [32, 64, 64, 16, 16], [16, 16, 32, 64, 64])
    tuning = {(w, h): {"rows": r, "cols": cols} for (w, h, _, _), r in zip(SOURCES, rows)}
    batch, bacc, _ = run_batch(cuda, module, steps, tuning=tuning)
    compare(plain, pacc, batch, bacc)


def test_batch_skipped_source_cambi_uses_the_cached_value(cuda, module, steps):
    rng = np.random.default_rng(5)
    flags = [[bool(rng.integers(0, 2)) for _ in SOURCES] for _ in range(FRAMES)]
    flags[15] = [False] * len(SOURCES)  # a graph with every source skipped
    plain, pacc = run_plain(cuda, module, steps, source_cambi=flags)
    batch, bacc, graphs = run_batch(cuda, module, steps, source_cambi=flags)
    compare(plain, pacc, batch, bacc)
    for s in range(len(SOURCES)):
        for f in range(FRAMES):
            if not flags[f][s]:
                assert all(r[1] == 1.25 for r in batch[s][0][f])


def test_batch_rejects_bad_arguments(cuda, module):
    with pytest.raises(es_b200.EsError):
        es_b200.Batch(module, [(15, 16, 10, 1)])
    with pytest.raises(es_b200.EsError):
        es_b200.Batch(module, [(64, 64, 10, 16)] * 4)  # 68 pictures
    with pytest.raises(es_b200.EsError):
        es_b200.Batch(module, [(64, 64, 10, 1)] * 33)  # 33 sources
    with pytest.raises(es_b200.EsError):
        es_b200.Batch(module, [(64, 64, 10, 1)], tuning={(64, 64): {"rows": [64] * 5, "cols": [96] * 5}})
    # the largest batch: 32 sources and 64 pictures
    big = es_b200.Batch(module, [(64, 64, 10, 1)] * 32, use_graphs=False)
    big.close()
    b = es_b200.Batch(module, [(64, 64, 10, 1)])
    with pytest.raises(es_b200.EsError):
        b.collect(0)
    b.close()


def test_host_frames_in_three_slots_equal_the_device_run(cuda, module, steps):
    """Frames in pinned host memory, copied on a second stream into three device slots with frame f + 1's copy queued
    before frame f - 1 is collected (the end-to-end pattern of bench.py), give the same results as
    frames resident on the device: no copy overwrites a slot that a queued step still reads."""
    from gpu_util import planar_view

    torch = cuda
    dev, dacc, _ = run_batch(cuda, module, steps)

    def pinned(a):
        a = np.ascontiguousarray(a)
        return torch.from_numpy(a.view(np.int16) if a.dtype == np.uint16 else a).pin_memory()

    pics = lambda f: [p for s in range(len(SOURCES)) for p in [steps[f][s].source] + list(steps[f][s].encodes)]
    host = [[[pinned(a) for a in (p.y, p.u, p.v)] for p in pics(f)] for f in range(FRAMES)]
    depths = [p.depth for p in pics(0)]
    slots = [[[torch.empty_like(t, device="cuda") for t in pic] for pic in host[0]] for _ in range(3)]
    views = [[planar_view(es_b200, *t, d) for t, d in zip(slot, depths)] for slot in slots]
    stream, copy_stream = torch.cuda.Stream(), torch.cuda.Stream()
    copied = [torch.cuda.Event() for _ in range(3)]
    free = [torch.cuda.Event() for _ in range(3)]

    def copy_in(f):
        s = f % 3
        with torch.cuda.stream(copy_stream):
            copy_stream.wait_event(free[s])
            for dst, src in zip(slots[s], host[f]):
                for d, h in zip(dst, src):
                    d.copy_(h, non_blocking=True)
            copied[s].record(copy_stream)

    b = es_b200.Batch(module, SOURCES)
    accs = [es_b200.new_accum() for _ in range(b.n_encodes)]
    results = {}

    def collect(f):
        r = b.collect(f, accs, accs)
        results[f] = [(x.cambi, x.cambi_source, tuple(x.psnr), tuple(x.color_source), tuple(x.color_encode), x.texture,
                       x.structure_windows, x.lasting_windows) for x in r]

    with torch.cuda.stream(stream):
        copy_in(0)
        for f in range(FRAMES):
            if f + 1 < FRAMES:
                copy_in(f + 1)
            stream.wait_event(copied[f % 3])
            b.queue(f, views[f % 3], stream.cuda_stream)
            free[f % 3].record(stream)
            if f > 0:
                collect(f - 1)
        collect(FRAMES - 1)
    b.close()
    for f in range(FRAMES):
        k = 0
        for s, (w, h, pd, n) in enumerate(SOURCES):
            assert results[f][k:k + n] == dev[s][0][f], (f, s)
            k += n
    assert [accum_bytes(x) for x in accs] == [accum_bytes(x) for x in dacc]
