"""Whole frame steps at the configured sizes against the CPU oracle: the reference's per-frame queue and collect
(src/main.cpp:518-643), at the picture sizes its own parity runs use (tests/test_native.py:83-130).

* 3840x2160 10-bit, one source and three encodes (blur 0.8/1.5/2.5, de-grain, requantised rectangles) through es_batch,
  with the autotuned c-value tile rows of that size and, from frame 14, the step replayed from a CUDA graph.
* 1920x1080 8-bit, one source and one encode (8-bit planar frames, anti-dithered to 10 bits for CAMBI) through
  es_frame.

Compared with the oracle on every frame: CAMBI of the source and of every encode, PSNR and color (bit for bit); the
window figures of every encode and, from frame 12, its lasting-texture figures (bit for bit); the structure windows;
and at the end the segment accumulators (histograms bit for bit, sums within 1e-12 relative: a different but fixed
order of additions). On frame 0 every computed c-value of every scale of every picture is compared bit for bit too.

The oracle's C calls release the GIL, so they run on a thread pool over the host's cores."""

import os
from concurrent.futures import ThreadPoolExecutor

import numpy as np
import pytest

import es_b200
import es_synth
import oracle
from gpu_util import from_dev, to_dev
from test_gpu_frame import assert_accum_equal

pytestmark = pytest.mark.gpu

FRAMES = 15  # frame 14 is the first step of ring phase 0 replayed from a CUDA graph


def _pool():
    return ThreadPoolExecutor(max_workers=max(2, min(32, os.cpu_count() or 2)))


def _scale_shapes(w, h):
    out = []
    for _ in range(es_b200.SCALES):
        out.append((h, w))
        w, h = (w + 1) >> 1, (h + 1) >> 1
    return out


class OracleSequence:
    """The oracle's side of a sequence of frame steps, planes already at the pipeline depth pd."""

    def __init__(self, steps, pd, pool):
        self.steps, self.pd, self.up = steps, pd, 10 - pd
        h, w = steps[0].source.y.shape
        self.w, self.h = w, h
        self.params = oracle.cambi_params(w, h)
        n_enc = len(steps[0].encodes)
        # CAMBI of every picture of every frame (frame 0 keeps its c-value planes), window figures of every encode
        jobs = {}
        for f, st in enumerate(steps):
            for i, pic in enumerate([st.source] + list(st.encodes)):
                jobs[("cambi", f, i)] = pool.submit(oracle.cambi, pic.y, pd, self.params, f == 0)
            for e, enc in enumerate(st.encodes):
                jobs[("win", f, e)] = pool.submit(oracle.window_stats, st.source.y, enc.y, self.up)
        for f in range(12, len(steps)):
            c = f - 6
            ring = [steps[c + k].source.y for k in range(-6, 7)]
            for e in range(n_enc):
                jobs[("persist", f, e)] = pool.submit(oracle.persist_stats, ring, steps[c].encodes[e].y, self.up)
        self.cambi = {k[1:]: v.result() for k, v in jobs.items() if k[0] == "cambi"}
        self.windows = {k[1:]: v.result()[1] for k, v in jobs.items() if k[0] == "win"}
        self.persist = {k[1:]: v.result()[1] for k, v in jobs.items() if k[0] == "persist"}

    def expect(self, f, e):
        """(CAMBI, source CAMBI, PSNR[3], source color, encode color) of encode e in frame f."""
        st = self.steps[f]
        src, enc = st.source, st.encodes[e]
        w, h, pd = self.w, self.h, self.pd
        sse = [oracle.plane_sse(a, b) for a, b in ((src.y, enc.y), (src.u, enc.u), (src.v, enc.v))]
        psnr = [oracle.psnr(sse[0], w * h, pd), oracle.psnr(sse[1], w * h // 4, pd), oracle.psnr(sse[2], w * h // 4, pd)]
        cs = oracle.color_sums(src.u, src.v, self.up) / (w * h // 4)
        ce = oracle.color_sums(enc.u, enc.v, self.up) / (w * h // 4)
        return self.cambi[(f, 1 + e)].score, self.cambi[(f, 0)].score, psnr, list(cs), list(ce)


def check_frame(orc, f, res, read_windows, want_acc, masks):
    """Compares frame f's per-encode results and figures with the oracle and adds the oracle's into want_acc."""
    n_enc = len(res)
    for e in range(n_enc):
        cam, cam_src, psnr, cs, ce = orc.expect(f, e)
        assert res[e].cambi == cam, f"frame {f} encode {e}: CAMBI {res[e].cambi!r} != {cam!r}"
        assert res[e].cambi_source == cam_src, f"frame {f}: source CAMBI"
        assert list(res[e].psnr) == psnr, f"frame {f} encode {e}: PSNR"
        assert list(res[e].color_source) == cs and list(res[e].color_encode) == ce, f"frame {f} encode {e}: color"
        st32 = orc.windows[(f, e)]
        got_st, got_ps = read_windows(e, f >= 12)
        assert np.array_equal(got_st.view(np.uint32), st32.view(np.uint32)), f"frame {f} encode {e}: window figures"
        a = want_acc[e]
        a.frames += 1
        a.cambi += cam
        a.cambi_source += cam_src
        a.psnr += psnr
        a.color_r += np.array(cs)
        a.color_d += np.array(ce)
        m = oracle.collect_frame(a, st32)
        masks[(e, f)] = m
        assert res[e].structure_windows == int(m.sum()), f"frame {f} encode {e}: structure windows"
        if f >= 12:
            ps32 = orc.persist[(f, e)]
            assert np.array_equal(got_ps.view(np.uint32), ps32.view(np.uint32)), f"frame {f} encode {e}: lasting figures"
            oracle.collect_lasting(a, ps32, masks[(e, f - 6)])


def check_cvalue_planes(torch, planes, result, what):
    for s, (t, want) in enumerate(zip(planes, result.cvalues)):
        got = from_dev(t, np.float32)
        bad = np.flatnonzero(got.view(np.uint32).ravel() != want.view(np.uint32).ravel())
        assert bad.size == 0, f"{what} scale {s}: {bad.size} c-values differ, first at {np.unravel_index(bad[0], want.shape)}"
    return any(float(c.max()) > 0 for c in result.cvalues)


@pytest.fixture(scope="module")
def c2_steps():
    with _pool() as pool:
        return list(pool.map(es_synth.c2_step, range(FRAMES)))


@pytest.fixture(scope="module")
def c1_steps():
    with _pool() as pool:
        return list(pool.map(es_synth.c1_step, range(FRAMES)))


def test_c2_4k10_three_encodes_batched_equals_the_oracle(cuda, module, c2_steps):
    torch = cuda
    w, h, n_enc = 3840, 2160, 3
    with _pool() as pool:
        orc = OracleSequence(c2_steps, 10, pool)
    b = es_b200.Batch(module, [(w, h, 10, n_enc)])
    tuned = es_b200.autotune_table().get((w, h), {"rows": [64] * 5, "cols": [0] * 5})
    assert b.tile_rows[0] == tuned["rows"] and b.tile_cols[0] == tuned["cols"], "the autotuned tile shapes of 4K are in use"
    planes = [[torch.zeros(shape, dtype=torch.float32, device="cuda") for shape in _scale_shapes(w, h)] for _ in range(1 + n_enc)]
    for p in range(1 + n_enc):
        b.set_cvalue_planes(p, [t.data_ptr() for t in planes[p]])
    acc = [es_b200.new_accum() for _ in range(n_enc)]
    want = [oracle.Accum() for _ in range(n_enc)]
    masks = {}
    stream = torch.cuda.current_stream().cuda_stream
    for f, st in enumerate(c2_steps):
        keep, views = es_b200.device_step(torch, st)
        b.queue(f, views, stream)
        res = b.collect(f, acc, acc)
        if f == 0:
            positive = [check_cvalue_planes(torch, planes[p], orc.cambi[(0, p)], f"picture {p}") for p in range(1 + n_enc)]
            assert all(positive[1:]), "every encode has positive c-values (banding is exercised)"
            for p in range(1 + n_enc):
                b.set_cvalue_planes(p, None)
        check_frame(orc, f, res, lambda e, persist: b.read_windows(0, e, persist=persist), want, masks)
        del keep
    assert b.graph_launches() == FRAMES - 14
    b.close()
    for e in range(n_enc):
        assert_accum_equal(acc[e], want[e])
    # the figures above were compared window by window; the seeded grain changes every frame, so few windows keep
    # their texture long enough for the lasting histogram
    assert want[2].cambi > 0 and sum(a.st_r[0] for a in want) > 0


def test_c1_1080p8_one_encode_equals_the_oracle(cuda, module, c1_steps):
    torch = cuda
    w, h = 1920, 1080
    with _pool() as pool:
        orc = OracleSequence(c1_steps, 8, pool)
    # every computed c-value of frame 0 through the kernels es_frame runs (an es_cambi instance per picture)
    for i, pic in enumerate([c1_steps[0].source, c1_steps[0].encodes[0]]):
        cam = es_b200.Cambi(module, w, h, 8)
        planes = [torch.zeros(shape, dtype=torch.float32, device="cuda") for shape in _scale_shapes(w, h)]
        cam.set_cvalue_planes([t.data_ptr() for t in planes])
        d = to_dev(torch, pic.y)
        cam.launch(d.data_ptr(), w, 0)
        assert cam.finish() == orc.cambi[(0, i)].score
        cam.close()
        positive = check_cvalue_planes(torch, planes, orc.cambi[(0, i)], f"1080p picture {i}")
        assert positive or i == 0
    fr = es_b200.Frame(module, w, h, 8, 1)
    acc = [es_b200.new_accum()]
    want = [oracle.Accum()]
    masks = {}
    stream = torch.cuda.current_stream().cuda_stream
    for f, st in enumerate(c1_steps):
        keep, views = [], []
        for pic in (st.source, st.encodes[0]):  # 8-bit planar frames, as a decoder hands them over
            t = [torch.from_numpy(np.ascontiguousarray(a.astype(np.uint8))).cuda() for a in (pic.y, pic.u, pic.v)]
            keep.append(t)
            views.append(es_b200.FrameView(t[0].data_ptr(), t[1].data_ptr(), t[2].data_ptr(), w, w // 2, 0, 1, 0, 8))
        fr.queue(f, views[0], views[1:], stream)
        res = fr.collect(f, acc, acc)
        check_frame(orc, f, res, lambda e, persist: fr.read_windows(e, persist=persist), want, masks)
    fr.close()
    assert_accum_equal(acc[0], want[0])
    assert want[0].cambi > 0 and want[0].st_r[0] > 0
