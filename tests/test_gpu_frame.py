"""The per-frame measures (src/main.cpp:518-643) on the GPU through the C ABI against the CPU oracle: every window
figure and lasting-texture figure bit for bit, PSNR, color and CAMBI per frame, and the per-segment accumulators."""

import math

import numpy as np
import pytest

import es_b200
import es_synth
import oracle
from gpu_util import to_dev

pytestmark = pytest.mark.gpu


def raw_frame(pic, fmt, x0=0, y0=0, extra=6):
    """A frame holding `pic` at offset (x0, y0) (even) in the given layout, with `extra` pixels of margin right and
    below and row padding, so that reading it needs the crop and the pitch."""
    y, u, v = pic.y, pic.u, pic.v
    h, w = y.shape
    H, W = h + y0 + extra, w + x0 + extra
    Y = np.zeros((H, W + extra), np.uint16)
    Y[y0:y0 + h, x0:x0 + w] = y
    cu, cv = np.zeros((H // 2, W // 2), np.uint16), np.zeros((H // 2, W // 2), np.uint16)
    cu[y0 // 2:y0 // 2 + h // 2, x0 // 2:x0 // 2 + w // 2] = u
    cv[y0 // 2:y0 // 2 + h // 2, x0 // 2:x0 // 2 + w // 2] = v
    if fmt in ("planar16", "planar8"):
        dt = np.uint16 if fmt == "planar16" else np.uint8
        Cu = np.zeros((H // 2, W // 2 + extra), dt)
        Cv = np.zeros_like(Cu)
        Cu[:, : W // 2], Cv[:, : W // 2] = cu, cv
        return dict(y=Y.astype(dt), u=Cu, v=Cv, semi=0, shift=0)
    if fmt == "nv12":
        UV = np.zeros((H // 2, 2 * (W // 2) + extra), np.uint8)
        UV[:, 0:2 * (W // 2):2], UV[:, 1:2 * (W // 2):2] = cu, cv
        return dict(y=Y.astype(np.uint8), u=UV, v=None, semi=1, shift=0)
    if fmt == "p010":
        UV = np.zeros((H // 2, 2 * (W // 2) + extra), np.uint16)
        UV[:, 0:2 * (W // 2):2], UV[:, 1:2 * (W // 2):2] = cu << 6, cv << 6
        return dict(y=Y << 6, u=UV, v=None, semi=1, shift=6)
    raise ValueError(fmt)


class DevFrame:
    def __init__(self, torch, raw, depth):
        self.t = [to_dev(torch, raw["y"]), to_dev(torch, raw["u"])] + ([to_dev(torch, raw["v"])] if raw["v"] is not None else [])
        b = raw["y"].dtype.itemsize
        self.view = es_b200.FrameView(self.t[0].data_ptr(), self.t[1].data_ptr(), self.t[2].data_ptr() if raw["v"] is not None else None,
                                      raw["y"].strides[0], raw["u"].strides[0], raw["semi"], b, raw["shift"], depth)


def oracle_planes(raw, depth, pd, w, h, x0=0, y0=0):
    Y, U, V = oracle.frame_planes(raw["y"], raw["u"], raw["v"], raw["semi"], raw["shift"], depth, x0, y0, pd, w, h)
    return Y, U, V


def run_sequence(torch, module, steps, pd, fmts, crops=None, check_windows=True):
    """Runs `steps` through es_frame and the oracle side by side; returns both accumulators per encode."""
    w, h = steps[0].source.y.shape[1], steps[0].source.y.shape[0]
    n_enc = len(steps[0].encodes)
    crops = crops or [(0, 0)] * (n_enc + 1)
    fr = es_b200.Frame(module, w, h, pd, n_enc)
    acc = [es_b200.new_accum() for _ in range(n_enc)]
    want = [oracle.Accum() for _ in range(n_enc)]
    ring, enc_ring, masks = {}, {}, {}
    up = 10 - pd
    cparams = oracle.cambi_params(w, h)
    stream = torch.cuda.current_stream().cuda_stream
    keep = []
    for f, step in enumerate(steps):
        pics = [step.source] + list(step.encodes)
        raws = [raw_frame(pic, fmts[i], *crops[i]) for i, pic in enumerate(pics)]
        devs = [DevFrame(torch, r, p.depth) for r, p in zip(raws, pics)]
        keep.append(devs)
        fr.queue(f, devs[0].view, [d.view for d in devs[1:]], stream, sx=crops[0][0], sy=crops[0][1],
                 ex=[c[0] for c in crops[1:]], ey=[c[1] for c in crops[1:]])
        res = fr.collect(f, acc, acc)
        # the oracle's figures of this frame
        planes = [oracle_planes(r, p.depth, pd, w, h, *crops[i]) for i, (r, p) in enumerate(zip(raws, pics))]
        ring[f] = planes[0][0]
        src_cambi = oracle.cambi(planes[0][0], pd, cparams).score
        for e in range(n_enc):
            Yd, Ud, Vd = planes[1 + e]
            enc_ring[(e, f)] = Yd
            _, st32 = oracle.window_stats(planes[0][0], Yd, up)
            cam = oracle.cambi(Yd, pd, cparams).score
            assert res[e].cambi == cam, f"frame {f} encode {e} CAMBI"
            assert res[e].cambi_source == src_cambi
            sse = [oracle.plane_sse(planes[0][k], planes[1 + e][k]) for k in range(3)]
            ps = [oracle.psnr(sse[0], w * h, pd), oracle.psnr(sse[1], w * h // 4, pd), oracle.psnr(sse[2], w * h // 4, pd)]
            assert list(res[e].psnr) == ps
            cs = oracle.color_sums(planes[0][1], planes[0][2], up) / (w * h // 4)
            ce = oracle.color_sums(Ud, Vd, up) / (w * h // 4)
            assert list(res[e].color_source) == list(cs) and list(res[e].color_encode) == list(ce)
            a = want[e]
            a.frames += 1
            a.cambi += cam
            a.cambi_source += src_cambi
            a.psnr += ps
            a.color_r += cs
            a.color_d += ce
            m = oracle.collect_frame(a, st32)
            masks[(e, f)] = m
            if check_windows:
                got_st, got_ps = fr.read_windows(e, persist=f >= 12)
                assert np.array_equal(got_st.view(np.uint32), st32.view(np.uint32)), f"frame {f} encode {e} window figures"
            if f >= 12:
                c = f - 6
                _, ps32 = oracle.persist_stats([ring[c + k] for k in range(-6, 7)], enc_ring[(e, c)], up)
                if check_windows:
                    assert np.array_equal(got_ps.view(np.uint32), ps32.view(np.uint32)), f"frame {f} encode {e} lasting figures"
                oracle.collect_lasting(a, ps32, masks[(e, c)])
            assert res[e].structure_windows == int(m.sum())
    fr.close()
    return acc, want


def assert_accum_equal(got, want, rel=1e-12):
    assert got.frames == want.frames
    for name in ("psnr", "color_r", "color_d", "all_r", "all_d", "st_r", "st_d", "sh_all_r", "sh_all_x", "sh_st_r", "sh_st_x"):
        g, w_ = np.array(list(getattr(got, name))), getattr(want, name)
        assert np.allclose(g, w_, rtol=rel, atol=0), name
    for name in ("cambi", "cambi_source", "own", "mine"):
        assert math.isclose(getattr(got, name), getattr(want, name), rel_tol=rel, abs_tol=1e-300), name
    for k in range(3):
        assert np.array_equal(np.array(got.amount[k].bins), want.amount[k].bins) and got.amount[k].n == want.amount[k].n
    for k in range(2):
        assert np.array_equal(np.array(got.matching[k].bins), want.matching[k].bins) and got.matching[k].n == want.matching[k].n
    assert np.array_equal(np.array(got.lasting.bins), want.lasting.bins) and got.lasting.n == want.lasting.n


def test_sequence_10bit_two_encodes(cuda, module):
    steps = [es_synth.c2_step(f, w=160, h=96, n_encodes=2) for f in range(16)]
    acc, want = run_sequence(cuda, module, steps, 10, ["planar16"] * 3)
    for e in range(2):
        assert_accum_equal(acc[e], want[e])
    assert want[0].lasting.n > 0


def test_sequence_8bit_nv12_with_crop(cuda, module):
    steps = [es_synth.c1_step(f, w=128, h=80) for f in range(14)]
    acc, want = run_sequence(cuda, module, steps, 8, ["nv12", "planar8"], crops=[(4, 2), (0, 0)])
    assert_accum_equal(acc[0], want[0])


def test_sequence_mixed_depths_p010(cuda, module):
    # an 8-bit encode in a 10-bit pipeline is shifted up (src/kernels.cu:295-296)
    steps = []
    for f in range(13):
        s = es_synth.c2_step(f, w=96, h=64, n_encodes=1)
        e8 = es_synth.c1_step(f, w=96, h=64).encodes[0]
        s.encodes.append(e8)
        steps.append(s)
    acc, want = run_sequence(cuda, module, steps, 10, ["p010", "planar16", "planar8"])
    for e in range(2):
        assert_accum_equal(acc[e], want[e])


def test_segment_json_matches_oracle(cuda, module):
    steps = [es_synth.c2_step(f, w=128, h=96, n_encodes=1) for f in range(14)]
    acc, want = run_sequence(cuda, module, steps, 10, ["planar16"] * 2, check_windows=False)
    import json

    got = json.loads(es_b200.accum_json(acc[0]))
    exp = oracle.parts_json(want[0])

    def close(a, b, path=""):
        if isinstance(b, dict):
            for k in b:
                close(a[k], b[k], path + "." + k)
        elif isinstance(b, list):
            for i, (x, y) in enumerate(zip(a, b)):
                close(x, y, f"{path}[{i}]")
        elif b is None or (isinstance(b, float) and math.isnan(b)):
            assert a is None, path
        else:
            assert a is not None and abs(a - b) <= 1e-3 + 1e-6 * abs(b), path

    close(got, exp)


def test_frames_must_come_in_order_and_be_collected(cuda, module):
    torch = cuda
    step = es_synth.c2_step(0, w=64, h=48, n_encodes=1)
    fr = es_b200.Frame(module, 64, 48, 10, 1)
    devs = [DevFrame(torch, raw_frame(p, "planar16"), 10) for p in (step.source, step.encodes[0])]
    with pytest.raises(es_b200.EsError):
        fr.queue(1, devs[0].view, [devs[1].view])
    fr.queue(0, devs[0].view, [devs[1].view])
    fr.queue(1, devs[0].view, [devs[1].view])
    with pytest.raises(es_b200.EsError) as e:
        fr.queue(2, devs[0].view, [devs[1].view])
    assert e.value.status == es_b200.ES_ERR_STATE
    fr.collect(0, None, None)
    fr.collect(1, None, None)
    with pytest.raises(es_b200.EsError):
        fr.collect(1, None, None)
    fr.close()


def _striped_step(w, h, seed=11):
    """A source whose right 70 % repeats one 16-pixel column profile (vertical stripes: the same oriented figure in
    every window there, so the 0.8 quantile falls inside a run of equal values) beside faint grain; one blurred
    encode."""
    from scipy import ndimage

    rng = np.random.Generator(np.random.PCG64(seed))
    y = np.tile(rng.integers(200, 800, 16).astype(np.float32), (h, w // 16))
    split = int(0.3 * (w // 16)) * 16
    y[:, :split] = 500 + rng.normal(0, 2, (h, split))
    src = np.clip(np.rint(y), 64, 940)
    enc = np.clip(np.rint(ndimage.gaussian_filter(src, 1.0, mode="nearest")), 64, 940)
    pic = lambda a: es_synth.Picture(a.astype(np.uint16), *(2 * [es_synth._chroma(a.astype(np.uint16))]), 10)
    return es_synth.Step(pic(src), [pic(enc)])


@pytest.mark.parametrize("w,h,kind", [(1920, 1088, "stripes"), (3840, 2160, "synth"), (4096, 2720, "synth"),
                                      (4096, 2720, "stripes")])
def test_structure_threshold_at_large_sizes(cuda, module, w, h, kind):
    """The frame's structure threshold (the exact 0.8 quantile of the source's oriented figures) and mask against the
    oracle's collect on the same window figures, with the figures staged in shared memory (up to 40960 windows) and
    read in place (4096 x 2720: 43520 windows), on distinct figures and on a long run of equal ones."""
    torch = cuda
    step = es_synth.c2_step(0, w=w, h=h, n_encodes=1) if kind == "synth" else _striped_step(w, h)
    fr = es_b200.Frame(module, w, h, 10, 1)
    keep, views = es_b200.device_step(torch, step)
    acc = [es_b200.new_accum()]
    fr.queue(0, views[0], views[1:], torch.cuda.current_stream().cuda_stream)
    res = fr.collect(0, acc, acc)
    st, _ = fr.read_windows(0)
    fr.close()
    o = np.sort(st[:, 6])
    lo = int(0.8 * (o.size - 1))
    if kind == "stripes":  # the premise: the two order statistics that make the quantile are equal
        assert o[lo] == o[lo + 1] and o[lo] > 0
    want = oracle.Accum()
    m = oracle.collect_frame(want, st)
    assert res[0].structure_windows == int(m.sum())
    for k in range(3):
        assert np.array_equal(np.array(acc[0].amount[k].bins), want.amount[k].bins) and acc[0].amount[k].n == want.amount[k].n
    for k in range(2):
        assert np.array_equal(np.array(acc[0].matching[k].bins), want.matching[k].bins)
    for name in ("st_r", "st_d", "sh_st_x"):
        assert np.allclose(np.array(list(getattr(acc[0], name))), getattr(want, name), rtol=1e-12, atol=0), name
