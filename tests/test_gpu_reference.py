"""The product against the reference's own GPU implementation (its kernels and class Cambi compiled from its sources
into oracle/_ref/), on the same inputs and the same CAMBI parameters:

* CAMBI: every scale's picture, mask and c-value bit for bit, and the score within the reference's own summation
  noise (it adds doubles in atomic order);
* PSNR squared errors and color value sums exactly; the color strength within FP32 rounding;
* window and lasting-texture figures within the reference's FP32 rounding, which the product does not share (it is
  exact), measured against the FP64 oracle.
"""

import numpy as np
import pytest

import es_b200
import es_synth
import oracle
from gpu_util import from_dev, to_dev, zeros_dev
from test_gpu_cambi import CASES, oracle_params, params_for

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("name,make,depth,over", [c for c in CASES if c[0] != "tiny"], ids=[c[0] for c in CASES if c[0] != "tiny"])
def test_cambi_steps_match_the_reference_kernels(cuda, module, ref, name, make, depth, over):
    torch = cuda
    img = make()
    h, w = img.shape
    p = params_for(img, over)
    if p.window > 65:
        pytest.skip("the reference's reciprocal table stops at window 65")
    sizes = oracle.scale_sizes(w, h)
    images = [zeros_dev(torch, (sh, sw), np.uint16) for sw, sh in sizes]
    masks = [zeros_dev(torch, (sh, sw), np.uint8) for sw, sh in sizes]
    cvals = [zeros_dev(torch, (sh, sw), np.float32) for sw, sh in sizes]
    scratch = zeros_dev(torch, (h, w), np.uint16)
    sums = zeros_dev(torch, (10,), np.float64)
    dimg = to_dev(torch, img)
    ref.cambi_steps(dimg.data_ptr(), w, w, h, depth, p.as_dict(), [t.data_ptr() for t in images], [t.data_ptr() for t in masks],
                    [t.data_ptr() for t in cvals], scratch.data_ptr(), sums.data_ptr())
    cam = es_b200.Cambi(module, w, h, depth, p)
    planes = [zeros_dev(torch, (sh, sw), np.float32) for sw, sh in sizes]
    cam.set_cvalue_planes([t.data_ptr() for t in planes])
    cam.launch(dimg.data_ptr(), w, 0)
    cam.finish()
    for s in range(oracle.SCALES):
        image, mask = cam.read_scale(s)
        assert np.array_equal(image, from_dev(images[s], np.uint16)), f"scale {s} picture"
        assert np.array_equal(mask, from_dev(masks[s], np.uint8)), f"scale {s} mask"
        assert np.array_equal(from_dev(planes[s], np.float32).view(np.uint32), from_dev(cvals[s], np.float32).view(np.uint32)), f"scale {s} c-values"
    ref_sums = from_dev(sums, np.float64)
    ref_counts = ref_sums[5:].view(np.uint64)
    _, fx, counts = cam.scale_stats()
    assert list(ref_counts) == counts
    assert np.allclose(ref_sums[:5], np.array(fx) / 2.0 ** 24, rtol=1e-12, atol=0)
    cam.close()


@pytest.mark.parametrize("w,h,depth", [(1920, 1080, 10), (1280, 720, 8), (640, 360, 10)])
def test_cambi_score_matches_the_reference_class(cuda, module, ref, w, h, depth):
    torch = cuda
    step = es_synth.c1_step(0, w=w, h=h) if depth == 8 else es_synth.c2_step(0, w=w, h=h, n_encodes=3)
    for pic in [step.source] + step.encodes:
        d = to_dev(torch, pic.y)
        want = ref.cambi_score(d.data_ptr(), w, h, depth)
        cam = es_b200.Cambi(module, w, h, depth)
        cam.launch(d.data_ptr(), w, 0)
        got = cam.finish()
        cam.close()
        assert abs(got - want) <= 1e-9 * max(1.0, abs(want)), (got, want)


def test_sums_match_the_reference_kernels(cuda, ref):
    torch = cuda
    step = es_synth.c2_step(3, w=320, h=192, n_encodes=1)
    a, b = to_dev(torch, step.source.y), to_dev(torch, step.encodes[0].y)
    s = zeros_dev(torch, (3,), np.float64)
    ref.plane_sse(a.data_ptr(), b.data_ptr(), 320 * 192, s.data_ptr())
    assert int(from_dev(s, np.uint64)[0]) == oracle.plane_sse(step.source.y, step.encodes[0].y)
    u, v = to_dev(torch, step.source.u), to_dev(torch, step.source.v)
    ref.color_sums(u.data_ptr(), v.data_ptr(), u.numel(), 0, s.data_ptr())
    got = from_dev(s, np.float64)
    want = oracle.color_sums(step.source.u, step.source.v, 0)
    assert got[0] == want[0] and got[1] == want[1]
    assert abs(got[2] - want[2]) <= 1e-6 * want[2]


def test_window_figures_against_the_reference_and_fp64(cuda, ref):
    """The reference's FP32 window figures and the product's exact ones, each against the FP64 oracle."""
    torch = cuda
    w, h = 640, 368
    step = es_synth.c2_step(1, w=w, h=h, n_encodes=1)
    yr, yd = to_dev(torch, step.source.y), to_dev(torch, step.encodes[0].y)
    ww, wh = w // 16, h // 16
    mid_r, mid_d = zeros_dev(torch, (h, w), np.float32), zeros_dev(torch, (h, w), np.float32)
    out = zeros_dev(torch, (ww * wh, 8), np.float32)
    ref.window_stats(yr.data_ptr(), yd.data_ptr(), 0, w, h, mid_r.data_ptr(), mid_d.data_ptr(), out.data_ptr())
    got_ref = from_dev(out, np.float32).astype(np.float64)
    exact, exact32 = oracle.window_stats(step.source.y, step.encodes[0].y, 0)
    scale = np.abs(exact).max(axis=0) + 1e-30
    ref_err = np.abs(got_ref - exact) / scale
    mine_err = np.abs(exact32.astype(np.float64) - exact) / scale
    # the product rounds each figure once; the reference's FP32 sums differ by more, but stay close
    assert mine_err.max() <= 2 ** -24
    assert ref_err.max() < 1e-3


def test_b200_cambi_is_faster_than_the_reference_kernels(cuda, module, ref):
    """The four 3840x2160 10-bit pictures of a c2 frame step scored by the reference's own Cambi class (its kernels
    compiled unmodified for sm_100a) and by es_cambi, each after a warm-up launch: scores equal to 1e-9 relative, and
    each picture scored faster here (wall time of launch + finish, which is what a caller waits for). Prints both."""
    import time

    import es_synth

    step = es_synth.c2_step(0)
    pics = [step.source] + list(step.encodes)
    stream = cuda.cuda.current_stream().cuda_stream
    rows = []
    c = es_b200.Cambi(module, 3840, 2160, 10)
    for i, pic in enumerate(pics):
        t = to_dev(cuda, pic.y)
        ref.cambi_score(t.data_ptr(), 3840, 2160, 10)  # warm-up
        t0 = time.perf_counter()
        want = ref.cambi_score(t.data_ptr(), 3840, 2160, 10)
        t_ref = time.perf_counter() - t0
        c.launch(t.data_ptr(), 3840, stream)
        c.finish()
        cuda.cuda.synchronize()
        t0 = time.perf_counter()
        c.launch(t.data_ptr(), 3840, stream)
        got = c.finish()
        t_b200 = time.perf_counter() - t0
        rows.append((i, want, got, 1000 * t_ref, 1000 * t_b200))
        assert abs(got - want) <= 1e-9 * max(abs(want), 1e-12), (i, got, want)
    c.close()
    print("\npicture  CAMBI (reference)  CAMBI (b200)  reference ms  b200 ms")
    for r in rows:
        print(f"{r[0]:7d}  {r[1]:17.9f}  {r[2]:12.9f}  {r[3]:12.3f}  {r[4]:7.3f}")
    assert all(r[4] < r[3] for r in rows)


def test_texture_kernels_at_4k_against_the_reference(cuda, module, ref):
    """A 3840x2160 10-bit c2 frame step (1 source, 3 encodes; every frame the same step, so the 13-frame texture
    window holds one picture) through the reference's window_stats, persist_stats, plane_sse and color_sums (compiled
    unmodified for sm_100a, launched as src/main.cpp:540-566 launches them) and through es_frame: the reference's FP32
    window and lasting figures within 1e-3 (of each figure's largest value) of the product's exact ones. Prints each
    group's device time per frame step: the reference's launches bracketed by CUDA events one by one, the product's
    kernels timed one by one by es_kernel_timing."""
    torch = cuda
    W, H, E = 3840, 2160, 3
    step = es_synth.c2_step(0, n_encodes=E)
    keep, views = es_b200.device_step(torch, step)
    stream = torch.cuda.current_stream().cuda_stream
    fr = es_b200.Frame(module, W, H, 10, E)
    acc = [es_b200.new_accum() for _ in range(E)]
    for f in range(16):
        fr.queue(f, views[0], views[1:], stream)
        fr.collect(f, acc, acc)
    es_b200.kernel_timing(True, serial=True)
    for f in range(16, 18):
        fr.queue(f, views[0], views[1:], stream)
        fr.collect(f, acc, acc)
    times = es_b200.kernel_times()
    es_b200.kernel_timing(False)
    mine = [fr.read_windows(e, persist=True) for e in range(E)]
    fr.close()
    ours = {k: times[k][0] / 2 for k in ("window_stats", "persist_stats", "pair_sums", "frame_unpack") if k in times}

    ys = to_dev(torch, step.source.y)
    us, vs = to_dev(torch, step.source.u), to_dev(torch, step.source.v)
    ring = torch.zeros((13, H, W), dtype=torch.float32, device="cuda")
    ws = (W // 16) * (H // 16)
    ev = [torch.cuda.Event(enable_timing=True) for _ in range(2)]
    ref_ms = {"window_stats": 0.0, "persist_stats": 0.0, "plane_sse + color_sums": 0.0}

    def timed(group, call):
        ev[0].record()
        call()
        ev[1].record()
        torch.cuda.synchronize()
        ref_ms[group] += ev[0].elapsed_time(ev[1])

    sse = zeros_dev(torch, (3,), np.float64)
    sums = zeros_dev(torch, (3,), np.float64)
    n = W * H
    timed("plane_sse + color_sums", lambda: ref.color_sums(us.data_ptr(), vs.data_ptr(), n // 4, 0, sums.data_ptr()))
    for e in range(E):
        enc = step.encodes[e]
        ye, ue, ve = to_dev(torch, enc.y), to_dev(torch, enc.u), to_dev(torch, enc.v)
        mid_d = torch.zeros((H, W), dtype=torch.float32, device="cuda")
        st = zeros_dev(torch, (ws, 8), np.float32)
        ps = zeros_dev(torch, (ws, 5), np.float32)
        ref.window_stats(ys.data_ptr(), ye.data_ptr(), 0, W, H, ring[0].data_ptr(), mid_d.data_ptr(), st.data_ptr())  # warm-up
        timed("window_stats", lambda: ref.window_stats(ys.data_ptr(), ye.data_ptr(), 0, W, H, ring[0].data_ptr(),
                                                       mid_d.data_ptr(), st.data_ptr()))
        ring[1:].copy_(ring[0].expand(12, H, W))
        timed("persist_stats", lambda: ref.persist_stats(ring.data_ptr(), n, 6, mid_d.data_ptr(), W, H, ps.data_ptr()))
        for a, b, m in ((ys, ye, n), (us, ue, n // 4), (vs, ve, n // 4)):
            timed("plane_sse + color_sums", lambda: ref.plane_sse(a.data_ptr(), b.data_ptr(), m, sse.data_ptr()))
        timed("plane_sse + color_sums", lambda: ref.color_sums(ue.data_ptr(), ve.data_ptr(), n // 4, 0, sums.data_ptr()))
        for got, want in ((from_dev(st, np.float32), mine[e][0]), (from_dev(ps, np.float32), mine[e][1])):
            scale = np.abs(want.astype(np.float64)).max(axis=0) + 1e-30
            err = np.abs(got.astype(np.float64) - want.astype(np.float64)) / scale
            assert err.max() < 1e-3, (e, err.max(axis=0))
    print("\nper 4K10 frame step (1 source, 3 encodes)   reference ms   b200 ms")
    print(f"window figures                               {ref_ms['window_stats']:12.3f}   {ours.get('window_stats', 0):7.3f}")
    print(f"lasting texture                              {ref_ms['persist_stats']:12.3f}   {ours.get('persist_stats', 0):7.3f}")
    print(f"PSNR squared errors + color                  {ref_ms['plane_sse + color_sums']:12.3f}   {ours.get('pair_sums', 0):7.3f}")
