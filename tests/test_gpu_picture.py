"""The VMAF picture feed (es_to_pictures: the reference's to_picture, src/kernels.cu:537-545, as src/main.cpp:506-512
uses it) against the reference's own kernel and a numpy restatement, bit for bit: 8-bit pictures (the low byte of
each value) and 16-bit ones, widths that are and are not multiples of 8, pitches that do and do not allow vector
stores; no byte outside a picture's rows is written. And es_frame_luma / es_batch_luma hand over the unpacked luma
planes the reference feeds to libvmaf: they equal the oracle's frame_planes."""

import numpy as np
import pytest

import es_b200
import es_synth
import oracle
from gpu_util import from_dev, to_dev

pytestmark = pytest.mark.gpu

SENTINEL = 0xA5

CASES = [(1920, 1080, 1, 1920), (1920, 1080, 2, 4096), (333, 17, 1, 341), (333, 17, 2, 670), (64, 9, 1, 77), (640, 360, 2, 1282)]


def want_picture(src, pitch, bytes_):
    h, w = src.shape
    out = np.full(pitch * h, SENTINEL, np.uint8).reshape(h, pitch)
    if bytes_ == 1:
        out[:, :w] = (src & 0xFF).astype(np.uint8)
    else:
        out[:, : 2 * w] = src.astype("<u2").view(np.uint8).reshape(h, 2 * w)
    return out


def test_pictures_equal_numpy_and_the_reference(cuda, ref):
    torch = cuda
    rng = np.random.default_rng(11)
    srcs, dsts, copies = [], [], []
    for w, h, b, pitch in CASES:
        src = rng.integers(0, 1024, (h, w), dtype=np.uint16)
        d_src = to_dev(torch, src)
        d_dst = torch.full((h * pitch + 16,), SENTINEL, dtype=torch.uint8, device="cuda")
        srcs.append((src, d_src))
        dsts.append(d_dst)
        copies.append((d_src.data_ptr(), d_dst.data_ptr() + (1 if b == 1 and w % 8 else 0), w, h, pitch, b))
    es_b200.to_pictures(copies, torch.cuda.current_stream().cuda_stream)
    torch.cuda.synchronize()
    for (w, h, b, pitch), (src, d_src), d_dst, c in zip(CASES, srcs, dsts, copies):
        off = c[1] - d_dst.data_ptr()
        got = from_dev(d_dst, np.uint8)
        want = want_picture(src, pitch, b)
        assert np.array_equal(got[off:off + h * pitch].reshape(h, pitch), want), (w, h, b, pitch)
        assert (got[:off] == SENTINEL).all() and (got[off + h * pitch:] == SENTINEL).all()
        r_dst = torch.full((h * pitch,), SENTINEL, dtype=torch.uint8, device="cuda")
        ref.to_picture(d_src.data_ptr(), w, h, r_dst.data_ptr(), pitch, b)
        assert np.array_equal(from_dev(r_dst, np.uint8).reshape(h, pitch), got[off:off + h * pitch].reshape(h, pitch))


def test_frame_and_batch_luma_are_the_unpacked_planes(cuda, module):
    torch = cuda
    w, h = 192, 128
    steps = [es_synth.c2_step(f, w=w, h=h, n_encodes=2) for f in range(9)]
    fr = es_b200.Frame(module, w, h, 10, 2)
    b = es_b200.Batch(module, [(w, h, 10, 2)])
    acc = [es_b200.new_accum() for _ in range(2)]
    stream = torch.cuda.current_stream().cuda_stream
    keep = []
    for f, st in enumerate(steps):
        k, views = es_b200.device_step(torch, st)
        keep.append(k)
        fr.queue(f, views[0], views[1:], stream)
        fr.collect(f, acc, acc)
        b.queue(f, views, stream)
        b.collect(f)
    torch.cuda.synchronize()
    # 9 frames queued: the source's ring (14) still holds every frame, the encodes' (7) frames 2 .. 8
    for f in (1, 2, 8):
        for p, pic in enumerate([steps[f].source] + list(steps[f].encodes)):
            if p > 0 and f < 2:
                for get in (fr.luma, b.luma):
                    with pytest.raises(es_b200.EsError):
                        get(p, f)
                continue
            Y, _, _ = oracle.frame_planes(pic.y, pic.u, pic.v, 0, 0, 10, 0, 0, 10, w, h)
            for addr in (fr.luma(p, f), b.luma(p, f)):
                t = torch.zeros((h, w), dtype=torch.int16, device="cuda")
                es_b200.to_pictures([(addr, t.data_ptr(), w, h, 2 * w, 2)], stream)
                torch.cuda.synchronize()
                assert np.array_equal(from_dev(t, np.uint16), Y), (f, p)
    with pytest.raises(es_b200.EsError):
        fr.luma(0, 9)  # not queued yet
    fr.close()
    b.close()
