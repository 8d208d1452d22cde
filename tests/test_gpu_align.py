"""The offset search on the GPU through the C ABI: es_thumbnails bit for bit against the oracle and against the
reference's own tiny_luma kernel (src/kernels.cu:502-520) on the same frames, es_offset_totals bit for bit against the
oracle's in-order double sums, and es_find_offset choosing the oracle's lag (src/main.cpp:336-353) or refusing a
picture that matches nowhere."""

import numpy as np
import pytest

import align
import es_b200
import refgpu
from gpu_util import to_dev
from test_align_cpu import moving

pytestmark = pytest.mark.gpu

FORMATS = {  # (bytes per sample, shift, depth)
    "planar16": (2, 0, 10),
    "planar8": (1, 0, 8),
    "nv12": (1, 0, 8),
    "p010": (2, 6, 10),
}


def frame(rng, w, h, fmt, t=0.0):
    """A luma plane of `fmt` with a pitch wider than the picture; returns (plane as stored, integer samples)."""
    b, shift, depth = FORMATS[fmt]
    yy, xx = np.mgrid[0:h, 0:w].astype(np.float32)
    top = (1 << depth) - 1
    v = 0.5 * top + 0.3 * top * np.sin(0.013 * xx + t) * np.cos(0.021 * yy - 0.5 * t) + rng.normal(0, 0.02 * top, (h, w))
    v = np.clip(np.rint(v), 0, top).astype(np.uint16)
    stored = np.zeros((h, w + 24), np.uint16 if b == 2 else np.uint8)
    stored[:, :w] = (v << shift) if b == 2 else v
    return stored, v


def views_of(cuda, planes, fmt):
    b, shift, depth = FORMATS[fmt]
    keep = [to_dev(cuda, p) for p in planes]
    views = [es_b200.FrameView(t.data_ptr(), t.data_ptr(), t.data_ptr(), p.strides[0], p.strides[0], int(fmt in ("nv12", "p010")),
                               b, shift, depth) for t, p in zip(keep, planes)]
    return keep, views


def same(a, b):
    """Equal as floats, NaN where the other is NaN."""
    return np.array_equal(np.isnan(a), np.isnan(b)) and np.array_equal(a[~np.isnan(a)], b[~np.isnan(b)])


# crops at multiples of 8 columns, at least 512 wide, take the row-band kernel with 16- / 8-byte loads; the others the
# cell-per-block kernel
@pytest.mark.parametrize("fmt,w,h,crop", [("planar16", 3840, 2160, (0, 0, 3840, 2160)), ("planar16", 3840, 2160, (4, 2, 3832, 2156)),
                                          ("planar8", 1920, 1080, (0, 0, 1920, 1080)),
                                          ("nv12", 1280, 720, (6, 4, 1270, 712)), ("p010", 1920, 1088, (0, 4, 1920, 1080)),
                                          ("planar16", 48, 30, (0, 0, 40, 30))])
def test_thumbnails_equal_the_oracle_and_the_reference(cuda, module, fmt, w, h, crop):
    rng = np.random.default_rng(w + h)
    frames = [frame(rng, w, h, fmt, t=0.3 * k) for k in range(3)]
    keep, views = views_of(cuda, [f[0] for f in frames], fmt)
    out = cuda.zeros(len(frames) * 2304, dtype=cuda.float32, device="cuda")
    es_b200.thumbnails(views, *crop, out.data_ptr())
    cuda.cuda.synchronize()
    got = out.cpu().numpy().reshape(-1, 36, 64)
    depth = FORMATS[fmt][2]
    for k, (_, v) in enumerate(frames):
        assert same(got[k], align.thumbnail(v, depth, *crop)), (fmt, k)
    ref = refgpu.load()
    if ref is None:
        pytest.skip("the reference's kernels (oracle/_ref) were not built")
    one = cuda.zeros(2304, dtype=cuda.float32, device="cuda")
    for k, view in enumerate(views):
        ref.tiny_luma(view, *crop, one.data_ptr())
        assert same(got[k], one.cpu().numpy().reshape(36, 64)), (fmt, k, "reference")


def test_thumbnails_of_more_frames_than_one_launch(cuda, module):
    rng = np.random.default_rng(5)
    frames = [frame(rng, 160, 96, "planar16", t=0.1 * k) for k in range(70)]  # two launches: 64 + 6 frames
    keep, views = views_of(cuda, [f[0] for f in frames], "planar16")
    out = cuda.zeros(70 * 2304, dtype=cuda.float32, device="cuda")
    es_b200.thumbnails(views, 0, 0, 160, 96, out.data_ptr())
    got = out.cpu().numpy().reshape(-1, 36, 64)
    for k, (_, v) in enumerate(frames):
        assert np.array_equal(got[k], align.thumbnail(v, 10, 0, 0, 160, 96)), k


def test_offset_totals_equal_the_oracle_bit_for_bit(cuda, module):
    ref = moving(40, seed=2)
    probe = ref[9:9 + 24] + np.random.default_rng(3).normal(0, 3, (24, 36, 64)).astype(np.float32)
    d_ref, d_probe = cuda.from_numpy(ref.ravel()).cuda(), cuda.from_numpy(probe.ravel().copy()).cuda()
    totals = cuda.zeros(40 - 24 + 1, dtype=cuda.float64, device="cuda")
    es_b200.offset_totals(d_ref.data_ptr(), 40, d_probe.data_ptr(), 24, totals.data_ptr())
    got = totals.cpu().numpy()
    assert np.array_equal(got.view(np.uint64), align.lag_totals(ref, probe).view(np.uint64))
    assert int(np.argmin(got)) == 9


def _rounding_case(kind, rng, n_ref, n_probe):
    shape = (n_ref, 36, 64)
    if kind == "tiny_differences":  # full mantissas, differences far below the total's unit, rare large ones
        ref = rng.random(shape, dtype=np.float32)
        probe = ref[5:5 + n_probe] * (np.float32(1) + np.ldexp(rng.integers(-4, 5, (n_probe, 36, 64)), -21).astype(np.float32))
        probe[:, :, ::61] += np.float32(500)
    elif kind == "exact_copy":  # lag 7 is every value zero
        ref = (rng.integers(0, 1024, shape) / 4).astype(np.float32)
        probe = ref[7:7 + n_probe].copy()
    else:  # magnitudes from 2^-40 to 2^40: totals that cross many binades, values far below and far above the unit
        ref = np.ldexp(rng.random(shape), rng.integers(-40, 41, shape)).astype(np.float32)
        probe = np.ldexp(rng.random((n_probe, 36, 64)), rng.integers(-40, 20, (n_probe, 36, 64))).astype(np.float32)
    return ref.astype(np.float32), probe.astype(np.float32)


@pytest.mark.parametrize("kind", ["tiny_differences", "exact_copy", "wide_range"])
@pytest.mark.parametrize("aligned", [True, False])
def test_offset_totals_of_rounding_cases_bit_for_bit(cuda, module, kind, aligned):
    """The lag totals where the in-order double sum rounds (exact halves among the cases), where a lag is all zeros,
    and where the totals cross many binades; with 16-byte aligned arrays and with arrays one float off (scalar
    loads), and a probe of an odd number of frames (the last chunk of each lag only part full)."""
    rng = np.random.default_rng(21)
    n_ref, n_probe = 31, 13
    ref, probe = _rounding_case(kind, rng, n_ref, n_probe)
    off = 0 if aligned else 1
    d_ref = cuda.zeros(ref.size + 4, dtype=cuda.float32, device="cuda")
    d_probe = cuda.zeros(probe.size + 4, dtype=cuda.float32, device="cuda")
    d_ref[off:off + ref.size] = cuda.from_numpy(ref.ravel())
    d_probe[off:off + probe.size] = cuda.from_numpy(probe.ravel())
    lags = n_ref - n_probe + 1
    totals = cuda.zeros(lags, dtype=cuda.float64, device="cuda")
    es_b200.offset_totals(d_ref.data_ptr() + 4 * off, n_ref, d_probe.data_ptr() + 4 * off, n_probe, totals.data_ptr())
    got = totals.cpu().numpy()
    want = align.lag_totals(ref, probe)
    bad = np.flatnonzero(got.view(np.uint64) != want.view(np.uint64))
    assert bad.size == 0, f"{bad.size} lags differ, first {bad[0]}: {got[bad[0]]!r} != {want[bad[0]]!r}"
    if kind == "exact_copy":
        assert got[7] == 0.0 and (np.delete(got, 7) > 0).all()


def test_find_offset_on_thumbnails_of_a_moving_sequence(cuda, module):
    """Source frames 0 .. 59 and an encode that starts 13 frames later (noisier): the thumbnails made on the GPU give
    the oracle's lag and offset; an encode of other pictures is refused."""
    rng = np.random.default_rng(7)
    w, h, n_src, n_enc, start = 320, 180, 60, 30, 13
    src = [frame(rng, w, h, "planar16", t=0.2 * k) for k in range(n_src)]
    enc = []
    for k in range(n_enc):
        stored, v = src[start + k]
        noisy = np.clip(v.astype(np.int32) + rng.integers(-6, 7, v.shape), 0, 1023).astype(np.uint16)
        s = stored.copy()
        s[:, :w] = noisy
        enc.append((s, noisy))
    other = []  # the same motion in negative: a different picture at every lag
    for stored, v in enc:
        s = stored.copy()
        s[:, :w] = 1023 - v
        other.append((s, 1023 - v))
    t_src = [1.0 + k / 25.0 for k in range(n_src)]
    t_enc = [k / 25.0 for k in range(n_enc)]
    thumbs = {}
    keep = []
    for name, fr in (("src", src), ("enc", enc), ("other", other)):
        k, views = views_of(cuda, [f[0] for f in fr], "planar16")
        keep.append(k)
        out = cuda.zeros(len(fr) * 2304, dtype=cuda.float32, device="cuda")
        es_b200.thumbnails(views, 0, 0, w, h, out.data_ptr())
        thumbs[name] = out
    host = {k: v.cpu().numpy().reshape(-1, 36, 64) for k, v in thumbs.items()}
    off, best = es_b200.find_offset(thumbs["src"].data_ptr(), t_src, thumbs["enc"].data_ptr(), t_enc)
    want_off, want_lag, want_best = align.find_offset(host["src"], t_src, host["enc"], t_enc)
    assert want_lag == start and off == want_off == t_src[start] - t_enc[0]
    assert best == want_best and best < 5
    with pytest.raises(es_b200.EsError) as e:
        es_b200.find_offset(thumbs["src"].data_ptr(), t_src, thumbs["other"].data_ptr(), t_enc)
    assert e.value.status == es_b200.ES_ERR_NO_MATCH
    with pytest.raises(align.NoMatch) as o:
        align.find_offset(host["src"], t_src, host["other"], t_enc)
    assert e.value.best_mean == o.value.best > 16


def test_find_offset_keeps_the_first_of_tied_lags(cuda, module):
    """Pictures that repeat with period 20 give lags 7 and 27 equal totals; the first is kept, as in the reference."""
    base = moving(20, seed=8)
    ref = np.concatenate([base, base, base])
    probe = ref[7:7 + 24] + np.random.default_rng(9).normal(0, 2, (24, 36, 64)).astype(np.float32)
    d_ref, d_probe = cuda.from_numpy(ref.ravel()).cuda(), cuda.from_numpy(probe.ravel().copy()).cuda()
    off, best = es_b200.find_offset(d_ref.data_ptr(), [k / 25.0 for k in range(60)], d_probe.data_ptr(), [0.0] * 24)
    want_off, want_lag, want_best = align.find_offset(ref, [k / 25.0 for k in range(60)], probe, [0.0] * 24)
    assert want_lag == 7 and off == want_off and best == want_best
