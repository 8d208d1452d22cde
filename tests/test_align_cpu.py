"""The offset search's oracle (src/kernels.cu:502-520, src/main.cpp:336-353) on known answers, and the C ABI's argument
checks of es_thumbnails / es_find_offset, which run before any device work."""

import ctypes

import numpy as np
import pytest

import align
import es_b200


def test_thumbnail_known_answers():
    y = np.full((72, 128), 700, np.uint16)
    assert np.all(align.thumbnail(y, 10, 0, 0, 128, 72) == 700)
    assert np.all(align.thumbnail((y // 4).astype(np.uint8), 8, 0, 0, 128, 72) == 175 * 4)
    # a ramp in x: cell tx of a 256-wide crop at x0 = 8 holds columns 8 + 4 tx .. 8 + 4 tx + 3, mean 8 + 4 tx + 1.5
    ramp = np.tile(np.arange(300, dtype=np.uint16), (80, 1))
    t = align.thumbnail(ramp, 10, 8, 4, 256, 72)
    assert np.array_equal(t, np.tile(np.float32(9.5) + 4 * np.arange(64, dtype=np.float32), (36, 1)))
    # uneven cells: w = 100 gives cells of 1 or 2 columns (tx w / 64), each the mean of its own columns
    t = align.thumbnail(ramp, 10, 0, 0, 100, 36)
    for tx in range(64):
        xa, xb = tx * 100 // 64, (tx + 1) * 100 // 64
        assert t[0, tx] == np.float32(np.arange(xa, xb).sum()) / np.float32(xb - xa)
    # a crop narrower than 64 columns leaves cells without pixels: NaN, as 0 / 0 in the reference
    t = align.thumbnail(ramp, 10, 0, 0, 40, 36)
    assert np.isnan(t[0, 0]) and not np.isnan(t[0, 1])


def moving(frames, seed=0, h=36, w=64):
    """Thumbnail-sized pictures of a pattern that moves from frame to frame, at 10-bit levels."""
    rng = np.random.default_rng(seed)
    yy, xx = np.mgrid[0:h, 0:w].astype(np.float32)
    out = []
    for t in range(frames):
        out.append(512 + 200 * np.sin(0.2 * xx + 0.35 * t) * np.cos(0.15 * yy - 0.25 * t) + rng.normal(0, 1, (h, w)))
    return np.array(out, np.float32)


def test_find_offset_finds_the_lag_and_refuses_other_pictures():
    ref = moving(60)
    times = [k / 24.0 for k in range(60)]
    probe = ref[17:17 + 30] + np.random.default_rng(1).normal(0, 2, (30, 36, 64)).astype(np.float32)
    off, lag, best = align.find_offset(ref, times, probe, [0.0] * 30)
    assert lag == 17 and off == times[17] and best < 5
    # the early stop does not change the choice: the first least of the full totals is the same lag
    assert int(np.argmin(align.lag_totals(ref, probe))) == 17
    with pytest.raises(align.NoMatch) as e:
        align.find_offset(ref, times, 1023 - probe, [0.0] * 30)
    assert e.value.best > 16
    with pytest.raises(ValueError):
        align.find_offset(ref, times, probe[:23], [0.0] * 23)
    with pytest.raises(ValueError):
        align.find_offset(ref[:20], times[:20], probe[:24], [0.0] * 24)


def test_abi_checks_arguments_before_the_device():
    L = es_b200.lib()
    times = (ctypes.c_double * 60)(*range(60))
    off, best = ctypes.c_double(), ctypes.c_double()
    st = L.es_find_offset(1, times, 60, 1, times, 23, None, ctypes.byref(off), ctypes.byref(best))
    assert st == es_b200.ES_ERR_INVALID and b"too few frames" in L.es_last_error()
    st = L.es_find_offset(1, times, 20, 1, times, 24, None, ctypes.byref(off), ctypes.byref(best))
    assert st == es_b200.ES_ERR_INVALID
    view = es_b200.FrameView(1, 1, 1, 128, 64, 0, 2, 0, 10)
    views = (es_b200.FrameView * 1)(view)
    assert L.es_thumbnails(views, 1, 0, 0, 0, 36, 1, None) == es_b200.ES_ERR_INVALID  # empty crop
    bad = (es_b200.FrameView * 1)(es_b200.FrameView(1, 1, 1, 128, 64, 0, 2, 0, 9))
    assert L.es_thumbnails(bad, 1, 0, 0, 64, 36, 1, None) == es_b200.ES_ERR_INVALID  # depth 9
    assert L.es_offset_totals(1, 10, 1, 11, 1, None) == es_b200.ES_ERR_INVALID  # more probe than reference frames


def test_c_restatement_of_the_lag_search_equals_the_python_one():
    import oracle

    ref = moving(60, seed=4)
    rng = np.random.default_rng(5)
    for start, probe in ((21, ref[21:21 + 30] + rng.normal(0, 2, (30, 36, 64)).astype(np.float32)), (None, 1023 - ref[5:35])):
        lag, best = oracle.find_offset_lag(ref, probe)
        if start is None:
            with pytest.raises(align.NoMatch) as e:
                align.find_offset(ref, list(range(60)), probe, [0] * 30)
            assert best == e.value.best > 16
        else:
            off, want_lag, want_best = align.find_offset(ref, list(range(60)), probe, [0] * 30)
            assert lag == want_lag == start and best == want_best


def test_ties_between_lags_keep_the_first():
    """A reference whose pictures repeat with period 20: lags 7 and 27 give equal totals, bit for bit, and every
    restatement keeps lag 7 (src/main.cpp:347 replaces the best only on a strictly smaller mean)."""
    import oracle

    base = moving(20, seed=8)
    ref = np.concatenate([base, base, base])  # 60 frames, period 20
    probe = ref[7:7 + 24] + np.random.default_rng(9).normal(0, 2, (24, 36, 64)).astype(np.float32)
    totals = align.lag_totals(ref, probe)
    assert totals[7] == totals[27] and int(np.argmin(totals)) == 7
    off, lag, best = align.find_offset(ref, [k / 25.0 for k in range(60)], probe, [0.0] * 24)
    assert lag == 7 and off == 7 / 25.0
    assert oracle.find_offset_lag(ref, probe) == (7, best)
