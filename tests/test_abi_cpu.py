"""The C-ABI library without a GPU: it loads, exports every function include/es_b200.h declares, fails loudly (no CPU
fallback) when asked for device work, and its host-side logic (parameters, Histogram / Accum / score, PSNR, the
segment JSON) matches the oracle's restatement of src/stats.hpp and src/main.cpp."""

import ctypes
import json
import math
import os
import re

import numpy as np
import pytest

import es_b200
import oracle

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_functions():
    text = open(os.path.join(ROOT, "include", "es_b200.h")).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(es_[a-z0-9_]+)\s*\(", text)))


def test_library_exports_every_declared_function():
    lib = es_b200.lib()
    names = declared_functions()
    assert len(names) >= 25
    for name in names:
        assert hasattr(lib, name), name
    assert set(names) == set(es_b200.SYMBOLS)


def test_version():
    assert es_b200.lib().es_version() == 10000


def test_no_device_fails_loudly():
    try:
        import torch

        if torch.cuda.is_available():
            pytest.skip("a GPU is present")
    except ImportError:
        pass
    with pytest.raises(es_b200.EsError) as e:
        es_b200.Module()
    assert e.value.status in (es_b200.ES_ERR_DEVICE, es_b200.ES_ERR_CUDA)


# the window / pad / mask index the reference derives (src/cambi.cpp:39-40) at the measured resolutions
RESOLUTIONS = [((1280, 720), 21, 10, 19), ((1920, 800), 29, 14, 21), ((1920, 1080), 33, 16, 21), ((3840, 1600), 59, 29, 24),
               ((3840, 2160), 65, 32, 24)]


@pytest.mark.parametrize("size,window,pad,index", RESOLUTIONS)
def test_derived_parameters(size, window, pad, index):
    p = es_b200.derive_params(*size).as_dict()
    assert (p["window"], p["pad"], p["mask_index"]) == (window, pad, index)
    o = oracle.cambi_params(*size).as_dict()
    assert p == o


def test_luminance_thresholds():
    p = es_b200.derive_params(1920, 1080)
    # BT.1886 (300 / 0.01 cd/m2) on 10-bit limited range with a Weber threshold of 0.019: increasing TVI per step size
    assert list(p.tvi) == [182, 309, 436, 563]
    assert p.vlt == 64 and p.band_base == 53 and p.band_size == 511
    assert list(p.weight) == [1, 2, 3, 4] and p.topk == 0.6


def test_psnr_matches_reference_formula():
    lib = es_b200.lib()
    for sse, n, d in [(0, 100, 10), (1, 100, 10), (12345678, 1920 * 1080, 10), (99, 64, 8), (10 ** 12, 4, 8)]:
        assert lib.es_psnr(sse, n, d) == oracle.psnr(sse, n, d)
    assert lib.es_psnr(0, 10, 10) == 72.0


def test_histogram_binning_and_quantile():
    lib = es_b200.lib()
    h = es_b200.Histogram()
    rng = np.random.default_rng(0)
    vals = np.concatenate([rng.normal(80, 30, 500), [-600, 600, 0.025, 0.075, -0.025, 499.975, 12.345]])
    for v in vals:
        lib.es_histogram_add(ctypes.byref(h), float(v))
    o = oracle.Histogram()
    o.add(vals)
    assert np.array_equal(np.array(h.bins), o.bins) and h.n == o.n
    for q in (0.0, 0.1, 0.5, 0.9, 1.0):
        assert lib.es_histogram_quantile(ctypes.byref(h), q) == o.quantile(q)
    assert math.isnan(lib.es_histogram_quantile(ctypes.byref(es_b200.Histogram()), 0.5))


def make_accum(rng, frames, lasting_n):
    a, o = es_b200.new_accum(), oracle.Accum()
    for acc in (a, o):
        acc.frames = frames
    vals = dict(vmaf=rng.uniform(50, 100) * frames, cambi=rng.uniform(0, 10), cambi_source=rng.uniform(0, 3))
    for k, v in vals.items():
        setattr(a, k, v)
        setattr(o, k, v)
    a.vmaf_min = o.vmaf_min = 40.0
    for name, n in (("psnr", 3), ("color_r", 3), ("color_d", 3), ("all_r", 3), ("all_d", 3), ("st_r", 3), ("st_d", 3), ("sh_all_r", 2),
                    ("sh_all_x", 2), ("sh_st_r", 2), ("sh_st_x", 2)):
        v = rng.uniform(1, 1000, n)
        getattr(a, name)[:] = list(v)
        getattr(o, name)[:] = v
    a.own, a.mine = o.own, o.mine = 500.0, 420.0
    for k in range(3):
        p = rng.normal(90, 20, 300)
        o.amount[k].add(p)
        for v in p:
            es_b200.lib().es_histogram_add(ctypes.byref(a.amount[k]), float(v))
    for k in range(2):
        p = rng.normal(70, 25, 300)
        o.matching[k].add(p)
        for v in p:
            es_b200.lib().es_histogram_add(ctypes.byref(a.matching[k]), float(v))
    p = rng.normal(85, 10, lasting_n)
    o.lasting.add(p)
    for v in p:
        es_b200.lib().es_histogram_add(ctypes.byref(a.lasting), float(v))
    return a, o


@pytest.mark.parametrize("lasting_n", [150, 20])
def test_score_and_json_match_oracle(lasting_n):
    rng = np.random.default_rng(lasting_n)
    a, o = make_accum(rng, 24, lasting_n)
    parts = es_b200.accum_score(a)
    want = o.score()
    for k in ("fidelity", "banding", "grain", "score"):
        assert getattr(parts, k) == pytest.approx(want[k], rel=1e-15, abs=1e-12)
    if lasting_n < 100:
        assert math.isnan(parts.texture) and math.isnan(want["texture"])
    else:
        assert parts.texture == want["texture"]
    got = json.loads(es_b200.accum_json(a))
    exp = oracle.parts_json(o)

    def cmp(x, y, path):
        if isinstance(y, dict):
            for k in y:
                cmp(x[k], y[k], path + "." + k)
        elif isinstance(y, list):
            for i in range(len(y)):
                cmp(x[i], y[i], f"{path}[{i}]")
        elif isinstance(y, float) and math.isnan(y):
            assert x is None, path
        else:
            assert x == pytest.approx(y, abs=1e-3), path

    cmp(got, exp, "")


def test_merge_adds_everything():
    rng = np.random.default_rng(3)
    a1, o1 = make_accum(rng, 10, 120)
    a2, o2 = make_accum(rng, 7, 130)
    es_b200.lib().es_accum_merge(ctypes.byref(a1), ctypes.byref(a2))
    o1.merge(o2)
    assert a1.frames == 17 and a1.lasting.n == o1.lasting.n
    assert np.array_equal(np.array(a1.amount[1].bins), o1.amount[1].bins)
    assert es_b200.accum_score(a1).score == pytest.approx(o1.score()["score"], rel=1e-14)


def test_score_known_answers():
    """The score arithmetic of reference/encode_score/compare.py:201-209 (tests/test_reference_compare.py:167-189)."""
    def accum(cambi, cambi_source, fine_kept=100.0, lasting=100.0, windows=500, vmaf=100.0):
        a = es_b200.new_accum()
        a.frames = 1
        a.vmaf = vmaf
        a.cambi, a.cambi_source = cambi, cambi_source
        a.all_r[0] = 1.0
        a.all_d[0] = (fine_kept / 100.0) ** 2
        for _ in range(windows):
            es_b200.lib().es_histogram_add(ctypes.byref(a.lasting), lasting)
        return es_b200.accum_score(a)

    p = accum(0.5, 0.5)
    assert (p.fidelity, p.texture, p.banding, p.grain) == (100.0, 100.0, 100.0, 100.0) and p.score == pytest.approx(100.0)
    p = accum(3.0, 0.5)
    assert p.banding == pytest.approx(50.0) and p.score == pytest.approx(100 - 50 * 0.25)
    assert accum(0.0, 0.5).banding == 100.0
    assert accum(0, 0, fine_kept=40.0).grain == pytest.approx(40.0)
    assert accum(0, 0, fine_kept=130.0).grain == pytest.approx(70.0)
    p = accum(0, 0, windows=3, vmaf=90.0)
    assert math.isnan(p.texture)
    assert p.score == pytest.approx((90 * 0.30 + 100 * 0.40) / 0.70)
