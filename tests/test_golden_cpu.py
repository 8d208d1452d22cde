"""The CPU oracle against golden outputs of the reference's numpy specification (reference/encode_score/compare.py,
run unmodified by tests/golden/make_golden.py on 14 seeded 160 x 96 frames):

* per-window fine, mid, oriented and shared energies equal the module's float64 run to 1e-12 relative, and its stock
  float32 run within float32 rounding;
* the oracle's per-frame reduction and per-segment figures (src/main.cpp:577-643 restated) match compare_frames with
  the tolerances of the reference's own test (tests/test_native.py:113-130): totals 0.01 points, medians and tenths
  0.1 (0.05-point bins), lasting-texture window count exact, color 1e-3.
"""

import json
import os

import numpy as np
import pytest

import oracle

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "compare_golden.npz")


@pytest.fixture(scope="module")
def golden():
    z = np.load(GOLDEN)
    g = {k: z[k] for k in z.files}
    g["figures"] = json.loads(bytes(g.pop("figures_json")).decode())
    return g


COLUMNS = {"src_fine": 0, "src_mid": 1, "enc_fine": 2, "enc_mid": 3, "cross_fine": 4, "cross_mid": 5, "src_oriented": 6, "enc_oriented": 7}


def test_window_energies_equal_the_module_in_float64(golden):
    o64, _ = oracle.window_stats(golden["src_y"][0], golden["enc_y"][0], 0)
    for name, col in COLUMNS.items():
        want = golden[f"f64_{name}"].ravel()
        np.testing.assert_allclose(o64[:, col], want, rtol=1e-12, atol=1e-9 * np.abs(want).max(), err_msg=name)


def test_window_energies_within_float32_rounding_of_the_stock_module(golden):
    _, o32 = oracle.window_stats(golden["src_y"][0], golden["enc_y"][0], 0)
    for name, col in COLUMNS.items():
        want = golden[f"f32_{name}"].ravel()
        np.testing.assert_allclose(o32[:, col].astype(np.float64), want, rtol=2e-3, atol=1e-3 * np.abs(want).max(), err_msg=name)


def run_oracle(golden):
    n, h, w = golden["src_y"].shape
    acc = oracle.Accum()
    masks = {}
    cn = (w // 2) * (h // 2)
    for f in range(n):
        _, st = oracle.window_stats(golden["src_y"][f], golden["enc_y"][f], 0)
        acc.frames += 1
        acc.color_r += oracle.color_sums(golden["src_u"][f], golden["src_v"][f], 0) / cn
        acc.color_d += oracle.color_sums(golden["enc_u"][f], golden["enc_v"][f], 0) / cn
        masks[f] = oracle.collect_frame(acc, st)
    last = oracle.Accum()
    for c in range(6, n - 6):
        _, ps = oracle.persist_stats([golden["src_y"][c + k] for k in range(-6, 7)], golden["enc_y"][c], 0)
        oracle.collect_lasting(last, ps, masks[c])
    return oracle.parts_json(acc), last


def test_segment_figures_match_compare_frames(golden):
    parts, last = run_oracle(golden)
    fig = golden["figures"]["whole"]
    keys = ("fine", "mid", "oriented")
    for region, tol in (("all", 0.01), ("structure", 0.01), ("median", 0.1), ("worst_tenth", 0.1)):
        for i, k in enumerate(keys):
            assert parts["amount"][region][i] == pytest.approx(fig[f"regions.{region}.{k}"], abs=tol), (region, k)
        for i, k in enumerate(keys[:2]):
            assert parts["matching"][region][i] == pytest.approx(fig[f"matching.{region}.{k}"], abs=tol), (region, k)
    for i, k in enumerate(("cb", "cr", "strength")):
        assert parts["color_source"][i] == pytest.approx(fig[f"color_ref.{k}"], abs=1e-3)
        assert parts["color_encode"][i] == pytest.approx(fig[f"color_dist.{k}"], abs=1e-3)
    lasting = golden["figures"]["lasting"]
    assert last.lasting.n == int(lasting["windows"]) > 0
    assert 100.0 * last.mine / last.own == pytest.approx(lasting["total"], abs=0.01)
    assert last.lasting.quantile(0.5) == pytest.approx(lasting["median"], abs=0.1)


# ---- CAMBI against the reference's own GPU implementation ---------------------------------------------------------
# tests/golden/make_cambi_golden.py ran the reference's src/kernels.cu and src/cambi.cpp (compiled unmodified) on four
# seeded pictures and saved every scale's picture, mask and c-values, the sums and counts of positive c-values, and
# the score of its Cambi class.

CAMBI_GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "cambi_ref_golden.npz")


@pytest.fixture(scope="module")
def cambi_golden():
    z = np.load(CAMBI_GOLDEN)
    g = {k: z[k] for k in z.files}
    return g, json.loads(bytes(g.pop("meta_json")).decode())


def oracle_params(d):
    p = oracle.CambiParams()
    for k, v in d.items():
        if isinstance(v, list):
            getattr(p, k)[:] = v
        else:
            setattr(p, k, v)
    return p


@pytest.mark.parametrize("case", ["banded10", "banded8", "blocks10", "grainy10"])
def test_oracle_cambi_equals_the_reference_kernels(cambi_golden, case):
    g, meta = cambi_golden
    m = meta[case]
    img = g[f"{case}_input"]
    got = oracle.cambi(img, m["depth"], oracle_params(m["params"]), keep=True)
    for s in range(oracle.SCALES):
        assert np.array_equal(got.images[s], g[f"{case}_image{s}"]), f"scale {s} picture"
        assert np.array_equal(got.masks[s], g[f"{case}_mask{s}"]), f"scale {s} mask"
        assert np.array_equal(got.cvalues[s].view(np.uint32), g[f"{case}_cvalues{s}"].view(np.uint32)), f"scale {s} c-values"
    assert got.counts == [int(c) for c in g[f"{case}_counts"]]
    np.testing.assert_allclose(np.array(got.sums_fx) / 2.0 ** 24, g[f"{case}_sums"], rtol=1e-12)
    # the reference's Cambi class with its own derived parameters
    score = oracle.cambi(img, m["depth"], oracle_params(m["class_params"])).score
    assert score == pytest.approx(m["class_score"], rel=1e-12, abs=1e-12)
