"""CAMBI on the GPU through the C ABI against the CPU oracle: every scale's picture and mask, every c-value, the exact
sums, the pooled values and the score bit for bit; the launch / finish contract of src/cambi.hpp:15-20."""

import numpy as np
import pytest

import es_b200
import oracle
from gpu_util import from_dev, to_dev, zeros_dev

pytestmark = pytest.mark.gpu


def banded(w, h, seed, lo=80, hi=200, step=1, grain=0.0, depth=10):
    rng = np.random.default_rng(seed)
    yy, xx = np.mgrid[0:h, 0:w]
    a = rng.uniform(0, 2 * np.pi)
    g = (np.cos(a) * xx / w + np.sin(a) * yy / h)
    g = (g - g.min()) / max(np.ptp(g), 1e-9)
    v = lo + (hi - lo) * g + (rng.normal(0, grain, (h, w)) if grain else 0)
    v = np.round(v / step) * step
    top = 255 if depth == 8 else 1023
    return np.clip(v, 0, top).astype(np.uint16)


def blocks(w, h, seed, lo=90, hi=170, size=6):
    rng = np.random.default_rng(seed)
    b = rng.integers(lo, hi, ((h + size - 1) // size, (w + size - 1) // size))
    return np.kron(b, np.ones((size, size), np.int64))[:h, :w].astype(np.uint16)


def stripes(w, h, v0=120, period=10):
    xx = np.arange(w)[None, :].repeat(h, 0)
    return (v0 + ((xx // period) % 2)).astype(np.uint16)


def plateaus(w, h, size=4, seed=11):
    """size x size plateaus of 10-bit values 60 .. 559 (a seeded permutation, block (bx, by) takes entry bx + 16 by
    mod 500): the 16 x 16 plateaus of an aligned 64 x 64 tile all differ, so with a window of 65 a tile has more than
    255 codes whose c-values are needed, more than a byte of ranks can hold."""
    perm = np.random.default_rng(seed).permutation(500) + 60
    by, bx = np.mgrid[0:(h + size - 1) // size, 0:(w + size - 1) // size]
    b = perm[(bx + 16 * by) % 500]
    return np.kron(b, np.ones((size, size), np.int64))[:h, :w].astype(np.uint16)


def test_plateaus_hold_more_than_255_codes_in_one_tile():
    assert len(np.unique(plateaus(320, 256)[64:128, 64:128])) > 255


CASES = [
    # (name, image, depth, params override)
    ("banded-1080-like", lambda: banded(320, 180, 1, step=2), 10, {"window": 33}),
    ("banded-odd", lambda: banded(203, 131, 2, step=3, grain=0.3), 10, {"window": 17}),
    ("blocks-multipass", lambda: blocks(256, 160, 3), 10, {"window": 33}),
    ("stripes-topk", lambda: stripes(192, 96), 10, {"window": 21, "topk": 0.2}),
    ("noise", lambda: np.random.default_rng(5).integers(64, 400, (90, 150)).astype(np.uint16), 10, None),
    ("flat", lambda: np.full((64, 96), 300, np.uint16), 10, None),
    ("8bit-banded", lambda: banded(240, 136, 6, lo=20, hi=60, step=1, depth=8), 8, {"window": 25}),
    ("tiny", lambda: banded(7, 5, 7), 10, None),
    ("window65", lambda: banded(400, 260, 8, step=2), 10, {"window": 65}),
    ("derived", lambda: banded(640, 360, 9, step=1, grain=0.2), 10, None),
    ("plateaus-many-ranks", lambda: plateaus(320, 256), 10, {"window": 65}),
]


def params_for(img, over):
    h, w = img.shape
    p = es_b200.derive_params(w, h)
    if over:
        if "window" in over:
            p.window = over["window"]
            p.pad = p.window // 2
        if "topk" in over:
            p.topk = over["topk"]
    return p


def oracle_params(p):
    q = oracle.CambiParams()
    for k, v in p.as_dict().items():
        if isinstance(v, list):
            getattr(q, k)[:] = v
        else:
            setattr(q, k, v)
    return q


@pytest.mark.parametrize("name,make,depth,over", CASES, ids=[c[0] for c in CASES])
def test_cambi_matches_oracle_bit_for_bit(cuda, module, name, make, depth, over):
    torch = cuda
    img = make()
    h, w = img.shape
    p = params_for(img, over)
    cam = es_b200.Cambi(module, w, h, depth, p)
    sizes = oracle.scale_sizes(w, h)
    planes = [zeros_dev(torch, (sh, sw), np.float32) for sw, sh in sizes]
    cam.set_cvalue_planes([t.data_ptr() for t in planes])
    dimg = to_dev(torch, img)
    cam.launch(dimg.data_ptr(), w, torch.cuda.current_stream().cuda_stream)
    score = cam.finish()
    want = oracle.cambi(img, depth, oracle_params(p), keep=True)
    for s in range(oracle.SCALES):
        image, mask = cam.read_scale(s)
        assert np.array_equal(image, want.images[s]), f"scale {s} picture"
        assert np.array_equal(mask, want.masks[s]), f"scale {s} mask"
        got = from_dev(planes[s], np.float32)
        assert np.array_equal(got.view(np.uint32), want.cvalues[s].view(np.uint32)), f"scale {s} c-values"
    pooled, sums, counts = cam.scale_stats()
    assert sums == want.sums_fx and counts == want.counts
    assert pooled == want.pooled
    assert score == want.score
    cam.close()


def test_cambi_without_cvalue_planes_gives_the_same_score(cuda, module):
    torch = cuda
    img = banded(300, 200, 11, step=2)
    p = params_for(img, {"window": 33})
    cam = es_b200.Cambi(module, 300, 200, 10, p)
    dimg = to_dev(torch, img)
    scores = []
    for _ in range(3):
        cam.launch(dimg.data_ptr(), 300, 0)
        scores.append(cam.finish())
    assert scores[0] == scores[1] == scores[2] == oracle.cambi(img, 10, oracle_params(p)).score
    cam.close()


def test_pitched_plane(cuda, module):
    torch = cuda
    img = banded(130, 70, 12, step=2)
    padded = np.zeros((70, 160), np.uint16)
    padded[:, :130] = img
    p = params_for(img, {"window": 15})
    cam = es_b200.Cambi(module, 130, 70, 10, p)
    d = to_dev(torch, padded)
    cam.launch(d.data_ptr(), 160, 0)
    assert cam.finish() == oracle.cambi(img, 10, oracle_params(p)).score
    cam.close()


def test_launch_finish_contract(cuda, module):
    torch = cuda
    img = banded(64, 64, 13)
    cam = es_b200.Cambi(module, 64, 64, 10)
    with pytest.raises(es_b200.EsError) as e:
        cam.finish()
    assert e.value.status == es_b200.ES_ERR_STATE
    d = to_dev(torch, img)
    cam.launch(d.data_ptr(), 64, 0)
    with pytest.raises(es_b200.EsError) as e:
        cam.launch(d.data_ptr(), 64, 0)
    assert e.value.status == es_b200.ES_ERR_STATE
    cam.finish()
    with pytest.raises(es_b200.EsError) as e:
        cam.launch(d.data_ptr(), 32, 0)
    assert e.value.status == es_b200.ES_ERR_INVALID
    cam.close()


def test_bad_sizes_are_refused(cuda, module):
    with pytest.raises(es_b200.EsError):
        es_b200.Cambi(module, 1, 10, 10)
    with pytest.raises(es_b200.EsError):
        es_b200.Cambi(module, 10, 10, 12)
    p = es_b200.derive_params(100, 100)
    p.window, p.pad = 131, 65
    with pytest.raises(es_b200.EsError):
        es_b200.Cambi(module, 100, 100, 10, p)
