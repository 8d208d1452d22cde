"""The learned tile proposal's CUDA kernels through the C ABI against the FP64 oracle (oracle/proposal.py): crop
features bit for bit, the training step's loss and gradients (FP32 on the device against FP64, tolerance stated per
check), Adam's update, the fused tensor-core prediction per tile, and the per-tile c-value sums that label the tiles."""

import numpy as np
import pytest

import es_b200
import es_synth
import oracle
import proposal
from gpu_util import from_dev, to_dev, zeros_dev

pytestmark = pytest.mark.gpu


def words_of(cuda, module, y, depth=10):
    """A CAMBI instance run on picture y; returns (instance, scale-0 words as numpy)."""
    h, w = y.shape
    c = es_b200.Cambi(module, w, h, depth)
    t = to_dev(cuda, y)
    c.launch(t.data_ptr(), w, cuda.cuda.current_stream().cuda_stream)
    c.finish()
    img, mask = c.read_scale(0)
    return c, (img.astype(np.uint16) | (mask.astype(np.uint16) << 15)), t


def needs_cvalue(words, p):
    code = (words & 0x7FFF).astype(np.int64) - p.band_base
    ok = ((words & 0x8000) != 0) & (code >= 0) & (code < p.band_size)
    value = code + p.band_base + 4
    need = np.zeros(words.shape, bool)
    for d in range(4):
        need |= (value <= p.tvi[d]) & (value + d + 1 > p.vlt)
    return ok & need


def random_params(seed):
    rng = np.random.default_rng(seed)
    params = proposal.init_params(seed)
    return [(w, (0.05 * rng.normal(size=b.shape)).astype(np.float32)) for w, b in params]


def test_features_match_the_oracle(cuda, module):
    step = es_synth.c2_step(0, w=300, h=200, n_encodes=1)
    c, words, keep = words_of(cuda, module, step.encodes[0].y)
    wd = to_dev(cuda, words)
    xy = np.array([[0, 0], [-16, -16], [100, 40], [290, 190], [-8, 120]], np.int32)
    n, fw, fh = len(xy), 24, 24
    out = zeros_dev(cuda, (n, 2, fh, fw), np.float32)
    es_b200.proposal_features(wd.data_ptr(), 300, 200, to_dev(cuda, xy).data_ptr(), n, fw, fh, out.data_ptr())
    got = from_dev(out, np.float32)
    for i, (x0, y0) in enumerate(xy):
        want = proposal.features_fast(words, int(x0), int(y0), fw, fh).astype(np.float32)
        assert np.array_equal(got[i], want), i
    c.close()


def test_training_step_gradients_match_the_oracle(cuda, module):
    rng = np.random.default_rng(11)
    n, size = 3, 8 + 2 * 16
    x = rng.normal(0, 1, (n, 2, size, size)).astype(np.float32)
    labels = rng.normal(0.5, 0.5, (n, 2, 2)).astype(np.float32)
    params = random_params(5)
    net = es_b200.ProposalNet(proposal.flatten(params))
    xd, ld = to_dev(cuda, x), to_dev(cuda, labels)
    loss, grads = net.train_step(xd.data_ptr(), ld.data_ptr(), n, size, size, 0.0, want_grads=True)
    want_loss, want = proposal.loss_and_grads(x.astype(np.float64), labels.astype(np.float64), params)
    assert abs(loss - want_loss) <= 1e-5 * abs(want_loss)
    want_flat = proposal.flatten([(gw, gb) for gw, gb in want]).astype(np.float64)
    # FP32 sums of ~4000 products against FP64: within 1e-3 of the largest gradient of the same layer
    at = 0
    for (gw, gb) in want:
        for g in (gw, gb):
            seg = slice(at, at + g.size)
            scale = np.abs(want_flat[seg]).max()
            assert np.abs(grads[seg] - want_flat[seg]).max() <= 1e-3 * scale + 1e-9
            at += g.size
    # the Adam step of the device from those gradients equals the oracle's Adam on the same gradients
    loss2, _ = net.train_step(xd.data_ptr(), ld.data_ptr(), n, size, size, 1e-3)
    got = net.params()
    opt = proposal.Adam(params, lr=1e-3)
    new = opt.step(params, proposal.unflatten(grads.astype(np.float64)))
    want_p = proposal.flatten(new)
    assert np.allclose(got, want_p, rtol=0, atol=2e-7)
    net.close()


def test_training_lowers_the_loss_on_the_device(cuda, module):
    rng = np.random.default_rng(3)
    n, size = 8, 8 + 2 * 16
    x = rng.normal(0, 1, (n, 2, size, size)).astype(np.float32)
    labels = np.tanh(x[:, 0, 8:-8:16, 8:-8:16] + 0.5 * x[:, 1, 8:-8:16, 8:-8:16]).astype(np.float32)  # a learnable target
    net = es_b200.ProposalNet(seed=1)
    xd, ld = to_dev(cuda, x), to_dev(cuda, labels)
    first, _ = net.train_step(xd.data_ptr(), ld.data_ptr(), n, size, size, 3e-3)
    for _ in range(150):
        last, _ = net.train_step(xd.data_ptr(), ld.data_ptr(), n, size, size, 3e-3)
    assert last < 0.3 * first
    net.close()


def test_prediction_matches_the_oracle(cuda, module):
    w, h = 330, 200
    step = es_synth.c2_step(1, w=w, h=h, n_encodes=3)
    c, words, keep = words_of(cuda, module, step.encodes[2].y)
    p = oracle.cambi_params(w, h)
    params = random_params(7)
    net = es_b200.ProposalNet(proposal.flatten(params))
    wd = to_dev(cuda, words)
    tx, ty = (w + 63) // 64, (h + 63) // 64
    pred = zeros_dev(cuda, (ty, tx), np.float32)
    net.predict(wd.data_ptr(), w, h, pred.data_ptr())
    got = from_dev(pred, np.float32)
    need = needs_cvalue(words, p)
    errs = []
    for j in range(ty):
        for i in range(tx):
            if not need[64 * j:64 * j + 64, 64 * i:64 * i + 64].any():
                assert got[j, i] == -np.inf, (i, j)
                continue
            f = proposal.features_fast(words, 64 * i - 16, 64 * j - 16, 24, 24)[None]
            z = proposal.forward(f.astype(np.float32).astype(np.float64), params, round_acts=True)[-1]
            want = z[0, 0].mean()
            errs.append(abs(got[j, i] - want))
    assert errs, "no tile needs c-values"
    # bfloat16 activations: an FP32 sum on either side of a rounding tie can move an activation by one bfloat16 step
    assert max(errs) <= 2e-2 and np.median(errs) <= 1e-3, (max(errs), np.median(errs))
    net.close()
    c.close()


def test_tile_masses_sum_the_cvalues_of_each_tile(cuda, module):
    w, h = 260, 150
    step = es_synth.c2_step(2, w=w, h=h, n_encodes=3)
    y = step.encodes[2].y
    n_tiles = es_b200.cambi_tile_count(w, h)
    c = es_b200.Cambi(module, w, h, 10)
    mass = zeros_dev(cuda, (n_tiles,), np.uint64)
    sizes = []
    ww, hh = w, h
    for _ in range(5):
        sizes.append((ww, hh))
        ww, hh = (ww + 1) >> 1, (hh + 1) >> 1
    planes = [zeros_dev(cuda, (sh, sw), np.float32) for sw, sh in sizes]
    c.set_tile_mass(mass.data_ptr())
    c.set_cvalue_planes([t.data_ptr() for t in planes])
    t = to_dev(cuda, y)
    c.launch(t.data_ptr(), w, cuda.cuda.current_stream().cuda_stream)
    c.finish()
    got = from_dev(mass, np.uint64)
    _, sums, _ = c.scale_stats()
    at = 0
    for s, (sw, sh) in enumerate(sizes):
        cv = from_dev(planes[s], np.float32).astype(np.float64)
        nx, ny = (sw + 63) // 64, (sh + 63) // 64
        for j in range(ny):
            for i in range(nx):
                blk = cv[64 * j:64 * j + 64, 64 * i:64 * i + 64]
                assert got[at + j * nx + i] == int(round((blk[blk > 0] * 16777216.0).sum())), (s, i, j)
        assert int(got[at:at + nx * ny].sum()) == sums[s]
        at += nx * ny
    assert at == n_tiles and got.sum() > 0
    c.close()
