"""The window-energy oracle of the precision study (oracle/precision.py) on the CPU, pinned on 16 x 16 windows to the
C oracle of the reference's window figures (es_oracle.c, exact integer numerators rounded once to float)."""

import numpy as np

import es_synth
import oracle
import precision


def test_16_pixel_windows_equal_the_c_oracle():
    step = es_synth.c4_step(0, w=208, h=144)
    yr, yd = step.source.y, step.encodes[0].y
    _, want = oracle.window_stats(yr, yd, 0)
    got = precision.window_figures(yr, yd, 0, 16).astype(np.float32)
    assert np.array_equal(got[:, :6], want[:, :6])
    # oriented: same exact sums, the square root's operand grouped differently: within one float step
    assert np.allclose(got[:, 6:], want[:, 6:], rtol=2 ** -23, atol=0)


def test_larger_windows_sum_the_16_pixel_numerators():
    step = es_synth.c4_step(1, w=256, h=192)
    yr, yd = step.source.y, step.encodes[0].y
    f16 = precision.window_figures(yr, yd, 0, 16)
    f64 = precision.window_figures(yr, yd, 0, 64)
    # the first six figures are sums: a 64-pixel window is the sum of its 16 blocks (exact in int64, one rounding)
    b = f16[:, :6].reshape(12, 16, 6)
    blocks = b.reshape(3, 4, 4, 4, 6).transpose(0, 2, 1, 3, 4).reshape(3 * 4, 16, 6).sum(axis=1)
    assert np.allclose(f64[:, :6], blocks, rtol=1e-12)
