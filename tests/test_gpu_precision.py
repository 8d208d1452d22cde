"""Texture window energies on larger windows (es_windows_*) against the FP64 oracle (oracle/precision.py): the integer
summed-area tables give every figure exactly (bit-equal doubles); compensated FP32 stays within 1e-5 relative; plain
FP32 is reported by its error, which the compensation must not exceed. Windows of 16, 32 and 64 pixels, 10- and 8-bit."""

import numpy as np
import pytest

import es_b200
import es_synth
import precision
from gpu_util import from_dev, to_dev, zeros_dev

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("w,h,depth", [(224, 160, 10), (200, 130, 8)])
def test_window_energies_in_three_arithmetics(cuda, module, w, h, depth):
    step = es_synth.c4_step(0, w=w, h=h) if depth == 10 else es_synth.c1_step(0, w=w, h=h)
    yr, yd = step.source.y, step.encodes[0].y
    up = 10 - depth
    win = es_b200.Windows(w, h)
    r, d = to_dev(cuda, yr), to_dev(cuda, yd)
    win.compute(r.data_ptr(), d.data_ptr(), up)
    for window in (16, 32, 64):
        want = precision.window_figures(yr, yd, up, window)
        n = want.shape[0]
        outs = []
        for mode in range(3):
            o = zeros_dev(cuda, (max(n, 1), 8), np.float64)
            win.figures(window, mode, o.data_ptr())
            outs.append(from_dev(o, np.float64)[:n])
        assert np.array_equal(outs[0], want), window
        scale = np.maximum(np.abs(want), 1e-3 * np.abs(want).max(axis=0, keepdims=True))
        rel_c = np.abs(outs[1] - want) / scale
        rel_p = np.abs(outs[2] - want) / scale
        assert rel_c.max() <= 1e-5, (window, rel_c.max())
        assert rel_c.max() <= rel_p.max() + 1e-12
    win.close()
