"""The reference's own calling pattern (src/main.cpp: Kernels::load, Cambi(k, w, h, depth), launch, finish) compiled
against include/gpu.hpp and include/cambi.hpp, in a driver-API context that is not the primary one: the scores equal
the CPU oracle's and those of the C ABI called from Python."""

import os
import subprocess

import numpy as np
import pytest

import oracle
from test_gpu_cambi import banded

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
PKG = os.path.join(ROOT, "encode-score_b200")
BIN = os.path.join(PKG, "_build", "dropin")


@pytest.mark.parametrize("w,h,depth", [(640, 360, 10), (1280, 720, 8)])
def test_cpp_dropin_matches_oracle(cuda, tmp_path, w, h, depth):
    if not os.path.exists(BIN):
        subprocess.run(["make", "-s", "-C", PKG, "dropin"], check=True)
    img = banded(w, h, 21, lo=20 if depth == 8 else 80, hi=60 if depth == 8 else 200, step=1, depth=depth)
    path = tmp_path / "plane.u16"
    img.astype("<u2").tofile(path)
    out = subprocess.run([BIN, str(path), str(w), str(h), str(depth)], capture_output=True, text=True, timeout=120)
    assert out.returncode == 0, out.stderr
    scores = [float(x) for x in out.stdout.split()]
    want = oracle.cambi(img, depth).score
    assert scores == [want, want]
    assert want > 0
