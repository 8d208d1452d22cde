"""Shared test set-up: import paths, the `gpu` marker and fixtures for the CUDA library and the oracles.

Tests marked `gpu` need an sm_100 device and run the product through its C ABI (libes_b200.so); the rest run on the
CPU: the oracle against the reference's golden vectors, the host logic, and the library's exported symbols.
"""

import os
import subprocess
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
PKG = os.path.join(ROOT, "encode-score_b200")
ORACLE = os.path.join(ROOT, "oracle")
GOLDEN = os.path.join(ROOT, "tests", "golden")
for p in (PKG, ORACLE, os.path.join(ROOT, "tests")):
    if p not in sys.path:
        sys.path.insert(0, p)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs an sm_100 (B200) GPU; runs the CUDA path through the C ABI")


def _build_if_missing():
    if not os.path.exists(os.path.join(PKG, "libes_b200.so")):
        subprocess.run(["make", "-s", "-C", PKG], check=True)
    if not os.path.exists(os.path.join(ORACLE, "liboracle.so")):
        subprocess.run(["make", "-s", "-C", ORACLE], check=True)


_build_if_missing()


@pytest.fixture(scope="session")
def cuda():
    """torch with a CUDA device (the tests use it only to hold device buffers and streams)."""
    import torch

    if not torch.cuda.is_available():
        pytest.skip("needs a CUDA device")
    torch.cuda.init()
    return torch


@pytest.fixture(scope="session")
def module(cuda):
    import es_b200

    m = es_b200.Module()
    yield m
    m.close()


@pytest.fixture(scope="session")
def ref(cuda):
    """The reference's own GPU implementation (oracle/_ref/libref.so), or skip when it was not built."""
    import refgpu

    r = refgpu.load()
    if r is None:
        pytest.skip("oracle/_ref/libref.so was not built (it needs the reference's sources at build time)")
    return r
