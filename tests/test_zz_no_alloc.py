"""es_cambi_score_noalloc, the CAMBI entry point that allocates no device memory (for callers that must not, such as
plugins whose host application owns the device memory budget): through the C ABI, two calls in a row on different
pictures give exactly the scores of the allocating entry point (es_cambi_create / launch / finish), which the other
CAMBI tests hold bit-equal to the CPU oracle; the same holds when the calls alternate between the primary CUDA context
and one made with the driver API's cuCtxCreate (as a host application such as FFmpeg makes its own); a picture larger
than the fixed scratch array is refused.

Collected last on purpose, so that a run stopping at the first failure has already run every other test; it also
passes alone in a fresh process."""

import ctypes

import numpy as np
import pytest

import es_b200
from gpu_util import from_dev, to_dev
from test_gpu_cambi import banded

pytestmark = pytest.mark.gpu


def allocating_score(torch, module, img, depth):
    h, w = img.shape
    cam = es_b200.Cambi(module, w, h, depth)
    d = to_dev(torch, img)
    cam.launch(d.data_ptr(), w, 0)
    s = cam.finish()
    cam.close()
    return s


def test_no_alloc_entry_point_matches_the_allocating_one(cuda, module):
    torch = cuda
    pictures = [(banded(1920, 1080, 31, lo=80, hi=200, step=2), 10), (banded(1280, 720, 32, lo=20, hi=60, step=1, depth=8), 8)]
    stream = torch.cuda.Stream()
    out = torch.zeros(2, dtype=torch.float64, device="cuda")
    dev = [to_dev(torch, img) for img, _ in pictures]
    torch.cuda.synchronize()
    # two calls in a row on one stream, then read both results
    for i, ((img, depth), d) in enumerate(zip(pictures, dev)):
        h, w = img.shape
        es_b200.cambi_score_noalloc(d.data_ptr(), w, w, h, depth, out.data_ptr() + 8 * i, stream.cuda_stream)
    stream.synchronize()
    got = from_dev(out, np.float64)
    want = [allocating_score(torch, module, img, depth) for img, depth in pictures]
    assert list(got) == want
    assert want[0] > 0 and want[1] > 0


def test_no_alloc_refuses_pictures_beyond_its_scratch(cuda, module):
    torch = cuda
    d = torch.zeros((2160, 3840), dtype=torch.int16, device="cuda")
    out = torch.zeros(1, dtype=torch.float64, device="cuda")
    with pytest.raises(es_b200.EsError) as e:
        es_b200.cambi_score_noalloc(d.data_ptr(), 3840, 3840, 2160, 10, out.data_ptr(), 0)
    assert e.value.status == es_b200.ES_ERR_INVALID
    assert "scratch" in str(e.value)


def _driver():
    cu = ctypes.CDLL("libcuda.so.1")

    def ok(status, what):
        assert status == 0, f"{what}: CUresult {status}"

    return cu, ok


def test_no_alloc_in_a_created_context_matches_the_primary_one(cuda, module):
    """Primary context, then a cuCtxCreate context on the same device, then the primary one again: each call finds the
    scratch array in the context it runs in, and all three scores equal the allocating entry point's."""
    torch = cuda
    img = banded(1280, 720, 32, lo=80, hi=200, step=2)
    h, w = img.shape
    want = allocating_score(torch, module, img, 10)
    assert want > 0

    def primary_score():
        d = to_dev(torch, img)
        out = torch.zeros(1, dtype=torch.float64, device="cuda")
        torch.cuda.synchronize()
        es_b200.cambi_score_noalloc(d.data_ptr(), w, w, h, 10, out.data_ptr(), 0)
        torch.cuda.synchronize()
        return float(from_dev(out, np.float64)[0])

    assert primary_score() == want
    cu, ok = _driver()
    dev = ctypes.c_int()
    ok(cu.cuDeviceGet(ctypes.byref(dev), torch.cuda.current_device()), "cuDeviceGet")
    ctx = ctypes.c_void_p()
    ok(cu.cuCtxCreate_v2(ctypes.byref(ctx), 0, dev), "cuCtxCreate")  # now current on this thread
    got = []
    try:
        plane = np.ascontiguousarray(img, dtype=np.uint16)
        d_img, d_score = ctypes.c_uint64(), ctypes.c_uint64()
        ok(cu.cuMemAlloc_v2(ctypes.byref(d_img), ctypes.c_size_t(plane.nbytes)), "cuMemAlloc")
        ok(cu.cuMemAlloc_v2(ctypes.byref(d_score), ctypes.c_size_t(8)), "cuMemAlloc")
        ok(cu.cuMemcpyHtoD_v2(d_img, plane.ctypes.data_as(ctypes.c_void_p), ctypes.c_size_t(plane.nbytes)), "upload")
        for _ in range(2):
            es_b200.cambi_score_noalloc(d_img.value, w, w, h, 10, d_score.value, 0)
            ok(cu.cuCtxSynchronize(), "cuCtxSynchronize")
            s = ctypes.c_double()
            ok(cu.cuMemcpyDtoH_v2(ctypes.byref(s), d_score, ctypes.c_size_t(8)), "download")
            got.append(s.value)
        ok(cu.cuMemFree_v2(d_img), "cuMemFree")
        ok(cu.cuMemFree_v2(d_score), "cuMemFree")
    finally:
        ok(cu.cuCtxDestroy_v2(ctx), "cuCtxDestroy")  # pops it: the primary context is current again
    assert got == [want, want]
    assert primary_score() == want
