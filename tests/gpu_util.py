"""Helpers for the GPU tests: numpy arrays to and from CUDA memory (held by torch tensors) and frame views."""

from __future__ import annotations

import numpy as np


def to_dev(torch, a: np.ndarray):
    """A CUDA tensor holding the bytes of `a` (uint16 travels as int16, uint8 as uint8)."""
    a = np.ascontiguousarray(a)
    if a.dtype == np.uint16:
        return torch.from_numpy(a.view(np.int16)).cuda()
    return torch.from_numpy(a).cuda()


def from_dev(t, dtype) -> np.ndarray:
    return t.cpu().numpy().view(dtype)


def zeros_dev(torch, shape, dtype):
    tdt = {np.uint16: torch.int16, np.uint8: torch.uint8, np.float32: torch.float32, np.float64: torch.float64, np.uint64: torch.int64,
           np.int32: torch.int32}[dtype]
    return torch.zeros(shape, dtype=tdt, device="cuda")


def planar_view(es_b200, y, u, v, depth: int):
    """es_frame_view of planar device planes (torch tensors of uint16 bits or uint8)."""
    b = y.element_size()
    return es_b200.FrameView(y.data_ptr(), u.data_ptr(), v.data_ptr(), y.stride(0) * b, u.stride(0) * b, 0, b, 0, depth)


def step_to_dev(torch, es_b200, step):
    """Device planes and views of a synthetic step (source and encodes as planar 16-bit frames)."""
    keep = []
    views = []
    for pic in [step.source] + list(step.encodes):
        t = [to_dev(torch, p) for p in (pic.y, pic.u, pic.v)]
        keep.append(t)
        views.append(planar_view(es_b200, *t, pic.depth))
    return keep, views[0], views[1:]
