"""TEST INFRASTRUCTURE: ctypes bindings of oracle/_ref/libref.so, the reference's own GPU implementation (its
src/kernels.cu, src/cambi.cpp and src/gpu.cpp compiled unmodified, driven by oracle/ref_shim.cpp).

Used only by tests and measurement scripts, as the GPU-side checker of the product's kernels.
"""

from __future__ import annotations

import ctypes
import os

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "_ref", "libref.so")


class RefGpu:
    def __init__(self, lib: ctypes.CDLL):
        self.lib = lib
        P, I, U64 = ctypes.c_void_p, ctypes.c_int, ctypes.c_uint64
        lib.ref_error.restype = ctypes.c_char_p
        lib.ref_kernels.restype = P
        lib.ref_cambi_create.restype = P
        lib.ref_cambi_create.argtypes = [P, I, I, I]
        lib.ref_cambi_launch.argtypes = [P, U64, I, U64]
        lib.ref_cambi_finish.argtypes = [P, ctypes.POINTER(ctypes.c_double)]
        lib.ref_cambi_destroy.argtypes = [P]
        lib.ref_cambi_steps.argtypes = [P, U64, I, I, I, I, ctypes.POINTER(I), ctypes.POINTER(U64), ctypes.POINTER(U64), ctypes.POINTER(U64), U64, U64]
        lib.ref_frame_planes.argtypes = [P, P, I, I, I, U64, U64, U64, I, I]
        lib.ref_window_stats.argtypes = [P, U64, U64, I, I, I, U64, U64, U64]
        lib.ref_persist_stats.argtypes = [P, U64, U64, I, U64, I, I, U64]
        lib.ref_plane_sse.argtypes = [P, U64, U64, U64, U64]
        lib.ref_color_sums.argtypes = [P, U64, U64, U64, I, U64]
        lib.ref_tiny_luma.argtypes = [P, P, I, I, I, I, U64]
        lib.ref_to_picture.argtypes = [P, U64, I, I, U64, I, I]
        self._check(lib.ref_init())
        self.k = lib.ref_kernels()
        if not self.k:
            raise RuntimeError("reference kernels: " + lib.ref_error().decode())

    def _check(self, r: int) -> None:
        if r:
            raise RuntimeError("reference: " + self.lib.ref_error().decode())

    def cambi_score(self, img: int, w: int, h: int, depth: int, pitch: int | None = None) -> float:
        c = self.lib.ref_cambi_create(self.k, w, h, depth)
        if not c:
            raise RuntimeError("reference Cambi: " + self.lib.ref_error().decode())
        try:
            self._check(self.lib.ref_cambi_launch(c, img, pitch or w, 0))
            s = ctypes.c_double()
            self._check(self.lib.ref_cambi_finish(c, ctypes.byref(s)))
            return s.value
        finally:
            self.lib.ref_cambi_destroy(c)

    def cambi_steps(self, img: int, pitch: int, w: int, h: int, depth: int, params: dict, images: list, masks: list, cvalues: list,
                    scratch: int, sums: int) -> None:
        p = [params["pad"], params["band_base"], params["band_size"], params["vlt"], *params["tvi"], *params["weight"], params["mask_index"]]
        arr = (ctypes.c_int * 13)(*p)
        u = lambda xs: (ctypes.c_uint64 * 5)(*xs)  # noqa: E731
        self._check(self.lib.ref_cambi_steps(self.k, img, pitch, w, h, depth, arr, u(images), u(masks), u(cvalues), scratch, sums))

    def frame_planes(self, view, x0, y0, pd, y16, u, v, w, h):
        self._check(self.lib.ref_frame_planes(self.k, ctypes.byref(view), x0, y0, pd, y16, u, v, w, h))

    def window_stats(self, yr, yd, up, w, h, mid_r, mid_d, out):
        self._check(self.lib.ref_window_stats(self.k, yr, yd, up, w, h, mid_r, mid_d, out))

    def persist_stats(self, ring, plane, centre, mid_d, w, h, out):
        self._check(self.lib.ref_persist_stats(self.k, ring, plane, centre, mid_d, w, h, out))

    def plane_sse(self, a, b, n, sse):
        self._check(self.lib.ref_plane_sse(self.k, a, b, n, sse))

    def color_sums(self, u, v, n, up, sums):
        self._check(self.lib.ref_color_sums(self.k, u, v, n, up, sums))

    def tiny_luma(self, view, x0: int, y0: int, w: int, h: int, out: int) -> None:
        """The reference's thumbnail of one frame (view: an es_frame_view-layout structure) into 2304 device floats."""
        self._check(self.lib.ref_tiny_luma(self.k, ctypes.byref(view), x0, y0, w, h, out))

    def to_picture(self, src: int, w: int, h: int, dst: int, pitch: int, bytes_: int) -> None:
        """The reference's VMAF picture feed of one plane."""
        self._check(self.lib.ref_to_picture(self.k, src, w, h, dst, pitch, bytes_))


_ref = None


def load() -> RefGpu | None:
    """The reference on the current CUDA device, or None when libref.so was not built."""
    global _ref
    if _ref is None and os.path.exists(LIB_PATH):
        _ref = RefGpu(ctypes.CDLL(LIB_PATH))
    return _ref
