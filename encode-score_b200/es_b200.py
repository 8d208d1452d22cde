"""ctypes binding of libes_b200.so, the C ABI in include/es_b200.h.

The library is built in-tree (``make -C encode-score_b200``). There is no fallback: if the library or a CUDA device
is missing, loading or the first call raises.

Device buffers are passed as integer addresses (``tensor.data_ptr()`` of a CUDA tensor works), streams as integer
handles (``torch.cuda.current_stream().cuda_stream``).
"""

from __future__ import annotations

import ctypes
import os

HERE = os.path.dirname(os.path.abspath(__file__))
# ES_B200_LIB selects another build of the library (another optimisation level, a profiling build)
LIB_PATH = os.environ.get("ES_B200_LIB") or os.path.join(HERE, "libes_b200.so")

ES_OK, ES_ERR_INVALID, ES_ERR_CUDA, ES_ERR_ALLOC, ES_ERR_STATE, ES_ERR_DEVICE, ES_ERR_NO_MATCH = range(7)
THUMB_W, THUMB_H = 64, 36
HIST_BINS = 20001
SCALES = 5

# every symbol include/es_b200.h declares, for the load check
SYMBOLS = (
    "es_last_error", "es_version", "es_launch_count", "es_kernel_timing", "es_kernel_times", "es_module_load", "es_module_unload", "es_module_get", "es_module_launch",
    "es_cambi_create", "es_cambi_create_with", "es_cambi_derive_params", "es_cambi_get_params", "es_cambi_launch",
    "es_cambi_finish", "es_cambi_destroy", "es_cambi_scale_stats", "es_cambi_read_scale", "es_cambi_set_cvalue_planes",
    "es_cambi_score_noalloc", "es_cambi_tile_count", "es_cambi_set_tile_mass", "es_cambi_scale_words",
    "es_proposal_net_create", "es_proposal_net_get", "es_proposal_net_train_step", "es_proposal_features",
    "es_proposal_predict", "es_proposal_net_destroy",
    "es_histogram_add", "es_histogram_quantile", "es_accum_init", "es_accum_merge", "es_accum_score", "es_accum_json",
    "es_psnr", "es_frame_create", "es_frame_queue", "es_frame_collect", "es_frame_read_windows", "es_frame_destroy",
    "es_batch_create", "es_batch_queue", "es_batch_collect", "es_batch_read_windows", "es_batch_scale_pooled",
    "es_batch_set_cvalue_planes", "es_batch_luma", "es_frame_luma", "es_to_pictures",
    "es_windows_create", "es_windows_compute", "es_windows_figures", "es_windows_destroy",
    "es_per_frame_json", "es_cambi_cache_open", "es_cambi_cache_find", "es_cambi_cache_add", "es_cambi_cache_file",
    "es_cambi_cache_close",
    "es_batch_graph_launches", "es_batch_destroy", "es_batch_set_proposal", "es_batch_proposal_stats",
    "es_thumbnails", "es_offset_totals", "es_find_offset",
)


class EsError(RuntimeError):
    def __init__(self, status: int, message: str):
        super().__init__(f"{message} (status {status})")
        self.status = status


class CambiParams(ctypes.Structure):
    _fields_ = [("w", ctypes.c_int), ("h", ctypes.c_int), ("window", ctypes.c_int), ("pad", ctypes.c_int), ("mask_index", ctypes.c_int),
                ("band_base", ctypes.c_int), ("band_size", ctypes.c_int), ("vlt", ctypes.c_int), ("tvi", ctypes.c_int * 4),
                ("weight", ctypes.c_int * 4), ("topk", ctypes.c_double)]

    def as_dict(self) -> dict:
        return {"w": self.w, "h": self.h, "window": self.window, "pad": self.pad, "mask_index": self.mask_index, "band_base": self.band_base,
                "band_size": self.band_size, "vlt": self.vlt, "tvi": list(self.tvi), "weight": list(self.weight), "topk": self.topk}


class FrameView(ctypes.Structure):
    _fields_ = [("y", ctypes.c_void_p), ("u", ctypes.c_void_p), ("v", ctypes.c_void_p), ("ypitch", ctypes.c_int), ("cpitch", ctypes.c_int),
                ("semi", ctypes.c_int), ("bytes", ctypes.c_int), ("shift", ctypes.c_int), ("depth", ctypes.c_int)]


class Histogram(ctypes.Structure):
    _fields_ = [("bins", ctypes.c_uint64 * HIST_BINS), ("n", ctypes.c_uint64)]


class Accum(ctypes.Structure):
    _fields_ = [("frames", ctypes.c_uint64), ("vmaf", ctypes.c_double), ("vmaf_min", ctypes.c_double), ("psnr", ctypes.c_double * 3),
                ("cambi", ctypes.c_double), ("cambi_source", ctypes.c_double), ("color_r", ctypes.c_double * 3), ("color_d", ctypes.c_double * 3),
                ("all_r", ctypes.c_double * 3), ("all_d", ctypes.c_double * 3), ("st_r", ctypes.c_double * 3), ("st_d", ctypes.c_double * 3),
                ("amount", Histogram * 3), ("sh_all_r", ctypes.c_double * 2), ("sh_all_x", ctypes.c_double * 2), ("sh_st_r", ctypes.c_double * 2),
                ("sh_st_x", ctypes.c_double * 2), ("matching", Histogram * 2), ("own", ctypes.c_double), ("mine", ctypes.c_double),
                ("lasting", Histogram)]


class Weights(ctypes.Structure):
    _fields_ = [("fidelity", ctypes.c_double), ("texture", ctypes.c_double), ("banding", ctypes.c_double), ("grain", ctypes.c_double)]


class Parts(ctypes.Structure):
    _fields_ = [("fidelity", ctypes.c_double), ("texture", ctypes.c_double), ("banding", ctypes.c_double), ("grain", ctypes.c_double),
                ("score", ctypes.c_double)]


class FrameResult(ctypes.Structure):
    _fields_ = [("cambi", ctypes.c_double), ("cambi_source", ctypes.c_double), ("psnr", ctypes.c_double * 3),
                ("color_source", ctypes.c_double * 3), ("color_encode", ctypes.c_double * 3), ("texture", ctypes.c_int),
                ("structure_windows", ctypes.c_uint32), ("lasting_windows", ctypes.c_uint32)]


_lib = None


class BatchSource(ctypes.Structure):
    _fields_ = [("w", ctypes.c_int), ("h", ctypes.c_int), ("pd", ctypes.c_int), ("n_encodes", ctypes.c_int),
                ("cv_tile_rows", ctypes.c_int * 5), ("cv_tile_cols", ctypes.c_int * 5)]


class PictureCopy(ctypes.Structure):
    _fields_ = [("src", ctypes.c_uint64), ("dst", ctypes.c_uint64), ("w", ctypes.c_int), ("h", ctypes.c_int),
                ("pitch", ctypes.c_int), ("bytes", ctypes.c_int)]


def to_pictures(copies: list, stream: int = 0) -> None:
    """es_to_pictures: copies [(src, dst, w, h, pitch, bytes), ...] planes into pictures, one launch."""
    arr = (PictureCopy * len(copies))(*[PictureCopy(*c) for c in copies])
    check(lib().es_to_pictures(arr, len(copies), ctypes.c_void_p(stream)))


class ProposalOptions(ctypes.Structure):
    _fields_ = [("threshold", ctypes.c_float), ("audit_permille", ctypes.c_int * 2), ("tolerance", ctypes.c_double),
                ("budget", ctypes.c_double)]


class ProposalStats(ctypes.Structure):
    _fields_ = [("estimate", ctypes.c_float), ("fallback", ctypes.c_int), ("run", ctypes.c_uint32 * 2), ("audited", ctypes.c_uint32 * 2),
                ("skipped", ctypes.c_uint32 * 2)]


class BatchOptions(ctypes.Structure):
    _fields_ = [("use_graphs", ctypes.c_int)]


def lib() -> ctypes.CDLL:
    """The loaded library (raises OSError with the path if it was not built)."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise OSError(f"{LIB_PATH} is missing: build it with `make -C {HERE}`")
        L = ctypes.CDLL(LIB_PATH)
        P, I, U64 = ctypes.c_void_p, ctypes.c_int, ctypes.c_uint64
        L.es_last_error.restype = ctypes.c_char_p
        L.es_launch_count.restype = U64
        L.es_kernel_timing.argtypes = [I]
        L.es_kernel_times.argtypes = [P, P, P, I, ctypes.POINTER(I)]
        L.es_module_load.argtypes = [ctypes.POINTER(P)]
        L.es_module_unload.argtypes = [P]
        L.es_module_get.argtypes = [P, ctypes.c_char_p, ctypes.POINTER(P)]
        L.es_module_launch.argtypes = [P, ctypes.c_uint, ctypes.c_uint, ctypes.POINTER(P), P]
        L.es_cambi_create.argtypes = [P, I, I, I, ctypes.POINTER(P)]
        L.es_cambi_create_with.argtypes = [P, I, I, I, ctypes.POINTER(CambiParams), ctypes.POINTER(P)]
        L.es_cambi_derive_params.argtypes = [I, I, ctypes.POINTER(CambiParams)]
        L.es_cambi_get_params.argtypes = [P, ctypes.POINTER(CambiParams)]
        L.es_cambi_launch.argtypes = [P, U64, I, P]
        L.es_cambi_finish.argtypes = [P, ctypes.POINTER(ctypes.c_double)]
        L.es_cambi_destroy.argtypes = [P]
        L.es_cambi_scale_stats.argtypes = [P, ctypes.POINTER(ctypes.c_double), ctypes.POINTER(U64), ctypes.POINTER(U64)]
        L.es_cambi_read_scale.argtypes = [P, I, P, P]
        L.es_cambi_set_cvalue_planes.argtypes = [P, ctypes.POINTER(P)]
        L.es_cambi_score_noalloc.argtypes = [U64, I, I, I, I, P, P]
        L.es_histogram_add.argtypes = [ctypes.POINTER(Histogram), ctypes.c_double]
        L.es_histogram_quantile.argtypes = [ctypes.POINTER(Histogram), ctypes.c_double]
        L.es_histogram_quantile.restype = ctypes.c_double
        L.es_accum_init.argtypes = [ctypes.POINTER(Accum)]
        L.es_accum_merge.argtypes = [ctypes.POINTER(Accum), ctypes.POINTER(Accum)]
        L.es_accum_score.argtypes = [ctypes.POINTER(Accum), ctypes.POINTER(Weights), ctypes.POINTER(Parts)]
        L.es_accum_json.argtypes = [ctypes.POINTER(Accum), ctypes.c_char_p, ctypes.c_size_t]
        L.es_accum_json.restype = ctypes.c_size_t
        L.es_psnr.argtypes = [U64, U64, I]
        L.es_psnr.restype = ctypes.c_double
        L.es_frame_create.argtypes = [P, I, I, I, I, ctypes.POINTER(P)]
        L.es_frame_queue.argtypes = [P, ctypes.c_long, ctypes.POINTER(FrameView), I, I, I, ctypes.POINTER(FrameView), ctypes.POINTER(I),
                                     ctypes.POINTER(I), P]
        L.es_frame_collect.argtypes = [P, ctypes.c_long, ctypes.POINTER(ctypes.c_double), ctypes.POINTER(ctypes.POINTER(Accum)),
                                       ctypes.POINTER(ctypes.POINTER(Accum)), ctypes.POINTER(FrameResult)]
        L.es_frame_read_windows.argtypes = [P, I, P, P]
        L.es_frame_destroy.argtypes = [P]
        L.es_cambi_tile_count.argtypes = [I, I, ctypes.POINTER(I)]
        L.es_cambi_set_tile_mass.argtypes = [P, P]
        L.es_cambi_scale_words.argtypes = [P, I, ctypes.POINTER(U64)]
        L.es_proposal_net_create.argtypes = [P, U64, ctypes.POINTER(P)]
        L.es_proposal_net_get.argtypes = [P, P]
        L.es_proposal_net_train_step.argtypes = [P, P, P, I, I, I, ctypes.c_float, ctypes.POINTER(ctypes.c_double), P, P]
        L.es_proposal_features.argtypes = [U64, I, I, P, I, I, I, P, P]
        L.es_proposal_predict.argtypes = [P, U64, I, I, P, P]
        L.es_proposal_net_destroy.argtypes = [P]
        L.es_per_frame_json.argtypes = [P, P, P, P, ctypes.c_long, ctypes.c_char_p, ctypes.c_size_t]
        L.es_per_frame_json.restype = ctypes.c_size_t
        L.es_cambi_cache_open.argtypes = [ctypes.c_char_p, I, I, I, I, I, ctypes.c_char_p, ctypes.POINTER(P)]
        L.es_cambi_cache_find.argtypes = [P, ctypes.c_int64, ctypes.POINTER(ctypes.c_double)]
        L.es_cambi_cache_add.argtypes = [P, ctypes.c_int64, ctypes.c_double]
        L.es_cambi_cache_file.argtypes = [P]
        L.es_cambi_cache_file.restype = ctypes.c_char_p
        L.es_cambi_cache_close.argtypes = [P]
        L.es_windows_create.argtypes = [I, I, ctypes.POINTER(P)]
        L.es_windows_compute.argtypes = [P, U64, U64, I, P]
        L.es_windows_figures.argtypes = [P, I, I, P, P]
        L.es_windows_destroy.argtypes = [P]
        L.es_batch_create.argtypes = [P, I, ctypes.POINTER(BatchSource), ctypes.POINTER(BatchOptions), ctypes.POINTER(P)]
        L.es_batch_queue.argtypes = [P, ctypes.c_long, ctypes.POINTER(FrameView), ctypes.POINTER(I), ctypes.POINTER(I), P]
        L.es_batch_collect.argtypes = [P, ctypes.c_long, ctypes.POINTER(ctypes.c_double), ctypes.POINTER(ctypes.POINTER(Accum)),
                                       ctypes.POINTER(ctypes.POINTER(Accum)), ctypes.POINTER(FrameResult)]
        L.es_batch_read_windows.argtypes = [P, I, I, P, P]
        L.es_batch_scale_pooled.argtypes = [P, I, ctypes.POINTER(ctypes.c_double)]
        L.es_batch_set_cvalue_planes.argtypes = [P, I, ctypes.POINTER(P)]
        L.es_batch_luma.argtypes = [P, I, ctypes.c_long, ctypes.POINTER(U64)]
        L.es_frame_luma.argtypes = [P, I, ctypes.c_long, ctypes.POINTER(U64)]
        L.es_to_pictures.argtypes = [ctypes.POINTER(PictureCopy), I, P]
        L.es_batch_graph_launches.argtypes = [P]
        L.es_batch_graph_launches.restype = U64
        L.es_batch_destroy.argtypes = [P]
        L.es_batch_set_proposal.argtypes = [P, P, ctypes.POINTER(ProposalOptions)]
        L.es_batch_proposal_stats.argtypes = [P, I, ctypes.POINTER(ProposalStats)]
        D = ctypes.POINTER(ctypes.c_double)
        L.es_thumbnails.argtypes = [ctypes.POINTER(FrameView), I, I, I, I, I, U64, P]
        L.es_offset_totals.argtypes = [U64, I, U64, I, U64, P]
        L.es_find_offset.argtypes = [U64, D, I, U64, D, I, P, D, D]
        _lib = L
    return _lib


def check(status: int) -> None:
    if status != ES_OK:
        raise EsError(status, lib().es_last_error().decode(errors="replace"))


def launch_count() -> int:
    return int(lib().es_launch_count())


def kernel_timing(on: bool, serial: bool = False) -> None:
    """Brackets each later kernel launch with CUDA events; with serial=True the CAMBI work also stays on the caller's
    stream, so each event pair times one kernel running alone."""
    check(lib().es_kernel_timing(2 if (on and serial) else int(bool(on))))


def kernel_times() -> dict:
    """{kernel name: (total ms, launches)} of the launches timed since kernel_timing(True)."""
    n = ctypes.c_int()
    check(lib().es_kernel_times(None, None, None, 0, ctypes.byref(n)))
    m = n.value
    names = ctypes.create_string_buffer(32 * max(m, 1))
    ms = (ctypes.c_double * max(m, 1))()
    cnt = (ctypes.c_uint64 * max(m, 1))()
    check(lib().es_kernel_times(names, ms, cnt, m, ctypes.byref(n)))
    out = {}
    for i in range(min(m, n.value)):
        name = names.raw[32 * i:32 * i + 32].split(b"\0", 1)[0].decode()
        out[name] = (ms[i], int(cnt[i]))
    return out


def derive_params(w: int, h: int) -> CambiParams:
    p = CambiParams()
    check(lib().es_cambi_derive_params(w, h, ctypes.byref(p)))
    return p


class Module:
    """Kernels (src/gpu.hpp:15-23): binds to the current device, which must be sm_100."""

    def __init__(self):
        self.handle = ctypes.c_void_p()
        check(lib().es_module_load(ctypes.byref(self.handle)))

    def get(self, name: str) -> int:
        f = ctypes.c_void_p()
        check(lib().es_module_get(self.handle, name.encode(), ctypes.byref(f)))
        return f.value

    def close(self) -> None:
        if self.handle:
            lib().es_module_unload(self.handle)
            self.handle = ctypes.c_void_p()


class Cambi:
    """class Cambi (src/cambi.hpp:9-21) through the C ABI."""

    def __init__(self, module: Module, w: int, h: int, depth: int, params: CambiParams | None = None):
        self.handle = ctypes.c_void_p()
        self.w, self.h = w, h
        if params is None:
            check(lib().es_cambi_create(module.handle, w, h, depth, ctypes.byref(self.handle)))
        else:
            check(lib().es_cambi_create_with(module.handle, w, h, depth, ctypes.byref(params), ctypes.byref(self.handle)))

    def params(self) -> CambiParams:
        p = CambiParams()
        check(lib().es_cambi_get_params(self.handle, ctypes.byref(p)))
        return p

    def launch(self, img: int, pitch: int, stream: int = 0) -> None:
        check(lib().es_cambi_launch(self.handle, img, pitch, ctypes.c_void_p(stream)))

    def finish(self) -> float:
        s = ctypes.c_double()
        check(lib().es_cambi_finish(self.handle, ctypes.byref(s)))
        return s.value

    def scale_stats(self) -> tuple[list, list, list]:
        pooled = (ctypes.c_double * SCALES)()
        sums = (ctypes.c_uint64 * SCALES)()
        counts = (ctypes.c_uint64 * SCALES)()
        check(lib().es_cambi_scale_stats(self.handle, pooled, sums, counts))
        return list(pooled), list(sums), list(counts)

    def read_scale(self, s: int):
        import numpy as np
        w, h = self.w, self.h
        for _ in range(s):
            w, h = (w + 1) >> 1, (h + 1) >> 1
        image = np.zeros((h, w), np.uint16)
        mask = np.zeros((h, w), np.uint8)
        check(lib().es_cambi_read_scale(self.handle, s, image.ctypes.data, mask.ctypes.data))
        return image, mask

    def set_tile_mass(self, ptr: int | None) -> None:
        """Per-tile exact c-value sums (2^-24 units) of later launches into the device array at ptr."""
        check(lib().es_cambi_set_tile_mass(self.handle, ctypes.c_void_p(ptr) if ptr else None))

    def scale_words(self, s: int) -> int:
        out = ctypes.c_uint64()
        check(lib().es_cambi_scale_words(self.handle, s, ctypes.byref(out)))
        return out.value

    def set_cvalue_planes(self, ptrs: list | None) -> None:
        arr = (ctypes.c_void_p * SCALES)(*(ptrs or [None] * SCALES))
        check(lib().es_cambi_set_cvalue_planes(self.handle, arr if ptrs else None))

    def close(self) -> None:
        if self.handle:
            lib().es_cambi_destroy(self.handle)
            self.handle = ctypes.c_void_p()


class Windows:
    """Texture window energies in three arithmetics (es_windows_*): mode 0 integer, 1 compensated FP32, 2 FP32."""

    INTEGER, COMPENSATED, FP32 = 0, 1, 2

    def __init__(self, w: int, h: int):
        self.handle = ctypes.c_void_p()
        self.w, self.h = w, h
        check(lib().es_windows_create(w, h, ctypes.byref(self.handle)))

    def compute(self, src: int, enc: int, up: int, stream: int = 0) -> None:
        check(lib().es_windows_compute(self.handle, src, enc, up, ctypes.c_void_p(stream)))

    def figures(self, window: int, mode: int, out: int, stream: int = 0) -> None:
        check(lib().es_windows_figures(self.handle, window, mode, ctypes.c_void_p(out), ctypes.c_void_p(stream)))

    def close(self) -> None:
        if self.handle:
            lib().es_windows_destroy(self.handle)
            self.handle = ctypes.c_void_p()


def per_frame_json(cambi, cambi_source, psnr_y, vmaf=None) -> str:
    """The per_frame JSON object of the reference's report (src/main.cpp:767-774)."""
    import numpy as np
    arrs = [None if a is None else np.ascontiguousarray(a, np.float64) for a in (vmaf, cambi, cambi_source, psnr_y)]
    n = len(arrs[1])
    ptrs = [None if a is None else a.ctypes.data for a in arrs]
    size = lib().es_per_frame_json(*ptrs, n, None, 0)
    buf = ctypes.create_string_buffer(size + 1)
    lib().es_per_frame_json(*ptrs, n, buf, size + 1)
    return buf.value.decode()


class CambiCache:
    """class CambiCache (src/cache.hpp) through the C ABI: the source's CAMBI per frame on disk."""

    def __init__(self, path: str, x0: int, y0: int, w: int, h: int, depth: int, directory: str | None = None):
        self.handle = ctypes.c_void_p()
        check(lib().es_cambi_cache_open(path.encode(), x0, y0, w, h, depth, directory.encode() if directory else None,
                                        ctypes.byref(self.handle)))

    def find(self, pts: int):
        v = ctypes.c_double()
        return v.value if lib().es_cambi_cache_find(self.handle, pts, ctypes.byref(v)) else None

    def add(self, pts: int, score: float) -> None:
        check(lib().es_cambi_cache_add(self.handle, pts, score))

    @property
    def file(self) -> str:
        return lib().es_cambi_cache_file(self.handle).decode()

    def close(self) -> None:
        if self.handle:
            lib().es_cambi_cache_close(self.handle)
            self.handle = ctypes.c_void_p()


def cambi_tile_count(w: int, h: int) -> int:
    out = ctypes.c_int()
    check(lib().es_cambi_tile_count(w, h, ctypes.byref(out)))
    return out.value


PROPOSAL_PARAMS = 5089


class ProposalNet:
    """The tile-proposal network on the device (es_proposal_net_*)."""

    def __init__(self, params=None, seed: int = 0):
        import numpy as np
        self.handle = ctypes.c_void_p()
        arr = None
        if params is not None:
            self._p = np.ascontiguousarray(params, np.float32)
            assert self._p.size == PROPOSAL_PARAMS
            arr = self._p.ctypes.data
        check(lib().es_proposal_net_create(arr, seed, ctypes.byref(self.handle)))

    def params(self):
        import numpy as np
        out = np.zeros(PROPOSAL_PARAMS, np.float32)
        check(lib().es_proposal_net_get(self.handle, out.ctypes.data))
        return out

    def train_step(self, x: int, labels: int, n: int, h: int, w: int, lr: float, stream: int = 0, want_loss: bool = True,
                   want_grads: bool = False):
        """x, labels: device addresses. Returns (loss or None, grads or None)."""
        import numpy as np
        loss = ctypes.c_double()
        grads = np.zeros(PROPOSAL_PARAMS, np.float32) if want_grads else None
        check(lib().es_proposal_net_train_step(self.handle, ctypes.c_void_p(x), ctypes.c_void_p(labels), n, h, w, lr,
                                               ctypes.byref(loss) if want_loss else None,
                                               grads.ctypes.data if want_grads else None, ctypes.c_void_p(stream)))
        return (loss.value if want_loss else None), grads

    def predict(self, words: int, w: int, h: int, pred: int, stream: int = 0) -> None:
        check(lib().es_proposal_predict(self.handle, words, w, h, ctypes.c_void_p(pred), ctypes.c_void_p(stream)))

    def close(self) -> None:
        if self.handle:
            lib().es_proposal_net_destroy(self.handle)
            self.handle = ctypes.c_void_p()


def proposal_features(words: int, w: int, h: int, xy: int, n: int, fw: int, fh: int, out: int, stream: int = 0) -> None:
    check(lib().es_proposal_features(words, w, h, ctypes.c_void_p(xy), n, fw, fh, ctypes.c_void_p(out), ctypes.c_void_p(stream)))


def cambi_score_noalloc(img: int, pitch: int, w: int, h: int, depth: int, score_dev: int, stream: int = 0) -> None:
    """es_cambi_score_noalloc: queues the CAMBI score of a device plane into the device double at `score_dev`,
    allocating nothing (fixed internal scratch; pictures up to about 1920 x 1080)."""
    check(lib().es_cambi_score_noalloc(img, pitch, w, h, depth, ctypes.c_void_p(score_dev), ctypes.c_void_p(stream)))


def new_accum() -> Accum:
    a = Accum()
    lib().es_accum_init(ctypes.byref(a))
    return a


def accum_json(a: Accum) -> str:
    n = lib().es_accum_json(ctypes.byref(a), None, 0)
    buf = ctypes.create_string_buffer(n + 1)
    lib().es_accum_json(ctypes.byref(a), buf, n + 1)
    return buf.value.decode()


def accum_score(a: Accum, weights: Weights | None = None) -> Parts:
    p = Parts()
    lib().es_accum_score(ctypes.byref(a), ctypes.byref(weights) if weights else None, ctypes.byref(p))
    return p


class Frame:
    """The per-frame queue / collect of src/main.cpp:518-643 through the C ABI."""

    def __init__(self, module: Module, w: int, h: int, pd: int, n_encodes: int):
        self.handle = ctypes.c_void_p()
        self.w, self.h, self.n = w, h, n_encodes
        check(lib().es_frame_create(module.handle, w, h, pd, n_encodes, ctypes.byref(self.handle)))

    def queue(self, f: int, source: FrameView, encodes: list, stream: int = 0, sx: int = 0, sy: int = 0, source_cambi: bool = True,
              ex: list | None = None, ey: list | None = None) -> None:
        encs = (FrameView * self.n)(*encodes)
        exa = (ctypes.c_int * self.n)(*(ex or [0] * self.n))
        eya = (ctypes.c_int * self.n)(*(ey or [0] * self.n))
        check(lib().es_frame_queue(self.handle, f, ctypes.byref(source), sx, sy, int(source_cambi), encs, exa, eya, ctypes.c_void_p(stream)))

    def collect(self, f: int, frame_acc: list | None, centre_acc: list | None, cached_source_cambi: float | None = None) -> list:
        out = (FrameResult * self.n)()
        fa = (ctypes.POINTER(Accum) * self.n)(*[ctypes.pointer(a) for a in frame_acc]) if frame_acc else None
        ca = (ctypes.POINTER(Accum) * self.n)(*[ctypes.pointer(a) for a in centre_acc]) if centre_acc else None
        cached = ctypes.byref(ctypes.c_double(cached_source_cambi)) if cached_source_cambi is not None else None
        check(lib().es_frame_collect(self.handle, f, cached, fa, ca, out))
        return list(out)

    def luma(self, p: int, f: int) -> int:
        """Device address of picture p's unpacked luma of frame f (0: the source, 1 + e: encode e)."""
        out = ctypes.c_uint64()
        check(lib().es_frame_luma(self.handle, p, f, ctypes.byref(out)))
        return out.value

    def read_windows(self, encode: int, persist: bool = False):
        import numpy as np
        windows = (self.w // 16) * (self.h // 16)
        st = np.zeros((windows, 8), np.float32)
        ps = np.zeros((windows, 5), np.float32) if persist else None
        check(lib().es_frame_read_windows(self.handle, encode, st.ctypes.data, ps.ctypes.data if persist else None))
        return st, ps

    def close(self) -> None:
        if self.handle:
            lib().es_frame_destroy(self.handle)
            self.handle = ctypes.c_void_p()


def device_step(torch, step) -> tuple:
    """A synthetic frame step (es_synth.Step) copied to the device as planar 16-bit frames: (tensors to keep alive,
    [source view, encode views ...])."""
    import numpy as np
    keep, views = [], []
    for pic in [step.source] + list(step.encodes):
        t = [torch.from_numpy(np.ascontiguousarray(a).view(np.int16)).cuda() for a in (pic.y, pic.u, pic.v)]
        keep.append(t)
        views.append(FrameView(t[0].data_ptr(), t[1].data_ptr(), t[2].data_ptr(), t[0].stride(0) * 2, t[1].stride(0) * 2, 0, 2, 0,
                               pic.depth))
    return keep, views


AUTOTUNE_PATH = os.path.join(HERE, "autotune.json")


def autotune_table(path: str = AUTOTUNE_PATH) -> dict:
    """{(w, h): {"rows": c-value tile rows per scale, "cols": tile columns per scale}} from the autotuner's table
    (empty when there is none; columns 0 where the table has none, the library's default)."""
    import json
    try:
        with open(path) as f:
            t = json.load(f)
    except (OSError, ValueError):
        return {}
    out = {}
    for key, entry in t.get("classes", {}).items():
        w, h = (int(v) for v in key.split("x"))
        out[(w, h)] = {"rows": list(entry["cv_tile_rows"]), "cols": list(entry.get("cv_tile_cols", [0] * 5))}
    return out


def _tile_shape(entry) -> tuple:
    """(rows, cols) per scale from a tuning entry: a list of rows, or a dict with "rows" and optionally "cols"."""
    if entry is None:
        return [64] * 5, [0] * 5
    if isinstance(entry, dict):
        return list(entry.get("rows", [64] * 5)), list(entry.get("cols", [0] * 5))
    return list(entry), [0] * 5


class Batch:
    """Batched frame steps of several sources (es_batch_*): one launch per stage for all pictures, CUDA graphs from
    frame 14 on. ``sources`` is a list of (w, h, pd, n_encodes); pictures and encodes are numbered source by source.
    ``tuning``: None for the autotuned c-value tile shapes of autotune.json (by picture size; the library's defaults
    where absent), False for the defaults everywhere, or a dict {(w, h): rows per scale, or {"rows": [...], "cols":
    [...]}} (cols 0: the library's default width)."""

    def __init__(self, module: Module, sources: list, use_graphs: bool = True, tuning=None):
        self.handle = ctypes.c_void_p()
        self.sources = [tuple(s) for s in sources]
        self.n_pictures = sum(1 + s[3] for s in self.sources)
        self.n_encodes = sum(s[3] for s in self.sources)
        table = autotune_table() if tuning is None else (tuning or {})
        shapes = [_tile_shape(table.get((s[0], s[1]))) for s in self.sources]
        self.tile_rows = [r for r, _ in shapes]
        self.tile_cols = [c for _, c in shapes]
        arr = (BatchSource * len(self.sources))(*[BatchSource(*s, (ctypes.c_int * 5)(*r), (ctypes.c_int * 5)(*c))
                                                  for s, (r, c) in zip(self.sources, shapes)])
        opt = BatchOptions(int(use_graphs))
        check(lib().es_batch_create(module.handle, len(self.sources), arr, ctypes.byref(opt), ctypes.byref(self.handle)))

    def queue(self, f: int, views: list, stream: int = 0, crops: list | None = None, source_cambi: list | None = None) -> None:
        va = (FrameView * self.n_pictures)(*views)
        ca = (ctypes.c_int * (2 * self.n_pictures))(*[c for xy in crops for c in xy]) if crops else None
        sa = (ctypes.c_int * len(self.sources))(*[int(x) for x in source_cambi]) if source_cambi is not None else None
        check(lib().es_batch_queue(self.handle, f, va, ca, sa, ctypes.c_void_p(stream)))

    def collect(self, f: int, frame_acc: list | None = None, centre_acc: list | None = None,
                cached_source_cambi: list | None = None) -> list:
        n = self.n_encodes
        out = (FrameResult * n)()
        fa = (ctypes.POINTER(Accum) * n)(*[ctypes.pointer(a) for a in frame_acc]) if frame_acc else None
        ca = (ctypes.POINTER(Accum) * n)(*[ctypes.pointer(a) for a in centre_acc]) if centre_acc else None
        cached = (ctypes.c_double * len(self.sources))(*cached_source_cambi) if cached_source_cambi is not None else None
        check(lib().es_batch_collect(self.handle, f, cached, fa, ca, out))
        return list(out)

    def read_windows(self, source: int, encode: int, persist: bool = False):
        import numpy as np
        w, h = self.sources[source][0], self.sources[source][1]
        windows = (w // 16) * (h // 16)
        st = np.zeros((windows, 8), np.float32)
        ps = np.zeros((windows, 5), np.float32) if persist else None
        check(lib().es_batch_read_windows(self.handle, source, encode, st.ctypes.data, ps.ctypes.data if persist else None))
        return st, ps

    def luma(self, picture: int, f: int) -> int:
        out = ctypes.c_uint64()
        check(lib().es_batch_luma(self.handle, picture, f, ctypes.byref(out)))
        return out.value

    def scale_pooled(self, picture: int) -> list:
        out = (ctypes.c_double * SCALES)()
        check(lib().es_batch_scale_pooled(self.handle, picture, out))
        return list(out)

    def set_cvalue_planes(self, picture: int, ptrs: list | None) -> None:
        """Later steps also write every computed c-value of `picture` into the zeroed device float planes `ptrs` (one
        per scale); None switches it off."""
        arr = (ctypes.c_void_p * SCALES)(*(ptrs or [None] * SCALES))
        check(lib().es_batch_set_cvalue_planes(self.handle, picture, arr if ptrs else None))

    def set_proposal(self, net, threshold: float = 0.05, audit=(50, 200), tolerance: float = 0.025, budget: float = 0.0) -> None:
        """Switches the learned tile proposal on (net: ProposalNet) or off (net None); budget > 0 also skips, per
        picture, the lowest-predicted scale-0 tiles while their predicted contribution to the score stays within it."""
        opt = ProposalOptions(threshold, (ctypes.c_int * 2)(*audit), tolerance, budget)
        check(lib().es_batch_set_proposal(self.handle, net.handle if net is not None else None, ctypes.byref(opt)))

    def proposal_stats(self, picture: int) -> dict:
        st = ProposalStats()
        check(lib().es_batch_proposal_stats(self.handle, picture, ctypes.byref(st)))
        return {"estimate": st.estimate, "fallback": st.fallback, "run": list(st.run), "audited": list(st.audited),
                "skipped": list(st.skipped)}

    def graph_launches(self) -> int:
        return int(lib().es_batch_graph_launches(self.handle))

    def close(self) -> None:
        if self.handle:
            lib().es_batch_destroy(self.handle)
            self.handle = ctypes.c_void_p()


# ---- temporal alignment (src/kernels.cu:502-520, src/main.cpp:301-353) ----------------------------------------------
def thumbnails(views: list, x0: int, y0: int, w: int, h: int, out: int, stream: int = 0) -> None:
    """64 x 36 luma thumbnails of the frames `views` cropped to w x h at (x0, y0), into the device floats at `out`
    (2304 per frame, row by row)."""
    arr = (FrameView * max(len(views), 1))(*views)
    check(lib().es_thumbnails(arr, len(views), x0, y0, w, h, out, ctypes.c_void_p(stream)))


def offset_totals(ref: int, n_ref: int, probe: int, n_probe: int, totals: int, stream: int = 0) -> None:
    """Per lag, the double total of |ref[l + i][p] - probe[i][p]| over the probe's frames (device arrays)."""
    check(lib().es_offset_totals(ref, n_ref, probe, n_probe, totals, ctypes.c_void_p(stream)))


def find_offset(ref: int, ref_times, probe: int, probe_times, stream: int = 0) -> tuple:
    """(offset, least mean difference) of the probe's thumbnails against the reference's (device arrays of
    len(times) thumbnails each); raises EsError with status ES_ERR_NO_MATCH when they match at no lag."""
    rt = (ctypes.c_double * len(ref_times))(*ref_times)
    pt = (ctypes.c_double * len(probe_times))(*probe_times)
    off, best = ctypes.c_double(), ctypes.c_double()
    status = lib().es_find_offset(ref, rt, len(ref_times), probe, pt, len(probe_times), ctypes.c_void_p(stream),
                                  ctypes.byref(off), ctypes.byref(best))
    if status != ES_OK:
        err = EsError(status, lib().es_last_error().decode(errors="replace"))
        err.best_mean = best.value  # written for a failed match too
        raise err
    return off.value, best.value
