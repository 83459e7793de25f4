"""compute-vp9 reconstruction on B200: Python host mirror of the C ABI.

The product is libcvp9_cuda.so (CUDA kernels for sm_100a + a C host
backend). This module binds it with ctypes so tests, the bench and the
serving loop drive exactly the entry points a C caller uses
(include/cuda_backend.h, include/cvp9_batch.h). There is no Python or CPU
fallback: if the library is missing, loading raises.
"""
import ctypes as C
import os

import numpy as np

from .cvp9_ctypes import (  # noqa: F401
    ARITH_FULL, ARITH_REFCPU, ARITH_SPEC, CVP9_ERR_AGAIN, CVP9_ERR_GPU, CVP9_ERR_INVALID_DATA,
    CVP9_ERR_UNSUPPORTED, CVP9_OK, ERR_NAMES, BlockInfo, DmabufFrame, ExportBuffer,
    FrameHeader, FrameInfo, MV, ParsedFrame, SynthConfig, i420_size, layout_offsets,
)

HERE = os.path.dirname(os.path.abspath(__file__))
LIBDIR = os.path.join(HERE, "lib")
CUDA_LIB = os.path.join(LIBDIR, "libcvp9_cuda.so")
SYNTH_LIB = os.path.join(LIBDIR, "libcvp9_synth.so")

# Every symbol include/*.h declares for the product library.
EXPORTED_SYMBOLS = [
    "cuda_backend_init", "cuda_backend_destroy", "cuda_decode_frame", "cuda_get_frame",
    "cuda_get_frame_dmabuf", "cuda_export_buffer_alloc", "cuda_export_buffer_free",
    "cuda_set_render_target", "cuda_backend_init_ex", "cuda_backend_last_timing",
    "cuda_backend_last_error", "cuda_backend_selftest_wait_limit",
    "cvp9_batch_create", "cvp9_batch_destroy", "cvp9_batch_stream_bytes",
    "cvp9_batch_open_stream", "cvp9_batch_close_stream", "cvp9_batch_reserve", "cvp9_batch_submit",
    "cvp9_batch_wait", "cvp9_batch_poll", "cvp9_batch_get_frame", "cvp9_batch_get_frame_at", "cvp9_batch_stats",
    "cvp9_batch_last_error", "cvp9_batch_timer_start", "cvp9_batch_timer_stop",
    "cvp9_batch_last_seq", "cvp9_batch_step_latency", "cvp9_batch_step_timeline", "cvp9_batch_tune_count",
    "cvp9_batch_tune_entry", "cvp9_batch_submit_sparse", "cvp9_pack_bound_words",
    "cvp9_pack_coeffs",
    "cvp9_hbd_create", "cvp9_hbd_destroy", "cvp9_hbd_open_stream", "cvp9_hbd_close_stream",
    "cvp9_hbd_submit", "cvp9_hbd_submit_sparse", "cvp9_hbd_wait", "cvp9_hbd_get_frame", "cvp9_hbd_step_times",
    "cvp9_hbd_timer_start", "cvp9_hbd_timer_stop",
]


class Cvp9Error(RuntimeError):
    def __init__(self, code, what=""):
        self.code = code
        super().__init__("%s: %s (%d)" % (what, ERR_NAMES.get(code, "?"), code))


_cuda = None
_synth = None


def _load(path, what):
    if not os.path.exists(path):
        raise RuntimeError("%s not built (%s missing); run python -m compute_vp9_b200.build"
                           % (what, path))
    return C.CDLL(path)


def cuda_lib():
    """The product library; raises if it is not built (no fallback)."""
    global _cuda
    if _cuda is None:
        lib = _load(CUDA_LIB, "CUDA backend")
        vp = C.c_void_p
        lib.cuda_backend_init.argtypes = [C.POINTER(vp)]
        lib.cuda_backend_init_ex.argtypes = [C.POINTER(vp), C.c_void_p]
        lib.cuda_backend_destroy.argtypes = [vp]
        lib.cuda_backend_destroy.restype = None
        lib.cuda_decode_frame.argtypes = [vp, C.POINTER(ParsedFrame), C.c_int64]
        lib.cuda_get_frame.argtypes = [vp, C.POINTER(FrameInfo), C.c_int]
        lib.cuda_get_frame_dmabuf.argtypes = [vp, C.POINTER(DmabufFrame)]
        lib.cuda_export_buffer_alloc.argtypes = [vp, C.c_uint64, C.POINTER(ExportBuffer)]
        lib.cuda_export_buffer_free.argtypes = [vp, C.POINTER(ExportBuffer)]
        lib.cuda_export_buffer_free.restype = None
        lib.cuda_set_render_target.argtypes = [vp, C.POINTER(ExportBuffer)]
        lib.cuda_backend_last_timing.argtypes = [vp, C.POINTER(C.c_float), C.POINTER(C.c_float)]
        lib.cuda_backend_last_error.argtypes = [vp]
        lib.cuda_backend_last_error.restype = C.c_char_p
        try:
            from . import batch as _b
            _b._bind(lib)
        except ImportError:
            pass
        _cuda = lib
    return _cuda


def synth_lib():
    global _synth
    if _synth is None:
        lib = _load(SYNTH_LIB, "synthetic generator")
        lib.cvp9_synth_preset.argtypes = [C.POINTER(SynthConfig), C.c_int, C.c_uint32,
                                          C.c_uint32, C.c_uint64]
        lib.cvp9_synth_preset.restype = None
        lib.cvp9_synth_create.argtypes = [C.POINTER(SynthConfig)]
        lib.cvp9_synth_create.restype = C.c_void_p
        lib.cvp9_synth_destroy.argtypes = [C.c_void_p]
        lib.cvp9_synth_destroy.restype = None
        lib.cvp9_synth_frame.argtypes = [C.c_void_p, C.c_int]
        lib.cvp9_synth_frame.restype = C.POINTER(ParsedFrame)
        lib.cvp9_fnv1a64.argtypes = [C.c_void_p, C.c_size_t, C.c_uint64]
        lib.cvp9_fnv1a64.restype = C.c_uint64
        _synth = lib
    return _synth


def synth_config(preset=1, width=0, height=0, seed=0, **overrides):
    cfg = SynthConfig()
    synth_lib().cvp9_synth_preset(C.byref(cfg), preset, width, height, seed)
    for k, v in overrides.items():
        if k == "tx_weights":
            for i, w in enumerate(v):
                cfg.tx_weights[i] = w
        else:
            setattr(cfg, k, v)
    return cfg


class Synth:
    """Seeded synthetic stream: frame(i) -> pointer to a vp9_parsed_frame_t."""

    def __init__(self, cfg):
        self.cfg = cfg
        self._h = synth_lib().cvp9_synth_create(C.byref(cfg))
        if not self._h:
            raise ValueError("invalid synthetic stream configuration")

    def frame(self, index):
        pf = synth_lib().cvp9_synth_frame(self._h, index)
        if not pf:
            raise RuntimeError("synthetic frame %d failed" % index)
        return pf

    def close(self):
        if self._h:
            synth_lib().cvp9_synth_destroy(self._h)
            self._h = None

    def __del__(self):
        self.close()


def fnv1a64(buf):
    arr = np.ascontiguousarray(buf)
    return int(synth_lib().cvp9_fnv1a64(arr.ctypes.data, arr.nbytes, 0))


class BackendOptions(C.Structure):
    _fields_ = [("device", C.c_int), ("arith", C.c_int), ("autotune", C.c_int)]


class CudaBackend:
    """One decoder stream on the CUDA backend (the drop-in ABI)."""

    def __init__(self, device=-1, arith=-1, autotune=0):
        lib = cuda_lib()
        self._lib = lib
        self._ctx = C.c_void_p()
        opt = BackendOptions(device, arith, autotune)
        rc = lib.cuda_backend_init_ex(C.byref(self._ctx), C.byref(opt))
        if rc != CVP9_OK:
            raise Cvp9Error(rc, "cuda_backend_init")

    @property
    def handle(self):
        return self._ctx

    def decode(self, pf, pts=0):
        return self._lib.cuda_decode_frame(self._ctx, pf, pts)

    def get_frame(self, wait=1):
        """(rc, FrameInfo)."""
        info = FrameInfo()
        rc = self._lib.cuda_get_frame(self._ctx, C.byref(info), wait)
        return rc, info

    def get_frame_array(self, wait=1):
        rc, info = self.get_frame(wait)
        if rc != CVP9_OK:
            return rc, None, None
        n = i420_size(info.width, info.height)
        arr = np.ctypeslib.as_array(info.plane_y, shape=(n,)).copy()
        return rc, arr, info

    def last_error(self):
        return self._lib.cuda_backend_last_error(self._ctx).decode()

    def last_timing(self):
        t, k = C.c_float(), C.c_float()
        self._lib.cuda_backend_last_timing(self._ctx, C.byref(t), C.byref(k))
        return t.value, k.value

    def close(self):
        if self._ctx:
            self._lib.cuda_backend_destroy(self._ctx)
            self._ctx = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
