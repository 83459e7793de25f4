"""ctypes binding of the multi-stream engine (include/cvp9_batch.h)."""
import ctypes as C

import numpy as np

from .cvp9_ctypes import CVP9_OK, ERR_NAMES, FrameInfo, ParsedFrame, i420_size

DEVICE_INPUTS = 1
NO_OUTPUT = 2


class BatchConfig(C.Structure):
    _fields_ = [("device", C.c_int), ("arith", C.c_int), ("hbm_budget", C.c_uint64),
                ("max_streams", C.c_int), ("use_graphs", C.c_int), ("autotune", C.c_int),
                ("pack", C.c_int)]


class CoeffList(C.Structure):
    """cvp9_coeff_list_t: a frame's nonzero coefficients (index, value)."""
    _fields_ = [("n", C.c_uint32), ("pos", C.c_void_p), ("val", C.c_void_p)]


class TuneEntry(C.Structure):
    _fields_ = [("key", C.c_uint64), ("frames", C.c_int), ("settled", C.c_int),
                ("inter_path", C.c_int), ("lf_tile_h", C.c_int), ("half_width", C.c_int),
                ("trials", C.c_int), ("best_ms", C.c_float)]


class BatchStats(C.Structure):
    _fields_ = [("step_ms", C.c_float), ("kernels_ms", C.c_float), ("h2d_ms", C.c_float),
                ("h2d_bytes", C.c_uint64), ("d2h_bytes", C.c_uint64),
                ("reserved_bytes", C.c_uint64), ("open_streams", C.c_int),
                ("graph_replays", C.c_int), ("kernel_launches", C.c_uint32),
                ("scan_ms", C.c_float), ("recon_ms", C.c_float), ("filter_ms", C.c_float),
                ("packed_frames", C.c_uint32), ("submit_pack_ms", C.c_float),
                ("submit_wait_ms", C.c_float), ("submit_stage_ms", C.c_float), ("dev_held_bytes", C.c_uint64),
                ("host_held_bytes", C.c_uint64)]


def _bind(lib):
    vp = C.c_void_p
    lib.cvp9_batch_create.argtypes = [C.POINTER(BatchConfig), C.POINTER(vp)]
    lib.cvp9_batch_destroy.argtypes = [vp]
    lib.cvp9_batch_destroy.restype = None
    lib.cvp9_batch_tune_count.argtypes = [vp]
    lib.cvp9_batch_submit_sparse.argtypes = [vp, C.c_int, C.POINTER(C.c_int),
                                             C.POINTER(C.POINTER(ParsedFrame)), C.POINTER(CoeffList),
                                             C.POINTER(C.c_int64), C.c_uint32]
    lib.cvp9_batch_tune_entry.argtypes = [vp, C.c_int, C.POINTER(TuneEntry)]
    lib.cvp9_batch_stream_bytes.argtypes = [C.c_uint32, C.c_uint32]
    lib.cvp9_batch_stream_bytes.restype = C.c_uint64
    lib.cvp9_batch_open_stream.argtypes = [vp, C.c_uint32, C.c_uint32]
    lib.cvp9_batch_close_stream.argtypes = [vp, C.c_int]
    lib.cvp9_batch_reserve.argtypes = [vp, C.c_uint32, C.c_uint32, C.c_int]
    lib.cvp9_batch_submit.argtypes = [vp, C.c_int, C.POINTER(C.c_int),
                                      C.POINTER(C.POINTER(ParsedFrame)), C.POINTER(C.c_int64),
                                      C.c_uint32]
    lib.cvp9_batch_wait.argtypes = [vp]
    lib.cvp9_batch_poll.argtypes = [vp]
    lib.cvp9_batch_get_frame.argtypes = [vp, C.c_int, C.POINTER(FrameInfo)]
    lib.cvp9_batch_get_frame_at.argtypes = [vp, C.c_int, C.c_uint64, C.POINTER(FrameInfo)]
    lib.cvp9_batch_stats.argtypes = [vp, C.POINTER(BatchStats)]
    lib.cvp9_batch_last_error.argtypes = [vp]
    lib.cvp9_batch_last_error.restype = C.c_char_p
    lib.cvp9_batch_timer_start.argtypes = [vp]
    lib.cvp9_batch_timer_stop.argtypes = [vp, C.POINTER(C.c_float)]
    lib.cvp9_batch_last_seq.argtypes = [vp]
    lib.cvp9_batch_last_seq.restype = C.c_uint64
    lib.cvp9_batch_step_latency.argtypes = [vp, C.c_uint64, C.POINTER(C.c_double)]
    lib.cvp9_batch_step_timeline.argtypes = [vp, C.c_uint64, C.POINTER(C.c_float)]
    lib.cvp9_pack_bound_words.argtypes = [C.c_uint32]
    lib.cvp9_pack_bound_words.restype = C.c_size_t
    lib.cvp9_pack_coeffs.argtypes = [C.c_int, C.POINTER(ParsedFrame), vp, C.c_size_t]
    lib.cvp9_pack_coeffs.restype = C.c_int64


def pack_coeffs(pf, arith=0):
    """The engine's host-side packing of one parsed frame's coefficients
    (cvp9_pack_coeffs) as a numpy uint32 array, or None when the frame is
    not packable. pf: a ParsedFrame pointer."""
    import numpy as np
    from . import cuda_lib
    lib = cuda_lib()
    cap = int(lib.cvp9_pack_bound_words(pf.contents.num_coeffs))
    out = np.zeros(cap, dtype=np.uint32)
    w = lib.cvp9_pack_coeffs(arith, pf, out.ctypes.data, cap)
    return None if w < 0 else out[:w].copy()


class BatchError(RuntimeError):
    def __init__(self, code, what, detail=""):
        self.code = code
        super().__init__("%s: %s (%d) %s" % (what, ERR_NAMES.get(code, "?"), code, detail))


class Batch:
    """Engine handle (cvp9_batch_*). Streams are admitted by HBM budget
    (open_stream returns None when the budget is full); submit() enqueues
    one frame per listed stream, reconstructed in one launch chain, up to
    three steps in flight.

    autotune: time the kernel configurations on the first steps of each
    shape bucket and keep the fastest (tuning() reports them).
    pack: host-side packing of dense host coefficient arrays before the
    upload — 0 for steps moving at least 64 MB of them, with the packed
    share balanced against the link; 1 always; -1 never."""

    def __init__(self, device=-1, arith=-1, hbm_budget=0, max_streams=0, use_graphs=1, autotune=1, pack=0):
        from . import cuda_lib
        self._lib = cuda_lib()
        self._h = C.c_void_p()
        cfg = BatchConfig(device, arith, hbm_budget, max_streams, use_graphs, autotune, pack)
        rc = self._lib.cvp9_batch_create(C.byref(cfg), C.byref(self._h))
        if rc != CVP9_OK:
            raise BatchError(rc, "cvp9_batch_create")

    def stream_bytes(self, w, h):
        return int(self._lib.cvp9_batch_stream_bytes(w, h))

    def open_stream(self, w, h):
        sid = self._lib.cvp9_batch_open_stream(self._h, w, h)
        return sid if sid >= 0 else None

    def reserve(self, w, h, nstreams):
        """Take device and pinned memory now for `nstreams` streams of w x h
        (cvp9_batch_reserve), so that opening them later allocates nothing."""
        rc = self._lib.cvp9_batch_reserve(self._h, w, h, nstreams)
        if rc != CVP9_OK:
            raise BatchError(rc, "cvp9_batch_reserve", self.last_error())

    def close_stream(self, sid):
        rc = self._lib.cvp9_batch_close_stream(self._h, sid)
        if rc != CVP9_OK:
            raise BatchError(rc, "cvp9_batch_close_stream", self.last_error())

    def submit(self, sids, pfs, pts=None, flags=0):
        n = len(sids)
        arr_s = (C.c_int * n)(*sids)
        arr_p = (C.POINTER(ParsedFrame) * n)(*pfs)
        arr_t = (C.c_int64 * n)(*(pts if pts is not None else [0] * n))
        rc = self._lib.cvp9_batch_submit(self._h, n, arr_s, arr_p, arr_t, flags)
        if rc != CVP9_OK:
            raise BatchError(rc, "cvp9_batch_submit", self.last_error())

    def submit_sparse(self, sids, pfs, lists, pts=None, flags=0):
        """Like submit, with each frame's coefficients as a CoeffList."""
        n = len(sids)
        arr_s = (C.c_int * n)(*sids)
        arr_p = (C.POINTER(ParsedFrame) * n)(*pfs)
        arr_l = (CoeffList * n)(*lists)
        arr_t = (C.c_int64 * n)(*(pts if pts is not None else [0] * n))
        rc = self._lib.cvp9_batch_submit_sparse(self._h, n, arr_s, arr_p, arr_l, arr_t, flags)
        if rc != CVP9_OK:
            raise BatchError(rc, "cvp9_batch_submit_sparse", self.last_error())

    def wait(self):
        return self._lib.cvp9_batch_wait(self._h)

    def poll(self):
        return self._lib.cvp9_batch_poll(self._h)

    def get_frame(self, sid):
        info = FrameInfo()
        rc = self._lib.cvp9_batch_get_frame(self._h, sid, C.byref(info))
        return rc, info

    def get_frame_array(self, sid):
        rc, info = self.get_frame(sid)
        if rc != CVP9_OK:
            return rc, None
        n = i420_size(info.width, info.height)
        return rc, np.ctypeslib.as_array(info.plane_y, shape=(n,)).copy()

    def get_frame_at(self, sid, seq):
        """The frame stream `sid` got from step `seq` (cvp9_batch_get_frame_at)."""
        info = FrameInfo()
        rc = self._lib.cvp9_batch_get_frame_at(self._h, sid, seq, C.byref(info))
        return rc, info

    def get_frame_array_at(self, sid, seq):
        rc, info = self.get_frame_at(sid, seq)
        if rc != CVP9_OK:
            return rc, None
        n = i420_size(info.width, info.height)
        return rc, np.ctypeslib.as_array(info.plane_y, shape=(n,)).copy()

    def stats(self):
        st = BatchStats()
        self._lib.cvp9_batch_stats(self._h, C.byref(st))
        return st

    def last_error(self):
        return self._lib.cvp9_batch_last_error(self._h).decode()

    def timer_start(self):
        rc = self._lib.cvp9_batch_timer_start(self._h)
        if rc != CVP9_OK:
            raise BatchError(rc, "cvp9_batch_timer_start", self.last_error())

    def timer_stop(self):
        ms = C.c_float()
        rc = self._lib.cvp9_batch_timer_stop(self._h, C.byref(ms))
        if rc != CVP9_OK:
            raise BatchError(rc, "cvp9_batch_timer_stop", self.last_error())
        return ms.value

    def last_seq(self):
        return int(self._lib.cvp9_batch_last_seq(self._h))

    def tuning(self):
        """The tuner's buckets: list of dicts (key, frames, settled, inter_path,
        lf_tile_h, half_width, trials, best_ms)."""
        out = []
        for i in range(self._lib.cvp9_batch_tune_count(self._h)):
            e = TuneEntry()
            if self._lib.cvp9_batch_tune_entry(self._h, i, C.byref(e)) == CVP9_OK:
                out.append({k: getattr(e, k) for k, _ in TuneEntry._fields_})
        return out

    def step_latency_ms(self, seq):
        ms = C.c_double()
        rc = self._lib.cvp9_batch_step_latency(self._h, seq, C.byref(ms))
        return ms.value if rc == CVP9_OK else None

    def step_timeline(self, seq):
        """Device timeline of completed step `seq` after timer_start: ms to
        its (upload start, upload end, kernels start, kernels end, download
        end), or None."""
        t = (C.c_float * 5)()
        rc = self._lib.cvp9_batch_step_timeline(self._h, seq, t)
        return tuple(t) if rc == CVP9_OK else None

    def close(self):
        if self._h:
            self._lib.cvp9_batch_destroy(self._h)
            self._h = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
