"""Profile 2 (10-bit 4:2:0): ctypes mirror of include/cvp9_hbd.h and seeded
10-bit synthetic frames.

A 10-bit frame crosses the boundary as the 8-bit path's parsed frame (header
with bit_depth = 10, block records) plus its coefficients dequantised as
int32 in the dense layout of pf->coeffs. `HbdEngine` binds the engine;
`hbd_frames` turns a synthetic 8-bit stream into 10-bit frames.
"""
import ctypes as C

import numpy as np

from . import Cvp9Error, Synth, cuda_lib, synth_config
from .cvp9_ctypes import CVP9_OK, ParsedFrame

HBD_DEVICE_INPUTS = 1 << 0
HBD_NO_OUTPUT = 1 << 1


class HbdFrame(C.Structure):
    _fields_ = [("pf", C.POINTER(ParsedFrame)), ("coeffs", C.c_void_p)]


class HbdCoeffList(C.Structure):
    _fields_ = [("n", C.c_uint32), ("pos", C.c_void_p), ("val", C.c_void_p)]


class HbdFrameInfo(C.Structure):
    _fields_ = [("width", C.c_uint32), ("height", C.c_uint32),
                ("stride_y", C.c_uint32), ("stride_uv", C.c_uint32),
                ("plane_y", C.POINTER(C.c_uint16)), ("plane_u", C.POINTER(C.c_uint16)),
                ("plane_v", C.POINTER(C.c_uint16)), ("pts", C.c_int64)]


_bound = False


def _lib():
    global _bound
    lib = cuda_lib()
    if not _bound:
        vp = C.c_void_p
        lib.cvp9_hbd_create.argtypes = [C.c_int, C.POINTER(vp)]
        lib.cvp9_hbd_destroy.argtypes = [vp]
        lib.cvp9_hbd_destroy.restype = None
        lib.cvp9_hbd_open_stream.argtypes = [vp, C.c_uint32, C.c_uint32]
        lib.cvp9_hbd_close_stream.argtypes = [vp, C.c_int]
        lib.cvp9_hbd_submit.argtypes = [vp, C.c_int, C.POINTER(C.c_int), C.POINTER(HbdFrame),
                                        C.POINTER(C.c_int64), C.c_uint]
        lib.cvp9_hbd_submit_sparse.argtypes = [vp, C.c_int, C.POINTER(C.c_int), C.POINTER(HbdFrame),
                                               C.POINTER(HbdCoeffList), C.POINTER(C.c_int64), C.c_uint]
        lib.cvp9_hbd_wait.argtypes = [vp]
        lib.cvp9_hbd_get_frame.argtypes = [vp, C.c_int, C.POINTER(HbdFrameInfo)]
        lib.cvp9_hbd_step_times.argtypes = [vp, C.POINTER(C.c_float)]
        lib.cvp9_hbd_timer_start.argtypes = [vp]
        lib.cvp9_hbd_timer_stop.argtypes = [vp, C.POINTER(C.c_float)]
        _bound = True
    return lib


def i420_samples(w, h):
    return w * h + 2 * ((w + 1) // 2) * ((h + 1) // 2)


class HbdEngine:
    """Many 10-bit streams, one launch chain per step (cvp9_hbd_*)."""

    def __init__(self, device=-1):
        self._lib = _lib()
        self._h = C.c_void_p()
        rc = self._lib.cvp9_hbd_create(device, C.byref(self._h))
        if rc != CVP9_OK:
            raise Cvp9Error(rc, "cvp9_hbd_create")

    def open_stream(self, w, h):
        sid = self._lib.cvp9_hbd_open_stream(self._h, w, h)
        if sid < 0:
            raise Cvp9Error(sid, "cvp9_hbd_open_stream")
        return sid

    def close_stream(self, sid):
        return self._lib.cvp9_hbd_close_stream(self._h, sid)

    def submit(self, sids, frames, pts=None, flags=0):
        """frames: [(pf pointer, coefficient address)]; returns the C status."""
        n = len(sids)
        s = (C.c_int * n)(*sids)
        f = (HbdFrame * n)()
        for i, (pf, co) in enumerate(frames):
            f[i].pf = pf
            f[i].coeffs = co
        p = (C.c_int64 * n)(*(pts if pts is not None else range(n)))
        return self._lib.cvp9_hbd_submit(self._h, n, s, f, p, flags)

    def submit_sparse(self, sids, pfs, lists, pts=None, flags=0):
        """pfs: parsed-frame pointers; lists: [(n, pos address, val address)]."""
        n = len(sids)
        s = (C.c_int * n)(*sids)
        f = (HbdFrame * n)()
        ls = (HbdCoeffList * n)()
        for i, pf in enumerate(pfs):
            f[i].pf = pf
            ls[i].n, ls[i].pos, ls[i].val = lists[i]
        p = (C.c_int64 * n)(*(pts if pts is not None else range(n)))
        return self._lib.cvp9_hbd_submit_sparse(self._h, n, s, f, ls, p, flags)

    def wait(self):
        return self._lib.cvp9_hbd_wait(self._h)

    def get_frame(self, sid):
        """The stream's latest frame as one uint16 I420 array (a copy)."""
        info = HbdFrameInfo()
        rc = self._lib.cvp9_hbd_get_frame(self._h, sid, C.byref(info))
        if rc != CVP9_OK:
            raise Cvp9Error(rc, "cvp9_hbd_get_frame")
        n = i420_samples(info.width, info.height)
        return np.ctypeslib.as_array(info.plane_y, shape=(n,)).copy()

    def step_times(self):
        ms = (C.c_float * 5)()
        self._lib.cvp9_hbd_step_times(self._h, ms)
        return list(ms)

    def timer_start(self):
        return self._lib.cvp9_hbd_timer_start(self._h)

    def timer_stop(self):
        ms = C.c_float()
        rc = self._lib.cvp9_hbd_timer_stop(self._h, C.byref(ms))
        if rc != CVP9_OK:
            raise Cvp9Error(rc, "cvp9_hbd_timer_stop")
        return ms.value

    def close(self):
        if self._h:
            self._lib.cvp9_hbd_destroy(self._h)
            self._h = C.c_void_p()

    def __del__(self):
        self.close()


def dequantise10(pf, step):
    """Synthetic 10-bit dequantised coefficients of a parsed frame: its
    quantised levels times `step` (synthetic content only: a 10-bit parser
    multiplies by the 10-bit quantiser steps, which sit near four times the
    8-bit ones). Returns an int32 array of pf.num_coeffs values."""
    n = pf.contents.num_coeffs
    if n == 0:
        return np.zeros(1, np.int32)
    src = np.ctypeslib.as_array(pf.contents.coeffs, shape=(n,))
    return src.astype(np.int32) * np.int32(step)


def hbd_frames(preset, w, h, frames, seed=0, step=4, **overrides):
    """Seeded 10-bit frames: (parsed frame with bit_depth 10, int32
    coefficients) for frame 0..frames-1 of a synthetic stream. The parsed
    frame is the generator's and is overwritten by the next frame."""
    syn = Synth(synth_config(preset, w, h, seed, **overrides))
    try:
        for f in range(frames):
            pf = syn.frame(f)
            pf.contents.hdr.bit_depth = 10
            pf.contents.hdr.profile = 2
            yield pf, dequantise10(pf, step)
    finally:
        syn.close()
