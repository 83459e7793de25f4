"""ctypes wrapper of the CPU checkers. TEST INFRASTRUCTURE ONLY: imported by
tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg, never by the
product package.

    OracleStream(profile)   the restatement in oracle/*.c (REFCPU, SPEC or FULL)
    RefStream()             the reference's own vp9_reconstruct_frame compiled
                            from its sources (oracle/_ref), REFCPU only
"""
import ctypes as C
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ORACLE_LIB = os.path.join(HERE, "liboracle.so")
REF_LIB = os.path.join(HERE, "_ref", "libvp9ref.so")

REFCPU = 0
SPEC = 1
FULL = 2

_orc = None
_ref = None


def build():
    subprocess.check_call(["make", "-s", "-C", HERE])


def oracle_lib():
    global _orc
    if _orc is None:
        if not os.path.exists(ORACLE_LIB):
            build()
        from compute_vp9_b200.cvp9_ctypes import ParsedFrame
        lib = C.CDLL(ORACLE_LIB)
        lib.oracle_stream_create.argtypes = [C.c_int]
        lib.oracle_stream_create.restype = C.c_void_p
        lib.oracle_stream_destroy.argtypes = [C.c_void_p]
        lib.oracle_stream_destroy.restype = None
        lib.oracle_stream_decode.argtypes = [C.c_void_p, C.POINTER(ParsedFrame), C.c_void_p]
        lib.oracle_refcpu_idct2d.argtypes = [C.c_void_p, C.c_void_p, C.c_int]
        lib.oracle_refcpu_idct2d.restype = None
        lib.oracle_spec_idct2d.argtypes = [C.c_void_p, C.c_void_p, C.c_int, C.c_int, C.c_int]
        lib.oracle_spec_idct2d.restype = None
        lib.oracle_loopfilter.argtypes = [C.c_void_p, C.c_uint32, C.c_uint32, C.c_uint32,
                                          C.c_int, C.c_int, C.c_int]
        lib.oracle_loopfilter.restype = None
        lib.oracle_nv12_pack.argtypes = [C.c_void_p, C.c_void_p, C.c_uint32, C.c_uint32]
        lib.oracle_nv12_pack.restype = None
        lib.oracle_refcpu_basis.argtypes = [C.c_void_p]
        lib.oracle_refcpu_basis.restype = None
        lib.oracle_spec_intra_block.argtypes = [C.c_void_p] + [C.c_int] * 8
        lib.oracle_spec_intra_block.restype = None
        lib.oracle_spec_mc_block.argtypes = [C.c_void_p, C.c_int, C.c_int, C.c_int, C.c_void_p] + [C.c_int] * 10
        lib.oracle_spec_mc_block.restype = None
        lib.oracle_full_itx2d.argtypes = [C.c_void_p, C.c_void_p] + [C.c_int] * 5
        lib.oracle_full_itx2d.restype = None
        lib.oracle_full_mc_block.argtypes = [C.c_void_p, C.c_void_p, C.c_int, C.c_int, C.c_int, C.c_void_p] + \
            [C.c_int] * 14
        lib.oracle_full_mc_block.restype = None
        lib.oracle_full_intra_tx.argtypes = [C.c_void_p] + [C.c_int] * 10
        lib.oracle_full_intra_tx.restype = None
        lib.oracle_hbd_stream_create.restype = C.c_void_p
        lib.oracle_hbd_stream_destroy.argtypes = [C.c_void_p]
        lib.oracle_hbd_stream_destroy.restype = None
        lib.oracle_hbd_stream_decode.argtypes = [C.c_void_p, C.POINTER(ParsedFrame), C.c_void_p, C.c_void_p]
        lib.oracle_hbd_itx1d.argtypes = [C.c_int, C.c_int, C.c_void_p, C.c_void_p]
        lib.oracle_hbd_itx1d.restype = None
        lib.oracle_hbd_itx2d.argtypes = [C.c_void_p, C.c_void_p] + [C.c_int] * 3
        lib.oracle_hbd_itx2d.restype = None
        lib.oracle_hbd_intra_tx.argtypes = [C.c_void_p] + [C.c_int] * 10
        lib.oracle_hbd_intra_tx.restype = None
        lib.oracle_hbd_mc_block.argtypes = [C.c_void_p, C.c_void_p, C.c_int, C.c_int, C.c_int, C.c_void_p] + \
            [C.c_int] * 14
        lib.oracle_hbd_mc_block.restype = None
        lib.oracle_idct1d.argtypes = [C.c_int, C.c_void_p, C.c_void_p]
        lib.oracle_idct1d.restype = None
        lib.oracle_dc_quant.argtypes = [C.c_int]
        lib.oracle_ac_quant.argtypes = [C.c_int]
        _orc = lib
    return _orc


def ref_available():
    return os.path.exists(REF_LIB)


def ref_lib():
    global _ref
    if _ref is None:
        if not ref_available():
            raise RuntimeError("oracle/_ref not built (needs the reference sources)")
        from compute_vp9_b200.cvp9_ctypes import ParsedFrame
        lib = C.CDLL(REF_LIB)
        lib.ref_stream_create.restype = C.c_void_p
        lib.ref_stream_destroy.argtypes = [C.c_void_p]
        lib.ref_stream_destroy.restype = None
        lib.ref_stream_decode.argtypes = [C.c_void_p, C.POINTER(ParsedFrame), C.c_void_p]
        lib.ref_layout.argtypes = [C.c_void_p, C.c_int]
        _ref = lib
    return _ref


def _i420_size(w, h):
    return w * h + 2 * ((w + 1) // 2) * ((h + 1) // 2)


class OracleStream:
    """Restated reconstruction + reference pool for one stream."""

    def __init__(self, profile=REFCPU):
        self._lib = oracle_lib()
        self._h = self._lib.oracle_stream_create(profile)

    def decode(self, pf):
        w, h = pf.contents.hdr.width, pf.contents.hdr.height
        out = np.empty(_i420_size(w, h), np.uint8)
        if not self._lib.oracle_stream_decode(self._h, pf, out.ctypes.data):
            raise RuntimeError("oracle decode failed")
        return out

    def close(self):
        if self._h:
            self._lib.oracle_stream_destroy(self._h)
            self._h = None

    def __del__(self):
        self.close()


class RefStream:
    """The reference's compiled CPU reconstruction + its pool rules."""

    def __init__(self):
        self._lib = ref_lib()
        self._h = self._lib.ref_stream_create()

    def decode(self, pf):
        w, h = pf.contents.hdr.width, pf.contents.hdr.height
        out = np.empty(_i420_size(w, h), np.uint8)
        if not self._lib.ref_stream_decode(self._h, pf, out.ctypes.data):
            raise RuntimeError("reference decode failed")
        return out

    def close(self):
        if self._h:
            self._lib.ref_stream_destroy(self._h)
            self._h = None

    def __del__(self):
        self.close()


def refcpu_basis():
    out = np.empty(16 + 64 + 256 + 1024, np.float64)
    oracle_lib().oracle_refcpu_basis(out.ctypes.data)
    return out


def refcpu_idct2d(coeffs):
    n = coeffs.shape[0]
    x = np.ascontiguousarray(coeffs, np.int16)
    out = np.empty((n, n), np.int16)
    oracle_lib().oracle_refcpu_idct2d(x.ctypes.data, out.ctypes.data, n)
    return out


def spec_idct2d(coeffs, q_dc, q_ac):
    n = coeffs.shape[0]
    x = np.ascontiguousarray(coeffs, np.int16)
    out = np.empty((n, n), np.int32)
    oracle_lib().oracle_spec_idct2d(x.ctypes.data, out.ctypes.data, n, q_dc, q_ac)
    return out


def loopfilter(plane, level, sharpness, profile):
    p = np.ascontiguousarray(plane, np.uint8).copy()
    h, w = p.shape
    oracle_lib().oracle_loopfilter(p.ctypes.data, w, h, w, level, sharpness, profile)
    return p


def nv12_pack(i420, w, h):
    src = np.ascontiguousarray(i420, np.uint8)
    dst = np.empty(_i420_size(w, h), np.uint8)
    oracle_lib().oracle_nv12_pack(src.ctypes.data, dst.ctypes.data, w, h)
    return dst


def spec_intra_block(plane, x, y, bw, bh, mode):
    """SPEC intra prediction of one block; returns the plane after it."""
    p = np.ascontiguousarray(plane, np.uint8).copy()
    h, w = p.shape
    oracle_lib().oracle_spec_intra_block(p.ctypes.data, w, h, w, x, y, bw, bh, mode)
    return p


def spec_mc_block(ref, dst_shape, x, y, bw, bh, mvx, mvy, chroma=0):
    """SPEC inter prediction of one block from ref into a zeroed plane of
    dst_shape; returns that plane."""
    r = np.ascontiguousarray(ref, np.uint8)
    d = np.zeros(dst_shape, np.uint8)
    oracle_lib().oracle_spec_mc_block(r.ctypes.data, r.shape[1], r.shape[0], r.shape[1],
                                      d.ctypes.data, d.shape[1], d.shape[0], d.shape[1],
                                      x, y, bw, bh, mvx, mvy, chroma)
    return d


def full_itx2d(coeffs, tx_type, q_dc, q_ac, lossless=0):
    n = coeffs.shape[0]
    x = np.ascontiguousarray(coeffs, np.int16)
    out = np.empty((n, n), np.int32)
    oracle_lib().oracle_full_itx2d(x.ctypes.data, out.ctypes.data, n, tx_type, lossless, q_dc, q_ac)
    return out


def full_intra_tx(plane, x0, y0, n, mode, have_top, have_left, have_right):
    """FULL intra prediction of one TX; returns the plane after it."""
    p = np.ascontiguousarray(plane, np.uint8).copy()
    h, w = p.shape
    oracle_lib().oracle_full_intra_tx(p.ctypes.data, w, h, w, x0, y0, n, mode, have_top, have_left, have_right)
    return p


def full_mc_block(ref0, ref1, dst_shape, x, y, bw, bh, mv0, mv1=(0, 0), compound=0, filt=0, chroma=0):
    r0 = np.ascontiguousarray(ref0, np.uint8)
    r1 = np.ascontiguousarray(ref1 if ref1 is not None else ref0, np.uint8)
    d = np.zeros(dst_shape, np.uint8)
    oracle_lib().oracle_full_mc_block(r0.ctypes.data, r1.ctypes.data, r0.shape[1], r0.shape[0], r0.shape[1],
                                      d.ctypes.data, d.shape[1], d.shape[0], d.shape[1], x, y, bw, bh,
                                      mv0[0], mv0[1], mv1[0], mv1[1], compound, filt, chroma)
    return d


class HbdOracleStream:
    """The 10-bit restatement (oracle_hbd.c) + its reference pool."""

    def __init__(self):
        self._lib = oracle_lib()
        self._h = self._lib.oracle_hbd_stream_create()

    def decode(self, pf, coeffs32):
        w, h = pf.contents.hdr.width, pf.contents.hdr.height
        out = np.empty(_i420_size(w, h), np.uint16)
        c = np.ascontiguousarray(coeffs32, np.int32)
        if not self._lib.oracle_hbd_stream_decode(self._h, pf, c.ctypes.data, out.ctypes.data):
            raise RuntimeError("oracle 10-bit decode failed")
        return out

    def close(self):
        if self._h:
            self._lib.oracle_hbd_stream_destroy(self._h)
            self._h = None

    def __del__(self):
        self.close()


def hbd_itx1d(vec, adst=0):
    x = np.ascontiguousarray(vec, np.int64)
    out = np.empty_like(x)
    oracle_lib().oracle_hbd_itx1d(len(x), adst, x.ctypes.data, out.ctypes.data)
    return out


def idct1d(vec):
    """The shader profiles' 32-bit 1-D inverse DCT (oracle_spec.c)."""
    x = np.ascontiguousarray(vec, np.int32)
    out = np.empty_like(x)
    oracle_lib().oracle_idct1d(len(x), x.ctypes.data, out.ctypes.data)
    return out


def hbd_itx2d(coeffs, tx_type=0, lossless=0):
    n = coeffs.shape[0]
    x = np.ascontiguousarray(coeffs, np.int32)
    out = np.empty((n, n), np.int64)
    oracle_lib().oracle_hbd_itx2d(x.ctypes.data, out.ctypes.data, n, tx_type, lossless)
    return out


def hbd_intra_tx(plane, x0, y0, n, mode, have_top, have_left, have_right):
    p = np.ascontiguousarray(plane, np.uint16).copy()
    h, w = p.shape
    oracle_lib().oracle_hbd_intra_tx(p.ctypes.data, w, h, w, x0, y0, n, mode, have_top, have_left, have_right)
    return p


def hbd_mc_block(ref0, ref1, dst_shape, x, y, bw, bh, mv0, mv1=(0, 0), compound=0, filt=0, chroma=0):
    r0 = np.ascontiguousarray(ref0, np.uint16)
    r1 = np.ascontiguousarray(ref1 if ref1 is not None else ref0, np.uint16)
    d = np.zeros(dst_shape, np.uint16)
    oracle_lib().oracle_hbd_mc_block(r0.ctypes.data, r1.ctypes.data, r0.shape[1], r0.shape[0], r0.shape[1],
                                     d.ctypes.data, d.shape[1], d.shape[0], d.shape[1], x, y, bw, bh,
                                     mv0[0], mv0[1], mv1[0], mv1[1], compound, filt, chroma)
    return d
