"""The allocation-free entry point (cuda_reconstruct_noalloc) against the
existing per-stream entry point (cuda_decode_frame / cuda_get_frame).

It serves callers that may not allocate GPU memory while decoding (a host
framework that owns all device memory, or a real-time decode thread): they
hand in device inputs, reference frames and the output frame, and the
kernels' scratch comes from a fixed array inside the library. Two calls in a
row — a key frame, then an inter frame predicting from the first call's
output — must reproduce the existing entry point's frames byte for byte (the
tolerance every parity test here uses: none). This file is collected last.
"""
import ctypes as C

import numpy as np
import pytest

from compute_vp9_b200 import (CVP9_OK, BlockInfo, CudaBackend, ParsedFrame, Synth, cuda_lib,
                              i420_size, synth_config)

pytestmark = pytest.mark.gpu


def _bind():
    lib = cuda_lib()
    fn = lib.cuda_reconstruct_noalloc
    fn.argtypes = [C.POINTER(ParsedFrame), C.POINTER(C.c_void_p), C.POINTER(C.c_uint32),
                   C.POINTER(C.c_uint32), C.c_void_p, C.c_int, C.c_void_p, C.c_void_p]
    fn.restype = C.c_int
    return fn


def _device_frame(pf, keep):
    """Copy a parsed frame's arrays to the GPU (the caller's own memory)."""
    import torch
    src = pf.contents
    nb, nc = src.num_blocks, src.num_coeffs
    bt = torch.from_numpy(np.ctypeslib.as_array(C.cast(src.blocks, C.POINTER(C.c_uint8)),
                                                shape=(nb * 32,)).copy()).cuda()
    ct = torch.from_numpy(np.ctypeslib.as_array(src.coeffs, shape=(nc,)).copy()).cuda()
    d = ParsedFrame()
    C.memmove(C.byref(d), C.byref(src), C.sizeof(ParsedFrame))
    d.blocks = C.cast(C.c_void_p(bt.data_ptr()), C.POINTER(BlockInfo))
    d.coeffs = C.cast(C.c_void_p(ct.data_ptr()), C.POINTER(C.c_int16))
    keep += [bt, ct]
    return d


# 352x288 runs the tiled loop filter; 353x289 (8k+1 in both directions) the
# frame-wide one; 251x131 has odd luma and chroma sizes on the tiled path.
@pytest.mark.parametrize("size", [(352, 288), (353, 289), (251, 131)])
@pytest.mark.parametrize("arith", [0, 1])
def test_noalloc_two_calls_match_existing_entry_point(arith, size):
    import torch
    fn = _bind()
    w, h = size
    # the shader profile (arith 1) reconstructs regular-filter frames only
    syn = Synth(synth_config(2, w, h, seed=21, gop=60, intra_in_inter=0.1, interp_filter=0))

    be = CudaBackend(arith=arith)
    want = []
    for f in range(2):
        assert be.decode(syn.frame(f), f) == CVP9_OK, be.last_error()
        rc, arr, _ = be.get_frame_array(wait=1)
        assert rc == CVP9_OK, be.last_error()
        want.append(arr)
    be.close()

    keep = []
    n = i420_size(w, h)
    outs = [torch.empty(n, dtype=torch.uint8, device="cuda") for _ in range(2)]
    status = torch.full((2,), 0xFFFF, dtype=torch.int32, device="cuda")
    stream = torch.cuda.Stream()
    widths = (C.c_uint32 * 8)(*([w] * 8))
    heights = (C.c_uint32 * 8)(*([h] * 8))
    for f in range(2):
        dpf = _device_frame(syn.frame(f), keep)
        torch.cuda.synchronize()
        if f == 0:
            refs = (C.c_void_p * 8)()          # key frame: empty pool
        else:
            refs = (C.c_void_p * 8)(*([outs[0].data_ptr()] * 8))   # key frame fills all 8 slots
        rc = fn(C.byref(dpf), refs, widths, heights, C.c_void_p(outs[f].data_ptr()), arith,
                C.c_void_p(status.data_ptr() + 4 * f), C.c_void_p(stream.cuda_stream))
        assert rc == CVP9_OK
    stream.synchronize()
    assert status.cpu().tolist() == [0, 0]
    for f in range(2):
        got = outs[f].cpu().numpy()
        assert np.array_equal(got, want[f]), "call %d: %d bytes differ" % (f, int((got != want[f]).sum()))


def test_noalloc_rejects_oversize_frame():
    fn = _bind()
    pf = ParsedFrame()
    pf.hdr.width, pf.hdr.height = 8192, 4352      # 128 x 68 = 8704 superblocks > 8160
    rc = fn(C.byref(pf), None, None, None, C.c_void_p(1), 0, None, None)
    assert rc == -3   # CVP9_ERR_INVALID_DATA, nothing launched
