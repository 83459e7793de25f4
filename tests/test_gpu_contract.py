"""The drop-in backend's delivery contract on the GPU, through the C ABI.

- NV12 render target: cuda_export_buffer_alloc + cuda_set_render_target arm a
  one-shot target that the next decode packs into (the Vulkan backend packs
  into its armed target each frame, src/backend/vulkan/vulkan_backend.c:
  1059-1062 and 1278-1291; layout of shaders/vp9_nv12_pack.comp.glsl:33-59).
  Both packing paths run: fused into the tiled loop filter, and the separate
  pack kernel on the frame-wide filter path (width or height of the form
  8k+1). The NV12 bytes must equal the oracle's frame packed by the oracle.
- The in-flight ring (vulkan_backend.c:1045-1047, 1391-1455): AGAIN when all
  three slots hold undelivered frames, non-blocking get returns AGAIN or the
  frame (and blocks when the ring is full), UNSUPPORTED on an empty ring,
  frames in submission order, plane pointers valid for the next two decodes.
- Interpolation filters: the shader profile rejects frames whose header asks
  for a filter other than the regular 8-tap one; the CPU profile never reads
  the field (src/decoder/vp9_reconstruct.c:94-131).
Tolerance: none — every byte must match.
"""
import ctypes as C

import numpy as np
import pytest

from compute_vp9_b200 import (CVP9_ERR_AGAIN, CVP9_ERR_INVALID_DATA, CVP9_ERR_UNSUPPORTED, CVP9_OK,
                              CudaBackend, DmabufFrame, ExportBuffer, Synth, cuda_lib,
                              i420_size, synth_config)
from compute_vp9_b200.batch import Batch, BatchError
from oracle.oracle_py import REFCPU, SPEC, OracleStream, nv12_pack
from profiles import overrides_for

pytestmark = pytest.mark.gpu


def _stream(profile, w, h, seed=7, **ov):
    return Synth(synth_config(2, w, h, seed, **overrides_for(profile, dict(gop=3, intra_in_inter=0.1, **ov))))


def _planes(info):
    n = i420_size(info.width, info.height)
    return np.ctypeslib.as_array(info.plane_y, shape=(n,)).copy()


@pytest.mark.parametrize("profile", [REFCPU, SPEC])
@pytest.mark.parametrize("size", [(1280, 720), (1920, 1080), (257, 129), (250, 130)])
def test_nv12_render_target(profile, size):
    w, h = size
    lib = cuda_lib()
    gpu = CudaBackend(arith=profile)
    orc = OracleStream(profile)
    syn = _stream(profile, w, h)
    nbytes = i420_size(w, h)
    buf = ExportBuffer()
    assert lib.cuda_export_buffer_alloc(gpu.handle, nbytes, C.byref(buf)) == CVP9_OK, gpu.last_error()
    assert buf.fd == -1 and buf.mapped and buf.size == nbytes
    target = np.ctypeslib.as_array(C.cast(buf.mapped, C.POINTER(C.c_uint8)), shape=(nbytes,))
    try:
        for f in range(3):
            want = orc.decode(syn.frame(f))
            if f != 1:                                   # frame 1: target not armed
                target[:] = 0xA5
                assert lib.cuda_set_render_target(gpu.handle, C.byref(buf)) == CVP9_OK
            before = target.copy()
            assert gpu.decode(syn.frame(f), f) == CVP9_OK, gpu.last_error()
            rc, got, info = gpu.get_frame_array(wait=1)
            assert rc == CVP9_OK, (rc, gpu.last_error())
            assert np.array_equal(got, want), "frame %d: I420 output differs" % f
            if f == 1:
                # one-shot: the previous decode consumed the target
                assert np.array_equal(target, before), "frame 1 wrote an unarmed target"
            else:
                nv = nv12_pack(want, w, h)
                if not np.array_equal(target, nv):
                    bad = np.nonzero(target != nv)[0]
                    pytest.fail("frame %d: %d NV12 bytes differ, first at %d" % (f, bad.size, bad[0]))
        # disarming with NULL leaves the target untouched
        before = target.copy()
        assert lib.cuda_set_render_target(gpu.handle, C.byref(buf)) == CVP9_OK
        assert lib.cuda_set_render_target(gpu.handle, None) == CVP9_OK
        assert gpu.decode(syn.frame(3), 3) == CVP9_OK
        assert gpu.get_frame_array(wait=1)[0] == CVP9_OK
        assert np.array_equal(target, before)
    finally:
        lib.cuda_export_buffer_free(gpu.handle, C.byref(buf))
        gpu.close()


def test_render_target_too_small_is_rejected():
    lib = cuda_lib()
    gpu = CudaBackend(arith=REFCPU)
    w, h = 320, 192
    buf = ExportBuffer()
    assert lib.cuda_export_buffer_alloc(gpu.handle, i420_size(w, h) - 1, C.byref(buf)) == CVP9_OK
    try:
        assert lib.cuda_set_render_target(gpu.handle, C.byref(buf)) == CVP9_OK
        syn = _stream(REFCPU, w, h)
        assert gpu.decode(syn.frame(0), 0) == CVP9_ERR_INVALID_DATA
        # nothing was queued
        assert gpu.get_frame(wait=0)[0] == CVP9_ERR_UNSUPPORTED
    finally:
        lib.cuda_export_buffer_free(gpu.handle, C.byref(buf))
        gpu.close()


def test_dmabuf_is_unsupported():
    lib = cuda_lib()
    gpu = CudaBackend(arith=REFCPU)
    out = DmabufFrame()
    assert lib.cuda_get_frame_dmabuf(gpu.handle, C.byref(out)) == CVP9_ERR_UNSUPPORTED
    gpu.close()


@pytest.mark.parametrize("profile", [REFCPU, SPEC])
def test_inflight_ring(profile):
    w, h = 640, 360
    gpu = CudaBackend(arith=profile)
    orc = OracleStream(profile)
    syn = _stream(profile, w, h, seed=9)
    want = [orc.decode(syn.frame(f)) for f in range(8)]

    # empty ring
    assert gpu.get_frame(wait=0)[0] == CVP9_ERR_UNSUPPORTED
    assert gpu.get_frame(wait=1)[0] == CVP9_ERR_UNSUPPORTED

    # three frames fill the ring; a fourth is refused and nothing is lost
    for f in range(3):
        assert gpu.decode(syn.frame(f), 100 + f) == CVP9_OK, gpu.last_error()
    assert gpu.decode(syn.frame(3), 103) == CVP9_ERR_AGAIN

    # full ring: the non-blocking get blocks and delivers the oldest frame
    rc, info = gpu.get_frame(wait=0)
    assert rc == CVP9_OK and info.pts == 100
    first = info.plane_y
    assert np.array_equal(_planes(info), want[0])

    # the frame's pointers stay valid for the next two decodes
    assert gpu.decode(syn.frame(3), 103) == CVP9_OK
    delivered = [100]
    polls = 0
    while len(delivered) < 4:
        rc, info = gpu.get_frame(wait=0)
        if rc == CVP9_ERR_AGAIN:
            polls += 1
            assert polls < 10_000_000
            continue
        assert rc == CVP9_OK, (rc, gpu.last_error())
        f = info.pts - 100
        assert np.array_equal(_planes(info), want[f]), "frame %d" % f
        delivered.append(info.pts)
        if len(delivered) == 2:
            assert gpu.decode(syn.frame(4), 104) == CVP9_OK
    assert delivered == [100, 101, 102, 103]
    n = i420_size(w, h)
    kept = np.ctypeslib.as_array(first, shape=(n,)).copy()
    assert np.array_equal(kept, want[0]), "frame 0's planes changed within two decodes"

    # drain: frame 4, then the ring is empty again
    rc, info = gpu.get_frame(wait=1)
    assert rc == CVP9_OK and info.pts == 104
    assert np.array_equal(_planes(info), want[4])
    assert gpu.get_frame(wait=1)[0] == CVP9_ERR_UNSUPPORTED
    gpu.close()


@pytest.mark.parametrize("filt", [1, 2, 3, 4])
def test_spec_rejects_filters_it_does_not_hold(filt):
    """Inter frames only: a key frame carries no filter."""
    w, h = 192, 128
    gpu = CudaBackend(arith=SPEC)
    syn = Synth(synth_config(2, w, h, 3, gop=4, interp_filter=filt))
    assert gpu.decode(syn.frame(0), 0) == CVP9_OK, gpu.last_error()
    assert gpu.get_frame(wait=1)[0] == CVP9_OK
    assert gpu.decode(syn.frame(1), 1) == CVP9_ERR_UNSUPPORTED
    assert "filter" in gpu.last_error()
    assert gpu.get_frame(wait=1)[0] == CVP9_ERR_UNSUPPORTED     # nothing queued
    gpu.close()

    eng = Batch(arith=SPEC)
    sid = eng.open_stream(w, h)
    eng.submit([sid], [syn.frame(0)], [0])
    assert eng.wait() == CVP9_OK
    with pytest.raises(BatchError) as e:
        eng.submit([sid], [syn.frame(1)], [1])
    assert e.value.code == CVP9_ERR_UNSUPPORTED
    assert "filter" in eng.last_error()
    eng.close()


def test_refcpu_ignores_the_filter_field():
    """The CPU path predicts bilinearly whatever the header says: frames that
    differ only in interp_filter reconstruct to the same bytes."""
    w, h = 256, 144
    outs = []
    for filt in (0, 2):
        gpu = CudaBackend(arith=REFCPU)
        orc = OracleStream(REFCPU)
        syn = Synth(synth_config(2, w, h, 4, gop=3, interp_filter=filt))
        frames = []
        for f in range(3):
            assert gpu.decode(syn.frame(f), f) == CVP9_OK, gpu.last_error()
            rc, got, _ = gpu.get_frame_array(wait=1)
            assert rc == CVP9_OK
            assert np.array_equal(got, orc.decode(syn.frame(f)))
            frames.append(got)
        outs.append(frames)
        gpu.close()
    for f in range(3):
        assert np.array_equal(outs[0][f], outs[1][f])
