"""The FULL profile on the GPU against its CPU restatement (oracle/oracle_full.c),
through the C ABI: compound prediction, every frame-level interpolation
filter, per-TX intra prediction with all ten modes and ADST, the header's
delta_q values, lossless frames (Walsh-Hadamard) and the VP9 loop filter.
Tolerance: none — every byte of every plane must match. The restatement
itself is unpinned (no VP9 decoder or conformance stream is present); what
ties it to the reference is checked on the CPU in tests/test_full_oracle.py.
"""
import ctypes as C

import numpy as np
import pytest

from compute_vp9_b200 import ARITH_FULL, CVP9_ERR_UNSUPPORTED, CVP9_OK, CudaBackend, Synth, synth_config
from compute_vp9_b200.batch import Batch, BatchError
from oracle.oracle_py import FULL, OracleStream

pytestmark = pytest.mark.gpu

CASES = {
    # name: (preset, w, h, frames, overrides, header edits)
    "mixed": (2, 352, 288, 6, {"gop": 3, "intra_in_inter": 0.2, "all_intra_modes": 1,
                               "compound_prob": 0.3}, {}),
    "sub8_skip_bilinear": (2, 200, 120, 5, {"gop": 2, "min_bsize": 4, "skip_prob": 0.3, "all_intra_modes": 1,
                                            "intra_in_inter": 0.3, "compound_prob": 0.5,
                                            "interp_filter": 3}, {}),
    "tiles_sharp": (2, 512, 256, 4, {"gop": 2, "log2_tile_cols": 1, "all_intra_modes": 1,
                                     "intra_in_inter": 0.3, "interp_filter": 2, "sharpness": 5}, {}),
    "big_tx_smooth": (2, 256, 256, 4, {"gop": 2, "tx_weights": [0, 0, 20, 80], "density_max": 0.5,
                                       "all_intra_modes": 1, "interp_filter": 1, "compound_prob": 0.5}, {}),
    "small_tx_lf63": (2, 320, 192, 4, {"gop": 2, "tx_weights": [80, 20, 0, 0], "all_intra_modes": 1,
                                       "intra_in_inter": 0.4, "lf_level": 63}, {}),
    "lossless": (2, 256, 128, 3, {"gop": 2, "qindex": 0, "tx_weights": [100, 0, 0, 0],
                                  "all_intra_modes": 1, "intra_in_inter": 0.3}, {}),
    "delta_q": (2, 256, 192, 3, {"gop": 2, "all_intra_modes": 1, "intra_in_inter": 0.3},
                {"y_dc_delta_q": -5, "uv_dc_delta_q": 7, "uv_ac_delta_q": -3}),
    "c1_720p": (1, 1280, 720, 3, {"compound_prob": 0.2, "intra_in_inter": 0.05, "all_intra_modes": 1}, {}),
    "c2_1080p": (2, 1920, 1080, 3, {"gop": 2, "intra_in_inter": 0.1, "all_intra_modes": 1,
                                    "compound_prob": 0.3}, {}),
}


def _frames(preset, w, h, frames, ov, edits, seed=11):
    syn = Synth(synth_config(preset, w, h, seed, **ov))
    out = []
    for f in range(frames):
        pf = syn.frame(f)
        for k, v in edits.items():
            setattr(pf.contents.hdr, k, v)
        out.append(pf)
        yield pf


def _check(got, want, w, h, f):
    if np.array_equal(got, want):
        return
    bad = np.nonzero(got != want)[0]
    ny, nc = w * h, ((w + 1) // 2) * ((h + 1) // 2)
    first = int(bad[0])
    plane = "Y" if first < ny else ("U" if first < ny + nc else "V")
    where = (first % w, first // w) if plane == "Y" else ((first - ny) % nc % ((w + 1) // 2),
                                                         (first - ny) % nc // ((w + 1) // 2))
    pytest.fail("frame %d: %d bytes differ, first in %s at %s (got %d want %d)"
                % (f, bad.size, plane, where, got[first], want[first]))


@pytest.mark.parametrize("name", list(CASES))
def test_full_parity_per_stream(name):
    preset, w, h, frames, ov, edits = CASES[name]
    gpu = CudaBackend(arith=ARITH_FULL)
    orc = OracleStream(FULL)
    for f, pf in enumerate(_frames(preset, w, h, frames, ov, edits)):
        want = orc.decode(pf)
        assert gpu.decode(pf, f) == CVP9_OK, gpu.last_error()
        rc, got, info = gpu.get_frame_array(wait=1)
        assert rc == CVP9_OK, (rc, gpu.last_error())
        _check(got, want, w, h, f)
    gpu.close()


def test_full_parity_batched_mix():
    """Several FULL streams of different sizes in one step, graphs on."""
    names = ["mixed", "sub8_skip_bilinear", "tiles_sharp", "big_tx_smooth"]
    eng = Batch(arith=ARITH_FULL)
    gens, orcs, sids, sizes = [], [], [], []
    for name in names:
        preset, w, h, frames, ov, edits = CASES[name]
        gens.append(_frames(preset, w, h, 4, ov, edits, seed=23))
        orcs.append(OracleStream(FULL))
        sids.append(eng.open_stream(w, h))
        sizes.append((w, h))
    for f in range(4):
        pfs = [next(g) for g in gens]
        eng.submit(sids, pfs, [f] * len(sids))
        assert eng.wait() == CVP9_OK, eng.last_error()
        for i, pf in enumerate(pfs):
            rc, got = eng.get_frame_array(sids[i])
            assert rc == CVP9_OK
            _check(got, orcs[i].decode(pf), sizes[i][0], sizes[i][1], f)
    eng.close()


def test_full_rejects_what_it_does_not_take():
    gpu = CudaBackend(arith=ARITH_FULL)
    syn = Synth(synth_config(2, 250, 130, 1, gop=2))
    assert gpu.decode(syn.frame(0), 0) == CVP9_ERR_UNSUPPORTED     # not a multiple of 8
    syn = Synth(synth_config(2, 256, 128, 1, gop=4, interp_filter=4))
    assert gpu.decode(syn.frame(0), 0) == CVP9_OK                  # key frame: no filter read
    assert gpu.get_frame(wait=1)[0] == CVP9_OK
    assert gpu.decode(syn.frame(1), 1) == CVP9_ERR_UNSUPPORTED     # SWITCHABLE inter frame
    assert "SWITCHABLE" in gpu.last_error()
    gpu.close()
    eng = Batch(arith=ARITH_FULL)
    sid = eng.open_stream(256, 128)
    eng.submit([sid], [syn.frame(0)], [0])
    assert eng.wait() == CVP9_OK
    with pytest.raises(BatchError) as e:
        eng.submit([sid], [syn.frame(1)], [1])
    assert e.value.code == CVP9_ERR_UNSUPPORTED
    eng.close()
