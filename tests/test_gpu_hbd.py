"""Profile 2 (10-bit) on the GPU against its CPU restatement
(oracle/oracle_hbd.c), through the C ABI of include/cvp9_hbd.h: k_hbd_recon
and k_lf_full<uint16_t>. Tolerance: none — every 16-bit sample of every plane
must match. The restatement is unpinned (no 10-bit VP9 decoder or
conformance stream is present); its transforms are tied to the 8-bit ones on
the CPU in tests/test_hbd_oracle.py.
"""
import numpy as np
import pytest

from compute_vp9_b200 import CVP9_ERR_UNSUPPORTED, CVP9_OK
from compute_vp9_b200.hbd import HbdEngine, hbd_frames
from oracle.oracle_py import HbdOracleStream

pytestmark = pytest.mark.gpu

CASES = {
    # name: (preset, w, h, frames, step, overrides)
    "mixed": (2, 352, 288, 6, 4, {"gop": 3, "intra_in_inter": 0.2, "all_intra_modes": 1, "compound_prob": 0.3}),
    "sub8_skip_bilinear": (2, 200, 120, 5, 4, {"gop": 2, "min_bsize": 4, "skip_prob": 0.3, "all_intra_modes": 1,
                                               "intra_in_inter": 0.3, "compound_prob": 0.5, "interp_filter": 3}),
    "tiles_sharp_full_range": (2, 512, 256, 4, 288, {"gop": 2, "log2_tile_cols": 1, "all_intra_modes": 1,
                                                     "intra_in_inter": 0.3, "interp_filter": 2, "sharpness": 5}),
    "big_tx_smooth": (2, 256, 256, 4, 64, {"gop": 2, "tx_weights": [0, 0, 20, 80], "density_max": 0.5,
                                          "all_intra_modes": 1, "interp_filter": 1, "compound_prob": 0.5}),
    "small_tx_lf63": (2, 320, 192, 4, 16, {"gop": 2, "tx_weights": [80, 20, 0, 0], "all_intra_modes": 1,
                                          "intra_in_inter": 0.4, "lf_level": 63}),
    "lossless": (2, 256, 128, 3, 4, {"gop": 2, "qindex": 0, "tx_weights": [100, 0, 0, 0],
                                     "all_intra_modes": 1, "intra_in_inter": 0.3}),
}

# the 10-bit 2160p workload's content: 32x32 TX on half the blocks, 10%
# coefficients, +-256 px MVs, the sharp filter, three references, dequantised
# values up to +-2^17
C4 = dict(gop=120, tx_weights=[10, 15, 25, 50], density_min=0.10, density_max=0.10, mv_range_px=256,
          interp_filter=2, nrefs=3, lf_level=-1, all_intra_modes=1, compound_prob=0.2, intra_in_inter=0.02)


def _check(got, want, w, h, what):
    if np.array_equal(got, want):
        return
    bad = np.nonzero(got != want)[0]
    ny, nc = w * h, ((w + 1) // 2) * ((h + 1) // 2)
    first = int(bad[0])
    plane = "Y" if first < ny else ("U" if first < ny + nc else "V")
    raise AssertionError("%s: %d samples differ, first in %s at %d (%d vs %d)"
                         % (what, len(bad), plane, first, int(got[first]), int(want[first])))


def _run(engine, cases, together=True, seed=11):
    """Decode every case's stream, all streams in one step per frame index
    (together) or one step per stream; check each frame against the oracle.
    Returns the frames."""
    streams = []
    for name, (preset, w, h, frames, step, ov) in cases.items():
        streams.append((name, w, h, frames, engine.open_stream(w, h),
                        hbd_frames(preset, w, h, frames, seed=seed, step=step, **ov), HbdOracleStream()))
    got_all = {}
    for f in range(max(s[3] for s in streams)):
        live = [s for s in streams if f < s[3]]
        inputs, wants = [], []
        for name, w, h, frames, sid, gen, orc in live:
            pf, c32 = next(gen)
            inputs.append((sid, pf, c32))
            wants.append(orc.decode(pf, c32))
        groups = [inputs] if together else [[x] for x in inputs]
        for g in groups:
            rc = engine.submit([x[0] for x in g], [(x[1], x[2].ctypes.data) for x in g])
            assert rc == CVP9_OK, rc
            assert engine.wait() == CVP9_OK
        for (name, w, h, frames, sid, gen, orc), want in zip(live, wants):
            got = engine.get_frame(sid)
            assert got.max() > got.min()            # real content, not a flat fill
            _check(got, want, w, h, "%s frame %d" % (name, f))
            got_all[(name, f)] = got
    for s in streams:
        engine.close_stream(s[4])
    return got_all


def test_hbd_cases_batched_match_oracle():
    e = HbdEngine()
    _run(e, CASES, together=True)
    ms = e.step_times()
    assert all(t >= 0 for t in ms) and ms[2] > 0


def test_hbd_alone_equals_in_the_mix():
    e = HbdEngine()
    sub = {k: CASES[k] for k in ("mixed", "tiles_sharp_full_range", "lossless")}
    alone = _run(e, sub, together=False, seed=4)
    mixed = _run(e, sub, together=True, seed=4)
    assert alone.keys() == mixed.keys()
    for k in alone:
        assert np.array_equal(alone[k], mixed[k]), k


def test_hbd_sparse_lists_equal_dense_arrays():
    """(index, value) lists scattered on the device give the frames of the
    dense int32 arrays."""
    e = HbdEngine()
    cases = {k: CASES[k] for k in ("mixed", "tiles_sharp_full_range", "big_tx_smooth")}
    dense = _run(e, cases, together=True, seed=6)
    sids, gens, nf = [], [], []
    for name, (preset, w, h, frames, step, ov) in cases.items():
        sids.append(e.open_stream(w, h))
        gens.append(hbd_frames(preset, w, h, frames, seed=6, step=step, **ov))
        nf.append(frames)
    for f in range(max(nf)):
        live = [i for i in range(len(sids)) if f < nf[i]]
        pfs, lists, keep = [], [], []
        for i in live:
            pf, c32 = next(gens[i])
            pos = np.nonzero(c32[:pf.contents.num_coeffs])[0].astype(np.uint32)
            val = c32[pos].astype(np.int32)
            keep += [pos, val]
            pfs.append(pf)
            lists.append((pos.size, pos.ctypes.data, val.ctypes.data))
        assert e.submit_sparse([sids[i] for i in live], pfs, lists) == CVP9_OK
        assert e.wait() == CVP9_OK
        for i in live:
            assert np.array_equal(e.get_frame(sids[i]), dense[(list(cases)[i], f)]), (list(cases)[i], f)


def test_hbd_blocks_out_of_decode_order():
    """The blocks of every superblock listed in reverse: intra blocks then
    read samples of blocks that come later in the list, so those
    superblocks run block by block in list order; the frames must still be
    the list-order oracle's."""
    import ctypes as C
    from compute_vp9_b200 import BlockInfo
    e = HbdEngine()
    sid = e.open_stream(256, 128)
    orc = HbdOracleStream()
    gen = hbd_frames(2, 256, 128, 3, seed=8, step=16, gop=3, intra_in_inter=0.4, all_intra_modes=1)
    for f in range(3):
        pf, c32 = next(gen)
        p = pf.contents
        nb = p.num_blocks
        raw = np.ctypeslib.as_array(C.cast(p.blocks, C.POINTER(C.c_uint8)), shape=(nb * 32,)).reshape(nb, 32)
        x = raw[:, 0].astype(int) | (raw[:, 1].astype(int) << 8)
        y = raw[:, 2].astype(int) | (raw[:, 3].astype(int) << 8)
        sb = (y >> 6) * 1000 + (x >> 6)
        order, i = [], 0
        while i < nb:
            j = i
            while j < nb and sb[j] == sb[i]:
                j += 1
            order += list(range(j - 1, i - 1, -1))
            i = j
        rev = np.ascontiguousarray(raw[order])
        orig = C.cast(p.blocks, C.c_void_p).value       # the address (a field read aliases the struct)
        p.blocks = C.cast(C.c_void_p(rev.ctypes.data), C.POINTER(BlockInfo))
        try:
            want = orc.decode(pf, c32)
            assert e.submit([sid], [(pf, c32.ctypes.data)]) == CVP9_OK
            assert e.wait() == CVP9_OK
            _check(e.get_frame(sid), want, 256, 128, "reversed frame %d" % f)
        finally:
            p.blocks = C.cast(C.c_void_p(orig), C.POINTER(BlockInfo))   # the generator writes the next frame there


def test_hbd_two_steps_in_flight():
    """Steps submitted back to back (two in flight: the next step's upload
    and the previous one's download around the kernels) give the frames of
    steps waited for one at a time; dense and sparse submits mixed."""
    e = HbdEngine()
    cases = {k: CASES[k] for k in ("mixed", "small_tx_lf63")}
    sids, gens, orcs = [], [], []
    for name, (preset, w, h, frames, step, ov) in cases.items():
        sids.append(e.open_stream(w, h))
        gens.append(hbd_frames(preset, w, h, 4, seed=13, step=step, **ov))
        orcs.append(HbdOracleStream())
    keep = []
    for f in range(4):
        fr = [next(g) for g in gens]
        want = [o.decode(pf, c) for o, (pf, c) in zip(orcs, fr)]
        if f % 2:
            lists = []
            for pf, c in fr:
                pos = np.nonzero(c[:pf.contents.num_coeffs])[0].astype(np.uint32)
                val = c[pos].astype(np.int32)
                keep += [pos, val, c]
                lists.append((pos.size, pos.ctypes.data, val.ctypes.data))
            assert e.submit_sparse(sids, [pf for pf, _ in fr], lists) == CVP9_OK
        else:
            keep += [c for _, c in fr]
            assert e.submit(sids, [(pf, c.ctypes.data) for pf, c in fr]) == CVP9_OK
        if f % 2:
            # two steps in flight: check the second, which read the first
            for sid, w, (name, (preset, ww, hh, *_)) in zip(sids, want, cases.items()):
                _check(e.get_frame(sid), w, ww, hh, "%s frame %d" % (name, f))
            assert e.wait() == CVP9_OK


def test_hbd_4k_config_content():
    e = HbdEngine()
    _run(e, {"c4_2160p": (2, 3840, 2160, 2, 288, C4)}, seed=1)


def test_hbd_rejects_what_it_does_not_take():
    e = HbdEngine()
    sid = e.open_stream(64, 64)
    gen = hbd_frames(2, 64, 64, 1, seed=2)
    pf, c32 = next(gen)      # the generator owns the frame: keep it alive
    pf.contents.hdr.bit_depth = 8
    assert e.submit([sid], [(pf, c32.ctypes.data)]) == CVP9_ERR_UNSUPPORTED
    pf.contents.hdr.bit_depth = 10
    gen = hbd_frames(2, 64, 64, 2, seed=2, gop=0)
    next(gen)
    pf2, c2 = next(gen)
    pf2.contents.hdr.interp_filter = 4          # SWITCHABLE: no per-block filter in the record
    assert e.submit([sid], [(pf2, c2.ctypes.data)]) == CVP9_ERR_UNSUPPORTED
    with pytest.raises(Exception):
        e.open_stream(100, 60)                  # not a multiple of 8
