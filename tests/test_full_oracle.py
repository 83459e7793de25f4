"""CPU checks of the FULL profile's restatement (oracle/oracle_full.c).

FULL has no counterpart to run here (no VP9 decoder or conformance stream),
so these tests pin what can be pinned: the parts FULL shares with the shader
profile give the shader profile's bytes, the added tables have the
properties every VP9 sub-pel filter has, and the loop filter leaves flat
content alone. The GPU tests then hold the CUDA FULL path to this oracle.
"""
import ctypes as C

import numpy as np
import pytest

from compute_vp9_b200 import Synth, synth_config
from oracle import oracle_py as O


def _filters():
    import re
    import os
    src = open(os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))),
                            "compute_vp9_b200", "csrc", "vp9_tables.h")).read()
    out = {}
    for name in ("REGULAR", "SMOOTH", "SHARP", "BILINEAR"):
        m = re.search(r"#define CVP9_SUBPEL_%s_INIT \{(.*?)\}\s*\}" % name, src, re.S)
        rows = re.findall(r"\{([^{}]*)\}", m.group(1) + "}")
        out[name] = np.array([[int(v) for v in r.split(",")] for r in rows])
    return out


@pytest.mark.parametrize("name", ["REGULAR", "SMOOTH", "SHARP", "BILINEAR"])
def test_subpel_tables_are_vp9_shaped(name):
    t = _filters()[name]
    assert t.shape == (16, 8)
    assert (t.sum(axis=1) == 128).all()
    assert (t[0] == [0, 0, 0, 128, 0, 0, 0, 0]).all()
    for k in range(1, 16):
        # the position k/16 mirrored about the half-sample point is (16-k)/16
        assert (t[16 - k] == t[k][::-1]).all(), (name, k)


def test_full_intra_equals_shader_rules_inside_the_frame():
    """DC, V, H and TM with both edges available inside the frame follow the
    same formulas in both profiles."""
    rng = np.random.default_rng(3)
    plane = rng.integers(0, 256, (96, 96)).astype(np.uint8)
    for n in (4, 8, 16, 32):
        for mode in (0, 1, 2, 9):
            x0, y0 = 32, 40
            a = O.full_intra_tx(plane, x0, y0, n, mode, 1, 1, 0)
            b = O.spec_intra_block(plane, x0, y0, n, n, mode)
            assert np.array_equal(a, b), (n, mode)


def test_full_intra_edge_fills():
    """No neighbours: V reads 127s, H reads 129s, TM gives the left fill,
    DC is 128."""
    plane = np.full((32, 32), 50, np.uint8)
    assert (O.full_intra_tx(plane, 0, 0, 8, 1, 0, 0, 0)[:8, :8] == 127).all()
    assert (O.full_intra_tx(plane, 0, 0, 8, 2, 0, 0, 0)[:8, :8] == 129).all()
    assert (O.full_intra_tx(plane, 0, 0, 8, 9, 0, 0, 0)[:8, :8] == 129).all()
    assert (O.full_intra_tx(plane, 0, 0, 8, 0, 0, 0, 0)[:8, :8] == 128).all()
    for mode in range(3, 9):   # directional modes over flat neighbours stay flat
        out = O.full_intra_tx(plane, 8, 8, 8, mode, 1, 1, 1)
        assert (out[8:16, 8:16] == 50).all(), mode


def test_full_intra_above_right_only_for_4x4():
    """D45 reads the above-right samples of a 4x4 TX that has them; larger
    TXs repeat the last above sample instead."""
    plane = np.full((32, 32), 100, np.uint8)
    plane[7, 12:24] = 200           # above-right of the TXs at (8, 8)
    a4 = O.full_intra_tx(plane, 8, 8, 4, 3, 1, 1, 1)
    a4_no = O.full_intra_tx(plane, 8, 8, 4, 3, 1, 1, 0)
    assert a4[11, 11] == 200 and a4_no[11, 11] == 100
    a8 = O.full_intra_tx(plane, 8, 8, 8, 3, 1, 1, 1)
    assert (a8[8:16, 8:16] <= 200).all() and a8[15, 15] == 200   # above[8..15] not read...
    plane2 = plane.copy()
    plane2[7, 8:16] = 100
    plane2[7, 16:24] = 7
    a8b = O.full_intra_tx(plane2, 8, 8, 8, 3, 1, 1, 1)
    assert (a8b[8:16, 8:16] == 100).all()                      # ...the 7s past it are ignored


def test_full_transform_dc_equals_shader_transform():
    """A DC-only TX gives the same residual whatever the pass order."""
    for n in (4, 8, 16):
        for dc in (-300, -7, 1, 64, 511):
            x = np.zeros((n, n), np.int16)
            x[0, 0] = dc
            a = O.full_itx2d(x, 0, 57, 67)
            b = O.spec_idct2d(x, 57, 67)
            assert np.array_equal(a, b), (n, dc)


def test_full_adst_is_not_dct_and_is_linear_in_sign():
    rng = np.random.default_rng(5)
    for n in (4, 8, 16):
        x = np.where(rng.random((n, n)) < 0.3, rng.integers(-40, 41, (n, n)), 0).astype(np.int16)
        x[0, 0] = 30
        base = O.full_itx2d(x, 0, 20, 20)
        for t in (1, 2, 3):
            a = O.full_itx2d(x, t, 20, 20)
            assert not np.array_equal(a, base), (n, t)
            # negating the input negates the output up to rounding
            b = O.full_itx2d(-x, t, 20, 20)
            assert np.abs(a + b).max() <= 1, (n, t)


def test_full_lossless_walsh_hadamard():
    """Lossless frames use the 4x4 Walsh-Hadamard transform: the quantiser
    step 4 is undone by its first shift, a DC coefficient d spreads d/4 to
    every sample, and no final rounding shift is applied."""
    x = np.zeros((4, 4), np.int16)
    x[0, 0] = 8
    assert (O.full_itx2d(x, 0, 4, 4, lossless=1) == 2).all()
    assert not np.array_equal(O.full_itx2d(x, 0, 4, 4, lossless=1), O.full_itx2d(x, 0, 4, 4, lossless=0))


def _stream_pair(ov, w=256, h=192, frames=3):
    syn = Synth(synth_config(2, w, h, 9, **ov))
    full, spec = O.OracleStream(O.FULL), O.OracleStream(O.SPEC)
    return [(full.decode(syn.frame(f)), spec.decode(syn.frame(f))) for f in range(frames)]


def test_full_inter_prediction_equals_shader_mc_without_additions():
    """With the regular filter and one reference FULL predicts exactly as the
    shader profile (whose luma MC is pinned to the shader translation), luma
    and chroma, MVs at every phase and far outside the frame."""
    rng = np.random.default_rng(11)
    ref = rng.integers(0, 256, (48, 64)).astype(np.uint8)
    for chroma in (0, 1):
        for mv in [(a, b) for a in (-700, -13, -1, 0, 5, 8, 21) for b in (-9, 0, 3, 15, 600)]:
            a = O.full_mc_block(ref, None, (48, 64), 8, 4, 40, 36, mv, chroma=chroma)
            b = O.spec_mc_block(ref, (48, 64), 8, 4, 40, 36, mv[0], mv[1], chroma)
            assert np.array_equal(a, b), (chroma, mv)


def test_full_compound_is_the_rounded_average():
    rng = np.random.default_rng(12)
    r0 = rng.integers(0, 256, (40, 40)).astype(np.uint8)
    r1 = rng.integers(0, 256, (40, 40)).astype(np.uint8)
    for filt in range(4):
        p0 = O.full_mc_block(r0, None, (40, 40), 4, 4, 16, 16, (13, -6), filt=filt).astype(int)
        p1 = O.full_mc_block(r1, None, (40, 40), 4, 4, 16, 16, (-3, 27), filt=filt).astype(int)
        c = O.full_mc_block(r0, r1, (40, 40), 4, 4, 16, 16, (13, -6), (-3, 27), compound=1, filt=filt)
        assert np.array_equal(c[4:20, 4:20], ((p0 + p1 + 1) >> 1)[4:20, 4:20]), filt


def test_full_compound_and_filters_change_prediction():
    ov = dict(gop=100, intra_in_inter=0.0, lf_level=0, interp_filter=0)
    base = _stream_pair(ov, frames=3)
    comp = _stream_pair(dict(ov, compound_prob=1.0), frames=3)
    assert not np.array_equal(base[2][0], comp[2][0])
    for filt in (1, 2, 3):
        other = _stream_pair(dict(ov, interp_filter=filt), frames=3)
        assert not np.array_equal(base[2][0], other[2][0]), filt


def test_full_loop_filter_changes_edges_and_level_zero_is_off():
    ov = dict(gop=2, intra_in_inter=0.2)
    on = _stream_pair(dict(ov, lf_level=40), frames=2)
    off = _stream_pair(dict(ov, lf_level=0), frames=2)
    assert not np.array_equal(on[0][0], off[0][0])
    # level 0: FULL reconstructs, then filters nothing
    syn = Synth(synth_config(2, 256, 192, 9, lf_level=0, **ov))
    a = O.OracleStream(O.FULL).decode(syn.frame(0))
    assert np.array_equal(a, off[0][0])


def test_full_rejects_what_it_does_not_take():
    syn = Synth(synth_config(2, 250, 130, 1, gop=2))
    with pytest.raises(RuntimeError):
        O.OracleStream(O.FULL).decode(syn.frame(0))
    syn = Synth(synth_config(2, 256, 128, 1, gop=2, interp_filter=4))
    s = O.OracleStream(O.FULL)
    s.decode(syn.frame(0))                       # key frame: no filter read
    with pytest.raises(RuntimeError):
        s.decode(syn.frame(1))
