"""CPU: the synthetic generator produces parsed frames with the tile
parser's layout (vp9_kf_tile.c:320-396, :1153-1182), deterministically."""
import ctypes as C

import numpy as np
import pytest

from compute_vp9_b200 import Synth, fnv1a64, synth_config


def _blocks(pf):
    p = pf.contents
    raw = np.ctypeslib.as_array(C.cast(p.blocks, C.POINTER(C.c_uint8)), shape=(p.num_blocks * 32,))
    return raw.reshape(-1, 32)


def _max_tx(w, h):
    m = min(w, h)
    return 3 if m >= 32 else 2 if m >= 16 else 1 if m >= 8 else 0


def _coded(blk, W, H):
    """Coefficients the parser appends for one block (all planes)."""
    x = int(blk[0]) | int(blk[1]) << 8
    y = int(blk[2]) | int(blk[3]) << 8
    w, h, tx, skip = int(blk[4]), int(blk[5]), int(blk[6]), int(blk[20])
    if skip:
        return 0
    sub8 = w < 8 or h < 8
    ew, eh = (8, 8) if sub8 else (w, h)
    mi_cols, mi_rows = (W + 7) // 8, (H + 7) // 8
    tot = 0
    for p in range(3):
        ss = p > 0
        pw, ph = max(4, ew >> ss), max(4, eh >> ss)
        t = tx if not ss else (0 if sub8 else min(tx, _max_tx(pw, ph)))
        t4 = 1 << t
        o4x, o4y = ((x // 8) * 2) >> ss, ((y // 8) * 2) >> ss
        mw = min(pw // 4, ((mi_cols * 2) >> ss) - o4x)
        mh = min(ph // 4, ((mi_rows * 2) >> ss) - o4y)
        nx = -(-mw // t4) if mw > 0 else 0
        ny = -(-mh // t4) if mh > 0 else 0
        tot += nx * ny * (16 << (2 * t))
    return tot


@pytest.mark.parametrize("preset,w,h,ov", [
    (1, 320, 192, {}),
    (2, 352, 288, {"gop": 3}),
    (2, 200, 120, {"min_bsize": 4, "skip_prob": 0.3}),
    (2, 250, 130, {"log2_tile_cols": 1}),
])
def test_layout_and_coverage(preset, w, h, ov):
    syn = Synth(synth_config(preset, w, h, 5, **ov))
    for f in range(3):
        pf = syn.frame(f)
        b = _blocks(pf)
        off = 0
        cover = np.zeros((h + 64, w + 64), np.int32)
        for blk in b:
            coff = int.from_bytes(bytes(blk[24:28]), "little")
            assert coff == off                      # runs are back to back, in block order
            off += _coded(blk, w, h)
            x = int(blk[0]) | int(blk[1]) << 8
            y = int(blk[2]) | int(blk[3]) << 8
            bw, bh = int(blk[4]), int(blk[5])
            assert x < w and y < h and (x % 64) + bw <= 64 and (y % 64) + bh <= 64
            cover[y:y + bh, x:x + bw] += 1
        assert off == pf.contents.num_coeffs
        assert cover.max() == 1                     # no overlaps
        if not ov.get("min_bsize"):
            assert (cover[:h, :w] == 1).all()       # the partition tiles the frame


def test_deterministic_and_seeded():
    a = Synth(synth_config(2, 256, 144, 9))
    b = Synth(synth_config(2, 256, 144, 9))
    c = Synth(synth_config(2, 256, 144, 10))
    for f in (0, 3, 1):
        ca = a.frame(f).contents
        cb = b.frame(f).contents
        ha = fnv1a64(np.ctypeslib.as_array(ca.coeffs, shape=(ca.num_coeffs,)))
        hb = fnv1a64(np.ctypeslib.as_array(cb.coeffs, shape=(cb.num_coeffs,)))
        assert ha == hb
    cc = c.frame(0).contents
    assert cc.num_blocks != ca.num_blocks or fnv1a64(np.ctypeslib.as_array(cc.coeffs, shape=(cc.num_coeffs,))) != ha


def test_mv_grid_matches_blocks():
    syn = Synth(synth_config(2, 192, 128, 4, gop=4))
    pf = syn.frame(1)
    p = pf.contents
    grid = np.ctypeslib.as_array(C.cast(p.mv_grid, C.POINTER(C.c_int32)),
                                 shape=(p.mv_grid_height, p.mv_grid_width, 4))
    for blk in _blocks(pf):
        if blk[7]:      # intra
            continue
        x = int(blk[0]) | int(blk[1]) << 8
        y = int(blk[2]) | int(blk[3]) << 8
        mvx = int(np.frombuffer(bytes(blk[12:14]), np.int16)[0])
        mvy = int(np.frombuffer(bytes(blk[14:16]), np.int16)[0])
        cell = grid[y // 4, x // 4]
        assert (cell[0], cell[1], cell[2]) == (mvx, mvy, int(blk[10]) - 1)
