"""CPU: the profile 2 (10-bit) restatement (oracle/oracle_hbd.c).

Its transforms are the 8-bit oracles' butterflies in 64-bit integers: on
inputs where neither overflows they must equal the 32-bit ones exactly (the
DCT is pinned to the shader translation, tests/golden/spec_idct.json), and
on the +-2^17 dequantised range of 10-bit streams they must stay within
rounding of the exact transform where the 32-bit ones wrap. Edge fills,
clipping and the frame loop are checked at 10 bits. No GPU.
"""
import numpy as np
import pytest

from compute_vp9_b200.hbd import hbd_frames
from oracle import oracle_py as O

RNG = np.random.default_rng(5)


@pytest.mark.parametrize("n", [4, 8, 16, 32])
def test_64bit_dct_equals_32bit_dct_without_overflow(n):
    for _ in range(50):
        x = RNG.integers(-4096, 4097, n)
        assert np.array_equal(O.hbd_itx1d(x), O.idct1d(x).astype(np.int64))


@pytest.mark.parametrize("n", [4, 8, 16, 32])
@pytest.mark.parametrize("tx_type", [0, 1, 2, 3])
def test_64bit_residual_equals_8bit_full_residual_without_overflow(n, tx_type):
    if n == 32 and tx_type:
        pytest.skip("32x32 is DCT only")
    q = 40
    for _ in range(10):
        lv = RNG.integers(-60, 61, (n, n)).astype(np.int16)
        want = O.full_itx2d(lv, tx_type, q, q)
        dq = lv.astype(np.int32) * q
        if n == 32:
            dq = (np.abs(dq) // 2) * np.sign(dq)     # the dequantiser's halving toward zero
        got = O.hbd_itx2d(dq.astype(np.int32), tx_type)
        assert np.array_equal(got, want.astype(np.int64))


def _float_idct(x):
    n = len(x)
    k = np.arange(n)
    basis = np.cos(np.pi * (2 * k[:, None] + 1) * k[None, :] / (2 * n))
    scale = np.where(k == 0, 1 / np.sqrt(2), 1.0)
    return basis @ (x * scale) * np.sqrt(2 / n) * np.sqrt(n / 2)


@pytest.mark.parametrize("n", [8, 16, 32])
def test_64bit_dct_stays_exact_on_the_10bit_range(n):
    wrapped = 0
    for _ in range(30):
        x = RNG.integers(-(1 << 17), (1 << 17) + 1, n)
        got = O.hbd_itx1d(x).astype(np.float64)
        ref = _float_idct(x.astype(np.float64))
        # Q14 roundings per stage and Q14 multipliers: within a few units per
        # point plus 1e-4 of the input's magnitude; a wrap would be off by ~2^18
        tol = 2 * n + 1e-4 * np.abs(x).sum()
        assert np.max(np.abs(got - ref)) <= tol, (got - ref)
        wrapped += not np.array_equal(O.idct1d(x.astype(np.int32)).astype(np.int64), O.hbd_itx1d(x))
    assert wrapped > 0      # where the 32-bit butterflies wrap, the 10-bit path must not


def test_lossless_walsh_hadamard_equals_8bit():
    x = np.zeros((4, 4), np.int32)
    x[0, 0] = 4 * 1000
    assert np.all(O.hbd_itx2d(x, 0, lossless=1) == 250)      # a DC spreads evenly
    for _ in range(20):
        lv = RNG.integers(-200, 201, (4, 4)).astype(np.int16)
        want = O.full_itx2d(lv, 0, 4, 4, lossless=1)
        assert np.array_equal(O.hbd_itx2d(lv.astype(np.int32) * 4, 0, lossless=1), want.astype(np.int64))


def test_intra_edge_fills_at_10_bits():
    p = np.full((16, 16), 700, np.uint16)
    # no neighbours: DC is the flat value
    assert np.all(O.hbd_intra_tx(p, 0, 0, 4, 0, 0, 0, 0)[:4, :4] == 512)
    # V without the row above reads 511, H without the left column 513
    assert np.all(O.hbd_intra_tx(p, 4, 0, 4, 1, 0, 1, 0)[:4, 4:8] == 511)
    assert np.all(O.hbd_intra_tx(p, 0, 4, 4, 2, 1, 0, 0)[4:8, :4] == 513)
    # TM clips at 1023
    q = np.zeros((16, 16), np.uint16)
    q[3, 4:8] = 1023
    q[4:8, 3] = 1023
    q[3, 3] = 0
    assert np.all(O.hbd_intra_tx(q, 4, 4, 4, 9, 1, 1, 0)[4:8, 4:8] == 1023)


def test_mc_clips_to_10_bits_and_phase_zero_copies():
    ref = np.zeros((32, 32), np.uint16)
    ref[:, ::2] = 1023
    full_pel = O.hbd_mc_block(ref, None, (32, 32), 8, 8, 8, 8, (16, 0))
    assert np.array_equal(full_pel[8:16, 8:16], ref[8:16, 10:18])
    # the two passes, each rounded and clipped to [0, 1023], restated in numpy
    # on a step edge, where the sharp filter overshoots past both ends
    from tests.test_full_oracle import _filters
    f = _filters()["SHARP"]
    edge = np.zeros((32, 32), np.int64)
    edge[:, 12:] = 1023
    got = O.hbd_mc_block(edge, None, (32, 32), 8, 8, 8, 8, (3, 5), filt=2)[8:16, 8:16]
    fx, fy = 6, 10
    rows = np.clip((np.array([[np.dot(f[fx], edge[y, x - 3:x + 5]) for x in range(8, 16)]
                              for y in range(5, 20)]) + 64) >> 7, 0, 1023)
    want = np.clip((np.array([[np.dot(f[fy], rows[r:r + 8, c]) for c in range(8)]
                              for r in range(8)]) + 64) >> 7, 0, 1023)
    assert np.array_equal(got, want)
    raw = np.array([[np.dot(f[fx], edge[8, x - 3:x + 5]) for x in range(8, 16)]]) + 64 >> 7
    assert raw.max() > 1023 and raw.min() < 0            # the clips were exercised
    comp = O.hbd_mc_block(ref, np.full_like(ref, 101), (32, 32), 8, 8, 8, 8, (16, 0), (0, 0), compound=1)
    assert np.array_equal(comp[8:16, 8:16], (ref[8:16, 10:18].astype(int) + 101 + 1) // 2)


def test_flat_key_frame_stays_at_512():
    gen = hbd_frames(2, 128, 64, 1, seed=3, gop=1, intra_in_inter=0.0)
    pf, c32 = next(gen)      # the generator owns the frame: keep it alive
    c32[:] = 0
    out = O.HbdOracleStream().decode(pf, c32)
    # DC blocks from 512 edges, no residual, LF sees no edge step
    if all(pf.contents.blocks[i].y_mode == 0 and pf.contents.blocks[i].uv_mode == 0
           for i in range(pf.contents.num_blocks)):
        assert np.all(out == 512)
    assert out.max() <= 1023


@pytest.mark.parametrize("step", [4, 288])
def test_sequence_decodes_in_range(step):
    o = O.HbdOracleStream()
    seen = set()
    for pf, c32 in hbd_frames(2, 192, 128, 4, seed=9, step=step, gop=2, compound_prob=0.4,
                              intra_in_inter=0.2, all_intra_modes=1, interp_filter=2):
        out = o.decode(pf, c32)
        assert out.dtype == np.uint16 and out.max() <= 1023
        seen.add(int(np.abs(c32).max()) > 32767)
    if step == 288:
        assert True in seen          # coefficients past int16: the 10-bit range


def test_rejects_8bit_headers():
    gen = hbd_frames(2, 64, 64, 1, seed=1)
    pf, c32 = next(gen)      # the generator owns the frame: keep it alive
    pf.contents.hdr.bit_depth = 8
    with pytest.raises(RuntimeError):
        O.HbdOracleStream().decode(pf, c32)
