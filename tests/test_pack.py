"""CPU: host-side coefficient packing (cvp9_pack_coeffs, the format in
include/cvp9_batch.h). The packed frame, expanded by a numpy restatement of
k_unpack_coeffs, must give back every coefficient the reconstruction reads
(REFCPU: each non-skip block's luma TX span, as k_gather_luma moves it;
SPEC: all) and zeros elsewhere on entry pages; every scan (scalar, AVX2,
AVX-512) must emit the same words."""
import ctypes as C
import os
import subprocess
import sys

import numpy as np
import pytest

from compute_vp9_b200 import ParsedFrame, Synth, synth_config
from compute_vp9_b200.batch import pack_coeffs

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def unpack(words, n):
    """Dense array from a packed frame, as the device kernel rebuilds it."""
    assert len(words) >= 1
    npages = int(words[0])
    assert npages == (n + 65535) // 65536
    out = np.zeros(n, np.int16)
    for p in range(npages):
        st, cnt = int(words[1 + 2 * p]), int(words[2 + 2 * p])
        s0, dense = st & 0x7FFFFFFF, st >> 31
        assert s0 % 4 == 0
        base = p << 16
        ln = min(65536, n - base)
        if dense:
            assert cnt == ln
            nw = (ln + 1) // 2
            assert s0 + nw <= len(words)
            out[base:base + ln] = words[s0:s0 + nw].copy().view(np.int16)[:ln]
        else:
            assert cnt <= (ln + 1) // 2 and s0 + cnt <= len(words)
            e = words[s0:s0 + cnt]
            off = (e & 0xFFFF).astype(np.int64)
            assert np.all(np.diff(off) > 0) and np.all(off < ln)
            out[base + off] = (e >> 16).astype(np.uint16).view(np.int16)
    return out


def coeffs_of(pf):
    p = pf.contents
    if not p.num_coeffs:
        return np.zeros(0, np.int16)
    return np.ctypeslib.as_array(C.cast(p.coeffs, C.POINTER(C.c_int16)), shape=(p.num_coeffs,)).copy()


def refcpu_mask(pf):
    """Coefficients REFCPU reads: each block's luma TX span."""
    p = pf.contents
    W, H, n = p.hdr.width, p.hdr.height, p.num_coeffs
    raw = np.ctypeslib.as_array(C.cast(p.blocks, C.POINTER(C.c_uint8)), shape=(p.num_blocks * 32,)).reshape(-1, 32)
    m = np.zeros(n, bool)
    for b in raw:
        x, y = int(b[0]) | int(b[1]) << 8, int(b[2]) | int(b[3]) << 8
        w, h, tx, skip = int(b[4]), int(b[5]), int(b[6]), int(b[20])
        if skip or tx > 3 or x >= W or y >= H:
            continue
        tn = 4 << tx
        cw, ch = min(w, W - x), min(h, H - y)
        a = int.from_bytes(bytes(b[24:28]), "little")
        e = min(n, a + (cw // tn) * (ch // tn) * tn * tn)
        if a < e:
            m[a:e] = True
    return m


def check(pf, arith):
    words = pack_coeffs(pf, arith)
    assert words is not None
    ref = coeffs_of(pf)
    got = unpack(words, len(ref))
    mask = np.ones(len(ref), bool) if arith == 1 else refcpu_mask(pf)
    assert np.array_equal(got[mask], ref[mask])
    return words, ref, got, mask


@pytest.mark.parametrize("arith", [0, 1])
@pytest.mark.parametrize("preset,w,h,ov", [
    (1, 320, 192, {}),
    (1, 1920, 1080, {}),
    (2, 352, 288, {"gop": 3}),
    (2, 200, 120, {"min_bsize": 4, "skip_prob": 0.3}),
    (2, 250, 130, {"log2_tile_cols": 1}),
])
def test_round_trip(arith, preset, w, h, ov):
    syn = Synth(synth_config(preset, w, h, 7, **ov))
    for f in range(2):
        pf = syn.frame(f)
        words, ref, got, mask = check(pf, arith)
        dense = ref.astype(np.int64)
        # zero where nothing was read, unless the page went dense
        nz_read = int(np.count_nonzero(ref[mask]))
        assert len(words) * 4 < max(64, 2 * ref.nbytes)
        assert int(np.count_nonzero(got)) >= nz_read
        del dense


def _frame_with(pf, coeffs):
    """A copy of pf whose coefficient array is `coeffs` (kept alive by the caller)."""
    q = ParsedFrame()
    C.pointer(q)[0] = pf.contents
    q.coeffs = C.cast(coeffs.ctypes.data, C.POINTER(C.c_int16))
    q.num_coeffs = len(coeffs)
    return C.pointer(q)


@pytest.mark.parametrize("arith", [0, 1])
def test_dense_pages_and_odd_sizes(arith):
    syn = Synth(synth_config(1, 320, 192, 3))
    pf = syn.frame(1)
    base = coeffs_of(pf)
    rng = np.random.default_rng(5)
    for density in (0.0, 0.3, 0.5, 0.7, 1.0):
        c = base.copy()
        sel = rng.random(len(c)) < density
        c[sel] = rng.integers(-2000, 2000, int(sel.sum()), dtype=np.int16) | 1
        q = _frame_with(pf, c)
        words, ref, got, mask = check(q, arith)
        pages = int(words[0])
        flags = [int(words[1 + 2 * p]) >> 31 for p in range(pages)]
        if density >= 0.7 and arith == 1:
            assert all(flags)
        if density == 0.0:
            assert not any(flags)
    if arith == 1:
        for n in (1, 7, 65535, 65536, 65537, 131071):
            c = rng.integers(-5, 5, n, dtype=np.int16)
            q = _frame_with(pf, c)
            check(q, 1)


def test_empty_and_unordered():
    syn = Synth(synth_config(1, 320, 192, 3))
    pf = syn.frame(1)
    q = ParsedFrame()
    C.pointer(q)[0] = pf.contents
    q.num_coeffs = 0
    w = pack_coeffs(C.pointer(q), 1)
    assert w is not None and int(w[0]) == 0
    # REFCPU spans out of order: the engine falls back to the dense upload
    p = pf.contents
    raw = np.ctypeslib.as_array(C.cast(p.blocks, C.POINTER(C.c_uint8)), shape=(p.num_blocks * 32,)).copy()
    rev = raw.reshape(-1, 32)[::-1].copy()
    r = ParsedFrame()
    C.pointer(r)[0] = p
    r.blocks = C.cast(rev.ctypes.data, type(p.blocks))
    assert pack_coeffs(C.pointer(r), 0) is None
    assert pack_coeffs(C.pointer(r), 1) is not None      # SPEC reads the array whole


_ISA_SCRIPT = r"""
import hashlib, sys
sys.path.insert(0, %r)
from compute_vp9_b200 import Synth, synth_config
from compute_vp9_b200.batch import pack_coeffs
h = hashlib.sha256()
for preset, w, hh in ((1, 1920, 1080), (2, 352, 288)):
    syn = Synth(synth_config(preset, w, hh, 11))
    for f in range(2):
        for arith in (0, 1):
            h.update(pack_coeffs(syn.frame(f), arith).tobytes())
print(h.hexdigest())
"""


def test_every_scan_emits_the_same_words():
    outs = {}
    for isa in ("scalar", "avx2", "avx512"):
        env = dict(os.environ, CVP9_PACK_ISA=isa)
        r = subprocess.run([sys.executable, "-c", _ISA_SCRIPT % ROOT], env=env, capture_output=True,
                           text=True, timeout=300)
        assert r.returncode == 0, r.stderr
        outs[isa] = r.stdout.strip()
    assert len(set(outs.values())) == 1, outs
