"""CPU: the oracle restatements against the committed golden fixtures (which
come from the reference's own compiled CPU reconstruction and from a
mechanical translation of the shader transforms), and against the compiled
reference itself when oracle/_ref is present."""
import json
import os

import numpy as np
import pytest

from compute_vp9_b200 import Synth, fnv1a64, synth_config
from oracle import oracle_py as O

GOLD = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


def _load(name):
    with open(os.path.join(GOLD, name)) as f:
        return json.load(f)


REF_CASES = _load("refcpu_frames.json")
SPEC_CASES = _load("spec_frames.json")


def _hashes(stream, case):
    syn = Synth(synth_config(case["preset"], case["w"], case["h"], case["seed"], **case["overrides"]))
    return ["%016x" % fnv1a64(stream.decode(syn.frame(f))) for f in range(case["frames"])]


@pytest.mark.parametrize("name", sorted(REF_CASES))
def test_refcpu_restatement_matches_reference_golden(name):
    assert _hashes(O.OracleStream(O.REFCPU), REF_CASES[name]) == REF_CASES[name]["hashes"]


@pytest.mark.parametrize("name", sorted(SPEC_CASES))
def test_spec_restatement_is_frozen(name):
    assert _hashes(O.OracleStream(O.SPEC), SPEC_CASES[name]) == SPEC_CASES[name]["hashes"]


@pytest.mark.skipif(not O.ref_available(), reason="oracle/_ref needs the reference sources")
@pytest.mark.parametrize("name", sorted(REF_CASES))
def test_compiled_reference_matches_golden(name):
    assert _hashes(O.RefStream(), REF_CASES[name]) == REF_CASES[name]["hashes"]


def test_spec_idct_matches_shader_translation():
    vecs = _load("spec_idct.json")
    assert len(vecs) == 24
    for v in vecs:
        got = O.spec_idct2d(np.array(v["in"], np.int16), v["q_dc"], v["q_ac"])
        assert np.array_equal(got, np.array(v["out"])), (v["n"], v["q_dc"], v["q_ac"])


def test_refcpu_idct_zero_and_dc():
    for n in (4, 8, 16, 32):
        z = np.zeros((n, n), np.int16)
        assert not O.refcpu_idct2d(z).any()
        x = z.copy()
        x[0, 0] = 64 * n // 8
        out = O.refcpu_idct2d(x)
        # DC alone spreads evenly: every sample is DC / N (orthonormal basis)
        assert (out == out[0, 0]).all() and abs(int(out[0, 0]) - x[0, 0] / n) <= 1


def test_loopfilter_level_zero_and_agreement():
    rng = np.random.default_rng(1)
    plane = (128 + rng.integers(-6, 7, (32, 40))).astype(np.uint8)
    # vp9_reconstruct.c:136 skips level 0; the shader floors the threshold at
    # 1 instead, which only admits p0 == q0 and then delta = 0: both no-ops
    assert np.array_equal(O.loopfilter(plane, 0, 0, O.REFCPU), plane)
    assert np.array_equal(O.loopfilter(plane, 0, 0, O.SPEC), plane)
    for level, sharp in ((20, 3), (63, 0), (5, 7)):
        a = O.loopfilter(plane, level, sharp, O.REFCPU)
        assert np.array_equal(a, O.loopfilter(plane, level, sharp, O.SPEC))
    assert not np.array_equal(O.loopfilter(plane, 63, 0, O.REFCPU), plane)


def test_nv12_pack():
    w, h = 6, 4
    y = np.arange(w * h, dtype=np.uint8)
    u = np.arange(100, 100 + 6, dtype=np.uint8)
    v = np.arange(200, 200 + 6, dtype=np.uint8)
    out = O.nv12_pack(np.concatenate([y, u, v]), w, h)
    assert np.array_equal(out[:w * h], y)
    assert np.array_equal(out[w * h::2], u) and np.array_equal(out[w * h + 1::2], v)


def _vectors():
    import sys
    if GOLD not in sys.path:
        sys.path.insert(0, GOLD)
    import vectors
    return vectors


def test_spec_intra_matches_shader_translation():
    """The restated shader intra predictor equals the shader's own main()
    (translated statement by statement) on every block size, the modes it
    implements (DC, V, H, TM), two it falls back on (D45, D207 -> V), and the
    four edge-availability cases."""
    V = _vectors()
    cases = _load("spec_intra.json")
    assert len(cases) == len(V.INTRA_SIZES) * len(V.INTRA_MODES) * len(V.INTRA_POS)
    for c in cases:
        plane = V.plane_bytes(c["seed"], V.INTRA_PLANE)
        got = O.spec_intra_block(plane, c["x"], c["y"], c["n"], c["n"], c["mode"])
        assert V.digest(got) == c["digest"], c


def test_spec_mc_matches_shader_translation():
    """The restated luma 8-tap prediction equals the shader's main() and
    fetch_ref on all 64 phase pairs and on MVs reaching far outside the
    frame (every fetch clamped)."""
    V = _vectors()
    cases = _load("spec_mc.json")
    assert len(cases) == 72
    h, w = V.MC_PLANE
    for c in cases:
        ref = V.plane_bytes(c["seed"], V.MC_PLANE)
        got = O.spec_mc_block(ref, (h, w), 0, 0, w, h, c["mvx"], c["mvy"], 0)
        assert V.digest(got) == c["digest"], c
