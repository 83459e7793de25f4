"""Bit-exact parity of the CUDA backend (through the C ABI) with the oracle.

REFCPU cases are the reference's CPU reconstruction (the restatement in
oracle/, itself pinned to the compiled reference and to tests/golden), run
with the warp-per-superblock inter path on (the default) and off; SPEC
cases are the shader-arithmetic restatement, also with the path on and off. Sizes keep the CPU oracle to
seconds. Tolerance: none — every byte of every plane must match.
"""
import numpy as np
import pytest

from compute_vp9_b200 import CVP9_OK, CudaBackend, Synth, synth_config
from oracle.oracle_py import REFCPU, SPEC, OracleStream
from profiles import overrides_for

pytestmark = pytest.mark.gpu

CASES = {
    # name: (preset, w, h, frames, overrides)
    "c1_small": (1, 320, 192, 4, {}),
    "c2_small": (2, 352, 288, 6, {"gop": 3}),
    "edges_sub8": (2, 200, 120, 5, {"gop": 2, "min_bsize": 4, "skip_prob": 0.2,
                                    "all_intra_modes": 1, "intra_in_inter": 0.3}),
    "odd_tiles": (2, 250, 130, 4, {"gop": 2, "log2_tile_cols": 1, "sharpness": 5}),
    "flat_lf": (2, 257, 129, 3, {"gop": 2, "intra_in_inter": 0.2}),
    "big_tx": (2, 256, 256, 4, {"gop": 2, "tx_weights": [0, 0, 20, 80], "density_max": 0.5}),
    "lf_zero": (1, 192, 128, 3, {"lf_level": 0}),
    "c1_720p": (1, 1280, 720, 3, {}),
    "c2_1080p": (2, 1920, 1080, 3, {"gop": 2, "intra_in_inter": 0.1}),
}


def run_case(profile, preset, w, h, frames, overrides, seed=11):
    cfg = synth_config(preset, w, h, seed, **overrides_for(profile, overrides))
    syn = Synth(cfg)
    gpu = CudaBackend(arith=profile)
    orc = OracleStream(profile)
    for f in range(frames):
        pf = syn.frame(f)
        expect = orc.decode(pf)
        assert gpu.decode(pf, f) == CVP9_OK, gpu.last_error()
        rc, got, info = gpu.get_frame_array(wait=1)
        assert rc == CVP9_OK, (rc, gpu.last_error())
        assert info.pts == f and info.width == w and info.height == h
        if not np.array_equal(got, expect):
            bad = np.nonzero(got != expect)[0]
            ny = w * h
            first = int(bad[0])
            plane = "Y" if first < ny else ("U" if first < ny + ((w + 1) // 2) * ((h + 1) // 2) else "V")
            where = (first % w, first // w) if plane == "Y" else first
            pytest.fail("frame %d: %d bytes differ, first in %s at %s (got %d want %d)"
                        % (f, bad.size, plane, where, got[first], expect[first]))
    gpu.close()


@pytest.mark.parametrize("name", list(CASES))
def test_refcpu_parity(name):
    run_case(REFCPU, *CASES[name])


@pytest.mark.parametrize("profile", [REFCPU, SPEC])
@pytest.mark.parametrize("name", ["c1_small", "c2_small", "edges_sub8", "big_tx", "flat_lf"])
def test_parity_without_inter_fast_path(name, profile, monkeypatch):
    """The general superblock kernel alone (CVP9_INTER_FAST=0) gives the same
    bytes as with the warp-per-superblock inter path."""
    monkeypatch.setenv("CVP9_INTER_FAST", "0")
    run_case(profile, *CASES[name])


@pytest.mark.parametrize("variant", ["3", "4", "5"])
@pytest.mark.parametrize("name", list(CASES))
def test_refcpu_parity_prediction_residual_split(name, variant, monkeypatch):
    """REFCPU's two-kernel inter path (k_pred into the frame, then k_resid in
    place; CVP9_INTER_FAST=3, 4 walking 8x8 TXs per TX, 5 with superblocks
    of 8x8 TXs only in a residual kernel of their own) gives the oracle's
    bytes on every case."""
    monkeypatch.setenv("CVP9_INTER_FAST", variant)
    run_case(REFCPU, *CASES[name])


@pytest.mark.parametrize("name", list(CASES))
def test_spec_parity_prediction_residual_split(name, monkeypatch):
    """SPEC through the two-kernel inter path (k_pred into the frame, then
    k_resid over every plane in place; CVP9_INTER_FAST=3) gives the
    restatement's bytes on every case, frame edges included (its TXs follow
    the MI grid past the edge, where nothing may be written)."""
    monkeypatch.setenv("CVP9_INTER_FAST", "3")
    run_case(SPEC, *CASES[name])


@pytest.mark.parametrize("name", list(CASES))
def test_spec_parity(name):
    run_case(SPEC, *CASES[name])
