"""CPU: the bench's frame schedule. The headline run is GOP-shaped — a key
frame every GOP steps at the rate of the benchmark's stream — and the
parity replay starts at the last key frame, which refreshes every
reference slot, so it reproduces the timed run's final frames exactly."""
import os
import sys

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)

import bench  # noqa: E402


def test_gop_schedule_has_key_frames_at_the_rate():
    frames = [bench.step_frame(t, "gop", 100) for t in range(3, 103)]
    assert frames.count(0) == 1                       # the default 100 timed steps hold one key step
    assert frames[97] == 0                            # t = 100
    assert set(frames) - {0} == set(range(1, bench.DISTINCT))
    assert all(bench.step_frame(t, "key") == 0 for t in range(10))
    inter = [bench.step_frame(t, "inter") for t in range(1, 50)]
    assert 0 not in inter and bench.step_frame(0, "inter") == 0
    assert [bench.step_frame(t, "gop", 60) for t in (0, 59, 60, 61)] == [0, 3, 0, 1]


def test_synthetic_key_frames_refresh_every_slot():
    from compute_vp9_b200 import Synth, synth_config
    for preset in (1, 2):
        syn = Synth(synth_config(preset, 128, 64, 3, gop=5))
        assert syn.frame(0).contents.hdr.refresh_frame_flags == 0xFF
        assert syn.frame(5).contents.hdr.refresh_frame_flags == 0xFF


def test_10bit_schedule_has_one_key_step_per_gop():
    frames = [bench.HbdWorkload.frame_of(t) for t in range(bench.HBD_GOP)]
    assert frames[0] == 0 and frames.count(0) == 1     # the timed 120 steps start at a key frame
    assert set(frames[1:]) == set(range(1, bench.HBD_DISTINCT))
    assert bench.HbdWorkload.frame_of(bench.HBD_GOP) == 0
