"""Continuous-batching serving loop: streams arrive while others decode,
are admitted by HBM budget, join the next step, and every delivered frame is
byte-identical to the same stream decoded alone by the oracle."""
import numpy as np
import pytest

from compute_vp9_b200 import serve
from oracle.oracle_py import REFCPU, SPEC, OracleStream

pytestmark = pytest.mark.gpu

SIZES = [(192, 128), (256, 144), (320, 192)]


@pytest.mark.parametrize("profile", [REFCPU, SPEC])
def test_served_frames_match_alone(profile):
    pool = serve.FramePool(SIZES, distinct=4, gop=5)
    expect = {}
    seen = []

    def hook(req, fi, arr):
        assert arr is not None, "frame not delivered"
        seen.append((req, fi))
        o = expect.setdefault(req, {"stream": OracleStream(profile), "size": None, "next": 0})
        assert fi == o["next"], "frames delivered out of order"
        o["next"] += 1
        size = sizes_of[req]
        want = o["stream"].decode(__import__("ctypes").pointer(pool.frame(size, fi)))
        assert np.array_equal(arr, want), "stream %d frame %d" % (req, fi)

    # admission: a budget for about three streams at a time forces queueing
    from compute_vp9_b200.batch import Batch
    budget = 3 * Batch(arith=profile).stream_bytes(320, 192)
    sizes_of = {}
    orig = serve.Stream.__init__

    def capture(self, req, size, *a):
        orig(self, req, size, *a)
        sizes_of[req] = size
    serve.Stream.__init__ = capture
    try:
        out = serve.run(streams=8, rate=400.0, frames=7, fps=100.0, speed=1.0, hbm_budget=budget,
                        arith=profile, seed=3, pool=pool, verify_hook=hook, sizes=SIZES, weights=[1, 1, 1])
    finally:
        serve.Stream.__init__ = orig
    assert out["frames"] == 8 * 7 and len(seen) == 8 * 7
    assert out["admission_waits"] > 0           # the budget made streams wait
    assert out["max_batch"] > 1                 # frames of several streams shared a step
    assert out["p99_ms"] is not None


@pytest.mark.parametrize("profile", [REFCPU])
def test_served_stream_pipelines_its_frames(profile):
    """Frames due faster than a step completes: a stream's next frame joins
    the next step while its previous one is still in flight, and every frame
    still equals the oracle's."""
    pool = serve.FramePool(SIZES, distinct=4, gop=6)
    orcs = {}
    sizes_of = {}
    orig = serve.Stream.__init__

    def capture(self, req, size, *a):
        orig(self, req, size, *a)
        sizes_of[req] = size
    serve.Stream.__init__ = capture

    def hook(req, fi, arr):
        assert arr is not None, "frame not delivered"
        o = orcs.setdefault(req, OracleStream(profile))
        want = o.decode(__import__("ctypes").pointer(pool.frame(sizes_of[req], fi)))
        assert np.array_equal(arr, want), "stream %d frame %d" % (req, fi)

    trace = []
    try:
        out = serve.run(streams=3, rate=1000.0, frames=30, fps=20000.0, speed=1.0, arith=profile, seed=5,
                        pool=pool, verify_hook=hook, sizes=SIZES, weights=[1, 1, 1], trace=trace, hold_ms=0)
    finally:
        serve.Stream.__init__ = orig
    assert out["frames"] == 3 * 30
    done = {(r[0], r[3]): r[6] for r in trace}
    overlapped = sum(1 for r in trace if (r[0], r[3] - 1) in done and r[5] < done[(r[0], r[3] - 1)])
    assert overlapped > 0, "no stream had two frames in flight"


def test_live_streams_batched_over_two_engines():
    """Real-time pacing with many streams live, due frames held also while
    an engine is idle, two engines: steps carry several streams, and every
    frame still equals the stream's oracle decode."""
    profile = REFCPU
    pool = serve.FramePool(SIZES, distinct=4, gop=6)
    orcs = {}
    sizes_of = {}
    orig = serve.Stream.__init__

    def capture(self, req, size, *a):
        orig(self, req, size, *a)
        sizes_of[req] = size
    serve.Stream.__init__ = capture

    def hook(req, fi, arr):
        assert arr is not None, "frame not delivered"
        o = orcs.setdefault(req, OracleStream(profile))
        want = o.decode(__import__("ctypes").pointer(pool.frame(sizes_of[req], fi)))
        assert np.array_equal(arr, want), "stream %d frame %d" % (req, fi)

    trace = []
    try:
        out = serve.run(streams=12, rate=400.0, frames=8, fps=200.0, speed=1.0, arith=profile, seed=6, pool=pool,
                        verify_hook=hook, sizes=SIZES, weights=[1, 1, 1], trace=trace, hold_ms=4.0,
                        hold_idle=True, engines=2, max_batch=6)
    finally:
        serve.Stream.__init__ = orig
    assert out["frames"] == 12 * 8 and out["engines"] == 2
    assert {r[9] for r in trace} == {0, 1}, "both engines served streams"
    assert out["max_batch"] > 1 and out["max_batch"] <= 6
