"""The engine's autotuner (host logic in backend_common.c), driven with
synthetic kernel times through the C ABI. CPU only: the library loads
without a GPU and the tuner makes no CUDA calls."""
import ctypes as C

import pytest

from compute_vp9_b200 import cuda_lib


class Cfg(C.Structure):
    _fields_ = [("inter", C.c_int8), ("lf32", C.c_int8), ("half", C.c_int8)]

    def t(self):
        return (self.inter, self.lf32, self.half)


@pytest.fixture()
def lib():
    lib = cuda_lib()
    lib.cvp9_tuner_init.argtypes = [C.c_void_p, C.c_int, C.c_int, Cfg]
    lib.cvp9_tuner_init.restype = None
    lib.cvp9_tuner_pick.argtypes = [C.c_void_p, C.c_uint64, C.c_int, C.POINTER(Cfg)]
    lib.cvp9_tuner_report.argtypes = [C.c_void_p, C.c_int, Cfg, C.c_float]
    lib.cvp9_tuner_report.restype = None
    lib.cvp9_tune_key.argtypes = [C.c_int, C.c_int, C.c_uint64]
    lib.cvp9_tune_key.restype = C.c_uint64
    return lib


def make(lib, arith=0, enabled=1, fixed=(1, 0, 0)):
    buf = C.create_string_buffer(1 << 16)
    lib.cvp9_tuner_init(buf, arith, enabled, Cfg(*fixed))
    return buf


def step(lib, t, key, ms_of):
    """One step of bucket `key`: pick, then report the time ms_of(cfg) twice
    (a candidate is judged on two samples)."""
    cfg = Cfg()
    idx = lib.cvp9_tuner_pick(t, key, 8, C.byref(cfg))
    if idx >= 0:
        lib.cvp9_tuner_report(t, idx, cfg, ms_of(cfg.t()))
    return idx, cfg.t()


def test_coordinate_descent_order_and_choice(lib):
    t = make(lib)
    times = {(1, 0, 0): 1.0, (0, 0, 0): 2.0, (2, 0, 0): 0.5, (3, 0, 0): 0.7, (4, 0, 0): 0.55, (5, 0, 0): 0.52,
             (2, 1, 0): 0.6, (2, 0, 1): 0.4}
    seen = []
    for _ in range(20):
        idx, cfg = step(lib, t, 7, lambda c: times[c])
        if idx < 0:
            break
        if not seen or seen[-1] != cfg:
            seen.append(cfg)
    # default, the other five inter paths (REFCPU has the two-kernel split,
    # in three forms), then lf tiles, then wavefront
    # width, each varied from the best
    assert seen == [(1, 0, 0), (0, 0, 0), (2, 0, 0), (3, 0, 0), (4, 0, 0), (5, 0, 0), (2, 1, 0), (2, 0, 1)]
    idx, cfg = step(lib, t, 7, lambda c: 9.0)
    assert idx == -1 and cfg == (2, 0, 1)


def test_stale_samples_are_ignored(lib):
    t = make(lib)
    cfg = Cfg()
    idx = lib.cvp9_tuner_pick(t, 3, 4, C.byref(cfg))
    assert idx >= 0 and cfg.t() == (1, 0, 0)
    # a sample from a configuration that is not under measurement
    lib.cvp9_tuner_report(t, idx, Cfg(0, 1, 1), 0.001)
    lib.cvp9_tuner_report(t, idx, cfg, 1.0)
    lib.cvp9_tuner_report(t, idx, cfg, 1.0)
    nxt = Cfg()
    lib.cvp9_tuner_pick(t, 3, 4, C.byref(nxt))
    assert nxt.t() == (0, 0, 0)


def test_spec_tunes_the_same_knobs(lib):
    t = make(lib, arith=1, fixed=(1, 0, 0))
    seen = []
    for _ in range(20):
        idx, cfg = step(lib, t, 5, lambda c: 1.0 + 0.1 * c[1] - 0.2 * c[2] + (0.5 if c[0] != 1 else 0))
        if idx < 0:
            break
        if not seen or seen[-1] != cfg:
            seen.append(cfg)
    assert seen == [(1, 0, 0), (0, 0, 0), (2, 0, 0), (3, 0, 0), (1, 1, 0), (1, 0, 1)]
    assert step(lib, t, 5, lambda c: 1.0) == (-1, (1, 0, 1))


def test_disabled_returns_the_fixed_configuration(lib):
    t = make(lib, enabled=0, fixed=(2, 1, 0))
    for k in range(5):
        assert step(lib, t, k, lambda c: 1.0) == (-1, (2, 1, 0))


def test_buckets_are_independent_and_recycled(lib):
    t = make(lib)
    a = step(lib, t, 100, lambda c: 1.0)[0]
    b = step(lib, t, 200, lambda c: 1.0)[0]
    assert a >= 0 and b >= 0 and a != b
    # more keys than buckets: the least recently used ones are reused
    for k in range(1000, 1100):
        assert step(lib, t, k, lambda c: 1.0)[0] >= 0


def test_bucket_key_rounding(lib):
    k = lib.cvp9_tune_key
    assert k(0, 60, 30000) == k(0, 64, 32768)
    assert k(0, 64, 32768) != k(0, 65, 32768)
    assert k(0, 64, 32768) != k(0, 64, 32769)
    assert k(0, 64, 32768) != k(1, 64, 32768)


def test_a_challenger_needs_a_clear_win(lib):
    # every alternative is 1% faster than the default: noise, the default stays
    t = make(lib)
    for _ in range(20):
        idx, cfg = step(lib, t, 9, lambda c: 1.0 if c == (1, 0, 0) else 0.99)
        if idx < 0:
            break
    assert step(lib, t, 9, lambda c: 1.0) == (-1, (1, 0, 0))


def test_full_tunes_only_the_wavefront_width(lib):
    """FULL sends every superblock through the general kernel and has one
    loop-filter layout: whatever the fixed configuration asks, the inter path
    stays 0 and only the wavefront width is tried."""
    t = make(lib, arith=2, fixed=(1, 1, 0))
    seen = []
    for _ in range(20):
        idx, cfg = step(lib, t, 9, lambda c: 1.0 - 0.2 * c[2])
        if idx < 0:
            break
        if not seen or seen[-1] != cfg:
            seen.append(cfg)
    assert seen == [(0, 0, 0), (0, 0, 1)]
    assert step(lib, t, 9, lambda c: 1.0) == (-1, (0, 0, 1))
    t = make(lib, arith=2, enabled=0, fixed=(3, 1, 0))
    assert step(lib, t, 1, lambda c: 1.0) == (-1, (0, 0, 0))
