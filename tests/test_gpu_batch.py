"""Multi-stream engine: every stream of a mixed-resolution batch decodes to the
oracle's bytes, and the same frames decode identically alone and in the mix
(with and without graph replay, with host and device-resident inputs)."""
import ctypes as C

import numpy as np
import pytest

from compute_vp9_b200 import CVP9_OK, Synth, synth_config
from compute_vp9_b200.batch import DEVICE_INPUTS, Batch
from oracle.oracle_py import REFCPU, SPEC, OracleStream
from profiles import mix_for

pytestmark = pytest.mark.gpu

MIX = [
    (1, 320, 192, {}),
    (2, 352, 288, {"gop": 3}),
    (2, 200, 120, {"gop": 2, "min_bsize": 4, "skip_prob": 0.2, "intra_in_inter": 0.3}),
    (1, 257, 129, {"intra_in_inter": 0.1}),
    (2, 640, 360, {"gop": 4, "log2_tile_cols": 1}),
]


def decode_mix(profile, streams, frames, graphs=1, order=None, seeds=None, tuning=None):
    eng = Batch(arith=profile, use_graphs=graphs)
    streams = mix_for(profile, streams)
    seeds = seeds or [10 + i for i in range(len(streams))]
    syns = [Synth(synth_config(p, w, h, seed=seeds[i], **ov)) for i, (p, w, h, ov) in enumerate(streams)]
    sids = [eng.open_stream(w, h) for (_, w, h, _) in streams]
    assert all(s is not None for s in sids)
    outs = [[] for _ in streams]
    for f in range(frames):
        idx = order(f) if order else list(range(len(streams)))
        eng.submit([sids[i] for i in idx], [syns[i].frame(f) for i in idx], [f] * len(idx))
        assert eng.wait() == CVP9_OK, eng.last_error()
        for i in idx:
            rc, arr = eng.get_frame_array(sids[i])
            assert rc == CVP9_OK, (rc, eng.last_error())
            outs[i].append(arr)
    if tuning is not None:
        tuning.extend(eng.tuning())
    eng.close()
    return outs


@pytest.mark.parametrize("profile", [REFCPU, SPEC])
def test_batch_matches_oracle(profile):
    outs = decode_mix(profile, MIX, 4)
    for i, (p, w, h, ov) in enumerate(mix_for(profile, MIX)):
        syn = Synth(synth_config(p, w, h, seed=10 + i, **ov))
        orc = OracleStream(profile)
        for f in range(4):
            want = orc.decode(syn.frame(f))
            assert np.array_equal(outs[i][f], want), "stream %d frame %d" % (i, f)


@pytest.mark.parametrize("profile,variant", [(REFCPU, "0"), (REFCPU, "2"), (REFCPU, "3"), (REFCPU, "4"), (REFCPU, "5"),
                                             (SPEC, "0"), (SPEC, "2"), (SPEC, "3")])
def test_every_inter_path_matches_oracle(profile, variant, monkeypatch):
    """Each fixed inter path the tuner can pick (general kernel only, the
    80-register k_inter, the k_pred + k_resid split, REFCPU's split walking
    8x8 TXs per TX) decodes the mixed batch to the oracle's bytes."""
    monkeypatch.setenv("CVP9_AUTOTUNE", "0")
    monkeypatch.setenv("CVP9_INTER_FAST", variant)
    outs = decode_mix(profile, MIX, 3)
    for i, (p, w, h, ov) in enumerate(mix_for(profile, MIX)):
        syn = Synth(synth_config(p, w, h, seed=10 + i, **ov))
        orc = OracleStream(profile)
        for f in range(3):
            assert np.array_equal(outs[i][f], orc.decode(syn.frame(f))), "stream %d frame %d" % (i, f)


@pytest.mark.parametrize("profile", [REFCPU, SPEC])
def test_alone_equals_in_mix(profile):
    mixed = decode_mix(profile, MIX, 3, graphs=1)
    for i in range(len(MIX)):
        alone = decode_mix(profile, [MIX[i]], 3, graphs=0, seeds=[10 + i])
        for f in range(3):
            assert np.array_equal(alone[0][f], mixed[i][f]), "stream %d frame %d" % (i, f)


def test_device_inputs_and_pipelining():
    """Two steps in flight, parsed frames already on the device."""
    import torch
    p, w, h, ov = 1, 256, 192, {}
    syn = Synth(synth_config(p, w, h, seed=5, **ov))
    from compute_vp9_b200 import ParsedFrame, BlockInfo
    keep = []
    pfs = []
    for f in range(5):
        src = syn.frame(f).contents
        nb, nc = src.num_blocks, src.num_coeffs
        bt = torch.from_numpy(np.ctypeslib.as_array(C.cast(src.blocks, C.POINTER(C.c_uint8)),
                                                    shape=(nb * 32,)).copy()).cuda()
        ct = torch.from_numpy(np.ctypeslib.as_array(src.coeffs, shape=(nc,)).copy()).cuda()
        d = ParsedFrame()
        C.memmove(C.byref(d), C.byref(src), C.sizeof(ParsedFrame))
        d.blocks = C.cast(C.c_void_p(bt.data_ptr()), C.POINTER(BlockInfo))
        d.coeffs = C.cast(C.c_void_p(ct.data_ptr()), C.POINTER(C.c_int16))
        keep += [bt, ct]
        pfs.append(d)
    torch.cuda.synchronize()
    eng = Batch(arith=REFCPU)
    sid = eng.open_stream(w, h)
    for f in range(5):
        eng.submit([sid], [C.pointer(pfs[f])], [f], DEVICE_INPUTS)
    assert eng.wait() == CVP9_OK, eng.last_error()
    rc, got = eng.get_frame_array(sid)
    assert rc == CVP9_OK
    orc = OracleStream(REFCPU)
    syn2 = Synth(synth_config(p, w, h, seed=5, **ov))
    for f in range(5):
        want = orc.decode(syn2.frame(f))
    assert np.array_equal(got, want)
    eng.close()


def test_admission_budget():
    eng = Batch(arith=REFCPU, hbm_budget=3 * Batch(arith=REFCPU).stream_bytes(1920, 1080))
    ids = [eng.open_stream(1920, 1080) for _ in range(4)]
    assert ids[:3] == [0, 1, 2] and ids[3] is None
    eng.close_stream(1)
    assert eng.open_stream(1920, 1080) is not None     # the freed reservation admits one more
    assert eng.open_stream(1920, 1080) is None
    eng.close()


@pytest.mark.parametrize("profile", [REFCPU, SPEC])
def test_autotune_settles_with_oracle_output(profile):
    """The tuner runs every candidate configuration on real steps: each of
    those steps still decodes to the oracle's bytes, and the bucket settles
    after all knobs were measured (the inter paths — 4, REFCPU 6 — then
    filter layout and wavefront width: 6 configurations, REFCPU 8)."""
    tuning = []
    frames = 22
    outs = decode_mix(profile, MIX, frames, tuning=tuning)
    for i, (p, w, h, ov) in enumerate(mix_for(profile, MIX)):
        syn = Synth(synth_config(p, w, h, seed=10 + i, **ov))
        orc = OracleStream(profile)
        for f in range(frames):
            want = orc.decode(syn.frame(f))
            assert np.array_equal(outs[i][f], want), "stream %d frame %d" % (i, f)
    assert len(tuning) == 1, tuning
    e = tuning[0]
    assert e["settled"] == 1 and e["trials"] == (8 if profile == REFCPU else 6), e
    assert e["best_ms"] > 0 and e["lf_tile_h"] in (16, 32)
    assert e["inter_path"] in ((0, 1, 2, 3, 4, 5) if profile == REFCPU else (0, 1, 2, 3))


def _pinned_copy(pf, keep):
    """The parsed frame with its block and coefficient arrays copied into
    page-locked host memory (the engine then DMAs them directly and, under
    REFCPU, moves only the luma coefficients with its gather kernel)."""
    import torch
    from compute_vp9_b200 import BlockInfo, ParsedFrame
    p = pf.contents
    nb, nc = p.num_blocks, p.num_coeffs
    bt = torch.empty(max(1, nb * 32), dtype=torch.uint8, pin_memory=True)
    ct = torch.empty(max(1, nc), dtype=torch.int16, pin_memory=True)
    C.memmove(bt.data_ptr(), C.cast(p.blocks, C.c_void_p), nb * 32)
    C.memmove(ct.data_ptr(), C.cast(p.coeffs, C.c_void_p), nc * 2)
    out = ParsedFrame()
    C.memmove(C.byref(out), C.byref(p), C.sizeof(ParsedFrame))
    out.blocks = C.cast(C.c_void_p(bt.data_ptr()), C.POINTER(BlockInfo))
    out.coeffs = C.cast(C.c_void_p(ct.data_ptr()), C.POINTER(C.c_int16))
    keep += [bt, ct, out]
    return C.pointer(out)


@pytest.mark.parametrize("profile", [REFCPU, SPEC])
def test_pinned_inputs_match_oracle(profile):
    """Page-locked inputs take the direct upload path (REFCPU: the luma-only
    coefficient gather from host memory); every frame equals the oracle."""
    eng = Batch(arith=profile)
    syns = [Synth(synth_config(p, w, h, seed=30 + i, **ov)) for i, (p, w, h, ov) in enumerate(mix_for(profile, MIX))]
    orcs = [OracleStream(profile) for _ in MIX]
    sids = [eng.open_stream(w, h) for (_, w, h, _) in MIX]
    for f in range(4):
        keep = []
        pfs = [syn.frame(f) for syn in syns]
        eng.submit(sids, [_pinned_copy(pf, keep) for pf in pfs], [f] * len(MIX))
        assert eng.wait() == CVP9_OK, eng.last_error()
        for i in range(len(MIX)):
            rc, arr = eng.get_frame_array(sids[i])
            assert rc == CVP9_OK
            assert np.array_equal(arr, orcs[i].decode(pfs[i])), "stream %d frame %d" % (i, f)
    st = eng.stats()
    assert st.h2d_bytes > 0
    eng.close()


@pytest.mark.parametrize("pinned", [True, False])
@pytest.mark.parametrize("profile", [REFCPU, SPEC])
def test_sparse_coefficients_match_oracle(profile, pinned):
    """Coefficients given as (index, value) lists (cvp9_batch_submit_sparse)
    decode to the oracle's bytes, from page-locked and from pageable memory."""
    import torch
    from compute_vp9_b200.batch import CoeffList
    eng = Batch(arith=profile)
    syns = [Synth(synth_config(p, w, h, seed=50 + i, **ov)) for i, (p, w, h, ov) in enumerate(mix_for(profile, MIX))]
    orcs = [OracleStream(profile) for _ in MIX]
    sids = [eng.open_stream(w, h) for (_, w, h, _) in MIX]
    for f in range(3):
        keep, lists = [], []
        pfs = [syn.frame(f) for syn in syns]
        for pf in pfs:
            p = pf.contents
            dense = np.ctypeslib.as_array(p.coeffs, shape=(p.num_coeffs,)) if p.num_coeffs else np.zeros(0, np.int16)
            pos = np.nonzero(dense)[0].astype(np.uint32)
            val = dense[pos].astype(np.int16)
            if pinned:
                tp = torch.empty(max(1, pos.size), dtype=torch.int32, pin_memory=True)
                tv = torch.empty(max(1, val.size), dtype=torch.int16, pin_memory=True)
                tp.numpy()[:pos.size] = pos.view(np.int32)
                tv.numpy()[:val.size] = val
                keep += [tp, tv]
                lists.append(CoeffList(pos.size, tp.data_ptr(), tv.data_ptr()))
            else:
                keep += [pos, val]
                lists.append(CoeffList(pos.size, pos.ctypes.data, val.ctypes.data))
        eng.submit_sparse(sids, pfs, lists, [f] * len(MIX))
        assert eng.wait() == CVP9_OK, eng.last_error()
        for i in range(len(MIX)):
            rc, arr = eng.get_frame_array(sids[i])
            assert rc == CVP9_OK
            assert np.array_equal(arr, orcs[i].decode(pfs[i])), "stream %d frame %d" % (i, f)
    eng.close()


@pytest.mark.parametrize("pinned", [True, False])
@pytest.mark.parametrize("profile", [REFCPU, SPEC])
def test_packed_coefficients_match_oracle(profile, pinned):
    """Dense coefficient arrays packed on the host (cvp9_pack_coeffs) and
    rebuilt on the device (k_unpack_coeffs) decode to the oracle's bytes,
    from page-locked and from pageable memory, and move fewer bytes."""
    eng = Batch(arith=profile, pack=1)
    syns = [Synth(synth_config(p, w, h, seed=70 + i, **ov)) for i, (p, w, h, ov) in enumerate(mix_for(profile, MIX))]
    orcs = [OracleStream(profile) for _ in MIX]
    sids = [eng.open_stream(w, h) for (_, w, h, _) in MIX]
    for f in range(4):
        keep = []
        pfs = [syn.frame(f) for syn in syns]
        sub = [_pinned_copy(pf, keep) for pf in pfs] if pinned else pfs
        eng.submit(sids, sub, [f] * len(MIX))
        assert eng.wait() == CVP9_OK, eng.last_error()
        for i in range(len(MIX)):
            rc, arr = eng.get_frame_array(sids[i])
            assert rc == CVP9_OK
            assert np.array_equal(arr, orcs[i].decode(pfs[i])), "stream %d frame %d" % (i, f)
        dense = sum(pf.contents.num_coeffs * 2 + pf.contents.num_blocks * 32 for pf in pfs)
        st = eng.stats()
        assert 0 < st.h2d_bytes < dense
        assert st.kernel_launches >= 1
    eng.close()


@pytest.mark.parametrize("profile", [REFCPU, SPEC])
def test_launch_count_follows_inter_path(profile, monkeypatch):
    """kernel_launches counts the inter path's kernels in both profiles:
    k_inter + k_compact (path 1) or k_pred + k_resid + k_compact (path 3)
    on top of the general chain (path 0)."""
    monkeypatch.setenv("CVP9_AUTOTUNE", "0")
    counts = {}
    for variant in ("0", "1", "3", "5"):
        monkeypatch.setenv("CVP9_INTER_FAST", variant)
        eng = Batch(arith=profile, use_graphs=0)
        p, w, h, ov = mix_for(profile, [MIX[1]])[0]
        syn = Synth(synth_config(p, w, h, seed=10, **ov))
        sid = eng.open_stream(w, h)
        for f in range(2):
            eng.submit([sid], [syn.frame(f)], [f])
            assert eng.wait() == CVP9_OK, eng.last_error()
        counts[variant] = eng.stats().kernel_launches
        eng.close()
    assert counts["1"] - counts["0"] == 2, counts
    assert counts["3"] - counts["0"] == 3, counts
    # path 5 adds the second residual kernel under REFCPU; SPEC runs its split
    assert counts["5"] - counts["0"] == (4 if profile == REFCPU else 3), counts


@pytest.mark.parametrize("profile", [REFCPU, SPEC])
def test_stream_in_several_steps_in_flight(profile):
    """One stream submitted in consecutive steps without waiting (three in
    flight, next to a second stream that skips every other step): each
    frame is read back by its step (cvp9_batch_get_frame_at) and equals the
    oracle's; a step without the stream reports INVALID_DATA, the two newest
    frames stay readable, and a frame whose output area went to a step five
    later reports INVALID_DATA."""
    from compute_vp9_b200 import CVP9_ERR_AGAIN, CVP9_ERR_INVALID_DATA
    streams = mix_for(profile, [(2, 352, 288, {"gop": 4}), (1, 320, 192, {})])
    syns = [Synth(synth_config(p, w, h, seed=40 + i, **ov)) for i, (p, w, h, ov) in enumerate(streams)]
    orcs = [OracleStream(profile) for _ in streams]
    eng = Batch(arith=profile)
    sids = [eng.open_stream(w, h) for (_, w, h, _) in streams]
    frames = 9
    seqs = []                                  # (step seq, [stream indices])
    nxt = [0, 0]
    for t in range(frames):
        idx = [0] if t % 2 else [0, 1]
        eng.submit([sids[i] for i in idx], [syns[i].frame(nxt[i]) for i in idx], [nxt[i] for i in idx])
        seqs.append((eng.last_seq(), [(i, nxt[i]) for i in idx]))
        for i in idx:
            nxt[i] += 1
        if t >= 2:
            # read the frames of the step submitted two steps ago, while the
            # two newer steps holding the same stream may still run
            q, items = seqs[t - 2]
            for i, f in items:
                rc, arr = eng.get_frame_array_at(sids[i], q)
                while rc == CVP9_ERR_AGAIN:
                    rc, arr = eng.get_frame_array_at(sids[i], q)
                assert rc == CVP9_OK, (rc, eng.last_error())
                assert np.array_equal(arr, orcs[i].decode(syns[i].frame(f))), "stream %d frame %d" % (i, f)
            if 1 not in [i for i, _ in items]:
                assert eng.get_frame_at(sids[1], q)[0] == CVP9_ERR_INVALID_DATA
    assert eng.wait() == CVP9_OK, eng.last_error()
    for q, items in seqs[frames - 2:]:
        for i, f in items:
            rc, arr = eng.get_frame_array_at(sids[i], q)
            assert rc == CVP9_OK
            assert np.array_equal(arr, orcs[i].decode(syns[i].frame(f)))
    # the two newest frames stay readable; the first step's output area has
    # been given to step 6, so its frames are gone
    assert eng.get_frame_at(sids[0], seqs[-1][0])[0] == CVP9_OK
    assert eng.get_frame_at(sids[0], seqs[-2][0])[0] == CVP9_OK
    assert eng.get_frame_at(sids[0], seqs[0][0])[0] == CVP9_ERR_INVALID_DATA
    eng.close()


def test_reserve_takes_memory_up_front():
    """After cvp9_batch_reserve for six streams, opening four of them and
    running steps that hold each stream in several steps in flight takes
    nothing more from the driver (device or page-locked memory), and the
    frames still equal the oracle's."""
    eng = Batch(arith=REFCPU)
    eng.reserve(320, 192, 6)
    st0 = eng.stats()
    held = (st0.dev_held_bytes, st0.host_held_bytes)
    assert held[0] > 0 and held[1] > 0
    syns = [Synth(synth_config(1, 320, 192, seed=70 + i)) for i in range(4)]
    orcs = [OracleStream(REFCPU) for _ in range(4)]
    sids = [eng.open_stream(320, 192) for _ in range(4)]
    seqs = []
    for f in range(8):
        eng.submit(sids, [s.frame(f) for s in syns], [f] * 4)
        seqs.append(eng.last_seq())
    assert eng.wait() == CVP9_OK, eng.last_error()
    st = eng.stats()
    assert (st.dev_held_bytes, st.host_held_bytes) == held
    for f in range(8):
        for i in range(4):
            want = orcs[i].decode(syns[i].frame(f))
            if f >= 6:          # the two newest frames of each stream stay readable
                rc, arr = eng.get_frame_array_at(sids[i], seqs[f])
                assert rc == CVP9_OK and np.array_equal(arr, want)
    for sid in sids:
        eng.close_stream(sid)
    eng.close()
