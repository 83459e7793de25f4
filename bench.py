#!/usr/bin/env python
"""Benchmark: batched VP9 reconstruction on B200 vs single stream vs the
reference's CPU reconstruction.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

Workload (one step): one frame of each of 64 independent 1920x1080 8-bit
4:2:0 streams (seeds 0..63), content as in the reference's synthetic
benchmark shape — every 64x64 superblock split to 8x8 blocks, 8x8 DCT, q60,
~5% Laplacian coefficients (|v| <= 512), MVs uniform +-64 px in 1/8 pel from
LAST, loop-filter level 32. A key (intra) frame every GOP steps (default
100: the reference benchmark's stream has frame 0 intra of 100 frames), inter
frames between; the default 100 timed steps hold one key step. Each stream
cycles through 8 distinct parsed frames (the key frame, then 1..7 repeated);
the reference chain keeps evolving, so every step is real decode work.
Per-step inputs (~460 MB) and outputs (~200 MB) exceed the 126 MB L2, so no
flush is needed between steps.

value        device-resident: parsed frames already in HBM, K GOP-shaped
             steps timed with CUDA events on the engine's streams, max over
             ranks; value_inter / value_key time inter or key steps alone.
e2e          the same K steps through cvp9_batch_submit with the parsed
             frames in pinned host memory: upload, kernels and the download
             of every reconstructed frame inside the timed region; every
             stream's final frame is then checked against the reference's
             own compiled reconstruction.
value_spec   the same steps in the shader arithmetic; value_full the VP9
             (FULL) profile on mixed block/TX/filter content.
value_hbd    profile 2 (10-bit): 16 x 3840x2160 streams of the 10-bit
             config's content through the cvp9_hbd engine, GOP 120.
Single-stream figures come from the plain per-stream path on stream 0.
Each rank decodes its own 64 streams (weak scaling, no data-path collective).
"""
import argparse
import ctypes as C
import json
import os
import statistics
import subprocess
import sys
import threading
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "recon Mpixel/s batched-serving vs single-stream, 1 B200, bit-exact; p50/p99 ms"
UNIT = "Mpixel/s"
DISTINCT = 8


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=100)
    ap.add_argument("--gop", type=int, default=100,
                    help="key frame every GOP steps (the reference benchmark's stream: frame 0 intra of 100)")
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--streams", type=int, default=64)
    ap.add_argument("--width", type=int, default=1920)
    ap.add_argument("--height", type=int, default=1080)
    ap.add_argument("--arith", default="refcpu", choices=["refcpu", "spec", "full"])
    ap.add_argument("--no-spec", action="store_true", help="skip the shader-arithmetic leg")
    ap.add_argument("--no-full", action="store_true", help="skip the VP9 (FULL) leg")
    ap.add_argument("--no-hbd", action="store_true", help="skip the profile 2 (10-bit) leg")
    ap.add_argument("--hbd-streams", type=int, default=16)
    ap.add_argument("--hbd-checks", action="store_true",
                    help="with --leg hbd: also the CPU baseline and the parity check of the 10-bit leg")
    ap.add_argument("--no-capacity", action="store_true", help="skip the serving capacity sweeps")
    ap.add_argument("--no-cpu", action="store_true", help="skip the CPU baseline leg")
    ap.add_argument("--no-single", action="store_true", help="skip the single-stream leg")
    ap.add_argument("--no-graphs", action="store_true")
    ap.add_argument("--no-serve", action="store_true", help="skip the serving run")
    ap.add_argument("--no-parity", action="store_true", help="skip the bit-exactness check of the e2e run")
    ap.add_argument("--no-mixed", action="store_true",
                    help="skip the second batched run on mixed block/TX-size content")
    ap.add_argument("--leg", default=None, choices=["gop", "inter", "key", "mixed", "link", "hbd"],
                    help="run one device-resident leg alone and print its timing (profiler captures); "
                         "mixed = the mixed block/TX-size content, GOP 60; link = the PCIe copy probe "
                         "(each direction alone and both at once, as single copies and as the "
                         "per-frame pieces of a 64 x 1080p step)")
    ap.add_argument("--no-tune", action="store_true", help="with --leg: the tuner off (default kernels)")
    ap.add_argument("--serve-speed", type=float, default=4.0,
                    help="pacing compression of the serving run (1 = the config's real time)")
    return ap.parse_args()


def step_frame(t, mode="inter", gop=100):
    """Distinct parsed frame used at step t. "gop": a key frame every `gop`
    steps (t % gop == 0), inter frames between; "inter": the key frame at
    t = 0 only; "key": key frames only."""
    if mode == "key":
        return 0
    if mode == "gop":
        t %= gop
    return 0 if t == 0 else 1 + (t - 1) % (DISTINCT - 1)


# ── distributed plumbing ─────────────────────────────────────────────────────

def dist_setup(backend=None):
    """One process per GPU (torchrun env). NCCL when CUDA is present, gloo
    otherwise; used only for barriers and the max-over-ranks of the timings."""
    ws = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if ws > 1:
        import datetime
        import torch
        import torch.distributed as dist
        if backend is None:
            backend = "nccl" if torch.cuda.is_available() else "gloo"
        if backend == "nccl":
            torch.cuda.set_device(local)
        dist.init_process_group(backend, timeout=datetime.timedelta(seconds=300))
    return ws, rank, local


def barrier(ws):
    if ws > 1:
        import torch.distributed as dist
        dist.barrier()


def allreduce_max(ws, v):
    if ws <= 1:
        return v
    import torch
    import torch.distributed as dist
    dev = "cuda" if dist.get_backend() == "nccl" else "cpu"
    t = torch.tensor([float(v)], device=dev)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def rank_seeds(rank, streams):
    """Stream seeds of a rank: ranks decode disjoint sets of streams."""
    return list(range(rank * streams, (rank + 1) * streams))


# ── workload ─────────────────────────────────────────────────────────────────

class Workload:
    """S streams x DISTINCT parsed frames, copied into one pinned host arena;
    optional device copy. pfs_host[s][f] / pfs_dev[s][f] are ParsedFrame
    structs whose arrays live in those arenas."""

    def __init__(self, streams, w, h, device_copy=True, seeds=None, preset=1, overrides=None, gop=100):
        import numpy as np
        import torch
        from compute_vp9_b200 import ParsedFrame, Synth, synth_config
        self.S, self.w, self.h = streams, w, h
        self.gop, self.mode = gop, "gop"
        self.seeds = list(seeds) if seeds is not None else list(range(streams))
        self.preset, self.overrides = preset, dict(overrides or {})
        t0 = time.time()
        # pass 1: generate and measure
        frames = []
        seeds = seeds if seeds is not None else list(range(streams))
        for s in range(streams):
            syn = Synth(synth_config(preset, w, h, seed=seeds[s], **(overrides or {})))
            per = []
            for f in range(DISTINCT):
                pf = syn.frame(f).contents
                nb, nc = pf.num_blocks, pf.num_coeffs
                blocks = np.ctypeslib.as_array(C.cast(pf.blocks, C.POINTER(C.c_uint8)), shape=(nb * 32,)).copy()
                coeffs = np.ctypeslib.as_array(pf.coeffs, shape=(nc,)).copy()
                hdr = ParsedFrame()
                C.memmove(C.byref(hdr), C.byref(pf), C.sizeof(ParsedFrame))
                per.append((hdr, blocks, coeffs))
            syn.close()
            frames.append(per)
        self.gen_s = time.time() - t0
        total = 0
        offs = []
        for per in frames:
            o = []
            for hdr, blocks, coeffs in per:
                ob = total
                total += (blocks.nbytes + 255) // 256 * 256
                oc = total
                total += (coeffs.nbytes + 255) // 256 * 256
                o.append((ob, oc))
            offs.append(o)
        self.arena_bytes = total
        self.host = torch.empty(total, dtype=torch.uint8, pin_memory=torch.cuda.is_available())
        hv = self.host.numpy()
        for per, o in zip(frames, offs):
            for (hdr, blocks, coeffs), (ob, oc) in zip(per, o):
                hv[ob:ob + blocks.nbytes] = blocks
                hv[oc:oc + coeffs.nbytes] = coeffs.view(np.uint8)
        self.dev = None
        if device_copy:
            self.dev = torch.empty(total, dtype=torch.uint8, device="cuda")
            self.dev.copy_(self.host)
            torch.cuda.synchronize()
        hbase, dbase = self.host.data_ptr(), (self.dev.data_ptr() if self.dev is not None else 0)
        from compute_vp9_b200 import BlockInfo
        self.pfs_host, self.pfs_dev = [], []
        self.nnz_luma, self.num_blocks = [], []
        for per, o in zip(frames, offs):
            ph, pd, nz, nbk = [], [], [], []
            for (hdr, blocks, coeffs), (ob, oc) in zip(per, o):
                a = ParsedFrame()
                C.memmove(C.byref(a), C.byref(hdr), C.sizeof(ParsedFrame))
                a.blocks = C.cast(C.c_void_p(hbase + ob), C.POINTER(BlockInfo))
                a.coeffs = C.cast(C.c_void_p(hbase + oc), C.POINTER(C.c_int16))
                ph.append(a)
                if dbase:
                    d = ParsedFrame()
                    C.memmove(C.byref(d), C.byref(hdr), C.sizeof(ParsedFrame))
                    d.blocks = C.cast(C.c_void_p(dbase + ob), C.POINTER(BlockInfo))
                    d.coeffs = C.cast(C.c_void_p(dbase + oc), C.POINTER(C.c_int16))
                    pd.append(d)
                nz.append(self._luma_nnz(blocks, coeffs))
                nbk.append(hdr.num_blocks)
            self.pfs_host.append(ph)
            self.pfs_dev.append(pd)
            self.nnz_luma.append(nz)
            self.num_blocks.append(nbk)
        del frames

    def _luma_nnz(self, blocks, coeffs):
        """Nonzero coefficients the REFCPU path reads: the luma TXs of each
        non-skip block that fit the frame (vp9_reconstruct.c:336-347)."""
        import numpy as np
        b = blocks.reshape(-1, 32)
        x = b[:, 0].astype(np.int64) | (b[:, 1].astype(np.int64) << 8)
        y = b[:, 2].astype(np.int64) | (b[:, 3].astype(np.int64) << 8)
        w = np.minimum(b[:, 4].astype(np.int64), self.w - x)
        h = np.minimum(b[:, 5].astype(np.int64), self.h - y)
        n = 4 << b[:, 6].astype(np.int64)
        skip = b[:, 20] != 0
        off = (b[:, 24].astype(np.int64) | (b[:, 25].astype(np.int64) << 8) |
               (b[:, 26].astype(np.int64) << 16) | (b[:, 27].astype(np.int64) << 24))
        ln = np.where(skip, 0, (w // n) * (h // n) * n * n)
        nzc = np.concatenate([[0], np.cumsum(coeffs != 0)])
        return int((nzc[off + ln] - nzc[off]).sum())

    def build_sparse(self):
        """(index, value) lists of every frame's nonzero coefficients in one
        page-locked arena — what a parser emitting coefficients as it decodes
        tokens would hand over; built once, outside any timed region."""
        import numpy as np
        import torch
        from compute_vp9_b200.batch import CoeffList
        hv = self.host.numpy()
        hbase = self.host.data_ptr()
        per_frame = []
        total = 0
        for s in range(self.S):
            row = []
            for f in range(DISTINCT):
                pf = self.pfs_host[s][f]
                oc = C.cast(pf.coeffs, C.c_void_p).value - hbase
                dense = hv[oc:oc + 2 * pf.num_coeffs].view(np.int16)
                pos = np.nonzero(dense)[0].astype(np.uint32)
                row.append((pos, dense[pos]))
                total += (pos.nbytes + 255) // 256 * 256 + (pos.size * 2 + 255) // 256 * 256
            per_frame.append(row)
        self.sparse_arena = torch.empty(max(1, total), dtype=torch.uint8, pin_memory=torch.cuda.is_available())
        av = self.sparse_arena.numpy()
        base = self.sparse_arena.data_ptr()
        off = 0
        self.lists = []
        for row in per_frame:
            lr = []
            for pos, val in row:
                op = off
                av[op:op + pos.nbytes] = pos.view(np.uint8)
                off += (pos.nbytes + 255) // 256 * 256
                ov = off
                av[ov:ov + val.nbytes] = val.view(np.uint8)
                off += (val.nbytes + 255) // 256 * 256
                lr.append(CoeffList(pos.size, base + op, base + ov))
            self.lists.append(lr)

    def frame_of(self, t):
        return step_frame(t, self.mode, self.gop)

    def step_lists(self, t):
        f = self.frame_of(t)
        return [self.lists[s][f] for s in range(self.S)]

    def step_pfs(self, t, device):
        f = self.frame_of(t)
        src = self.pfs_dev if device else self.pfs_host
        return [C.pointer(src[s][f]) for s in range(self.S)]

    def alg_bytes(self, t):
        """Algorithmic bytes of one step: recon write 1.5*W*H, reference read
        1.5*W*H on inter frames, 4 bytes per nonzero coefficient read, 32 per
        block descriptor (no NV12 target armed)."""
        f = self.frame_of(t)
        px = self.w * self.h
        inter = 1 if f != 0 else 0
        tot = 0
        for s in range(self.S):
            tot += 1.5 * px + 1.5 * px * inter + 4 * self.nnz_luma[s][f] + 32 * self.num_blocks[s][f]
        return tot


# ── clocks ───────────────────────────────────────────────────────────────────

class ClockSampler:
    QUERY = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index):
        self.gpu = gpu_index
        self.samples = []
        self._stop = threading.Event()
        self._t = None

    def _run(self):
        while not self._stop.is_set():
            try:
                out = subprocess.run(["nvidia-smi", "-i", str(self.gpu), "--query-gpu=" + self.QUERY,
                                      "--format=csv,noheader,nounits"], capture_output=True,
                                     text=True, timeout=5).stdout.strip()
                if out:
                    self.samples.append([x.strip() for x in out.split(",")])
            except Exception:
                pass
            self._stop.wait(0.2)

    def __enter__(self):
        # the first nvidia-smi of a fresh box is slow and was seen to stall
        # the GPU work beside it: take one sample before anything is timed
        self._stop.clear()
        t0 = time.perf_counter()
        self._t = threading.Thread(target=self._run, daemon=True)
        self._t.start()
        while not self.samples and self._t.is_alive() and time.perf_counter() - t0 < 10.0:
            time.sleep(0.01)
        return self

    def __exit__(self, *a):
        self._stop.set()
        self._t.join(timeout=10)

    def summary(self):
        if not self.samples:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}
        mhz = [float(s[1]) for s in self.samples if s[1].replace(".", "").isdigit()]
        mx = [float(s[2]) for s in self.samples if s[2].replace(".", "").isdigit()]
        reasons = set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for s in self.samples:
            for i, n in enumerate(names):
                if len(s) > 5 + i and s[5 + i].lower().startswith("active"):
                    reasons.add(n)
        return {"sm_mhz": statistics.median(mhz) if mhz else None,
                "sm_max_mhz": max(mx) if mx else None, "reasons": sorted(reasons),
                "samples": len(self.samples)}


# ── legs ─────────────────────────────────────────────────────────────────────

def run_batched(wl, steps, warmup, arith, device_inputs, graphs, ws, tuned=None, sparse=False, pack=0,
                final=False, tune=True):
    """K timed steps of all streams in the workload's schedule (wl.mode).
    The engine's tuner first settles this shape's kernel configuration on
    untimed steps; `tuned` receives its choice. Returns a dict: ms (timed
    region), stats (last timed step), prof (per-phase device times of three
    more steps), lat (host latencies), seq (the step indices submitted, in
    order) and, with final=True, outs: every stream's frame after one more
    step that downloads its outputs (the bit-exactness check replays seq)."""
    import torch
    from compute_vp9_b200.batch import DEVICE_INPUTS, NO_OUTPUT, Batch
    eng = Batch(arith=arith, use_graphs=1 if graphs else 0, autotune=1 if tune else 0, pack=pack)
    sids = [eng.open_stream(wl.w, wl.h) for _ in range(wl.S)]
    assert all(s is not None for s in sids), "admission refused"
    flags = (DEVICE_INPUTS | NO_OUTPUT) if device_inputs else 0
    seq = []

    def submit(t, fl=None):
        seq.append(t)
        if sparse:
            eng.submit_sparse(sids, wl.step_pfs(t, False), wl.step_lists(t), [t] * wl.S, flags)
        else:
            eng.submit(sids, wl.step_pfs(t, device_inputs), [t] * wl.S, flags if fl is None else fl)
    for t in range(40):
        submit(t)
        assert eng.wait() == 0, eng.last_error()
        if all(e["settled"] for e in eng.tuning()):
            break
    if tuned is not None:
        tuned.extend(eng.tuning())
    for t in range(warmup):
        submit(t)
    rc = eng.wait()
    assert rc == 0, eng.last_error()
    torch.cuda.synchronize()
    barrier(ws)
    torch.cuda.synchronize()
    seq0 = eng.last_seq()
    eng.timer_start()
    for t in range(warmup, warmup + steps):
        submit(t)
    ms = eng.timer_stop()
    rc = eng.wait()
    assert rc == 0, eng.last_error()
    torch.cuda.synchronize()
    barrier(ws)
    lat = [eng.step_latency_ms(q) for q in range(seq0 + 1, seq0 + steps + 1)]
    last = eng.stats()
    # per-kernel device times: a few more steps, each waited for
    prof = []
    t_next = warmup + steps
    for t in range(t_next, t_next + 3):
        submit(t)
        eng.wait()
        st = eng.stats()
        prof.append((st.scan_ms, st.recon_ms, st.filter_ms, st.kernels_ms, st.step_ms))
    t_next += 3
    outs = None
    if final:
        submit(t_next, DEVICE_INPUTS if device_inputs else 0)
        assert eng.wait() == 0, eng.last_error()
        outs = []
        for sid in sids:
            rc, arr = eng.get_frame_array(sid)
            outs.append(arr if rc == 0 else None)
    eng.close()
    return {"ms": ms, "stats": last, "prof": prof, "lat": [x for x in lat if x is not None],
            "seq": seq, "outs": outs}


def check_parity(wl, seq, outs, profile, streams, threads):
    """Replay each listed stream's submitted sequence on the CPU (from its
    last key frame, which refreshes every reference slot) and compare the
    final frame byte for byte. REFCPU replays through the reference's own
    compiled reconstruction (oracle/_ref) when it is built, otherwise and for
    SPEC/FULL through the restatement. Returns the JSON record."""
    from concurrent.futures import ThreadPoolExecutor
    from oracle.oracle_py import FULL, REFCPU, SPEC, OracleStream, RefStream, ref_available
    use_ref = profile == REFCPU and ref_available()
    frames = [wl.frame_of(t) for t in seq]
    start = max(i for i, f in enumerate(frames) if f == 0)

    def one(s):
        chk = RefStream() if use_ref else OracleStream(profile)
        want = None
        for f in frames[start:]:
            want = chk.decode(C.pointer(wl.pfs_host[s][f]))
        chk.close()
        return outs[s] is not None and bool((want == outs[s]).all())

    with ThreadPoolExecutor(max(1, min(threads, len(streams)))) as ex:
        ok = list(ex.map(one, streams))
    return {"streams_checked": len(streams), "streams_bit_exact": int(sum(ok)),
            "frames_replayed_per_stream": len(frames) - start,
            "checked": "final frame of each checked stream after the run's %d submitted steps, replayed "
                       "on the CPU from the last key frame" % len(frames),
            "against": "oracle/_ref (the reference's vp9_reconstruct_frame)" if use_ref
                       else "oracle restatement (%s)" % {REFCPU: "REFCPU", SPEC: "SPEC", FULL: "FULL"}[profile],
            "bit_exact": all(ok)}


def run_single_plain(wl, frames, arith):
    """Plain per-stream backend (the drop-in ABI) on stream 0, host inputs,
    frames in the workload's schedule."""
    from compute_vp9_b200 import CVP9_OK, CudaBackend
    be = CudaBackend(arith=arith)
    # warm-up: key frame + the frames the backend's tuner measures on
    warm = 14
    for t in range(warm):
        assert be.decode(C.pointer(wl.pfs_host[0][wl.frame_of(t)]), t) == CVP9_OK
        rc, _ = be.get_frame(1)
        assert rc == CVP9_OK, be.last_error()
    t0 = time.perf_counter()
    pending = 0
    for t in range(warm, warm + frames):
        rc = be.decode(C.pointer(wl.pfs_host[0][wl.frame_of(t)]), t)
        if rc == -6:  # ring full: deliver the oldest, then resubmit
            r2, _ = be.get_frame(1)
            assert r2 == CVP9_OK
            pending -= 1
            rc = be.decode(C.pointer(wl.pfs_host[0][wl.frame_of(t)]), t)
        assert rc == CVP9_OK, be.last_error()
        pending += 1
    while pending:
        r2, _ = be.get_frame(1)
        assert r2 == CVP9_OK
        pending -= 1
    dt = time.perf_counter() - t0
    total_ms, kern_ms = be.last_timing()
    be.close()
    return frames * wl.w * wl.h / dt / 1e6, kern_ms


def cpu_leg(wl, threads, target_s=12.0):
    """Reference CPU reconstruction (oracle/_ref, else the restatement) on host
    cores, one stream per thread; returns (Mpx/s, kind, cores, sample)."""
    from concurrent.futures import ThreadPoolExecutor
    from oracle import oracle_py as O
    kind = "reference" if O.ref_available() else "port"
    mk = (lambda: O.RefStream()) if kind == "reference" else (lambda: O.OracleStream(O.REFCPU))
    threads = max(1, min(threads, wl.S))
    # calibrate one inter frame
    s0 = mk()
    s0.decode(C.pointer(wl.pfs_host[0][0]))
    t = time.perf_counter()
    s0.decode(C.pointer(wl.pfs_host[0][1]))
    per = time.perf_counter() - t
    s0.close()
    per_thread = max(1, min(DISTINCT - 1, int(target_s / per / threads)))

    def work(s):
        st = mk()
        st.decode(C.pointer(wl.pfs_host[s][0]))
        t0 = time.perf_counter()
        for k in range(per_thread):
            st.decode(C.pointer(wl.pfs_host[s][1 + k % (DISTINCT - 1)]))
        dt = time.perf_counter() - t0
        st.close()
        return dt

    t0 = time.perf_counter()
    with ThreadPoolExecutor(threads) as ex:
        list(ex.map(work, range(threads)))
    wall = time.perf_counter() - t0
    px = threads * per_thread * wl.w * wl.h
    sample = ("%d streams x %d inter frames of %dx%d (one stream per thread, key frame untimed)"
              % (threads, per_thread, wl.w, wl.h))
    return px / wall / 1e6, kind, threads, sample


def host_cores():
    try:
        return len(os.sched_getaffinity(0))
    except Exception:
        return os.cpu_count() or 1


def read_peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    try:
        with open(p) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


def read_traffic(split=False):
    """Per-step DRAM bytes of the warp-per-superblock recon kernels (k_inter,
    or k_pred + k_resid) at the bench workload, from the committed ncu
    summary."""
    name = "k_pred_k_resid_refcpu_1080p_x16.md" if split else "k_inter_refcpu_1080p_x16.md"
    p = os.path.join(ROOT, "profiles", name)
    try:
        with open(p) as f:
            for line in f:
                if line.startswith("traffic_bytes_per_launch_full:"):
                    return float(line.split(":")[1].strip())
    except Exception:
        pass
    return None


# ── arms ─────────────────────────────────────────────────────────────────────

def reference_arm(args, ws, rank):
    if rank != 0:
        return
    from concurrent.futures import ThreadPoolExecutor
    from oracle import oracle_py as O
    kind = "reference" if O.ref_available() else "port"
    wl = Workload(args.streams, args.width, args.height, device_copy=False, gop=args.gop)
    cores = host_cores()
    threads = min(cores, wl.S)
    mk = (lambda: O.RefStream()) if kind == "reference" else (lambda: O.OracleStream(O.REFCPU))
    streams = [mk() for _ in range(wl.S)]

    def one(args_):
        s, t = args_
        streams[s].decode(C.pointer(wl.pfs_host[s][wl.frame_of(t)]))

    with ThreadPoolExecutor(threads) as ex:
        for t in range(args.warmup):
            list(ex.map(one, [(s, t) for s in range(wl.S)]))
        t0 = time.perf_counter()
        for t in range(args.warmup, args.warmup + args.steps):
            list(ex.map(one, [(s, t) for s in range(wl.S)]))
        dt = time.perf_counter() - t0
    for s in streams:
        s.close()
    value = args.steps * wl.S * wl.w * wl.h / dt / 1e6
    sample = "%d steps x %d streams x %dx%d inter frames on %d host threads" % (
        args.steps, wl.S, wl.w, wl.h, threads)
    line = {
        "impl": "reference", "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": args.gpus,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": dt * 1000 / args.steps,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "u8",
        "data": "synthetic", "config": workload_config(args),
        "cpu_baseline": {"value": value, "unit": UNIT, "cores": threads, "kind": kind, "sample": sample},
        "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


def workload_config(args):
    return {
        "workload": "batched: %d x %dx%d 8-bit 4:2:0 streams, one frame per stream per step "
                    "(8x8 blocks, TX 8x8, q60, 5%% coeffs, +-64 px MVs from LAST, LF 32; "
                    "seeds 0..%d; a key frame every %d steps, inter frames between; %d distinct parsed "
                    "frames per stream, cycled)"
                    % (args.streams, args.width, args.height, args.streams - 1, args.gop, DISTINCT),
        "streams_per_gpu": args.streams, "width": args.width, "height": args.height, "gop": args.gop,
        "arith": args.arith, "l2": "per-step inputs+outputs exceed L2 (no flush needed)",
        "parallelism": "streams sharded per GPU (replicas, no collective)",
    }


def px_rate(wl, steps, ms, ws=1):
    return ws * wl.S * wl.w * wl.h * steps / (ms / 1000.0) / 1e6


def leg_roofline(wl, r, steps, warmup, peak):
    """Achieved algorithmic GB/s of the recon phase of the three profiling
    steps after the timed region, and its fraction of the peak."""
    recon_ms = statistics.mean(p[1] for p in r["prof"])
    alg = statistics.mean(wl.alg_bytes(t) for t in range(warmup + steps, warmup + steps + 3))
    ach = alg / (recon_ms / 1000.0) / 1e9
    return {"recon_ms": recon_ms, "alg_bytes_per_launch": alg, "achieved_gbs": ach, "frac": ach / peak}


# ── profile 2 (10-bit) ───────────────────────────────────────────────────────

HBD_GOP = 120
HBD_DISTINCT = 3
# the 10-bit config's content: 3840x2160, 32x32 TX on half the blocks, 10%
# coefficients dequantised up to +-2^17, +-256 px MVs, the sharp filter,
# LAST/GOLDEN/ALTREF, loop-filter level per frame
HBD_CONTENT = dict(gop=HBD_GOP, tx_weights=[10, 15, 25, 50], density_min=0.10, density_max=0.10,
                   mv_range_px=256, interp_filter=2, nrefs=3, lf_level=-1, intra_in_inter=0.0)
HBD_STEP = 288      # dequantiser step of the synthetic levels: |level| <= 512 -> +-2^17


class HbdWorkload:
    """S streams x HBD_DISTINCT 10-bit frames (a key frame, then inter frames
    cycled), block records and int32 coefficients in one pinned host arena
    and one device copy."""

    def __init__(self, streams, w, h, seeds):
        import numpy as np
        import torch
        from compute_vp9_b200 import BlockInfo, ParsedFrame, Synth, synth_config
        from compute_vp9_b200.hbd import dequantise10
        self.S, self.w, self.h = streams, w, h
        per_stream = []
        for s in range(streams):
            syn = Synth(synth_config(2, w, h, seed=seeds[s], **HBD_CONTENT))
            per = []
            for f in range(HBD_DISTINCT):
                pfp = syn.frame(f)
                pfp.contents.hdr.bit_depth = 10
                pfp.contents.hdr.profile = 2
                pf = pfp.contents
                blocks = np.ctypeslib.as_array(C.cast(pf.blocks, C.POINTER(C.c_uint8)),
                                               shape=(pf.num_blocks * 32,)).copy()
                c32 = dequantise10(pfp, HBD_STEP)
                hdr = ParsedFrame()
                C.memmove(C.byref(hdr), C.byref(pf), C.sizeof(ParsedFrame))
                per.append((hdr, blocks, c32))
            syn.close()
            per_stream.append(per)
        total, offs = 0, []
        for per in per_stream:
            o = []
            for hdr, blocks, c32 in per:
                ob = total
                total += (blocks.nbytes + 255) // 256 * 256
                oc = total
                total += (c32.nbytes + 255) // 256 * 256
                o.append((ob, oc))
            offs.append(o)
        self.host = torch.empty(total, dtype=torch.uint8, pin_memory=True)
        hv = self.host.numpy()
        for per, o in zip(per_stream, offs):
            for (hdr, blocks, c32), (ob, oc) in zip(per, o):
                hv[ob:ob + blocks.nbytes] = blocks
                hv[oc:oc + c32.nbytes] = c32.view(np.uint8)
        self.dev = torch.empty(total, dtype=torch.uint8, device="cuda")
        self.dev.copy_(self.host)
        torch.cuda.synchronize()
        hb, db = self.host.data_ptr(), self.dev.data_ptr()
        self.frames = []        # [s][f] -> (pf host, pf device, coeffs host, coeffs device)
        self.nnz, self.nblocks = [], []
        for per, o in zip(per_stream, offs):
            row, nz, nb = [], [], []
            for (hdr, blocks, c32), (ob, oc) in zip(per, o):
                ph, pd = ParsedFrame(), ParsedFrame()
                for dst, base in ((ph, hb), (pd, db)):
                    C.memmove(C.byref(dst), C.byref(hdr), C.sizeof(ParsedFrame))
                    dst.blocks = C.cast(C.c_void_p(base + ob), C.POINTER(BlockInfo))
                    dst.coeffs = None
                row.append((ph, pd, hb + oc, db + oc))
                nz.append(int(np.count_nonzero(c32)))
                nb.append(hdr.num_blocks)
            self.frames.append(row)
            self.nnz.append(nz)
            self.nblocks.append(nb)
        # the int32 coefficients as views of the pinned arena (the CPU leg)
        self.c32 = [[hv[oc:oc + c32.nbytes].view(np.int32) for (_, _, c32), (ob, oc) in zip(per, o)]
                    for per, o in zip(per_stream, offs)]
        # the nonzero coefficients as (index, value) lists, in pinned memory
        # (what a parser emitting them as it decodes tokens would hand over)
        lists, total = [], 0
        for per in per_stream:
            row = []
            for hdr, blocks, c32 in per:
                pos = np.nonzero(c32[:hdr.num_coeffs])[0].astype(np.uint32)
                row.append((pos, c32[pos].astype(np.int32)))
                total += 2 * ((pos.nbytes + 255) // 256 * 256)
            lists.append(row)
        self.sparse = torch.empty(max(total, 1), dtype=torch.uint8, pin_memory=True)
        sv, sb, off = self.sparse.numpy(), self.sparse.data_ptr(), 0
        self.lists = []
        for row in lists:
            lr = []
            for pos, val in row:
                op = off
                sv[op:op + pos.nbytes] = pos.view(np.uint8)
                off += (pos.nbytes + 255) // 256 * 256
                ov = off
                sv[ov:ov + val.nbytes] = val.view(np.uint8)
                off += (val.nbytes + 255) // 256 * 256
                lr.append((pos.size, sb + op, sb + ov))
            self.lists.append(lr)

    @staticmethod
    def frame_of(t):
        t %= HBD_GOP
        return 0 if t == 0 else 1 + (t - 1) % (HBD_DISTINCT - 1)

    def step(self, t, device):
        f = self.frame_of(t)
        return [(C.pointer(self.frames[s][f][1 if device else 0]), self.frames[s][f][3 if device else 2])
                for s in range(self.S)]

    def step_lists(self, t):
        f = self.frame_of(t)
        return [C.pointer(self.frames[s][f][0]) for s in range(self.S)], [self.lists[s][f] for s in range(self.S)]

    def alg_bytes(self, t):
        """One step's algorithmic bytes: the 16-bit frame written (3*W*H), the
        reference read on inter frames (3*W*H), 4 bytes per nonzero
        dequantised coefficient, 32 per block record."""
        f = self.frame_of(t)
        px = self.w * self.h
        return sum(3 * px * (2 if f else 1) + 4 * self.nnz[s][f] + 32 * self.nblocks[s][f] for s in range(self.S))


def run_hbd(wl, steps, warmup, device_inputs, sparse=False):
    """W warm-up steps, then K timed steps t = 0..K-1 of the GOP schedule (a
    key frame at t = 0) submitted back to back — the engine keeps two in
    flight, so one step's download, the next one's kernels and the upload
    of the one after overlap — timed with the engine's CUDA events from
    before the first upload to after the last download. Then three inter
    steps one at a time give the per-phase device times."""
    from compute_vp9_b200.hbd import HBD_DEVICE_INPUTS, HBD_NO_OUTPUT, HbdEngine
    eng = HbdEngine()
    sids = [eng.open_stream(wl.w, wl.h) for _ in range(wl.S)]
    flags = (HBD_DEVICE_INPUTS | HBD_NO_OUTPUT) if device_inputs else 0

    def submit(t):
        if sparse:
            pfs, lists = wl.step_lists(t)
            return eng.submit_sparse(sids, pfs, lists, flags=flags)
        return eng.submit(sids, wl.step(t, device_inputs), flags=flags)
    for t in range(warmup):
        assert submit(t) == 0
    assert eng.wait() == 0
    assert eng.timer_start() == 0
    t0 = time.perf_counter()
    for t in range(steps):
        assert submit(t) == 0
    ms = eng.timer_stop()
    assert eng.wait() == 0
    wall = (time.perf_counter() - t0) * 1000.0
    parts, recon, alg = [0.0] * 5, [], []
    for t in range(HBD_GOP + 1, HBD_GOP + 4):
        assert submit(t) == 0
        assert eng.wait() == 0
        m = eng.step_times()
        parts = [a + b for a, b in zip(parts, m)]
        recon.append(m[2])
        alg.append(wl.alg_bytes(t))
    eng.close()
    return {"ms": ms, "wall_ms": wall, "parts": [p / 3 for p in parts], "recon": recon, "alg": alg}


def hbd_live(wl, steps=60, fps=30.0):
    """The streams served live: every 1/fps s one frame of each is due (a
    step through cvp9_hbd_submit_sparse from host memory, frames
    downloaded); latency = due time -> the step's frames in host memory
    (host clock)."""
    from compute_vp9_b200.hbd import HbdEngine
    eng = HbdEngine()
    sids = [eng.open_stream(wl.w, wl.h) for _ in range(wl.S)]
    for t in range(3):
        pfs, lists = wl.step_lists(t)
        assert eng.submit_sparse(sids, pfs, lists) == 0
    assert eng.wait() == 0
    lat = []
    t0 = time.perf_counter() + 0.05
    for t in range(steps):
        due = t0 + t / fps
        now = time.perf_counter()
        if now < due:
            time.sleep(due - now)
        pfs, lists = wl.step_lists(t)
        assert eng.submit_sparse(sids, pfs, lists) == 0
        assert eng.wait() == 0
        lat.append((time.perf_counter() - due) * 1000.0)
    eng.close()
    s = sorted(lat)
    return {"streams": wl.S, "fps": fps, "steps": steps, "p50_ms": statistics.median(s),
            "p99_ms": s[min(len(s) - 1, int(0.99 * len(s)))], "offered": wl.S * wl.w * wl.h * fps / 1e6,
            "unit": UNIT, "what": "every stream live at 30 fps, one step per frame period, inputs as "
                                  "(index, value) lists from host memory, frames downloaded"}


def hbd_cpu(wl, threads):
    """The 10-bit restatement (oracle/oracle_hbd.c; the reference has no 10-bit
    path) on host cores, one stream per thread: its key frame untimed, then
    one inter frame each, timed from the moment every thread has its key
    frame. Returns (Mpx/s, threads, sample)."""
    import threading
    from concurrent.futures import ThreadPoolExecutor
    from oracle.oracle_py import HbdOracleStream
    threads = max(1, min(threads, wl.S))
    ready = threading.Barrier(threads)

    def work(s):
        o = HbdOracleStream()
        o.decode(C.pointer(wl.frames[s][0][0]), wl.c32[s][0])
        ready.wait()
        t0 = time.perf_counter()
        o.decode(C.pointer(wl.frames[s][1][0]), wl.c32[s][1])
        t1 = time.perf_counter()
        o.close()
        return t0, t1
    with ThreadPoolExecutor(threads) as ex:
        spans = list(ex.map(work, range(threads)))
    wall = max(t1 for _, t1 in spans) - min(t0 for t0, _ in spans)
    return (threads * wl.w * wl.h / wall / 1e6, threads,
            "%d streams x 1 inter frame of %dx%d 10-bit (one stream per thread, key frame untimed)"
            % (threads, wl.w, wl.h))


def hbd_parity(streams=2, frames=3, seed0=1000):
    """Fresh 10-bit streams of the same content, every frame downloaded and
    compared with the 10-bit restatement (oracle/oracle_hbd.c)."""
    import numpy as np
    from compute_vp9_b200.hbd import HbdEngine, hbd_frames
    from oracle.oracle_py import HbdOracleStream
    eng = HbdEngine()
    sids = [eng.open_stream(3840, 2160) for _ in range(streams)]
    gens = [hbd_frames(2, 3840, 2160, frames, seed=seed0 + s, step=HBD_STEP, **HBD_CONTENT) for s in range(streams)]
    orcs = [HbdOracleStream() for _ in range(streams)]
    bad = 0
    for f in range(frames):
        fr = [next(g) for g in gens]
        want = [o.decode(pf, c) for o, (pf, c) in zip(orcs, fr)]
        assert eng.submit(sids, [(pf, c.ctypes.data) for pf, c in fr]) == 0
        assert eng.wait() == 0
        bad += sum(0 if np.array_equal(eng.get_frame(sid), w) else 1 for sid, w in zip(sids, want))
    eng.close()
    return {"streams_checked": streams, "frames_each": frames, "frames_mismatched": bad,
            "bit_exact": bad == 0, "against": "oracle/oracle_hbd.c (10-bit restatement, unpinned)"}


def hbd_leg(args, rank, peak, parity=True):
    seeds = [rank * args.hbd_streams + s for s in range(args.hbd_streams)]
    wl = HbdWorkload(args.hbd_streams, 3840, 2160, seeds)
    steps = max(args.steps, HBD_GOP) if not args.leg else args.steps
    R = run_hbd(wl, steps, args.warmup, True)
    E = run_hbd(wl, min(steps, 30), args.warmup, False)
    Es = run_hbd(wl, min(steps, 30), args.warmup, False, sparse=True)
    px = wl.S * wl.w * wl.h
    recon_ms = statistics.mean(R["recon"])            # inter steps
    alg = statistics.mean(R["alg"])
    out = {"workload": "%d x 3840x2160 10-bit 4:2:0 streams, TX 4x4..32x32 weighted 10/15/25/50, 10%% "
                       "coefficients dequantised up to +-2^17, +-256 px MVs, sharp filter, LAST/GOLDEN/ALTREF, "
                       "a key frame every %d steps; %d timed steps from a key frame" % (wl.S, HBD_GOP, steps),
           "value": px * steps / (R["ms"] / 1000.0) / 1e6, "unit": UNIT, "ms_per_step": R["ms"] / steps,
           "wall_ms_per_step": R["wall_ms"] / steps,
           "device_ms_per_inter_step": dict(zip(("upload", "scan", "recon", "filter", "download"), R["parts"])),
           "e2e": {"value": px * min(steps, 30) / (E["ms"] / 1000.0) / 1e6, "unit": UNIT,
                   "ms_per_step": E["ms"] / min(steps, 30),
                   "device_ms_per_inter_step": dict(zip(("upload", "scan", "recon", "filter", "download"),
                                                        E["parts"])),
                   "what": "cvp9_hbd_submit from page-locked host arrays (block records + dense int32 "
                           "coefficients up, every 16-bit frame down), two steps in flight, timed on the "
                           "engine's CUDA events"},
           "e2e_sparse_input": {"value": px * min(steps, 30) / (Es["ms"] / 1000.0) / 1e6, "unit": UNIT,
                                "ms_per_step": Es["ms"] / min(steps, 30),
                                "device_ms_per_inter_step": dict(zip(("upload", "scan", "recon", "filter",
                                                                      "download"), Es["parts"])),
                                "what": "as e2e, the coefficients as (index, value) lists through "
                                        "cvp9_hbd_submit_sparse (8 bytes per nonzero coefficient up)"},
           "roofline": {"bound": "hbm", "kernel": "k_hbd_recon (inter steps)", "achieved": alg / (recon_ms / 1e3) / 1e9,
                        "peak": peak, "unit": "GB/s", "frac": alg / (recon_ms / 1e3) / 1e9 / peak,
                        "alg_bytes_per_launch": alg, "launch_ms": recon_ms},
           "dtype": "u16 samples, int64 butterflies"}
    out["live"] = hbd_live(wl)
    if parity:
        v, th, sample = hbd_cpu(wl, host_cores())
        out["cpu_port"] = {"value": v, "unit": UNIT, "cores": th, "kind": "port", "sample": sample}
        out["parity"] = hbd_parity()
    return out


def hbd_leg_process(args):
    """The 10-bit leg (HBD_GOP timed steps, CPU baseline and parity) in a
    fresh process on this GPU; returns its JSON record."""
    cmd = [sys.executable, os.path.abspath(__file__), "--leg", "hbd", "--steps", str(max(args.steps, HBD_GOP)),
           "--warmup", str(args.warmup), "--hbd-streams", str(args.hbd_streams), "--hbd-checks"]
    env = dict(os.environ)
    for k in ("RANK", "WORLD_SIZE", "LOCAL_RANK", "MASTER_ADDR", "MASTER_PORT"):
        env.pop(k, None)
    p = subprocess.run(cmd, capture_output=True, text=True, timeout=1200, env=env)
    lines = [ln for ln in p.stdout.splitlines() if ln.startswith("{")]
    if p.returncode != 0 or not lines:
        return {"error": "10-bit leg exited %d" % p.returncode, "stderr_tail": p.stderr[-2000:]}
    out = json.loads(lines[-1])
    out["process"] = "its own (bench.py --leg hbd --hbd-checks)"
    return out


def link_probe(local):
    """PCIe host<->device throughput on this GPU: H2D alone, D2H alone and
    both at once on two streams, for one large copy per direction and for
    the sizes of a 64 x 1080p step (packed inputs up, I420 frames down) as
    single copies and as per-frame pieces. CUDA events; best of 4."""
    import torch
    torch.cuda.set_device(local)
    MB = 1 << 20
    big = 256 * MB
    h_up = torch.empty(big, dtype=torch.uint8, pin_memory=True)
    h_dn = torch.empty(big, dtype=torch.uint8, pin_memory=True)
    d_up = torch.empty(big, dtype=torch.uint8, device="cuda")
    d_dn = torch.empty(big, dtype=torch.uint8, device="cuda")
    s_up, s_dn = torch.cuda.Stream(), torch.cuda.Stream()

    def pieces(n, piece):
        return [(o, min(piece, n - o)) for o in range(0, n, piece)]

    def run(up, dn):
        best = None
        for r in range(5):
            torch.cuda.synchronize()
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record()
            s_up.wait_stream(torch.cuda.current_stream())
            s_dn.wait_stream(torch.cuda.current_stream())
            with torch.cuda.stream(s_dn):
                for o, n in dn:
                    h_dn[o:o + n].copy_(d_dn[o:o + n], non_blocking=True)
            with torch.cuda.stream(s_up):
                for o, n in up:
                    d_up[o:o + n].copy_(h_up[o:o + n], non_blocking=True)
            torch.cuda.current_stream().wait_stream(s_up)
            torch.cuda.current_stream().wait_stream(s_dn)
            e1.record()
            torch.cuda.synchronize()
            ms = e0.elapsed_time(e1)
            if r and (best is None or ms < best):
                best = ms
        return best

    UP, DN, FB = 102400000, 199065600, 3110400
    cases = [("one 256 MB copy each way", pieces(big, big), pieces(big, big)),
             ("a 64x1080p step, one copy each way", pieces(UP, UP), pieces(DN, DN)),
             ("a 64x1080p step, per-frame pieces (0.8 MB up, 3.1 MB down)", pieces(UP, 800000), pieces(DN, FB)),
             ("a 64x1080p step, 8 MB pieces", pieces(UP, 8 * MB), pieces(DN, 8 * MB))]
    out = []
    for name, up, dn in cases:
        bu, bd = sum(n for _, n in up), sum(n for _, n in dn)
        tu, td, tb = run(up, []), run([], dn), run(up, dn)
        out.append({"case": name, "up_MB": bu / 1e6, "down_MB": bd / 1e6, "up_GBps": bu / tu / 1e6,
                    "down_GBps": bd / td / 1e6, "both_ms": tb, "serial_ms": tu + td, "max_ms": max(tu, td),
                    "both_GBps": (bu + bd) / tb / 1e6})
    print(json.dumps({"leg": "link", "cases": out}), flush=True)


def leg_only(args, ws, rank, local):
    """One device-resident leg alone, for profiler captures: the tuner's
    settling steps (unless --no-tune), W warm-up steps, K timed steps and
    three profiling steps of the named schedule; prints one JSON line."""
    import torch
    torch.cuda.set_device(local)
    os.environ.setdefault("CVP9_CUDA_DEVICE", str(local))
    from compute_vp9_b200 import ARITH_FULL, ARITH_REFCPU, ARITH_SPEC
    arith = {"spec": ARITH_SPEC, "full": ARITH_FULL}.get(args.arith, ARITH_REFCPU)
    preset, gop, mode, ov = 1, args.gop, args.leg, {}
    if args.leg == "mixed":
        preset, gop, mode, ov = 2, 60, "gop", {"intra_in_inter": 0.0}
        if arith == ARITH_SPEC:
            ov["interp_filter"] = 0          # the shader profile holds the regular filter only
    wl = Workload(args.streams, args.width, args.height, device_copy=True,
                  seeds=rank_seeds(rank, args.streams), preset=preset, overrides=ov, gop=gop)
    wl.mode = mode
    tuned = []
    r = run_batched(wl, args.steps, args.warmup, arith, True, not args.no_graphs, ws, tuned,
                    tune=not args.no_tune)
    ms = allreduce_max(ws, r["ms"])
    if rank == 0:
        print(json.dumps({"leg": args.leg, "arith": args.arith, "streams": wl.S, "width": wl.w, "height": wl.h,
                          "steps": args.steps, "value": px_rate(wl, args.steps, ms, ws), "unit": UNIT,
                          "ms_per_step": ms / args.steps,
                          "kernels_ms": {k: statistics.mean(p[i] for p in r["prof"])
                                         for i, k in enumerate(("scan", "recon", "filter", "all", "step"))},
                          "tuning": [{k: e[k] for k in ("inter_path", "lf_tile_h", "half_width")}
                                     for e in tuned]}), flush=True)


def main():
    args = parse()
    ws, rank, local = dist_setup()
    if args.leg == "link":
        if rank == 0:
            link_probe(local)
        if ws > 1:
            import torch.distributed as dist
            dist.destroy_process_group()
        return
    if args.leg == "hbd":
        import torch
        torch.cuda.set_device(local)
        os.environ.setdefault("CVP9_CUDA_DEVICE", str(local))
        r = hbd_leg(args, rank, read_peaks()[0], parity=args.hbd_checks)
        if rank == 0:
            print(json.dumps(r), flush=True)
        if ws > 1:
            import torch.distributed as dist
            dist.destroy_process_group()
        return
    if args.leg:
        leg_only(args, ws, rank, local)
        if ws > 1:
            import torch.distributed as dist
            dist.destroy_process_group()
        return
    if args.impl == "reference":
        reference_arm(args, ws, rank)
        if ws > 1:
            import torch.distributed as dist
            dist.destroy_process_group()
        return
    import torch
    torch.cuda.set_device(local)
    os.environ.setdefault("CVP9_CUDA_DEVICE", str(local))
    if ws > 1:
        # the legs rank 0 runs alone while the other ranks wait at a barrier
        # (CPU baseline, single stream, serving and its sweeps, the mixed,
        # FULL and 10-bit legs) are measured at N = 1; at N > 1 every rank
        # runs the timed legs only, which keeps the wait well inside the
        # process group's timeout
        args.no_cpu = args.no_single = args.no_serve = args.no_capacity = True
        args.no_mixed = args.no_full = args.no_hbd = True
    from compute_vp9_b200 import ARITH_FULL, ARITH_REFCPU, ARITH_SPEC
    from oracle.oracle_py import FULL, REFCPU, SPEC
    arith = {"spec": ARITH_SPEC, "full": ARITH_FULL}.get(args.arith, ARITH_REFCPU)
    oracle_profile = {ARITH_SPEC: SPEC, ARITH_FULL: FULL}.get(arith, REFCPU)
    wl = Workload(args.streams, args.width, args.height, device_copy=True,
                  seeds=rank_seeds(rank, args.streams), gop=args.gop)
    px_step = wl.S * wl.w * wl.h
    graphs = not args.no_graphs
    peak, peak_kind = read_peaks()
    cores = host_cores()

    # device-resident legs: the GOP-shaped sequence (the headline), inter
    # steps only and key steps only
    clocks = ClockSampler(int(os.environ.get("CVP9_NVSMI_INDEX", str(local))))
    tuned = []
    with clocks:
        wl.mode = "gop"
        R = run_batched(wl, args.steps, args.warmup, arith, True, graphs, ws, tuned)
        wl.mode = "inter"
        Ri = run_batched(wl, args.steps, args.warmup, arith, True, graphs, ws)
        wl.mode = "key"
        key_steps = min(args.steps, 12)
        Rk = run_batched(wl, key_steps, args.warmup, arith, True, graphs, ws)
    wl.mode = "gop"
    ms_dev = allreduce_max(ws, R["ms"])
    value = px_rate(wl, args.steps, ms_dev, ws)
    ms_int = allreduce_max(ws, Ri["ms"])
    ms_key = allreduce_max(ws, Rk["ms"])
    timed_keys = sum(1 for t in range(args.warmup, args.warmup + args.steps) if wl.frame_of(t) == 0)

    # end to end through the public API from page-locked host arrays, every
    # frame downloaded; its final frames are checked against the reference
    E = run_batched(wl, args.steps, args.warmup, arith, False, graphs, ws, final=True)
    ms_e2e = allreduce_max(ws, E["ms"])
    e2e = px_rate(wl, args.steps, ms_e2e, ws)

    # the same without host-side coefficient packing (dense arrays over PCIe)
    Enp = run_batched(wl, args.steps, args.warmup, arith, False, graphs, ws, pack=-1)
    ms_np = allreduce_max(ws, Enp["ms"])
    e2e_np = px_rate(wl, args.steps, ms_np, ws)

    # the same, coefficients as (index, value) lists (cvp9_batch_submit_sparse)
    wl.build_sparse()
    Esp = run_batched(wl, args.steps, args.warmup, arith, False, graphs, ws, sparse=True)
    ms_sp = allreduce_max(ws, Esp["ms"])
    e2e_sp = px_rate(wl, args.steps, ms_sp, ws)

    # the shader arithmetic on the same workload (regular filter, as the
    # shaders hold), device-resident
    Rs = None
    if not args.no_spec and arith != ARITH_SPEC:
        Rs = run_batched(wl, args.steps, args.warmup, ARITH_SPEC, True, graphs, ws, final=True)
        Rs["ms"] = allreduce_max(ws, Rs["ms"])

    out = None
    if rank == 0:
        main_rf = leg_roofline(wl, R, args.steps, args.warmup, peak)
        recon_ms, alg, achieved = main_rf["recon_ms"], main_rf["alg_bytes_per_launch"], main_rf["achieved_gbs"]
        split = bool(tuned) and tuned[0].get("inter_path") in (3, 4, 5)
        traffic = read_traffic(split)
        parity = check_parity(wl, E["seq"], E["outs"], oracle_profile, list(range(wl.S)), cores)
        value_spec = None
        if Rs is not None:
            value_spec = {"value": px_rate(wl, args.steps, Rs["ms"], ws), "unit": UNIT,
                          "ms_per_step": Rs["ms"] / args.steps,
                          "roofline": leg_roofline(wl, Rs, args.steps, args.warmup, peak),
                          "parity": check_parity(wl, Rs["seq"], Rs["outs"], SPEC, list(range(min(16, wl.S))),
                                                 cores),
                          "what": "the same GOP-shaped device-resident steps in the shader arithmetic "
                                  "(8-tap MC, integer butterflies on every plane)"}
        # the 10-bit leg in a process of its own: run inside this one after
        # the other legs, its pipelined e2e steps and live loop measured two
        # to three times slower with unchanged per-phase device times (cause
        # not identified); alone it measures what a 10-bit user sees
        value_hbd = None if args.no_hbd else hbd_leg_process(args)
        single = None
        if not args.no_single:
            one = Workload(1, args.width, args.height, device_copy=True, gop=args.gop)
            r1 = run_batched(one, args.gop, args.warmup, arith, True, graphs, 1)
            single_dev = px_rate(one, args.gop, r1["ms"])
            plain_e2e, plain_kern = run_single_plain(one, args.gop, arith)
            single = {"value": single_dev, "e2e_plain_backend": plain_e2e, "unit": UNIT,
                      "kernel_ms_per_frame": plain_kern,
                      "workload": "stream 0 alone, %dx%d, %d frames holding one key frame; value "
                                  "device-resident, e2e through cuda_decode_frame/cuda_get_frame with host "
                                  "inputs" % (one.w, one.h, args.gop)}
        serving = None
        capacity = None
        capacity_streams = None
        if not args.no_serve:
            from compute_vp9_b200 import serve
            sv = serve.run(streams=256, rate=2.0, frames=120, fps=30.0, speed=args.serve_speed,
                           hbm_budget=150e9, arith=arith, seed=1)
            serving = {"workload": "256 streams, Poisson arrivals 2/s, 640x360/1280x720/1920x1080/"
                                   "3840x2160 in 4:3:2:1, 120 frames at 30 fps, GOP 60, 150 GB budget; "
                                   "arrivals and pacing compressed %gx" % args.serve_speed,
                       "speed": args.serve_speed, "frames": sv["frames"], "steps": sv["steps"],
                       "mean_batch": sv["mean_batch"], "p50_ms": sv["p50_ms"], "p99_ms": sv["p99_ms"],
                       "value": sv["mpx_per_s"], "unit": UNIT, "admission_waits": sv["admission_waits"],
                       "latency": "frame due -> its planes in host memory"}
            if not args.no_capacity:
                capacity = serve.capacity_sweep(arith=arith)
                capacity_streams = serve.stream_capacity_sweep(arith=arith)
        cpu = None
        if not args.no_cpu:
            v, kind, cthreads, sample = cpu_leg(wl, cores)
            cpu = {"value": v, "unit": UNIT, "cores": cthreads, "kind": kind, "sample": sample}
        launches_per_step = int(R["stats"].kernel_launches)
        lat = E["lat"]
        # the 1080p GOP-60 stream's content (blocks 8-64, TX 4x4-32x32 weighted
        # 30/30/25/15, 2-20% coefficients, +-128 px MVs over LAST/GOLDEN/
        # ALTREF, filters uniform over regular/smooth/sharp, GOP 60): REFCPU
        # and the VP9 (FULL) profile
        mixed = None
        value_full = None
        if not args.no_mixed or not args.no_full:
            n_steps = args.steps
            del wl
            wl = None
            wl2 = Workload(args.streams, args.width, args.height, device_copy=True,
                           seeds=rank_seeds(rank, args.streams), preset=2, gop=60,
                           overrides={"intra_in_inter": 0.0})
            wdesc = ("%d x %dx%d streams, blocks 8-64 (rectangular partitions), TX 4x4..32x32 weighted "
                     "30/30/25/15, 2-20%% coefficients, +-128 px MVs over LAST/GOLDEN/ALTREF, filter "
                     "uniform over regular/smooth/sharp, a key frame every 60 steps; device-resident inputs"
                     % (wl2.S, wl2.w, wl2.h))
            if not args.no_mixed:
                tuned2 = []
                r2 = run_batched(wl2, n_steps, args.warmup, ARITH_REFCPU, True, graphs, 1, tuned2)
                rf2 = leg_roofline(wl2, r2, n_steps, args.warmup, peak)
                mixed = {"workload": wdesc, "value": px_rate(wl2, n_steps, r2["ms"]), "unit": UNIT,
                         "ms_per_step": r2["ms"] / n_steps, "recon_ms": rf2["recon_ms"],
                         "roofline_frac": rf2["frac"], "arith": "refcpu",
                         "tuning": [{k: e[k] for k in ("inter_path", "lf_tile_h", "half_width")} for e in tuned2]}
            if not args.no_full:
                rf = run_batched(wl2, n_steps, args.warmup, ARITH_FULL, True, graphs, 1, final=True)
                value_full = {"workload": wdesc, "value": px_rate(wl2, n_steps, rf["ms"]), "unit": UNIT,
                              "ms_per_step": rf["ms"] / n_steps,
                              "roofline": leg_roofline(wl2, rf, n_steps, args.warmup, peak),
                              "kernels_ms_per_step": {"scan": statistics.mean(p[0] for p in rf["prof"]),
                                                      "recon": statistics.mean(p[1] for p in rf["prof"]),
                                                      "filter": statistics.mean(p[2] for p in rf["prof"])},
                              "parity": check_parity(wl2, rf["seq"], rf["outs"], FULL, [0, 1], cores),
                              "what": "the VP9 completion of the shader profile (compound, all frame "
                                      "filters, per-TX directional intra + ADST, the VP9 loop filter); "
                                      "parity against its from-spec restatement (unpinned)"}
            del wl2
        out = {
            "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": ws, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": ms_dev / args.steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "u8",
            "data": "synthetic (seeded parsed-frame streams)",
            "config": dict(workload_config(args), timed_key_steps=timed_keys),
            "value_inter": {"value": ws * px_step * args.steps / (ms_int / 1000.0) / 1e6, "unit": UNIT,
                            "ms_per_step": ms_int / args.steps, "what": "inter steps only"},
            "value_key": {"value": ws * px_step * key_steps / (ms_key / 1000.0) / 1e6, "unit": UNIT,
                          "ms_per_step": ms_key / key_steps, "steps": key_steps,
                          "recon_ms": statistics.mean(p[1] for p in Rk["prof"]),
                          "what": "key (intra) steps only: every superblock through the wavefront kernel"},
            "e2e": {"value": e2e, "unit": UNIT, "h2d_bytes_per_step": int(E["stats"].h2d_bytes),
                    "d2h_bytes_per_step": int(E["stats"].d2h_bytes),
                    "ms_per_step": ms_e2e / args.steps,
                    "packed_frames_per_step": int(E["stats"].packed_frames),
                    "host_pack_ms_per_step": float(E["stats"].submit_pack_ms),
                    "what": "cvp9_batch_submit from page-locked host arrays in the parser's dense layout; "
                            "the engine packs coefficients on host threads inside the timed region; the "
                            "same GOP-shaped sequence"},
            "e2e_without_packing": {"value": e2e_np, "unit": UNIT,
                                    "h2d_bytes_per_step": int(Enp["stats"].h2d_bytes),
                                    "d2h_bytes_per_step": int(Enp["stats"].d2h_bytes),
                                    "ms_per_step": ms_np / args.steps},
            "e2e_sparse_input": {"value": e2e_sp, "unit": UNIT,
                                 "h2d_bytes_per_step": int(Esp["stats"].h2d_bytes),
                                 "d2h_bytes_per_step": int(Esp["stats"].d2h_bytes),
                                 "ms_per_step": ms_sp / args.steps,
                                 "what": "as e2e, with each frame's coefficients handed over as (index, "
                                         "value) lists through cvp9_batch_submit_sparse (built before "
                                         "timing, as a parser emitting them would); outputs identical"},
            "latency_ms": {"p50": statistics.median(lat) if lat else None,
                           "p99": (sorted(lat)[min(len(lat) - 1, int(0.99 * len(lat)))] if lat else None),
                           "what": "host clock, submit to frame in pinned host memory, e2e steps (3 in flight)"},
            "roofline": {"bound": "hbm",
                         "kernel": ("recon phase (k_pred, k_resid, k_compact, k_recon)" if split
                                    else "recon phase (k_inter, k_compact, k_recon)"),
                         "achieved": achieved, "peak": peak,
                         "unit": "GB/s", "frac": achieved / peak, "traffic": traffic,
                         "peak_source": peak_kind + " (MEASURED_PEAKS.json hbm_gbs)"
                         if peak_kind == "measured" else "fallback 6650 GB/s",
                         "alg_bytes_per_launch": alg, "launch_ms": recon_ms},
            "kernels_ms_per_step": {"scan": statistics.mean(p[0] for p in R["prof"]),
                                    "recon": recon_ms, "filter": statistics.mean(p[2] for p in R["prof"])},
            "gpu_launches": launches_per_step * args.steps,
            "tuning": [{k: e[k] for k in ("settled", "inter_path", "lf_tile_h", "half_width", "trials",
                                          "best_ms")} for e in tuned],
            "clocks": clocks.summary(),
            "cpu_baseline": cpu,
            "parity": parity,
            "value_spec": value_spec,
            "value_mixed_content": mixed,
            "value_full": value_full,
            "value_hbd": value_hbd,
            "single_stream": single,
            "serving": serving,
            "serving_capacity": capacity,
            "serving_capacity_streams": capacity_streams,
            "batched_vs_single": (value / single["value"]) if single else None,
            "batched_vs_single_e2e": (e2e / single["e2e_plain_backend"]) if single else None,
        }
    barrier(ws)
    if rank == 0:
        print(json.dumps(out), flush=True)
    if ws > 1:
        import torch.distributed as dist
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
