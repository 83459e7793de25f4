"""CPU: the C ABI library loads and exports every function include/*.h
declares; boundary layouts and tables equal the reference's; host-side
logic (DCT basis, wavefront ticket order) is correct. No GPU calls."""
import ctypes as C
import hashlib
import json
import os
import re

import numpy as np

import compute_vp9_b200 as P
from compute_vp9_b200.cvp9_ctypes import layout_offsets
from oracle import oracle_py as O

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
GOLD = os.path.join(ROOT, "tests", "golden")


def _declared_functions(header):
    text = open(os.path.join(ROOT, "include", header)).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    names = re.findall(r"^[A-Za-z_][\w \*]*?\b(\w+)\s*\([^;{]*\)\s*;", text, flags=re.M)
    return [n for n in names if not n.startswith("if")]


def test_library_exports_every_declared_function():
    lib = P.cuda_lib()
    declared = (_declared_functions("cuda_backend.h") + _declared_functions("cvp9_batch.h") +
                _declared_functions("cvp9_hbd.h"))
    assert "cuda_decode_frame" in declared and "cvp9_batch_submit" in declared
    assert "cvp9_hbd_submit" in declared
    assert "cuda_reconstruct_noalloc" in declared
    missing = [n for n in declared if not hasattr(lib, n)]
    assert not missing, missing
    assert set(P.EXPORTED_SYMBOLS) <= set(declared)


def test_synth_library_exports():
    lib = P.synth_lib()
    for n in _declared_functions("cvp9_synth.h"):
        assert hasattr(lib, n), n


def test_struct_layout_matches_reference():
    want = json.load(open(os.path.join(GOLD, "layout.json")))["offsets"]
    assert layout_offsets() == want


def test_tables_match_reference():
    want = json.load(open(os.path.join(GOLD, "tables.json")))
    lib = O.oracle_lib()
    dc = np.array([lib.oracle_dc_quant(q) for q in range(256)], np.int32)
    ac = np.array([lib.oracle_ac_quant(q) for q in range(256)], np.int32)
    assert hashlib.sha256(dc.tobytes()).hexdigest() == want["dc_q_sha256"]
    assert hashlib.sha256(ac.tobytes()).hexdigest() == want["ac_q_sha256"]
    text = open(os.path.join(ROOT, "compute_vp9_b200", "csrc", "vp9_tables.h")).read()
    body = text[text.index("CVP9_SUBPEL_REGULAR_INIT") + len("CVP9_SUBPEL_REGULAR_INIT"):]
    body = body[:body.index("#define CVP9_QINDEX_CLAMP")]
    taps = [int(x) for x in re.findall(r"-?\d+", body)]
    assert len(taps) == 128
    assert hashlib.sha256(np.array(taps, np.int32).reshape(16, 8).tobytes()).hexdigest() == \
        want["subpel_regular_sha256"]
    m = re.search(r"CVP9_INTRA_TX_TYPE_INIT \{([^}]*)\}", text)
    txt = [int(x) for x in m.group(1).split(",")]
    assert hashlib.sha256(np.array(txt, np.int32).tobytes()).hexdigest() == want["intra_tx_type_sha256"]


def test_dct_basis_identical_to_oracle():
    lib = P.cuda_lib()
    lib.cvp9_build_dct_basis.argtypes = [C.c_void_p]
    lib.cvp9_build_dct_basis.restype = None
    mine = np.empty(1360, np.float64)
    lib.cvp9_build_dct_basis(mine.ctypes.data)
    assert np.array_equal(mine.view(np.uint64), O.refcpu_basis().view(np.uint64))


def test_wavefront_ticket_order():
    lib = P.cuda_lib()
    lib.cvp9_tickets_on_diagonal.argtypes = [C.c_int, C.c_int, C.c_int, C.c_int, C.c_void_p]
    for cols, rows in [(30, 17), (1, 1), (5, 1), (1, 7), (20, 12)]:
        out = (C.c_uint32 * (cols * rows))()
        n = 0
        order = []
        for d in range(cols + rows - 1):
            buf = (C.c_uint32 * (cols * rows))()
            k = lib.cvp9_tickets_on_diagonal(cols, rows, 3, d, buf)
            order += [buf[i] for i in range(k)]
        assert len(order) == cols * rows
        assert all(t >> 20 == 3 for t in order)
        pos = {t & 0xFFFFF: i for i, t in enumerate(order)}
        assert sorted(pos) == list(range(cols * rows))
        for sb, i in pos.items():
            r, c = divmod(sb, cols)
            for dr, dc in ((0, -1), (-1, 0), (-1, -1)):
                if r + dr >= 0 and c + dc >= 0:
                    assert pos[(r + dr) * cols + c + dc] < i   # dependencies come first


def test_job_struct_is_word_copyable():
    # the recon kernel copies the job descriptor into shared memory as 32-bit words
    text = open(os.path.join(ROOT, "compute_vp9_b200", "csrc", "recon_job.h")).read()
    assert "cvp9_ref_t ref[8]" in text


def test_parallel_memcpy_copies_every_byte():
    """The host copy pool the per-stream backend stages frames with: sizes
    around the 1 MB threshold and the chunk edges, and concurrent callers
    (one takes the pool, the others fall back to memcpy)."""
    import threading
    import numpy as np
    from compute_vp9_b200 import cuda_lib
    lib = cuda_lib()
    lib.cvp9_parallel_memcpy.argtypes = [C.c_void_p, C.c_void_p, C.c_size_t]
    lib.cvp9_parallel_memcpy.restype = None
    rng = np.random.default_rng(5)
    for n in (0, 17, (1 << 20) - 1, 1 << 20, (1 << 20) + 4097, 7_300_001, 16 << 20):
        src = rng.integers(0, 256, size=n, dtype=np.uint8)
        dst = np.zeros(n + 64, np.uint8)
        lib.cvp9_parallel_memcpy(dst.ctypes.data, src.ctypes.data, n)
        assert np.array_equal(dst[:n], src) and not dst[n:].any(), n
    srcs = [rng.integers(0, 256, size=3_000_000 + k, dtype=np.uint8) for k in range(6)]
    dsts = [np.zeros_like(s) for s in srcs]

    def work(k):
        for _ in range(20):
            lib.cvp9_parallel_memcpy(dsts[k].ctypes.data, srcs[k].ctypes.data, srcs[k].size)

    ts = [threading.Thread(target=work, args=(k,)) for k in range(6)]
    for t in ts:
        t.start()
    for t in ts:
        t.join()
    assert all(np.array_equal(d, s) for d, s in zip(dsts, srcs))


def test_parallel_for_runs_every_task_once():
    """The host worker pool the batch engine packs frames on: every task
    index runs exactly once, on more than one thread when the pool has
    workers, for task counts around the pool size; a second job started
    while one holds the pool runs its tasks on its own caller."""
    import threading
    from compute_vp9_b200 import cuda_lib
    lib = cuda_lib()
    CB = C.CFUNCTYPE(None, C.c_void_p, C.c_int)
    lib.cvp9_parallel_for.argtypes = [C.c_int, CB, C.c_void_p]
    lib.cvp9_parallel_for.restype = None
    lib.cvp9_pool_threads.restype = C.c_int
    threads = lib.cvp9_pool_threads()
    assert threads >= 1
    for ntasks in (0, 1, 2, threads - 1, threads, threads + 1, 3 * threads + 5, 200):
        if ntasks < 0:
            continue
        seen, tids = [], set()
        lock = threading.Lock()

        def task(ctx, k, seen=seen, tids=tids, lock=lock):
            with lock:
                seen.append(k)
                tids.add(threading.get_ident())

        cb = CB(task)
        lib.cvp9_parallel_for(ntasks, cb, None)
        assert sorted(seen) == list(range(ntasks)), ntasks
    # nested use from inside a task: the pool is held, so the inner job runs
    # serially on the calling worker and still covers every index
    inner_seen = []
    inner_lock = threading.Lock()

    def inner(ctx, k):
        with inner_lock:
            inner_seen.append(k)

    inner_cb = CB(inner)

    def outer(ctx, k):
        lib.cvp9_parallel_for(5, inner_cb, None)

    outer_cb = CB(outer)
    lib.cvp9_parallel_for(4, outer_cb, None)
    assert sorted(inner_seen) == sorted(list(range(5)) * 4)


def test_pack_share_balances_host_and_link():
    """The share of a large step's frames packed on the host, in 16ths:
    raised after a pipelined submit that waited for its slot, lowered after
    one that did not, untouched by callers that wait for every step."""
    from compute_vp9_b200 import cuda_lib
    lib = cuda_lib()
    f = lib.cvp9_pack_share_update
    f.argtypes = [C.c_int, C.c_int, C.c_double]
    f.restype = C.c_int
    assert f(16, 1, 1.0) == 16          # saturates
    assert f(0, 1, 0.0) == 0
    assert f(8, 1, 0.2) == 9
    assert f(8, 1, 0.01) == 7
    assert f(8, 0, 5.0) == 8            # nothing in flight: no signal
    # a host that is always behind drains the share, a link that is always
    # behind fills it, an alternation holds it near where it started
    q = 16
    for _ in range(40):
        q = f(q, 1, 0.0)
    assert q == 0
    for _ in range(40):
        q = f(q, 1, 3.0)
    assert q == 16
    q = 10
    for i in range(41):
        q = f(q, 1, 3.0 if i % 2 else 0.0)
    assert 9 <= q <= 10
