"""CPU, world size 2 over gloo: the multi-rank bench path. Ranks decode
disjoint stream sets (weak scaling, no collective on the data path); the only
collectives are the barrier and the max-over-ranks of the timings."""
import os
import socket

import pytest
import torch.multiprocessing as mp


def _port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _worker(rank, ws, port, q):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank),
                      WORLD_SIZE=str(ws), LOCAL_RANK=str(rank))
    import sys
    sys.path.insert(0, os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
    import bench
    import torch.distributed as dist
    w, r, _ = bench.dist_setup(backend="gloo")
    bench.barrier(w)
    t = bench.allreduce_max(w, 10.0 + r)
    seeds = bench.rank_seeds(r, 4)
    # each rank decodes one frame of its own first stream on the CPU oracle
    import ctypes as C
    from compute_vp9_b200 import Synth, fnv1a64, synth_config
    from oracle.oracle_py import OracleStream
    h = fnv1a64(OracleStream().decode(Synth(synth_config(1, 64, 64, seeds[0])).frame(0)))
    q.put((r, t, seeds, h))
    bench.barrier(w)
    dist.destroy_process_group()


def test_two_rank_gloo_path():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    out = sorted(q.get(timeout=120) for _ in procs)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    assert [o[1] for o in out] == [11.0, 11.0]          # max over ranks, seen by both
    assert set(out[0][2]).isdisjoint(out[1][2])          # disjoint stream shards
    assert out[0][3] != out[1][3]                        # different content per rank
