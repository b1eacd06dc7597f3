"""Host-side logic of the N > 1 paths, on CPU.

- bench.py's max-over-ranks timing and weak-scaling value with two gloo
  ranks (the same collective every rank runs under torchrun + nccl);
- the msm() C ABI's card split (core/src/msm/src/msm_impl.cuh:832-844): the
  two-phase size query plans each card's range on the host, so it runs
  without a GPU."""
import ctypes
import os
import socket

import pytest
import torch.distributed as dist
import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port() -> int:
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _rank_main(rank, world, port, q):
    import sys
    sys.path.insert(0, ROOT)
    import bench
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    ms = [12.5, 17.25][rank]
    got = bench.max_over_ranks(ms, dist)
    val = bench.replica_value(1 << 22, world, got)
    q.put((rank, got, val))
    dist.barrier()
    dist.destroy_process_group()


def test_max_over_ranks_gloo_two_ranks():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank_main, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(timeout=120)
        assert p.exitcode == 0
    out = sorted(q.get(timeout=10) for _ in range(2))
    for _, got, val in out:
        assert got == 17.25
        assert abs(val - 2 * (1 << 22) / 17.25e-3) < 1e-3


def test_msm_abi_card_split_sizes():
    from impeller_b200 import build, lib
    build.build()
    L = lib.load()
    n = 100_001
    sizes1 = (ctypes.c_ulong * 1)()
    sizes2 = (ctypes.c_ulong * 2)()
    rc = L.msm(None, sizes1, n, 1, 1, 1, 1, 1, (ctypes.c_uint * 1)(0), None, 0, None, None)
    assert rc == 0
    rc = L.msm(None, sizes2, n, 1, 1, 1, 1, 2, (ctypes.c_uint * 2)(0, 1), None, 0, None, None)
    assert rc == 0
    # each card plans ceil(n / 2) points: both halves smaller than the whole
    assert 0 < sizes2[0] < sizes1[0] and 0 < sizes2[1] <= sizes2[0]
    # parts bound the per-card buffer for large inputs (two staged parts plus
    # the bucket accumulators instead of the whole range)
    big = 1 << 22
    whole, split = (ctypes.c_ulong * 1)(), (ctypes.c_ulong * 1)()
    assert L.msm(None, whole, big, 1, 1, 1, 1, 1, (ctypes.c_uint * 1)(0), None, 0, None, None) == 0
    assert L.msm(None, split, big, 1, 8, 2, 2, 1, (ctypes.c_uint * 1)(0), None, 0, None, None) == 0
    assert split[0] < whole[0] // 2
