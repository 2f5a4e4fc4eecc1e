"""The multi-rank path of the benchmark on CPU: two gloo ranks (the GPU runs
use NCCL with the same calls)."""
from __future__ import annotations

import os
import socket

import pytest
import torch.multiprocessing as mp


def _free_port() -> int:
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _rank_main(rank: int, world: int, port: int, out):
    os.environ.update(RANK=str(rank), LOCAL_RANK=str(rank), WORLD_SIZE=str(world), MASTER_ADDR="127.0.0.1",
                      MASTER_PORT=str(port))
    from tups_b200 import replicas
    r = replicas.init("gloo", timeout_s=60)
    replicas.barrier(r)
    # each rank times its own replica; the job reports the slowest
    mx = replicas.max_over_ranks(r, [10.0 * (rank + 1), 3.0 - rank])
    out[rank] = (r.world, r.rank, mx, replicas.seconds_per_iteration(mx[0], 5, r.world))
    replicas.finish(r)


def test_two_gloo_ranks_reduce_max_and_aggregate():
    world = 2
    port = _free_port()
    with mp.Manager() as mgr:
        out = mgr.dict()
        mp.spawn(_rank_main, args=(world, port, out), nprocs=world, join=True)
        res = dict(out)
    for rank in range(world):
        ws, rk, mx, spi = res[rank]
        assert ws == world and rk == rank
        assert mx == [20.0, 3.0]
        # 2 ranks x 5 iterations in the slowest rank's 20 ms
        assert spi == pytest.approx(20e-3 / 10)


def test_single_rank_needs_no_process_group(monkeypatch):
    from tups_b200 import replicas
    for k in ("RANK", "LOCAL_RANK", "WORLD_SIZE"):
        monkeypatch.delenv(k, raising=False)
    r = replicas.init("gloo")
    assert r.world == 1 and r.pg is None
    assert replicas.max_over_ranks(r, [1.5, 2]) == [1.5, 2.0]
    replicas.finish(r)
