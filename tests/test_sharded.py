"""Slot sharding on the CPU: the reference's split of the Nred bosonic slots
over ranks (Nb = Nred/ntasks, contiguous blocks; SRC/parquet_ini.f90:336,
SRC/preprocessing.f90:95-98) and the exchange of the three all-slot buffers
over two gloo ranks."""
from __future__ import annotations

import multiprocessing as mp
import os
import socket

import pytest
import torch

from tups_b200.sharded import XCH_MAX, XCH_SUM, combine, slot_range


def test_slot_range_blocks():
    Nred = 36
    for ntasks in (1, 2, 3, 4, 6, 12, 36):
        seen = []
        for rank in range(ntasks):
            s0, nb = slot_range(Nred, rank, ntasks)
            assert nb == Nred // ntasks and s0 == rank * nb
            seen += list(range(s0, s0 + nb))
        assert seen == list(range(Nred))


def test_slot_range_rejects():
    with pytest.raises(ValueError, match="divides Nred"):
        slot_range(36, 0, 5)
    with pytest.raises(ValueError):
        slot_range(36, 2, 2)


def _free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank: int, world: int, port: int, out):
    import datetime

    import torch.distributed as dist
    dist.init_process_group("gloo", init_method=f"tcp://127.0.0.1:{port}", rank=rank, world_size=world,
                            timeout=datetime.timedelta(seconds=60))
    try:
        a = torch.arange(6, dtype=torch.float64) * (rank + 1)  # a partial sum per rank
        combine(a, XCH_SUM)
        m = torch.tensor([1.0 + rank, 5.0 - rank, 0.0, 0.0, float(rank)], dtype=torch.float64)  # max|F|, NaN flag
        combine(m, XCH_MAX)
        out.put((rank, a.tolist(), m.tolist()))
    finally:
        dist.destroy_process_group()


def test_exchange_two_gloo_ranks():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    ps = [ctx.Process(target=_rank_main, args=(r, 2, port, q)) for r in range(2)]
    for p in ps:
        p.start()
    res = sorted(q.get(timeout=120) for _ in ps)
    for p in ps:
        p.join(timeout=60)
        assert p.exitcode == 0
    for rank, a, m in res:
        assert a == [3.0 * i for i in range(6)]  # 1x + 2x
        assert m == [2.0, 5.0, 0.0, 0.0, 1.0]
