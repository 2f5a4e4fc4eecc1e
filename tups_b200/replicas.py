"""Multi-GPU plumbing of the benchmark: one process per GPU, independent
replicas of the loop.

The reference distributes the bosonic slots of one loop over MPI ranks
(Nb = Nred / ntasks, parquet_ini.f90:336).  This build runs the whole loop
on one GPU (every call here has one GPU), so N processes run N independent
replicas: no data-path collective, only a barrier around the timed region
and a max over ranks of the device times.  `torch.distributed` carries
both: NCCL between GPUs, gloo on CPU (the multi-rank tests).
"""
from __future__ import annotations

import os
from dataclasses import dataclass
from datetime import timedelta


@dataclass
class Ranks:
    world: int = 1
    rank: int = 0
    local: int = 0
    pg: object = None       # torch.distributed when world > 1
    device: str = "cpu"     # where reduction tensors live


def init(backend: str = "nccl", timeout_s: int = 120) -> Ranks:
    """Read RANK / LOCAL_RANK / WORLD_SIZE and join the process group when
    there is more than one rank (MASTER_ADDR / MASTER_PORT from the launcher)."""
    ws = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    r = Ranks(ws, rank, local)
    if ws > 1:
        import torch.distributed as dist
        dist.init_process_group(backend, timeout=timedelta(seconds=timeout_s))
        r.pg = dist
        r.device = f"cuda:{local}" if backend == "nccl" else "cpu"
    return r


def barrier(r: Ranks) -> None:
    if r.pg is not None:
        r.pg.barrier()


def max_over_ranks(r: Ranks, values):
    """Element-wise max of a list of floats over all ranks (every rank gets it)."""
    vals = [float(v) for v in values]
    if r.pg is None:
        return vals
    import torch
    t = torch.tensor(vals, dtype=torch.float64, device=r.device)
    r.pg.all_reduce(t, op=r.pg.ReduceOp.MAX)
    return [float(x) for x in t.tolist()]


def seconds_per_iteration(ms_max: float, iterations_per_rank: int, world: int) -> float:
    """Whole-job seconds per iteration: world x iterations done in the slowest rank's time."""
    return ms_max * 1e-3 / (iterations_per_rank * world)


def finish(r: Ranks) -> None:
    if r.pg is not None:
        r.pg.barrier()
        r.pg.destroy_process_group()
