"""Slot-sharded parquet loop over torch.distributed.

The reference distributes the Nred bosonic slots over its MPI ranks in
contiguous blocks of Nb = Nred / ntasks (SRC/parquet_ini.f90:336,
SRC/preprocessing.f90:95-116).  A sharded ``Solver`` keeps that split: its
vertices, chi and BSE cover its own slots, and three buffers are combined
over the ranks during an iteration (the exchange function of the C ABI):

* Phi(R) of each channel, summed over the ranks' momenta (the reference's
  communicatePhis + FTPhis, SRC/parquet_PhiR.f90:114-258);
* Sigma_V(k_IBZ, nu), summed over the slots (SRC/parquet_SDE.f90:221-258);
* max|F_r| and the NaN flag of conv, maximum (SRC/parquet_check.f90:109-117).

``TorchExchange`` does these with ``torch.distributed.all_reduce``: in place on
the device buffer with NCCL, through a host copy with gloo.
"""
from __future__ import annotations

import torch
import torch.distributed as dist

XCH_SUM, XCH_MAX = 0, 1


def slot_range(Nred: int, rank: int, ntasks: int) -> tuple[int, int]:
    """(first global slot, number of slots) of ``rank``; the rule of the
    library's sharded contexts."""
    if ntasks < 1 or not 0 <= rank < ntasks:
        raise ValueError("rank must lie in [0, ntasks)")
    if Nred % ntasks:
        raise ValueError(f"choose the number of tasks such that it divides Nred = {Nred}")
    nb = Nred // ntasks
    return rank * nb, nb


def combine(t: torch.Tensor, op: int, group=None) -> None:
    """All-reduce ``t`` in place over ``group`` (sum or max), on the device
    with NCCL, through host memory otherwise; complete when it returns."""
    rop = dist.ReduceOp.SUM if op == XCH_SUM else dist.ReduceOp.MAX
    if t.is_cuda and dist.get_backend(group) == "nccl":
        dist.all_reduce(t, op=rop, group=group)
        torch.cuda.synchronize(t.device)
        return
    h = t.cpu() if t.is_cuda else t
    dist.all_reduce(h, op=rop, group=group)
    if h is not t:
        t.copy_(h)
        torch.cuda.synchronize(t.device)


class _DeviceBuffer:
    """``count`` float64 at a raw device address, for torch.as_tensor."""

    def __init__(self, ptr: int, count: int):
        self.__cuda_array_interface__ = {"shape": (count,), "typestr": "<f8", "data": (ptr, False),
                                         "version": 3, "strides": None}


class TorchExchange:
    """The exchange function of a sharded ``Solver`` on ``device``."""

    def __init__(self, device: int, group=None):
        self.device = device
        self.group = group

    def __call__(self, what: int, ptr: int, count: int, op: int) -> None:
        t = torch.as_tensor(_DeviceBuffer(ptr, count), device=f"cuda:{self.device}")
        combine(t, op, self.group)
