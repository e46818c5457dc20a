"""Multi-process plumbing: one process per GPU, torch.distributed for the
control plane only.

Two multi-GPU modes:
  * replicas (the benchmark's mode): independent solves are sharded over
    ranks and advance with no data-path collective.  What crosses ranks is
    bookkeeping: a barrier around timed regions, the max of the ranks'
    device times, sums of throughput counters, which rank owns which solve.
  * z-slabs of one solve (slab_solver): the reference's domain
    decomposition (src/variables.f90:186-375) along z; the halo exchange and
    the reductions run inside the library over NCCL, and torch.distributed
    only carries the 128-byte NCCL id from rank 0 to the others.
"""
from __future__ import annotations

import datetime
import os
from dataclasses import dataclass


@dataclass(frozen=True)
class World:
    size: int
    rank: int
    local_rank: int


def world() -> World:
    return World(int(os.environ.get("WORLD_SIZE", "1")), int(os.environ.get("RANK", "0")),
                 int(os.environ.get("LOCAL_RANK", "0")))


def init(backend: str | None = None, timeout_s: float = 120.0):
    """Initialise the default process group when WORLD_SIZE > 1; returns the
    torch.distributed module or None for a single process."""
    w = world()
    if w.size <= 1:
        return None
    import torch
    import torch.distributed as dist

    if backend is None:
        backend = "nccl" if torch.cuda.is_available() else "gloo"
    if not dist.is_initialized():
        dist.init_process_group(backend, timeout=datetime.timedelta(seconds=timeout_s))
    return dist


def _reduce(x: float, op: str) -> float:
    import torch
    import torch.distributed as dist

    if not dist.is_available() or not dist.is_initialized() or dist.get_world_size() == 1:
        return float(x)
    dev = "cuda" if dist.get_backend() == "nccl" else "cpu"
    t = torch.tensor([float(x)], dtype=torch.float64, device=dev)
    dist.all_reduce(t, op=dist.ReduceOp.MAX if op == "max" else dist.ReduceOp.SUM)
    return float(t.item())


def max_over_ranks(x: float) -> float:
    """Max of a per-rank value (device times of a timed region)."""
    return _reduce(x, "max")


def sum_over_ranks(x: float) -> float:
    return _reduce(x, "sum")


def barrier() -> None:
    import torch.distributed as dist

    if dist.is_available() and dist.is_initialized():
        dist.barrier()


def shard(items, rank: int | None = None, size: int | None = None):
    """Round-robin ownership of independent solves: rank r owns items
    r, r+size, r+2*size, ..."""
    w = world()
    rank = w.rank if rank is None else rank
    size = w.size if size is None else size
    return list(items)[rank::size]


def finalize() -> None:
    import torch.distributed as dist

    if dist.is_available() and dist.is_initialized():
        dist.barrier()
        dist.destroy_process_group()


def slab_plan(nz: int):
    """(rank, nranks, nccl_id, k0, nzl) of this process for a z-slab solve of
    nz planes: rank 0 creates the NCCL id and broadcasts it; every rank
    derives its slab from the same partition rule as the library."""
    from . import slab

    w = world()
    nid = slab.nccl_unique_id() if w.rank == 0 else None
    if w.size > 1:
        import torch.distributed as dist

        box = [nid]
        dist.broadcast_object_list(box, src=0)
        nid = box[0]
    k0, nzl = slab.partition(nz, w.size, w.rank)
    return w.rank, w.size, nid, k0, nzl


def slab_solver(params):
    """This rank's z-slab of one solve (gpe_create_slab over NCCL)."""
    from .solver import Solver

    rank, size, nid, _, _ = slab_plan(params.nz)
    return Solver(params, rank=rank, nranks=size, nccl_id=nid)
