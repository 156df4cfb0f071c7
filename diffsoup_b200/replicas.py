"""Multi-GPU execution of the training step: independent replicas, one
process per GPU.

Views are independent in every kernel of the step and the reference has no
multi-GPU code, so N GPUs run N replicas of the step on their own views
(weak scaling) with no data-path collective.  This module is the host side
of that: rendezvous from the torchrun environment (RANK, LOCAL_RANK,
WORLD_SIZE, MASTER_ADDR/PORT), a barrier around timed regions, the job's
time as the maximum over ranks and the whole-job throughput.  NCCL on GPUs;
the same code runs on gloo for CPU tests.
"""

from __future__ import annotations

import datetime
import os
from dataclasses import dataclass
from typing import Optional

import torch
import torch.distributed as dist


@dataclass
class Replicas:
    rank: int
    world: int
    local_rank: int
    device: torch.device
    backend: Optional[str]  # None when world == 1 (no process group)


def init(backend: Optional[str] = None, timeout_s: float = 120.0) -> Replicas:
    """Reads the torchrun environment; with WORLD_SIZE > 1 joins the process
    group (NCCL when CUDA is available, else gloo) with a short timeout so
    that ranks waiting on a lost peer end with an error."""
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if torch.cuda.is_available():
        torch.cuda.set_device(local)
        dev = torch.device("cuda", local)
    else:
        dev = torch.device("cpu")
    be = None
    if world > 1:
        be = backend or ("nccl" if dev.type == "cuda" else "gloo")
        kw = dict(timeout=datetime.timedelta(seconds=timeout_s))
        if be == "nccl":
            kw["device_id"] = dev
        dist.init_process_group(be, **kw)
    return Replicas(rank, world, local, dev, be)


def barrier(r: Replicas) -> None:
    if r.world > 1:
        dist.barrier()


def max_over_ranks(r: Replicas, value: float) -> float:
    """The maximum of a per-rank scalar (a timed region's milliseconds)."""
    if r.world == 1:
        return float(value)
    dev = r.device if r.backend == "nccl" else torch.device("cpu")
    t = torch.tensor([float(value)], dtype=torch.float64, device=dev)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def job_throughput(r: Replicas, units_per_rank: float, ms_max: float) -> float:
    """Whole-job units per second: every rank processed units_per_rank in at
    most ms_max milliseconds."""
    return units_per_rank * r.world / (ms_max / 1000.0)


def shutdown(r: Replicas) -> None:
    if r.world > 1:
        barrier(r)
        dist.destroy_process_group()
