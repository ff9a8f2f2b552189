"""Process-group plumbing for running replicas of a box on several GPUs.

The single-GPU time step has no exchange step, so N GPUs run N independent
replicas (weak scaling).  The only cross-rank operations are a barrier around
the timed region and the maximum of the ranks' times; both work over NCCL
(CUDA tensors) and over gloo (CPU tensors, used by the multi-process tests).
"""
from __future__ import annotations

import datetime
import os


def init_from_env(backend: str | None = None, timeout_s: int = 120):
    """RANK / LOCAL_RANK / WORLD_SIZE / MASTER_* as set by torchrun."""
    import torch
    import torch.distributed as dist
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if world > 1 and not dist.is_initialized():
        if backend is None:
            backend = "nccl" if torch.cuda.is_available() else "gloo"
        dist.init_process_group(backend, timeout=datetime.timedelta(seconds=timeout_s))
    return rank, local, world


def _device():
    import torch
    import torch.distributed as dist
    if dist.is_initialized() and dist.get_backend() == "nccl":
        return torch.device("cuda", torch.cuda.current_device())
    return torch.device("cpu")


def barrier(world: int) -> None:
    if world > 1:
        import torch.distributed as dist
        dist.barrier()


def allmax(x: float, world: int) -> float:
    """Maximum of a scalar over ranks (every rank gets it)."""
    if world == 1:
        return float(x)
    import torch
    import torch.distributed as dist
    t = torch.tensor([float(x)], dtype=torch.float64, device=_device())
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def weak_scaling_value(nodes_per_rank: int, steps: int, ms_max: float, world: int) -> float:
    """Lattice updates of all ranks (millions) per second of the slowest rank."""
    return world * nodes_per_rank * steps / (ms_max * 1e-3) / 1e6


def shutdown(world: int) -> None:
    if world > 1:
        import torch.distributed as dist
        if dist.is_initialized():
            dist.destroy_process_group()
