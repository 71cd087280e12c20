"""Multi-GPU plumbing for the sweep: one process per GPU, energy-group slices.

Energy groups are independent in the sweep (the reference threads over them
with no communication, sweeper_kba_c_kernels.h:600-605), so N processes split
the groups and exchange nothing while sweeping. The only collective is the sum
of the two FP64 checksums (the reference's Env_sum_P after get_state_norms,
array_operations.c:105-106) and, for timing, the max over ranks.
"""
from __future__ import annotations


def group_slice(ne: int, world: int, rank: int) -> tuple[int, int]:
    """[ie0, ie1) of rank `rank` out of `world`: contiguous, sizes differ by at
    most one, whole group pairs where possible (the kernel pairs groups)."""
    if world <= 0 or not (0 <= rank < world) or ne <= 0:
        raise ValueError("invalid slice request")
    npair = (ne + 1) // 2
    p0 = rank * npair // world
    p1 = (rank + 1) * npair // world
    return min(2 * p0, ne), min(2 * p1, ne)


def sum_norms(normsq: float, normsqdiff: float, group=None) -> tuple[float, float]:
    """All-reduce (SUM) of the two FP64 checksums across the process group."""
    import torch
    import torch.distributed as dist

    if not dist.is_available() or not dist.is_initialized():
        return normsq, normsqdiff
    dev = torch.device("cuda", torch.cuda.current_device()) if dist.get_backend(group) == "nccl" else "cpu"
    t = torch.tensor([normsq, normsqdiff], dtype=torch.float64, device=dev)
    dist.all_reduce(t, op=dist.ReduceOp.SUM, group=group)
    return float(t[0]), float(t[1])


def max_over_ranks(seconds: float, group=None) -> float:
    """The slowest rank's time: whole-job throughput divides by it."""
    import torch
    import torch.distributed as dist

    if not dist.is_available() or not dist.is_initialized():
        return seconds
    dev = torch.device("cuda", torch.cuda.current_device()) if dist.get_backend(group) == "nccl" else "cpu"
    t = torch.tensor([seconds], dtype=torch.float64, device=dev)
    dist.all_reduce(t, op=dist.ReduceOp.MAX, group=group)
    return float(t[0])
