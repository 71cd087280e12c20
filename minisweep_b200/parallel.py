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


# ------------------------------------------------ KBA x/y decomposition
class TorchGroupComm:
    """The process group of a decomposed sweep (--nproc_x / --nproc_y > 1)
    over torch.distributed: one process per GPU, process number = rank.

    Holds the msb_comm table the library calls (msb_env_set_comm) and the
    face-message buffers (device tensors handed to the Sweeper with
    msb_kba_set_buffers), so that the exchange callback can post the
    messages on those tensors: NCCL point-to-point between GPUs, or, on a gloo
    group, copies through host tensors.  The collectives serve the whole group
    only (nactive == world size), the case of a grid that covers every rank.
    The counterpart of the reference's MPI transport (env_mpi.c:309-480)."""

    def __init__(self, group=None):
        import torch
        import torch.distributed as dist

        import minisweep_b200 as msb

        self.dist, self.torch, self.group = dist, torch, group
        self.rank = dist.get_rank(group)
        self.world = dist.get_world_size(group)
        self.nccl = dist.get_backend(group) == "nccl"
        self.coll_dev = torch.device("cuda", torch.cuda.current_device()) if self.nccl else "cpu"
        self.buffers = {}  # device address -> uint8 tensor
        self.comm = msb.make_comm(self._exchange, self._sum, self._allgather, self._barrier)

    def _whole(self, nactive):
        if nactive != self.world:
            raise RuntimeError(f"collective over {nactive} of {self.world} ranks is not served")

    def _sum(self, nactive, x):
        self._whole(nactive)
        t = self.torch.tensor([x], dtype=self.torch.float64, device=self.coll_dev)
        self.dist.all_reduce(t, op=self.dist.ReduceOp.SUM, group=self.group)
        return float(t[0])

    def _allgather(self, nactive, v):
        self._whole(nactive)
        t = self.torch.tensor([v], dtype=self.torch.int64, device=self.coll_dev)
        out = [self.torch.zeros_like(t) for _ in range(self.world)]
        self.dist.all_gather(out, t, group=self.group)
        return [int(x[0]) for x in out]

    def _barrier(self, nactive):
        self._whole(nactive)
        self.dist.barrier(group=self.group)

    def attach(self, problem) -> None:
        """Message buffers for a decomposed Problem: six device tensors of the
        sizes the Sweeper asks for, registered with it."""
        torch = self.torch
        _, bx, by = problem.kba_info()
        sizes = [bx, by, bx, bx, by, by]
        bufs = [torch.empty(max(int(s), 16), dtype=torch.uint8, device="cuda") for s in sizes]
        problem.kba_set_buffers(*[b.data_ptr() for b in bufs])
        self.buffers = {b.data_ptr(): b for b in bufs}

    def _exchange(self, nactive, msgs):
        """All of one step's messages; returns after they landed."""
        torch, dist = self.torch, self.dist
        self._whole(nactive)
        if not msgs:
            return
        views = [(m, self.buffers[m.buf][:m.bytes]) for m in msgs]
        if self.nccl:
            ops = [dist.P2POp(dist.isend if m.is_send else dist.irecv, t, m.peer, group=self.group)
                   for m, t in views]
            for w in dist.batch_isend_irecv(ops):
                w.wait()
            torch.cuda.current_stream().synchronize()
            return
        # gloo: point-to-point on host copies of the device buffers
        host = [(m, t, t.cpu() if m.is_send else torch.empty(t.numel(), dtype=torch.uint8)) for m, t in views]
        reqs = [(dist.isend if m.is_send else dist.irecv)(h, m.peer, group=self.group) for m, _, h in host]
        for r in reqs:
            r.wait()
        for m, t, h in host:
            if not m.is_send:
                t.copy_(h)
        if t.is_cuda:
            torch.cuda.synchronize()
