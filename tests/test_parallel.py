"""The N > 1 path on CPU: two gloo ranks, each sweeping its energy-group slice.

Checks the sharding the benchmark and a multi-GPU user rely on: slices cover
the groups exactly once, every slice's sweep equals the same groups of the
single-process sweep (groups are independent), and the all-reduced checksums
and the max-over-ranks time equal the single-process values.  The sweeps here
run the CPU oracle: this tests the plumbing, not the kernel.
"""
import os
import socket

import numpy as np
import pytest
import torch.multiprocessing as mp

from minisweep_b200.parallel import group_slice


def test_group_slices_cover_exactly_once():
    for ne in [1, 2, 3, 7, 8, 64, 65]:
        for world in [1, 2, 3, 4, 8]:
            seen = []
            for r in range(world):
                a, b = group_slice(ne, world, r)
                assert 0 <= a <= b <= ne
                seen += list(range(a, b))
                if b < ne and a < b:
                    assert b % 2 == 0  # slices start on group pairs
            assert seen == list(range(ne))


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _rank_main(rank, world, port, dims, out):
    import torch.distributed as dist

    import oracle
    from minisweep_b200.parallel import max_over_ranks, sum_norms

    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    import datetime
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    nx, ny, nz, ne, na, nm = dims
    a, m, vi = oracle.random_problem(nx, ny, nz, ne, nm, na, seed=9)
    g0, g1 = group_slice(ne, world, rank)
    vo = oracle.sweep(nx, ny, nz, ne, nm, na, a, m, vi, groups=(g0, g1))
    # this rank's share of the checksums: its groups only
    v_i = vi.reshape(nz, ne, -1)[:, g0:g1]
    v_o = vo.reshape(nz, ne, -1)[:, g0:g1]
    s = float(np.sum(v_o * v_o))
    d = float(np.sum((v_i - v_o) ** 2))
    s_all, d_all = sum_norms(s, d)
    t = max_over_ranks(0.5 + rank)
    out[rank] = (g0, g1, v_o.copy(), s_all, d_all, t)
    dist.barrier()
    dist.destroy_process_group()


@pytest.mark.timeout(300)
def test_two_rank_energy_split_matches_single_process():
    import oracle

    dims = (3, 4, 3, 5, 16, 16)
    nx, ny, nz, ne, na, nm = dims
    world = 2
    with mp.Manager() as man:
        out = man.dict()
        mp.start_processes(_rank_main, args=(world, _free_port(), dims, out), nprocs=world, join=True,
                           start_method="spawn")
        res = dict(out)
    a, m, vi = oracle.random_problem(nx, ny, nz, ne, nm, na, seed=9)
    full = oracle.sweep(nx, ny, nz, ne, nm, na, a, m, vi).reshape(nz, ne, -1)
    s_ref = float(np.sum(full * full))
    d_ref = float(np.sum((vi.reshape(nz, ne, -1) - full) ** 2))
    covered = []
    for r in range(world):
        g0, g1, v_o, s_all, d_all, t = res[r]
        assert np.array_equal(v_o, full[:, g0:g1])
        assert abs(s_all - s_ref) <= 1e-12 * s_ref and abs(d_all - d_ref) <= 1e-12 * d_ref
        assert t == 0.5 + (world - 1)
        covered += list(range(g0, g1))
    assert covered == list(range(ne))
