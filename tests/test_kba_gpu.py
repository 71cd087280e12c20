"""KBA x/y decomposition on the GPU, every process of the grid emulated in
one process on one GPU.

Each process of an nproc_x x nproc_y grid is a Problem of its own (its
subdomain, its Sweeper, its stream); the test drives the decomposed sweep step
by step and moves the face messages between the processes' buffers itself
after each step, so no kernel ever waits on another process's kernel.  The
subdomain results, put together, must equal the undecomposed sweep bit for bit
(the reference's test_mpi battery compares the norms of the same pairs,
tester.c:395-454, and test_mpi_cuda, tester.c:458-509).
"""
import numpy as np
import pytest

import minisweep_b200 as msb
import oracle

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")


def _parse(argstring):
    t = argstring.split()
    return {t[i]: int(t[i + 1]) for i in range(0, len(t), 2)}


def _group_comm(gx, gy, npx, npy):
    """Collectives of one emulated process, answered from the decomposition
    (the library gathers the local x sizes, then the y sizes)."""
    calls = []

    def allgather(nactive, v):
        axis = len(calls) % 2
        calls.append(v)
        n, np_ = (gx, npx) if axis == 0 else (gy, npy)
        return [msb.local_extent(n, np_, (q % npx) if axis == 0 else (q // npx))[1] for q in range(nactive)]

    return msb.make_comm(lambda nactive, msgs: None, lambda nactive, x: x, allgather, lambda nactive: None)


def sweep_decomposed(common, npx, npy, nblock_z, nm, vi_global, nsweep=1, extra=""):
    """vo of the global problem swept on an npx x npy grid of emulated
    processes (nsweep sweeps alternating vi -> vo -> vi as runner.c:148-155)."""
    kv = _parse(common)
    gx, gy, nz, ne, na = kv["--ncell_x"], kv["--ncell_y"], kv["--ncell_z"], kv["--ne"], kv["--na"]
    nproc = npx * npy
    args = f"{common} --nproc_x {npx} --nproc_y {npy} --nblock_z {nblock_z} {extra}"
    comms = [_group_comm(gx, gy, npx, npy) for _ in range(nproc)]
    probs = [msb.Problem(args, nm=nm, proc=p, nproc=nproc, comm=comms[p]) for p in range(nproc)]
    try:
        vg = vi_global.reshape(nz, ne, gy, gx, msb.NU, nm)
        a_d, b_d, bufs = [], [], []
        for pb in probs:
            x0, y0, nx, ny = pb.x0, pb.y0, pb.dims.ncell_x, pb.dims.ncell_y
            a_d.append(torch.from_numpy(np.ascontiguousarray(vg[:, :, y0:y0 + ny, x0:x0 + nx])).cuda().reshape(-1))
            b_d.append(torch.zeros_like(a_d[-1]))
            nstep, bx, by = pb.kba_info()
            sizes = [bx, by, bx, bx, by, by]
            bufs.append([torch.empty(max(s, 16), dtype=torch.uint8, device="cuda") for s in sizes])
            pb.kba_set_buffers(*[b.data_ptr() for b in bufs[-1]])
        torch.cuda.synchronize()
        nstep = probs[0].kba_info()[0]
        for it in range(nsweep):
            src, dst = (a_d, b_d) if it % 2 == 0 else (b_d, a_d)
            for p, pb in enumerate(probs):
                pb.kba_begin(dst[p].data_ptr(), src[p].data_ptr())
            for step in range(nstep):
                for pb in probs:
                    pb.kba_step(step)
                for p, pb in enumerate(probs):
                    for m in pb.kba_messages(step):
                        if not m.is_send:
                            continue
                        q = m.peer
                        recv = [r for r in probs[q].kba_messages(step)
                                if not r.is_send and r.peer == p and r.axis == m.axis]
                        assert len(recv) == 1 and recv[0].side == 1 - m.side and recv[0].bytes == m.bytes
                        slot = 2 + 2 * m.axis + recv[0].side
                        bufs[q][slot][:m.bytes].copy_(bufs[p][m.axis][:m.bytes])
                torch.cuda.synchronize()
                for pb in probs:
                    pb.kba_unpack(step)
            for pb in probs:
                pb.kba_end()
        out = (b_d if nsweep % 2 == 1 else a_d)
        vo = np.zeros_like(vg)
        for p, pb in enumerate(probs):
            x0, y0, nx, ny = pb.x0, pb.y0, pb.dims.ncell_x, pb.dims.ncell_y
            vo[:, :, y0:y0 + ny, x0:x0 + nx] = out[p].cpu().numpy().reshape(nz, ne, ny, nx, msb.NU, nm)
        return vo.reshape(-1)
    finally:
        for pb in probs:
            pb.close()


def sweep_single(common, nm, vi, nsweep=1, extra=""):
    with msb.Problem(f"{common} {extra}", nm=nm) as pb:
        v = vi
        for _ in range(nsweep):
            v = pb.sweep_host(v)
        return v


def init_global(common, nm):
    with msb.Problem(common, nm=nm) as pb:
        return pb.init_state()


# tester.c:417-453 (test_mpi) and :480-505 (test_mpi_cuda), plus larger cases
# with angle passes (na > 64), NM 4 and several z-blocks per process.
CASES = [
    ("--ncell_x 5 --ncell_y 4 --ncell_z 5 --ne 7 --na 10", 2, 1, 1, 16),
    ("--ncell_x 5 --ncell_y 4 --ncell_z 5 --ne 7 --na 10", 1, 2, 1, 16),
    ("--ncell_x 5 --ncell_y 4 --ncell_z 6 --ne 7 --na 10", 4, 4, 2, 16),
    ("--ncell_x 5 --ncell_y 8 --ncell_z 16 --ne 9 --na 12", 4, 4, 1, 16),
    ("--ncell_x 5 --ncell_y 8 --ncell_z 16 --ne 9 --na 12", 4, 4, 4, 16),
    ("--ncell_x 3 --ncell_y 5 --ncell_z 6 --ne 2 --na 5", 2, 2, 2, 16),
    ("--ncell_x 3 --ncell_y 5 --ncell_z 6 --ne 2 --na 5", 2, 1, 2, 4),
    ("--ncell_x 12 --ncell_y 10 --ncell_z 8 --ne 6 --na 96", 2, 3, 4, 16),
    ("--ncell_x 9 --ncell_y 7 --ncell_z 6 --ne 5 --na 40", 3, 2, 3, 4),
]


@pytest.mark.parametrize("common,npx,npy,nb,nm", CASES)
def test_decomposed_equals_single(common, npx, npy, nb, nm):
    vi = init_global(common, nm)
    ref = sweep_single(common, nm, vi)
    got = sweep_decomposed(common, npx, npy, nb, nm, vi)
    assert np.array_equal(got, ref), f"max abs diff {np.max(np.abs(got - ref))}"
    # the reference's check: the norms of both runs agree and the sweep
    # reproduces its input on the built-in problem (runner.c:187-241)
    with msb.Problem(common, nm=nm) as pb:
        n1, d1 = pb.state_norms(vi, ref)
        n2, d2 = pb.state_norms(vi, got)
    assert n1 == n2 and d1 == 0.0 and d2 == 0.0


def test_decomposed_matches_oracle_random_input():
    """Random state and matrices: the decomposed sweep against the oracle."""
    common = "--ncell_x 6 --ncell_y 5 --ncell_z 4 --ne 3 --na 32"
    nm = 4
    nx, ny, nz, ne, na = 6, 5, 4, 3, 32
    rng = np.random.default_rng(7)
    vi = rng.random(nx * ny * nz * ne * nm * msb.NU)
    a, m = msb.random_matrices(nm, na, seed=11)
    ref = oracle.sweep(nx, ny, nz, ne, nm, na, a.copy(), m.copy(), vi)
    # every emulated process gets the same matrices
    orig = msb.Problem.__init__

    def init(self, *args_, **kw):
        orig(self, *args_, **kw)
        self.set_matrices(a, m)

    msb.Problem.__init__ = init
    try:
        got = sweep_decomposed(common, 2, 2, 2, nm, vi)
    finally:
        msb.Problem.__init__ = orig
    assert np.allclose(got, ref, rtol=1e-12, atol=1e-12)


def test_decomposed_iterations_alternate():
    """Two sweeps (vi -> vo -> vi), as the driver's iteration loop runs them."""
    common = "--ncell_x 8 --ncell_y 6 --ncell_z 4 --ne 4 --na 16"
    vi = init_global(common, 16)
    ref = sweep_single(common, 16, vi, nsweep=2)
    got = sweep_decomposed(common, 2, 2, 2, 16, vi, nsweep=2)
    assert np.array_equal(got, ref)


def test_decomposed_refuses_other_kernels():
    common = "--ncell_x 4 --ncell_y 4 --ncell_z 4 --ne 2 --na 8 --nproc_x 2 --nproc_y 1"
    comm = _group_comm(4, 4, 2, 1)
    with pytest.raises(msb.SweepError) as e:
        msb.Problem(common + " --precision 1", nm=16, proc=0, nproc=2, comm=comm)
    assert e.value.code == msb.MSB_ERR_UNSUPPORTED


# ------------------------------------- the torch.distributed transport, 2 processes
def _torch_rank(rank, world, port, common, npx, npy, nm, out):
    import datetime
    import os

    import torch.distributed as dist

    from minisweep_b200.parallel import TorchGroupComm

    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=120))
    try:
        tg = TorchGroupComm()
        args = f"{common} --nproc_x {npx} --nproc_y {npy} --nblock_z 2"
        with msb.Problem(args, nm=nm, proc=rank, nproc=world, comm=tg.comm) as pb:
            # both processes drive this one GPU: their sweep kernels take turns
            pb.env.flags_ |= 1
            tg.attach(pb)
            vi = pb.init_state()
            vo = pb.sweep_host(vi)          # Sweeper_sweep: the library's step loop and the callbacks
            n2, d2 = pb.state_norms(vi, vo)  # Env_sum_P over the group
            out[rank] = (pb.x0, pb.y0, pb.dims.ncell_x, pb.dims.ncell_y, vo, n2, d2)
        dist.barrier()
    finally:
        dist.destroy_process_group()


@pytest.mark.timeout(600)
@pytest.mark.parametrize("npx,npy", [(2, 1), (1, 2)])
def test_torch_group_transport(npx, npy):
    import socket

    import torch.multiprocessing as mp

    common = "--ncell_x 7 --ncell_y 6 --ncell_z 4 --ne 3 --na 40"
    nm = 16
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    with mp.Manager() as man:
        out = man.dict()
        mp.start_processes(_torch_rank, args=(2, port, common, npx, npy, nm, out), nprocs=2, join=True,
                           start_method="spawn")
        res = dict(out)
    vi = init_global(common, nm)
    ref = sweep_single(common, nm, vi)
    kv = _parse(common)
    gx, gy, nz, ne = kv["--ncell_x"], kv["--ncell_y"], kv["--ncell_z"], kv["--ne"]
    got = np.zeros((nz, ne, gy, gx, msb.NU, nm))
    for r in range(2):
        x0, y0, nx, ny, vo, n2, d2 = res[r]
        got[:, :, y0:y0 + ny, x0:x0 + nx] = vo.reshape(nz, ne, ny, nx, msb.NU, nm)
        assert d2 == 0.0
    assert np.array_equal(got.reshape(-1), ref)
    with msb.Problem(common, nm=nm) as pb:
        n1, _ = pb.state_norms(vi, ref)
    assert all(res[r][5] == n1 for r in range(2))
