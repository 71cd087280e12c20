"""KBA x/y decomposition: host-side plan, message routing and subdomain
offsets (no GPU).

The reference's decomposed sweep (stepscheduler_kba.c:80-284, faces_kba.c,
quantities_testing_c.h:206-333) is checked here through its invariants: every
process sweeps every (octant, z-block) unit once, a unit starts only after the
upwind neighbours swept it, every face sent is received by the right
neighbour in the same step and arrives before that neighbour sweeps the unit.
"""
import ctypes
import subprocess
import sys

import numpy as np
import pytest

import minisweep_b200 as msb

GRIDS = [(1, 1, 1), (2, 1, 1), (1, 2, 1), (2, 2, 2), (4, 4, 1), (4, 4, 2), (4, 4, 4), (3, 5, 3), (8, 1, 2)]


@pytest.mark.parametrize("npx,npy,nb", GRIDS)
def test_plan_steps_and_dependencies(npx, npy, nb):
    nstep, oct_, zb, start = msb.kba_plan(npx, npy, nb)
    # the reference's step count for one octant per step (stepscheduler_kba.c:80-84)
    assert nstep == 8 * nb + 2 * (npx - 1) + 3 * (npy - 1)
    nunit = 8 * nb
    assert sorted(zip(oct_.tolist(), zb.tolist())) == [(o, b) for o in range(8) for b in range(nb)]
    for o in range(8):
        ks = [k for k in range(nunit) if oct_[k] == o]
        blocks = [int(zb[k]) for k in ks]
        # z-blocks of one octant in its upwind z order
        assert blocks == (list(range(nb)) if o & 4 == 0 else list(range(nb - 1, -1, -1)))
    for p in range(npx * npy):
        px, py = p % npx, p // npx
        assert np.all(np.diff(start[p]) >= 1), "one unit per process per step, in order"
        assert start[p].min() >= 0 and start[p].max() < nstep
        for k in range(nunit):
            dx = -1 if oct_[k] & 1 else 1
            dy = -1 if oct_[k] & 2 else 1
            if 0 <= px - dx < npx:
                assert start[p, k] > start[(px - dx) + npx * py, k]
            if 0 <= py - dy < npy:
                assert start[p, k] > start[px + npx * (py - dy), k]


@pytest.mark.parametrize("npx,npy,nb", GRIDS)
def test_messages_match_and_arrive_in_time(npx, npy, nb):
    nstep, oct_, zb, start = msb.kba_plan(npx, npy, nb)
    nproc = npx * npy
    msgs = {(p, s): msb.kba_plan_messages(npx, npy, nb, p, s) for p in range(nproc) for s in range(nstep)}
    received = set()
    for (p, s), lst in msgs.items():
        recv_slots = [(m["axis"], m["side"]) for m in lst if not m["is_send"]]
        assert len(recv_slots) == len(set(recv_slots)), "one receive per buffer per step"
        for m in lst:
            if m["is_send"]:
                assert start[p, m["unit"]] == s
                q = m["peer"]
                match = [r for r in msgs[(q, s)] if not r["is_send"] and r["peer"] == p]
                assert len(match) == 1
                r = match[0]
                assert (r["axis"], r["side"], r["unit"]) == (m["axis"], 1 - m["side"], m["unit"])
                assert start[q, m["unit"]] > s, "the face arrives before the neighbour sweeps the unit"
            else:
                q = m["peer"]
                assert any(x["is_send"] and x["peer"] == p and x["unit"] == m["unit"] for x in msgs[(q, s)])
                received.add((p, m["unit"], m["axis"]))
    # every unit with an upwind neighbour along an axis gets that axis's face
    for p in range(nproc):
        px, py = p % npx, p // npx
        for k in range(8 * nb):
            dx = -1 if oct_[k] & 1 else 1
            dy = -1 if oct_[k] & 2 else 1
            assert ((p, k, 0) in received) == (0 <= px - dx < npx)
            assert ((p, k, 1) in received) == (0 <= py - dy < npy)


def test_local_extent_matches_reference_split():
    # runner.c:95-106: ((p + 1) n) / P - (p n) / P
    for n in (1, 3, 5, 8, 17):
        for nproc in (1, 2, 3, 4):
            ext = [msb.local_extent(n, nproc, p) for p in range(nproc)]
            assert sum(e[1] for e in ext) == n
            assert all(ext[p][0] == sum(e[1] for e in ext[:p]) for p in range(nproc))


def _fake_comm(gx, gy, npx, npy):
    """Collectives of one process answered from the decomposition itself
    (the library gathers the local x sizes, then the y sizes)."""
    calls = []

    def allgather(nactive, v):
        axis = len(calls)
        calls.append(v)
        n, np_ = (gx, npx) if axis == 0 else (gy, npy)
        return [msb.local_extent(n, np_, (q % npx) if axis == 0 else (q // npx))[1] for q in range(nactive)]

    return msb.make_comm(lambda nactive, msgs: None, lambda nactive, x: x, allgather, lambda nactive: None)


@pytest.mark.parametrize("npx,npy", [(2, 1), (1, 3), (4, 4), (3, 2)])
def test_quantities_offsets_from_group(npx, npy):
    """Quantities_create on a decomposed grid sets ix_base / iy_base and the
    global sizes as the reference does (quantities_testing_c.h:206-333)."""
    L = msb.lib()
    gx, gy = 7, 5
    for p in range(npx * npy):
        comm = _fake_comm(gx, gy, npx, npy)
        env = msb.Env()
        L.Env_initialize(ctypes.byref(env), 0, None)
        assert L.msb_env_set_comm(ctypes.byref(env), p, npx * npy, ctypes.byref(comm)) == 0
        args = msb.Arguments()
        L.Arguments_create_from_string(ctypes.byref(args), f"--nproc_x {npx} --nproc_y {npy}".encode())
        L.Env_set_values(ctypes.byref(env), ctypes.byref(args))
        x0, nx = msb.local_extent(gx, npx, p % npx)
        y0, ny = msb.local_extent(gy, npy, p // npx)
        q = msb.Quantities()
        L.Quantities_create(ctypes.byref(q), msb.Dimensions(nx, ny, 3, 2, 4, 8), ctypes.byref(env))
        assert (q.ix_base, q.iy_base, q.ncell_x_g, q.ncell_y_g) == (x0, y0, gx, gy)
        # the initial state takes global coordinates (quantities_testing.h:60-90)
        v = np.zeros(nx * ny * 3 * 2 * 4 * 4)
        L.initialize_state(v.ctypes.data_as(ctypes.POINTER(ctypes.c_double)), msb.Dimensions(nx, ny, 3, 2, 4, 8),
                           4, ctypes.byref(q))
        L.Quantities_destroy(ctypes.byref(q))
        L.Arguments_destroy(ctypes.byref(args))
        L.Env_finalize(ctypes.byref(env))
        vg = np.zeros(gx * gy * 3 * 2 * 4 * 4)
        q1 = msb.Quantities()
        env1 = msb.Env()
        L.Env_initialize(ctypes.byref(env1), 0, None)
        L.Quantities_create(ctypes.byref(q1), msb.Dimensions(gx, gy, 3, 2, 4, 8), ctypes.byref(env1))
        L.initialize_state(vg.ctypes.data_as(ctypes.POINTER(ctypes.c_double)), msb.Dimensions(gx, gy, 3, 2, 4, 8),
                           4, ctypes.byref(q1))
        L.Quantities_destroy(ctypes.byref(q1))
        L.Env_finalize(ctypes.byref(env1))
        sub = vg.reshape(3, 2, gy, gx, 4, 4)[:, :, y0:y0 + ny, x0:x0 + nx]
        assert np.array_equal(v.reshape(3, 2, ny, nx, 4, 4), sub)


_INSIST = """
import ctypes, minisweep_b200 as msb
L = msb.lib()
env = msb.Env(); L.Env_initialize(ctypes.byref(env), 0, None)
args = msb.Arguments(); L.Arguments_create_from_string(ctypes.byref(args), b"--nproc_x 2 --nproc_y 1")
L.Env_set_values(ctypes.byref(env), ctypes.byref(args))
print("not reached")
"""


def test_grid_larger_than_group_is_refused():
    """env_mpi.c:119-126: more processes requested than there are -> Insist."""
    r = subprocess.run([sys.executable, "-c", _INSIST], capture_output=True, text=True, timeout=120)
    assert r.returncode != 0
    assert "Not enough processors available." in r.stderr
    assert "not reached" not in r.stdout


def test_set_comm_validates():
    L = msb.lib()
    env = msb.Env()
    assert L.msb_env_set_comm(ctypes.byref(env), 2, 2, None) == msb.MSB_ERR_ARG
    assert L.msb_env_set_comm(ctypes.byref(env), 0, 2, None) == msb.MSB_ERR_ARG  # a group needs callbacks
    assert L.msb_env_set_comm(ctypes.byref(env), 0, 1, None) == 0


# ------------------------------------------------ the group transport (gloo)
def _free_port():
    import socket

    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _group_rank(rank, world, port, npx, npy, out):
    import datetime
    import os

    import torch
    import torch.distributed as dist

    from minisweep_b200.parallel import TorchGroupComm

    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    L = msb.lib()
    tg = TorchGroupComm()
    env = msb.Env()
    L.Env_initialize(ctypes.byref(env), 0, None)
    assert L.msb_env_set_comm(ctypes.byref(env), rank, world, ctypes.byref(tg.comm)) == 0
    args = msb.Arguments()
    L.Arguments_create_from_string(ctypes.byref(args), f"--nproc_x {npx} --nproc_y {npy}".encode())
    L.Env_set_values(ctypes.byref(env), ctypes.byref(args))
    gx, gy = 9, 6
    x0, nx = msb.local_extent(gx, npx, rank % npx)
    y0, ny = msb.local_extent(gy, npy, rank // npx)
    dims = msb.Dimensions(nx, ny, 2, 3, 4, 8)
    q = msb.Quantities()
    L.Quantities_create(ctypes.byref(q), dims, ctypes.byref(env))  # allgather through the callbacks
    v = np.zeros(nx * ny * 2 * 3 * 4 * 4)
    DP = ctypes.POINTER(ctypes.c_double)
    L.initialize_state(v.ctypes.data_as(DP), dims, 4, ctypes.byref(q))
    s, d = ctypes.c_double(), ctypes.c_double()
    L.get_state_norms(v.ctypes.data_as(DP), np.zeros_like(v).ctypes.data_as(DP), dims, 4, ctypes.byref(s),
                      ctypes.byref(d), ctypes.byref(env))  # Env_sum_P through the callbacks
    # one step's messages: every rank sends its number to its x neighbours
    send = torch.full((64,), rank, dtype=torch.uint8)
    recv = torch.zeros(64, dtype=torch.uint8)
    tg.buffers = {send.data_ptr(): send, recv.data_ptr(): recv}
    msgs = []
    px = rank % npx
    if px + 1 < npx:
        msgs.append(msb.KbaMsg(rank + 1, 1, 0, 1, 64, send.data_ptr()))
    if px > 0:
        msgs.append(msb.KbaMsg(rank - 1, 0, 0, 0, 64, recv.data_ptr()))
    arr = (msb.KbaMsg * max(1, len(msgs)))(*msgs)
    rc = tg.comm.exchange(None, world, arr, len(msgs))  # the C entry point the library calls
    out[rank] = (q.ix_base, q.iy_base, q.ncell_x_g, q.ncell_y_g, s.value, d.value, rc, int(recv[0]), int(recv[-1]))
    L.Quantities_destroy(ctypes.byref(q))
    dist.barrier()
    dist.destroy_process_group()


@pytest.mark.timeout(300)
@pytest.mark.parametrize("npx,npy", [(2, 1), (2, 2)])
def test_group_transport_gloo(npx, npy):
    import torch.multiprocessing as mp

    world = npx * npy
    with mp.Manager() as man:
        out = man.dict()
        mp.start_processes(_group_rank, args=(world, _free_port(), npx, npy, out), nprocs=world, join=True,
                           start_method="spawn")
        res = dict(out)
    # the single-process norms of the whole initial state (vo = 0: normsq 0)
    L = msb.lib()
    env = msb.Env()
    L.Env_initialize(ctypes.byref(env), 0, None)
    q = msb.Quantities()
    dims = msb.Dimensions(9, 6, 2, 3, 4, 8)
    L.Quantities_create(ctypes.byref(q), dims, ctypes.byref(env))
    v = np.zeros(9 * 6 * 2 * 3 * 4 * 4)
    DP = ctypes.POINTER(ctypes.c_double)
    L.initialize_state(v.ctypes.data_as(DP), dims, 4, ctypes.byref(q))
    L.Quantities_destroy(ctypes.byref(q))
    d_ref = float(np.sum(v * v))
    for r in range(world):
        ixb, iyb, gx, gy, s, d, rc, r0, r1 = res[r]
        assert (ixb, iyb) == (msb.local_extent(9, npx, r % npx)[0], msb.local_extent(6, npy, r // npx)[0])
        assert (gx, gy) == (9, 6)
        assert s == 0.0 and d == d_ref  # every rank holds the group's sum
        assert rc == 0
        if r % npx > 0:
            assert r0 == r1 == r - 1


# ------------------------------------------------ the node-local group
@pytest.mark.timeout(300)
def test_node_group_collectives(tmp_path):
    """Four processes started by the launcher join one group in
    Env_initialize; grids of 1, 2, 3 and 4 of them run the library's
    allgather (subdomain offsets) and sum (norms) through shared memory,
    with the processes a grid leaves out going straight on to the next grid
    (per-size barriers keep them apart, as the reference's per-run
    communicators do)."""
    import json
    import os

    from minisweep_b200 import launch

    child = os.path.join(os.path.dirname(__file__), "kba_group_child.py")
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    env = dict(os.environ, CUDA_VISIBLE_DEVICES="", PYTHONPATH=root)
    assert launch.run(4, [sys.executable, child, str(tmp_path)], timeout=240, env=env) == 0
    import kba_group_child as kc

    # single-process reference: the whole initial state's sum of squares
    L = msb.lib()
    e1 = msb.Env()
    L.Env_initialize(ctypes.byref(e1), 0, None)
    q = msb.Quantities()
    dims = msb.Dimensions(kc.GX, kc.GY, kc.NZ, kc.NE, kc.NM, kc.NA)
    L.Quantities_create(ctypes.byref(q), dims, ctypes.byref(e1))
    v = np.zeros(kc.GX * kc.GY * kc.NZ * kc.NE * kc.NM * 4)
    L.initialize_state(v.ctypes.data_as(ctypes.POINTER(ctypes.c_double)), dims, 4, ctypes.byref(q))
    L.Quantities_destroy(ctypes.byref(q))
    d_ref = float(np.sum(v * v))
    for p in range(4):
        res = json.load(open(tmp_path / f"proc_{p}.json"))
        assert (res["proc"], res["nproc"]) == (p, 4)
        for (npx, npy), run in zip(kc.GRIDS, res["runs"]):
            if p >= npx * npy:
                assert run is None
                continue
            ixb, iyb, gx, gy, d = run
            assert (ixb, iyb) == (msb.local_extent(kc.GX, npx, p % npx)[0], msb.local_extent(kc.GY, npy, p // npx)[0])
            assert (gx, gy) == (kc.GX, kc.GY)
            assert d == d_ref
