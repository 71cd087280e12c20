"""msb_sweep_noalloc: the sweep for callers that cannot allocate device memory.

Callers whose device memory belongs to a pool or arena, or that must not
trigger the device synchronisation an allocation can cause, get a sweep whose
scratch (task table, progress counters, face planes) lives in a fixed
file-scope device array of the library.  This file checks, through the C ABI,
that its output equals the regular entry point's (Sweeper_sweep_device, which
allocates its scratch once in Sweeper_create) on two calls in a row -- the
built-in problem bit for bit, a random-input problem to the 1e-12 relative
tolerance of the other GPU tests -- and that sizes beyond the fixed array are
refused.  It is collected last so that a run stopping at the first failure has
run every other test; it also passes alone in a fresh process.
"""
import ctypes

import numpy as np
import pytest

import oracle

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu

import minisweep_b200 as msb  # noqa: E402

RTOL_FP64 = 1e-12


def noalloc():
    L = msb.lib()
    f = L.msb_sweep_noalloc
    f.argtypes = [ctypes.c_void_p] * 4 + [ctypes.c_int] * 6 + [ctypes.c_void_p]
    f.restype = ctypes.c_int
    return f


def regular_and_noalloc(nx, ny, nz, ne, na, nm, a=None, m=None, vi=None):
    """The same sweep through the regular entry point and the no-allocation
    one; returns both outputs (host arrays)."""
    dev = torch.device("cuda:0")
    with msb.Problem(f"--ncell_x {nx} --ncell_y {ny} --ncell_z {nz} --ne {ne} --na {na}", nm=nm) as pb:
        if a is not None:
            pb.set_matrices(a, m)
        if vi is None:
            vi = pb.init_state()
        a_h, m_h = pb.matrices()
        d_vi = torch.from_numpy(np.ascontiguousarray(vi)).to(dev)
        d_a = torch.from_numpy(a_h.copy()).to(dev)
        d_m = torch.from_numpy(m_h.copy()).to(dev)
        d_ref = torch.full_like(d_vi, float("nan"))
        d_out = torch.full_like(d_vi, float("nan"))
        torch.cuda.synchronize()
        pb.sweep_device(d_ref.data_ptr(), d_vi.data_ptr())
        pb.sync()
        stream = torch.cuda.current_stream(dev).cuda_stream
        rc = noalloc()(d_out.data_ptr(), d_vi.data_ptr(), d_a.data_ptr(), d_m.data_ptr(), nx, ny, nz, ne, nm, na,
                       stream)
        assert rc == msb.MSB_OK, msb.last_error()
        torch.cuda.synchronize()
        return d_ref.cpu().numpy(), d_out.cpu().numpy(), vi


def test_noalloc_matches_regular_builtin_twice():
    # two calls in a row: the second reuses the array the first left behind
    for nx, ny, nz, ne in [(8, 8, 8, 8), (6, 5, 7, 3)]:
        ref, out, vi = regular_and_noalloc(nx, ny, nz, ne, 32, 16)
        assert np.array_equal(out, ref)
        s, d = oracle.norms(vi, out)
        assert d == 0.0 and s == oracle.normsq_closed_form(nx, ny, nz, ne, 16)


def test_noalloc_matches_regular_random_twice():
    for seed in (5, 6):
        nx, ny, nz, ne, na, nm = 5, 4, 6, 5, 24, 16
        a, m, vi = oracle.random_problem(nx, ny, nz, ne, nm, na, seed=seed)
        ref, out, _ = regular_and_noalloc(nx, ny, nz, ne, na, nm, a, m, vi)
        assert np.max(np.abs(out - ref)) / np.max(np.abs(ref)) <= RTOL_FP64


def test_noalloc_nm4_matches_regular():
    ref, out, _ = regular_and_noalloc(7, 6, 5, 4, 32, 4)
    assert np.array_equal(out, ref)


def test_noalloc_refuses_sizes_beyond_the_array():
    f = noalloc()
    one = torch.zeros(8, dtype=torch.float64, device="cuda:0")
    p = one.data_ptr()
    # 64^3 cells x 64 groups: more tasks than the static schedule holds
    rc = f(p, p, p, p, 64, 64, 64, 64, 16, 32, None)
    assert rc == msb.MSB_ERR_ARG
    assert "schedule" in msb.last_error()
    # 16^3 cells x 8 groups: 2048 tasks fit the schedule, but the face planes
    # (3 x 16 MiB) do not fit the 32 MiB array
    rc = f(p, p, p, p, 16, 16, 16, 8, 16, 32, None)
    assert rc == msb.MSB_ERR_ARG
    assert "bytes of scratch" in msb.last_error()
    rc = f(p, p, p, p, 4, 4, 4, 2, 8, 32, None)  # NM 8: not in this entry point
    assert rc == msb.MSB_ERR_UNSUPPORTED


def test_noalloc_call_allocates_no_device_memory():
    # After one call on the device (which commits the array), further calls
    # -- here with another problem shape, so the schedule is rebuilt -- leave
    # the device's free memory unchanged.
    dev = torch.device("cuda:0")
    shapes = [(6, 5, 7, 3), (8, 8, 8, 8)]
    bufs = []
    for nx, ny, nz, ne in shapes:
        with msb.Problem(f"--ncell_x {nx} --ncell_y {ny} --ncell_z {nz} --ne {ne} --na 32", nm=16) as pb:
            vi = pb.init_state()
            a_h, m_h = pb.matrices()
            bufs.append((torch.from_numpy(vi).to(dev), torch.empty(vi.size, dtype=torch.float64, device=dev),
                         torch.from_numpy(a_h.copy()).to(dev), torch.from_numpy(m_h.copy()).to(dev)))
    torch.cuda.synchronize()
    f = noalloc()
    stream = torch.cuda.current_stream(dev).cuda_stream

    def call(i):
        nx, ny, nz, ne = shapes[i]
        d_vi, d_vo, d_a, d_m = bufs[i]
        assert f(d_vo.data_ptr(), d_vi.data_ptr(), d_a.data_ptr(), d_m.data_ptr(), nx, ny, nz, ne, 16, 32,
                 stream) == msb.MSB_OK, msb.last_error()

    call(0)
    free0 = torch.cuda.mem_get_info(dev)[0]
    call(1)
    call(0)
    assert torch.cuda.mem_get_info(dev)[0] == free0
    assert torch.equal(bufs[0][1], bufs[0][0])  # the built-in problem is a fixed point of the sweep


def test_noalloc_refuses_a_capturing_stream():
    dev = torch.device("cuda:0")
    one = torch.zeros(8, dtype=torch.float64, device=dev)
    p = one.data_ptr()
    f = noalloc()
    s = torch.cuda.Stream(dev)
    g = torch.cuda.CUDAGraph()
    with torch.cuda.stream(s):
        g.capture_begin()
        try:
            rc = f(p, p, p, p, 4, 4, 4, 2, 16, 32, s.cuda_stream)
        finally:
            g.capture_end()
    assert rc == msb.MSB_ERR_UNSUPPORTED
    assert "capturing" in msb.last_error()
