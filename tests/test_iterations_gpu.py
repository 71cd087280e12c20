"""Sweeper_sweep_iterations (host buffers in and out, the reference driver's
iteration loop of runner.c:148-155 in one call) against the same iterations
run sweep by sweep on device arrays.

On a large FP64 problem the call sweeps the energy groups in slices of group
pairs, so that one slice's host copies overlap another slice's sweeps; the
groups are independent in the sweep, so the results must be equal bit for
bit to the unsliced iterations.  Inputs are random (the built-in state is a
fixed point of the sweep, which would hide a missing or repeated sweep).
"""
import numpy as np
import pytest

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu

import minisweep_b200 as msb  # noqa: E402


def flags(nx, ny, nz, ne, na, extra=""):
    return f"--ncell_x {nx} --ncell_y {ny} --ncell_z {nz} --ne {ne} --na {na} {extra}"


def device_iterations(pb, vi_host, niter):
    """niter sweeps on device arrays through Sweeper_sweep_device."""
    dev = torch.device("cuda:0")
    a = torch.from_numpy(vi_host).to(dev)
    b = torch.empty_like(a)
    torch.cuda.synchronize()
    for _ in range(niter):
        pb.sweep_device(b.data_ptr(), a.data_ptr())
        pb.sync()
        a, b = b, a
    torch.cuda.synchronize()
    return a.cpu().numpy()


def host_iterations(pb, vi_host, niter, pinned=True):
    if pinned:
        hin = torch.from_numpy(vi_host).pin_memory()
        hout = torch.empty_like(hin).pin_memory()
        pb.sweep_iterations_host(hout.data_ptr(), hin.data_ptr(), niter)
        return hout.numpy().copy()
    hin = np.ascontiguousarray(vi_host)
    hout = np.empty_like(hin)
    pb.sweep_iterations_host(hout.ctypes.data, hin.ctypes.data, niter)
    return hout


def random_state(pb, seed):
    return np.random.default_rng(seed).random(pb.nstate)


@pytest.mark.parametrize("nx,ny,nz,ne,na,nm,niter,slices", [
    (6, 5, 4, 7, 32, 16, 3, 1),        # small: one piece
    (32, 32, 32, 32, 32, 16, 2, 2),    # 537 MB of state, 16 group pairs: 2 slices
    (32, 32, 32, 33, 80, 16, 1, 2),    # odd ne (the last slice ends in a single group), two angle passes
    (24, 24, 24, 64, 32, 16, 3, 4),    # 32 group pairs: 4 slices, odd iteration count (result in vo)
])
def test_iterations_match_device_sweeps(nx, ny, nz, ne, na, nm, niter, slices):
    with msb.Problem(flags(nx, ny, nz, ne, na), nm=nm) as pb:
        vi = random_state(pb, 5)
        ref = device_iterations(pb, vi, niter)
        got = host_iterations(pb, vi, niter)
        assert pb.iterations_slices() == slices
    assert np.array_equal(got, ref), f"max abs diff {np.max(np.abs(got - ref))}"


@pytest.mark.parametrize("nx,ny,nz,ne,na,prec,niter", [
    (32, 32, 32, 32, 32, 1, 2),   # FP16 halves, 2 slices
    (32, 32, 32, 33, 64, 2, 1),   # BF16 halves, odd ne, two angle passes (the partial sum adds)
])
def test_mixed_iterations_sliced(nx, ny, nz, ne, na, prec, niter):
    """The mixed-precision sweeper goes in slices too: the vi conversion and
    the partial sum cover each slice's groups, and the results are those of
    the whole-problem sweeps, bit for bit."""
    with msb.Problem(flags(nx, ny, nz, ne, na, f"--precision {prec}"), nm=16) as pb:
        vi = random_state(pb, 8)
        ref = device_iterations(pb, vi, niter)
        got = host_iterations(pb, vi, niter)
        assert pb.iterations_slices() == 2
        one = pb.sweep_host(vi)
        assert pb.iterations_slices() == 2
        ref1 = device_iterations(pb, vi, 1)
    assert np.array_equal(got, ref), f"max abs diff {np.max(np.abs(got - ref))}"
    assert np.array_equal(one, ref1)


def test_host_pointer_sweep_sliced():
    """Sweeper_sweep (host Pointers, the reference driver's call) goes in
    slices too."""
    with msb.Problem(flags(32, 32, 32, 32, 32), nm=16) as pb:
        vi = random_state(pb, 4)
        ref = device_iterations(pb, vi, 1)
        got = pb.sweep_host(vi)
        assert pb.iterations_slices() == 2
    assert np.array_equal(got, ref)


def test_sliced_run_from_pageable_buffers():
    with msb.Problem(flags(32, 32, 32, 32, 32), nm=16) as pb:
        vi = random_state(pb, 9)
        ref = device_iterations(pb, vi, 2)
        got = host_iterations(pb, vi, 2, pinned=False)
        assert pb.iterations_slices() == 2
    assert np.array_equal(got, ref)


def test_autotuning_sweeper_slices_once_tuned():
    """The first sweep of --autotune 1 times every plan on the whole problem;
    the slices are cut from the plan it keeps."""
    with msb.Problem(flags(32, 32, 32, 32, 32, "--autotune 1"), nm=16) as pb:
        vi = random_state(pb, 3)
        first = host_iterations(pb, vi, 2)
        assert pb.iterations_slices() == 1
        second = host_iterations(pb, vi, 2)
        assert pb.iterations_slices() == 2
        ref = device_iterations(pb, vi, 2)
    assert np.array_equal(first, ref) and np.array_equal(second, ref)


def test_zero_iterations_copy_through():
    with msb.Problem(flags(32, 32, 32, 32, 32), nm=16) as pb:
        vi = random_state(pb, 1)
        got = host_iterations(pb, vi, 0)
        assert pb.iterations_slices() == 1
    assert np.array_equal(got, vi)


def test_sliced_run_reports_timeout_and_recovers():
    """A forced 1 ns wait budget: the first wait that spins gives up, the
    error survives the later slices' sweeps (which end at once) and the call
    returns MSB_ERR_TIMEOUT; with the default budget the next call is right."""
    with msb.Problem(flags(32, 32, 32, 32, 32), nm=16) as pb:
        vi = random_state(pb, 6)
        ref = device_iterations(pb, vi, 2)
        pb.set_timeout_ns(1)
        with pytest.raises(msb.SweepError) as e:
            host_iterations(pb, vi, 2)
        assert e.value.code == msb.MSB_ERR_TIMEOUT
        assert pb.iterations_slices() == 2
        pb.set_timeout_ns(0)
        got = host_iterations(pb, vi, 2)
    assert np.array_equal(got, ref)
