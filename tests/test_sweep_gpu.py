"""GPU parity of the FP64 sweep against the CPU oracle (oracle/sweep_oracle.c).

* Built-in deterministic Quantities: the reference's own pass criterion is
  normsqdiff == 0 (sweep.c:53-56); here vo must also equal the oracle's vo
  bit for bit, and normsq must equal the closed form.
* Random inputs (vi ~ U[0,1), a_from_m ~ N(0, 1/nm), m_from_a = pinv): vo must
  match the oracle to 1e-12 relative (max |vo - vo_oracle| / max |vo_oracle|);
  the two differ only in the order of FP64 additions inside the transforms.
"""
import numpy as np
import pytest

import oracle

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu

import minisweep_b200 as msb  # noqa: E402

RTOL_FP64 = 1e-12


def flags(nx, ny, nz, ne, na, extra=""):
    return f"--ncell_x {nx} --ncell_y {ny} --ncell_z {nz} --ne {ne} --na {na} {extra}"


def run_builtin(nx, ny, nz, ne, na, nm, extra=""):
    with msb.Problem(flags(nx, ny, nz, ne, na, extra), nm=nm) as pb:
        vi = pb.init_state()
        vo = pb.sweep_host(vi)
    return vi, vo


# tester.c:46-99 (serial battery sizes) and tester.c:312-389 (CUDA battery, na 32)
BUILTIN = [
    (2, 1, 2, 3, 7, 16),
    (5, 4, 5, 3, 7, 16),
    (5, 4, 5, 3, 7, 4),
    (3, 4, 2, 5, 32, 16),
    (1, 1, 1, 1, 1, 4),
    (4, 3, 5, 20, 32, 16),
    (5, 5, 5, 30, 33, 16),   # the reference's default flags
    (7, 6, 5, 4, 64, 16),
    (6, 5, 4, 3, 100, 8),    # na > 32: passes over angle ranges, later passes add to vo
    (4, 4, 4, 2, 128, 16),
    (3, 4, 5, 3, 65, 16),    # a one-angle last pass
    (16, 16, 16, 16, 32, 4),  # the CPU-runnable headline case
]


@pytest.mark.parametrize("nx,ny,nz,ne,na,nm", BUILTIN)
def test_builtin_bitexact(nx, ny, nz, ne, na, nm):
    vi, vo = run_builtin(nx, ny, nz, ne, na, nm)
    a, m = oracle.am_matrices(nm, na)
    ref = oracle.sweep(nx, ny, nz, ne, nm, na, a, m, vi)
    assert np.array_equal(vo, ref), f"max abs diff {np.max(np.abs(vo - ref))}"
    normsq, normsqdiff = oracle.norms(vi, vo)
    assert normsqdiff == 0.0
    assert normsq == oracle.normsq_closed_form(nx, ny, nz, ne, nm)


@pytest.mark.parametrize("nx,ny,nz,ne,na,nm", BUILTIN)
def test_builtin_bitexact_chained_kernel(nx, ny, nz, ne, na, nm):
    # the chained-wavefront FP64 kernel (--fp64_kernel 1; 32-angle passes)
    vi, vo = run_builtin(nx, ny, nz, ne, na, nm, "--fp64_kernel 1")
    a, m = oracle.am_matrices(nm, na)
    ref = oracle.sweep(nx, ny, nz, ne, nm, na, a, m, vi)
    assert np.array_equal(vo, ref), f"max abs diff {np.max(np.abs(vo - ref))}"


@pytest.mark.parametrize("extra", ["--nblock_z 2", "--nthread_octant 8 --nthread_e 4",
                                   "--nthread_octant 2 --nsemiblock 2 --ncell_x_per_subblock 1",
                                   "--is_face_comm_async 0 --nthread_y 2 --nthread_z 2"])
def test_builtin_flags_invariant(extra):
    # compare_runs (runner.c:187-241): the result must not depend on the
    # sweeper's blocking/threading flags
    vi0, vo0 = run_builtin(4, 5, 6, 3, 32, 16)
    vi1, vo1 = run_builtin(4, 5, 6, 3, 32, 16, extra)
    assert np.array_equal(vo0, vo1)


@pytest.mark.parametrize("nx,ny,nz,ne,na,nm,extra", [
    (5, 4, 5, 3, 7, 16, "--tile 24"),
    (7, 6, 5, 4, 64, 16, "--tile 24"),
    (9, 7, 6, 5, 32, 4, "--tile 42"),
    (9, 7, 6, 5, 32, 16, "--autotune 1"),
    (6, 5, 4, 3, 40, 8, "--autotune 1 --tile 24"),
    (5, 4, 3, 3, 128, 16, "--tile 24"),      # several angle passes
    (4, 5, 3, 2, 100, 4, "--autotune 1"),    # a ragged last angle pass
    (7, 6, 5, 4, 64, 16, "--tile 24 --fp64_kernel 1"),
    (4, 5, 3, 2, 100, 4, "--autotune 1 --fp64_kernel 1"),
    (5, 4, 3, 3, 128, 16, "--angle_pass 32"),   # four 32-angle passes of the staged kernel
    (6, 5, 4, 3, 40, 8, "--angle_pass 32 --tile 24"),
    (4, 5, 3, 2, 20, 4, "--angle_pass 64"),     # a 64-angle pass over 20 angles
])
def test_tile_shapes_bitexact(nx, ny, nz, ne, na, nm, extra):
    # the 2 x 4 tile (and the autotuned choice, whose first sweep runs both
    # shapes) gives the same bits as the oracle, sweep after sweep
    with msb.Problem(flags(nx, ny, nz, ne, na, extra), nm=nm) as pb:
        vi = pb.init_state()
        vo1 = pb.sweep_host(vi)
        vo2 = pb.sweep_host(vi)
        t = pb.tile()
    a, m = oracle.am_matrices(nm, na)
    ref = oracle.sweep(nx, ny, nz, ne, nm, na, a, m, vi)
    assert np.array_equal(vo1, ref) and np.array_equal(vo2, ref)
    assert (t["tx"], t["ty"]) in ((4, 2), (2, 4))
    if "--autotune 1" in extra:
        assert 0.0 < t["ms_chosen"] <= t["ms_other"]
    elif "--tile 24" in extra:
        assert (t["tx"], t["ty"]) == (2, 4)
    if "--angle_pass" in extra:
        assert t["angle_pass"] == int(extra.split("--angle_pass ")[1].split()[0])


RANDOM = [
    (3, 2, 4, 3, 16, 16),
    (5, 4, 3, 4, 32, 16),
    (4, 4, 4, 5, 33, 16),
    (6, 3, 5, 2, 64, 8),
    (3, 5, 4, 3, 128, 16),
    (5, 5, 5, 4, 32, 4),
    (4, 3, 4, 3, 97, 8),
]


@pytest.mark.parametrize("kernel", [0, 1])
@pytest.mark.parametrize("nx,ny,nz,ne,na,nm", RANDOM)
def test_random_inputs(nx, ny, nz, ne, na, nm, kernel):
    a, m, vi = oracle.random_problem(nx, ny, nz, ne, nm, na, seed=1234)
    with msb.Problem(flags(nx, ny, nz, ne, na, f"--fp64_kernel {kernel}"), nm=nm) as pb:
        pb.set_matrices(a, m)
        vo = pb.sweep_host(vi)
    ref = oracle.sweep(nx, ny, nz, ne, nm, na, a, m, vi)
    err = np.max(np.abs(vo - ref)) / np.max(np.abs(ref))
    assert err <= RTOL_FP64, err
    s, _ = oracle.norms(vi, vo)
    s_ref, _ = oracle.norms(vi, ref)
    assert abs(s - s_ref) <= RTOL_FP64 * s_ref


def test_device_path_and_norms():
    nx, ny, nz, ne, na, nm = 8, 8, 8, 4, 32, 16
    with msb.Problem(flags(nx, ny, nz, ne, na), nm=nm) as pb:
        dev = torch.device("cuda:0")
        vi = torch.empty(pb.nstate, dtype=torch.float64, device=dev)
        vo = torch.empty_like(vi)
        pb.init_state_device(vi.data_ptr())
        torch.cuda.synchronize()
        pb.sweep_device(vo.data_ptr(), vi.data_ptr())
        pb.sync()
        s, d = pb.norms_device(vi.data_ptr(), vo.data_ptr())
        assert d == 0.0
        assert s == oracle.normsq_closed_form(nx, ny, nz, ne, nm)
        host_vi = pb.init_state()
        assert np.array_equal(vi.cpu().numpy(), host_vi)
        # two iterations with the vi/vo swap (runner.c:148-155)
        pb.sweep_device(vi.data_ptr(), vo.data_ptr())
        pb.sync()
        assert np.array_equal(vi.cpu().numpy(), host_vi)


def test_timeout_reports_error_and_recovers():
    # A forced 1 ns wait budget makes the first wait that has to spin give up:
    # the kernel records MSB_ERR_TIMEOUT and every CTA returns; the context
    # stays usable and the next sweep with the default budget is correct.
    # 16^3 cells x 4 group pairs is 2048 tasks for 148 CTAs: the tiles of the
    # first diagonal levels are grabbed together, and a downwind tile's first
    # plane always waits on its upwind neighbour, so a wait has to spin.
    nx, ny, nz, ne, na, nm = 16, 16, 16, 8, 32, 16
    with msb.Problem(flags(nx, ny, nz, ne, na), nm=nm) as pb:
        vi = pb.init_state()
        pb.set_timeout_ns(1)
        with pytest.raises(msb.SweepError) as e:
            pb.sweep_host(vi)
        assert e.value.code == msb.MSB_ERR_TIMEOUT
        assert "ran out of time" in str(e.value)
        pb.set_timeout_ns(0)
        vo = pb.sweep_host(vi)
        assert np.array_equal(vo, vi)


@pytest.mark.parametrize("prec", [0, 1])
def test_energy_slices_match_full_problem(prec):
    # The multi-GPU decomposition on one GPU: a 6-group problem swept whole
    # and as two energy-group slices (groups 0-3 and 4-5, --ie_base 4), each
    # slice with its own arrays and device-built initial state.  Groups are
    # independent in the sweep, so each slice equals its groups of the whole
    # sweep (FP64: bit for bit; mixed: the rows of a group pair do not mix,
    # so the same bits too), and the slices' checksums add up to the whole's.
    nx, ny, nz, ne, na, nm = 5, 4, 6, 6, 32, 16
    dev = torch.device("cuda:0")

    def sweep(ne_s, ie_base):
        with msb.Problem(flags(nx, ny, nz, ne_s, na, f"--ie_base {ie_base} --precision {prec}"), nm=nm) as pb:
            vi = torch.empty(pb.nstate, dtype=torch.float64, device=dev)
            vo = torch.empty_like(vi)
            pb.init_state_device(vi.data_ptr(), ie_base)
            torch.cuda.synchronize()
            pb.sweep_device(vo.data_ptr(), vi.data_ptr())
            pb.sync()
            s, d = pb.norms_device(vi.data_ptr(), vo.data_ptr())
            return vi.cpu().numpy().reshape(nz, ne_s, -1), vo.cpu().numpy().reshape(nz, ne_s, -1), s, d

    vi_f, vo_f, s_f, d_f = sweep(ne, 0)
    parts = [sweep(4, 0), sweep(2, 4)]
    vi_s = np.concatenate([p[0] for p in parts], axis=1)
    vo_s = np.concatenate([p[1] for p in parts], axis=1)
    assert np.array_equal(vi_s, vi_f)
    assert np.array_equal(vo_s, vo_f)
    # checksums: exact sums of integers for the FP64 sweep; the mixed result's
    # partial sums come in another order
    tol = 0.0 if prec == 0 else 1e-12
    assert abs(sum(p[2] for p in parts) - s_f) <= tol * s_f
    assert abs(sum(p[3] for p in parts) - d_f) <= tol * max(d_f, 1.0)
    if prec == 0:
        assert d_f == 0.0 and s_f == oracle.normsq_closed_form(nx, ny, nz, ne, nm)
