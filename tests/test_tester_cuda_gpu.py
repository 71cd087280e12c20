"""The reference tester's CUDA battery on the B200 library.

tester.c's CUDA case lists (test_cuda, tester.c:290-390, and the
single-process pairs of test_mpi_cuda, tester.c:431-476) only run in a build
with USE_MPI, which the drop-in tester binaries cannot have here, so the same
case lists are restated below and run through `compare_runs`, this package's
mirror of runner.c:187-241 (both runs normsqdiff == 0, equal normsq).  The
flag sets exercise the reference's device decomposition (--nthread_e,
--nthread_octant, subblock sizes, --nthread_y/z, --is_using_device); on the
B200 they are validated and recorded, and the result must not depend on them.
"""
import itertools

import pytest

import minisweep_b200 as msb

pytestmark = pytest.mark.gpu


def cuda_battery():
    """(common, string1, string2) of every pair of test_cuda, in tester.c's order."""
    pairs = []
    common1 = "--ncell_x 2 --ncell_y 3 --ncell_z 4 --ne 20 --na 5 --nblock_z 2"
    for key in range(4):  # tester.c:312-322
        pairs.append((common1, "", f"--is_using_device 1 --nthread_e 1 --nthread_octant {1 << key}"))
    for nthread_e in range(1, 21):  # tester.c:326-333
        pairs.append((common1, "", f"--is_using_device 1 --nthread_e {nthread_e} --nthread_octant 8"))
    nx, ny, nz = 3, 4, 2  # tester.c:337-389
    common2 = f"--ncell_x {nx} --ncell_y {ny} --ncell_z {nz}  --ne 2 --na 32"
    for sx, sy, sz, ty, tz, te, to in itertools.product(range(1, nx + 2), range(1, ny + 2), range(1, nz + 2),
                                                        (1, 2), (1, 2), (1, 2), (1, 2)):
        pairs.append((common2, "", f"--ncell_x_per_subblock {sx} --ncell_y_per_subblock {sy} "
                                   f"--ncell_z_per_subblock {sz} --nthread_y {ty} --nthread_z {tz} "
                                   f"--nthread_e {te} --nthread_octant {to} --is_using_device 1"))
    return pairs


def mpi_cuda_single_process():
    """The pairs of test_mpi_cuda with --nproc_x 1 --nproc_y 1 (tester.c:444-476)."""
    common = "--ncell_x 3 --ncell_y 5 --ncell_z 6 --ne 2 --na 5 --nblock_z 2"
    return [(common, "", f"--is_using_device 1 --nproc_x 1 --nproc_y 1 --nthread_e 3 --nthread_octant {1 << k}")
            for k in range(4)]


def run_battery(pairs, nm):
    failed = []
    for common, s1, s2 in pairs:
        a1, a2 = f"{common} {s1}", f"{common} {s2}"
        if not msb.compare_runs(a1, a2, nm):
            failed.append((a1, a2))
    return failed


def test_battery_size():
    # 4 + 20 + 4*5*3*2*2*2*2 pairs, as the reference's CUDA build counts them
    assert len(cuda_battery()) == 984


@pytest.mark.parametrize("nm", [16, 4])
def test_cuda_battery(nm):
    pairs = cuda_battery()
    failed = run_battery(pairs, nm)
    assert not failed, f"{len(failed)} of {len(pairs)} pairs failed, first: {failed[:3]}"


def test_mpi_cuda_single_process_pairs():
    assert not run_battery(mpi_cuda_single_process(), 16)
