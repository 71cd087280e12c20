"""The reference's own driver programs, unmodified, on the B200 library.

oracle/Makefile's `dropin` target compiles the reference's src/4_driver/
runner.c + sweep.c and runner.c + tester.c against include/ and links them
with libminisweep_b200.so in place of the reference's libsweeper.  Here they
run on the GPU: `sweep` must print the reference's result line with PASS and
the reference's normsq, and each `tester` build must pass its whole battery
(the compare_runs pairs of tester.c, each requiring normsqdiff == 0 and equal
normsq across two flag sets) with exactly the pair count the reference's own
build of that configuration runs (measured on the reference's CPU builds:
serial 54, OpenMP threads 981, OpenMP tasks 64, variants 2).
"""
import os
import re
import subprocess

import pytest

import oracle

pytestmark = pytest.mark.gpu
REF = os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "oracle", "_ref")


def binary(name):
    p = os.path.join(REF, name)
    if not os.access(p, os.X_OK):
        pytest.skip(f"{name} not built (make -C oracle dropin)")
    return p


@pytest.mark.parametrize("nm,flags", [
    (16, "--ncell_x 5 --ncell_y 4 --ncell_z 6 --ne 3 --na 32 --nblock_z 2"),
    (16, "--ncell_x 8 --ncell_y 8 --ncell_z 8 --ne 8 --na 32 --niterations 3"),
    (4, "--ncell_x 16 --ncell_y 16 --ncell_z 16 --ne 16 --na 32"),
    (16, "--ncell_x 3 --ncell_y 5 --ncell_z 4 --ne 5 --na 33 --is_using_device 1 --nthread_octant 8 --nthread_e 5"),
])
def test_reference_sweep_driver(nm, flags):
    out = subprocess.run([binary(f"sweep_b200_nm{nm}")] + flags.split(), capture_output=True, text=True,
                         timeout=300)
    assert out.returncode == 0, out.stderr
    m = re.search(r"Normsq result: ([0-9.e+]+)\s+diff: ([0-9.e+-]+)\s+(PASS|FAIL)", out.stdout)
    assert m, out.stdout
    assert m.group(3) == "PASS" and float(m.group(2)) == 0.0
    d = dict(zip(flags.split()[::2], flags.split()[1::2]))
    ref = oracle.normsq_closed_form(int(d["--ncell_x"]), int(d["--ncell_y"]), int(d["--ncell_z"]),
                                    int(d["--ne"]), nm)
    assert abs(float(m.group(1)) - ref) <= 5e-9 * ref


def test_reference_sweep_driver_rejects_bad_flags():
    # Insist -> message + exit(EXIT_FAILURE), as the reference does
    out = subprocess.run([binary("sweep_b200_nm16"), "--ncell_z", "5", "--nblock_z", "2"], capture_output=True,
                         text=True, timeout=120)
    assert out.returncode != 0
    assert "Insist" in out.stderr


# (binary, pairs): tester.c's batteries are chosen by the build macros of
# the reference's configurations (tester.c:46-99 test_serial, :104-212
# test_openmp, :217-285 test_openmp_tasks, :511-546 test_variants).
BATTERIES = [
    ("tester_b200_nm16", 2),
    ("tester_b200_serial_nm16", 54),
    ("tester_b200_serial_nm4", 54),
    ("tester_b200_omp_nm4", 981),
    ("tester_b200_omp_nm16", 981),
    ("tester_b200_tasks_nm16", 64),
]


@pytest.mark.parametrize("name,pairs", BATTERIES)
def test_reference_tester_battery(name, pairs):
    out = subprocess.run([binary(name)], capture_output=True, text=True, timeout=1200)
    assert out.returncode == 0, out.stderr[-2000:]
    m = re.search(r"TESTS\s+(\d+)\s+PASSED\s+(\d+)\s+FAILED\s+(\d+)", out.stdout)
    assert m, out.stdout[-2000:]
    assert (int(m.group(1)), int(m.group(2)), int(m.group(3))) == (pairs, pairs, 0), out.stdout[-2000:]


# --------------------------------------------- the MPI builds, as a process group
# The reference's MPI configurations (tester.c:395-454 test_mpi with 16
# processes; tester.c:290-391 test_cuda + :458-509 test_mpi_cuda with 4),
# started by the node launcher in place of mpirun: the library's Env joins the
# launcher's group, the decomposed sweeps exchange their faces between the
# processes (CUDA IPC device copies), and the processes sharing this one GPU
# take turns with their sweep kernels.
def _launch(n, argv, timeout):
    import sys

    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    env = dict(os.environ, PYTHONPATH=root)
    return subprocess.run([sys.executable, "-m", "minisweep_b200.launch", "-n", str(n), "--timeout",
                           str(timeout), "--"] + argv, capture_output=True, text=True, timeout=timeout + 120,
                          env=env)


@pytest.mark.parametrize("name,nproc,pairs", [
    ("tester_b200_mpi_nm16", 16, 6),
    ("tester_b200_mpi_cuda_nm16", 4, 984 + 16),
])
def test_reference_mpi_tester_battery(name, nproc, pairs):
    out = _launch(nproc, [binary(name)], 1500)
    assert out.returncode == 0, out.stderr[-3000:]
    m = re.search(r"TESTS\s+(\d+)\s+PASSED\s+(\d+)\s+FAILED\s+(\d+)", out.stdout)
    assert m, out.stdout[-2000:]
    assert (int(m.group(1)), int(m.group(2)), int(m.group(3))) == (pairs, pairs, 0), out.stdout[-3000:]


@pytest.mark.parametrize("nproc,grid", [(2, "--nproc_x 2 --nproc_y 1"), (4, "--nproc_x 2 --nproc_y 2"),
                                        (6, "--nproc_x 3 --nproc_y 2")])
def test_reference_sweep_driver_decomposed(nproc, grid):
    """sweep.c on a process grid prints the single-process normsq."""
    flags = "--ncell_x 12 --ncell_y 9 --ncell_z 8 --ne 6 --na 32 --nblock_z 4 --niterations 2"
    out = _launch(nproc, [binary("sweep_b200_nm16")] + (flags + " " + grid).split(), 600)
    assert out.returncode == 0, out.stderr[-3000:]
    m = re.search(r"Normsq result: ([0-9.e+]+)\s+diff: ([0-9.e+-]+)\s+(PASS|FAIL)", out.stdout)
    assert m, out.stdout
    assert m.group(3) == "PASS" and float(m.group(2)) == 0.0
    single = subprocess.run([binary("sweep_b200_nm16")] + flags.split(), capture_output=True, text=True,
                            timeout=300)
    m1 = re.search(r"Normsq result: ([0-9.e+]+)", single.stdout)
    assert m1 and m1.group(1) == m.group(1)
