"""GPU checks of the mixed-precision sweep (--precision 1: FP16 halves,
--precision 2: BF16 halves) against the FP64 CPU oracle.

The mixed kernel computes the two transforms on the tensor cores from
split 16-bit operands with FP32 accumulation, the face recurrence in FP32 and
the vo accumulation in FP64, so it is compared with stated tolerances rather
than bit for bit:

* random inputs (vi ~ U[0,1), a_from_m ~ N(0, 1/nm), m_from_a = pinv): the
  error of the split products dominates.  FP16 halves carry a 22-bit
  significand per operand, BF16 halves 16 bits:
  max |vo - vo_oracle| / max |vo_oracle| <= 1e-6 (FP16) and <= 2e-5 (BF16).
* na > 32 is swept in 32-angle passes whose octant sums add up in vo
  (angles are independent in the sweep); the same tolerances.
* the built-in problem: its faces are large integers that cancel in the
  second transform, which amplifies any rounding of psi.  psi = sm * cc + vs
  is therefore formed in FP64 with the FP64 reciprocal of (1 + octant) and
  rounded once to FP32; then max-rel <= 1e-5 and the relative normsq error
  <= 1e-5 on every geometry, including na 64 / 128 and NM 4 (formed in FP32
  the normsq error reached 3.3e-5 at na 128 and 8.3e-5 at NM 4, na 64).
"""
import numpy as np
import pytest

import oracle

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu

import minisweep_b200 as msb  # noqa: E402

RTOL_RANDOM = {1: 1e-6, 2: 2e-5}
RTOL_BUILTIN = 1e-5
NORMSQ_TOL = 1e-5


def flags(nx, ny, nz, ne, na, extra=""):
    return f"--ncell_x {nx} --ncell_y {ny} --ncell_z {nz} --ne {ne} --na {na} {extra}"


def run(nx, ny, nz, ne, na, nm, prec, a=None, m=None, vi=None):
    with msb.Problem(flags(nx, ny, nz, ne, na, f"--precision {prec}"), nm=nm) as pb:
        if a is not None:
            pb.set_matrices(a, m)
        if vi is None:
            vi = pb.init_state()
        vo = pb.sweep_host(vi)
    return vi, vo


def rel_errors(vo, ref):
    maxrel = np.max(np.abs(vo - ref)) / np.max(np.abs(ref))
    nq, nr = np.sum(vo * vo), np.sum(ref * ref)
    return maxrel, abs(nq - nr) / nr


BUILTIN = [
    (1, 1, 1, 1, 32, 16),
    (3, 2, 3, 3, 33, 16),   # na > 32: one pass per 32 angles, the last one ragged
    (4, 3, 2, 2, 128, 16),
    (2, 3, 4, 3, 70, 4),
    (2, 1, 2, 3, 7, 16),
    (5, 4, 5, 3, 7, 4),
    (3, 4, 2, 5, 32, 16),
    (4, 3, 5, 20, 32, 16),
    (6, 5, 4, 3, 24, 8),
    (9, 7, 6, 5, 32, 16),
    (16, 16, 16, 16, 32, 4),
    (16, 16, 16, 4, 128, 16),  # the dense case's angle count
    (16, 16, 16, 4, 64, 4),    # NM 4, na 64 (the batched workload's worst case)
    (12, 9, 20, 6, 64, 16),
]


@pytest.mark.parametrize("prec", [1, 2])
@pytest.mark.parametrize("nx,ny,nz,ne,na,nm", BUILTIN)
def test_mixed_builtin(nx, ny, nz, ne, na, nm, prec):
    vi, vo = run(nx, ny, nz, ne, na, nm, prec)
    a, m = oracle.am_matrices(nm, na)
    ref = oracle.sweep(nx, ny, nz, ne, nm, na, a, m, vi)
    maxrel, nrel = rel_errors(vo, ref)
    assert maxrel <= RTOL_BUILTIN, maxrel
    assert nrel <= NORMSQ_TOL, nrel


RANDOM = [
    (3, 2, 4, 3, 16, 16, 1),
    (5, 4, 3, 4, 32, 16, 2),
    (5, 5, 5, 4, 32, 4, 3),
    (6, 3, 5, 2, 24, 8, 4),
    (7, 6, 9, 6, 32, 16, 5),
    (3, 4, 3, 3, 64, 16, 6),   # two 32-angle passes
    (4, 3, 3, 2, 128, 16, 7),  # four passes (the dense geometry's na)
    (3, 3, 4, 3, 45, 8, 8),    # a ragged last pass
]


@pytest.mark.parametrize("prec", [1, 2])
@pytest.mark.parametrize("nx,ny,nz,ne,na,nm,seed", RANDOM)
def test_mixed_random(nx, ny, nz, ne, na, nm, seed, prec):
    a, m, vi = oracle.random_problem(nx, ny, nz, ne, nm, na, seed=seed)
    ref = oracle.sweep(nx, ny, nz, ne, nm, na, a, m, vi)
    _, vo = run(nx, ny, nz, ne, na, nm, prec, a, m, vi)
    maxrel, _ = rel_errors(vo, ref)
    assert maxrel <= RTOL_RANDOM[prec], maxrel


def test_mixed_repeatable():
    # the schedule is dynamic (tasks are grabbed at run time) but every vo
    # entry is accumulated in a fixed order: results repeat bit for bit
    a, m, vi = oracle.random_problem(8, 8, 8, 6, 16, 32, seed=11)
    _, vo1 = run(8, 8, 8, 6, 32, 16, 1, a, m, vi)
    _, vo2 = run(8, 8, 8, 6, 32, 16, 1, a, m, vi)
    assert np.array_equal(vo1, vo2)


@pytest.mark.parametrize("nx,ny,nz,ne,na,nm,prec", [
    (64, 64, 64, 64, 32, 16, 1),   # the headline geometry
    (64, 64, 64, 64, 32, 16, 2),
    (32, 32, 96, 8, 128, 16, 1),   # the dense geometry (8 of its 128 groups)
    (48, 40, 64, 16, 64, 4, 2),    # NM 4, na 64
])
def test_mixed_large_geometry_vs_fp64(nx, ny, nz, ne, na, nm, prec):
    # the mixed sweep against the FP64 sweep of the same problem, both on the
    # device
    dev = torch.device("cuda:0")
    out = {}
    for p in (0, prec):
        with msb.Problem(flags(nx, ny, nz, ne, na, f"--precision {p}"), nm=nm) as pb:
            vi = torch.empty(pb.nstate, dtype=torch.float64, device=dev)
            vo = torch.empty_like(vi)
            pb.init_state_device(vi.data_ptr())
            torch.cuda.synchronize()
            pb.sweep_device(vo.data_ptr(), vi.data_ptr())
            pb.sync()
            out[p] = vo
    f, r = out[0], out[prec]
    maxrel = (torch.max(torch.abs(r - f)) / torch.max(torch.abs(f))).item()
    nrel = abs((torch.sum(r * r) - torch.sum(f * f)) / torch.sum(f * f)).item()
    assert maxrel <= RTOL_BUILTIN, maxrel
    assert nrel <= NORMSQ_TOL, nrel
