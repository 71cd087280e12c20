"""The CPU oracle (oracle/sweep_oracle.c) pinned against the reference.

* the committed golden fixtures (tests/golden/*.npz, produced by the
  reference's own serial KBA sweeper, see tests/golden/make_golden.py):
  bit-exact for the built-in Quantities, 1e-13 relative for injected random
  inputs (the reference's KBA sweeper adds octant contributions and transform
  products in a different order than the simple sweeper the oracle follows);
* the closed form of normsq (vo == vi for the built-in Quantities);
* the reference build itself (oracle/_ref) when it is present.
"""
import glob
import os

import numpy as np
import pytest

import oracle

HERE = os.path.dirname(os.path.abspath(__file__))
GOLDEN = sorted(glob.glob(os.path.join(HERE, "golden", "*.npz")))
RTOL_RANDOM = 1e-13


def test_golden_fixtures_exist():
    assert len(GOLDEN) >= 6


@pytest.mark.parametrize("path", GOLDEN, ids=[os.path.basename(p)[:-4] for p in GOLDEN])
def test_oracle_matches_reference_fixture(path):
    g = np.load(path)
    nx, ny, nz, ne, na, nm = (int(v) for v in g["dims"])
    vo = oracle.sweep(nx, ny, nz, ne, nm, na, g["a_from_m"], g["m_from_a"], g["vi"])
    ref = g["vo"]
    if os.path.basename(path).startswith("builtin"):
        assert np.array_equal(vo, ref)
        s, d = oracle.norms(g["vi"], vo)
        assert d == 0.0 and float(g["normsqdiff"]) == 0.0
        assert s == float(g["normsq"]) == oracle.normsq_closed_form(nx, ny, nz, ne, nm)
        # the built-in inputs themselves
        a, m = oracle.am_matrices(nm, na)
        assert np.array_equal(a, g["a_from_m"]) and np.array_equal(m, g["m_from_a"])
        assert np.array_equal(oracle.init_state(nx, ny, nz, ne, nm), g["vi"])
    else:
        err = np.max(np.abs(vo - ref)) / np.max(np.abs(ref))
        assert err <= RTOL_RANDOM, err


# normsq values printed by the reference for these configurations
# (sweep.c:53-56); the closed form reproduces them exactly
KNOWN_NORMSQ = [
    ((5, 5, 5, 30, 4), 6.89525100e+09),
    ((16, 16, 16, 16, 4), 1.20741888e+11),
    ((8, 8, 8, 8, 16), 3.76312218e+11),
    ((32, 32, 32, 32, 16), 9.63359277e+13),
    ((64, 64, 64, 64, 16), 1.54137484e+15),
    ((32, 32, 96, 128, 16), 1.15603113e+15),
]


@pytest.mark.parametrize("dims,val", KNOWN_NORMSQ)
def test_closed_form_normsq(dims, val):
    s = oracle.normsq_closed_form(*dims)
    assert abs(s - val) <= 5e-9 * val
    assert s == float(int(s))  # an integer below 2^53: every summation order is exact


def test_scale_factors():
    L = oracle.lib()
    # powers of two in {1, 2, 4, 8} from the low two bits of the index hashes
    for ie in range(50):
        assert L.oracle_scalefactor_energy(ie) == 1 << (((ie * 1366 + 150889) % 714025) & 3)
    assert [L.oracle_scalefactor_unknown(u) for u in range(4)] == [1 << (((u * 741 + 66037) % 312500) & 3)
                                                                  for u in range(4)]
    assert L.oracle_scalefactor_space(-1, 0, 0) == 2 and L.oracle_scalefactor_space(0, 0, -1) == 8
    # boundary flux: (1+ia) 2^(ia&7) s_space s_energy s_unknown (1+octant)
    assert L.oracle_init_face(3, -1, 2, 1, 0, 0, 2) == 4 * 8 * L.oracle_scalefactor_space(-1, 2, 1) * \
        L.oracle_scalefactor_energy(0) * L.oracle_scalefactor_unknown(0) * 3


def test_oracle_group_subset_matches_full():
    nx, ny, nz, ne, na, nm = 3, 3, 2, 5, 16, 16
    a, m, vi = oracle.random_problem(nx, ny, nz, ne, nm, na, seed=3)
    full = oracle.sweep(nx, ny, nz, ne, nm, na, a, m, vi)
    part = oracle.sweep(nx, ny, nz, ne, nm, na, a, m, vi, groups=(1, 4))
    v = full.reshape(nz, ne, -1)
    p = part.reshape(nz, ne, -1)
    assert np.array_equal(v[:, 1:4], p[:, 1:4])


@pytest.mark.skipif(oracle.ref_lib(16) is None, reason="reference build (oracle/_ref) not present")
@pytest.mark.parametrize("nx,ny,nz,ne,na,nm,extra", [
    (4, 3, 5, 3, 24, 16, "--nblock_z 5"),
    (2, 5, 3, 2, 40, 16, ""),
    (5, 2, 2, 3, 12, 4, "--nblock_z 2"),
])
def test_oracle_against_reference_build(nx, ny, nz, ne, na, nm, extra):
    args = f"--ncell_x {nx} --ncell_y {ny} --ncell_z {nz} --ne {ne} --na {na} {extra}"
    a, m = oracle.am_matrices(nm, na)
    vi = oracle.init_state(nx, ny, nz, ne, nm)
    vo_ref, _, s, d = oracle.ref_run(args, nx, ny, nz, ne, nm)
    assert np.array_equal(oracle.sweep(nx, ny, nz, ne, nm, na, a, m, vi), vo_ref)
    assert d == 0.0
    a, m, vi = oracle.random_problem(nx, ny, nz, ne, nm, na, seed=11)
    vo_ref, _, _, _ = oracle.ref_run(args, nx, ny, nz, ne, nm, a, m, vi)
    vo = oracle.sweep(nx, ny, nz, ne, nm, na, a, m, vi)
    assert np.max(np.abs(vo - vo_ref)) / np.max(np.abs(vo_ref)) <= RTOL_RANDOM
