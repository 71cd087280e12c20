"""Regenerates the golden fixtures in this directory from the reference itself.

Runs the reference's own serial KBA sweeper (compiled from its sources into
oracle/_ref by `make -C oracle ref`, driven through oracle/ref_dump.c) and
stores small input/output vectors:

* builtin_*.npz  -- the reference's built-in Quantities; vo as the reference's
                    runner leaves it, normsq / normsqdiff;
* random_*.npz   -- vi ~ U[0,1), a_from_m ~ N(0, 1/nm), m_from_a = pinv
                    (oracle.random_problem, seed fixed) injected into the
                    reference's Quantities / state arrays; vo as the reference
                    computes it.

Only this script needs the reference tree; the fixtures travel with the repo.
Usage:  python tests/golden/make_golden.py
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))

import oracle  # noqa: E402

# (name, nx, ny, nz, ne, na, nm, extra reference flags)
CASES = [
    ("builtin_2x1x2_ne3_na7_nm16", 2, 1, 2, 3, 7, 16, ""),
    ("builtin_5x4x5_ne3_na7_nm4", 5, 4, 5, 3, 7, 4, "--nblock_z 5"),
    ("builtin_3x4x2_ne5_na33_nm16", 3, 4, 2, 5, 33, 16, "--nblock_z 2"),
    ("builtin_4x4x4_ne2_na32_nm16", 4, 4, 4, 2, 32, 16, ""),
    ("random_3x2x4_ne3_na16_nm16", 3, 2, 4, 3, 16, 16, ""),
    ("random_4x3x3_ne2_na32_nm16", 4, 3, 3, 2, 32, 16, "--nblock_z 3"),
    ("random_3x3x3_ne4_na32_nm4", 3, 3, 3, 4, 32, 4, ""),
    ("random_2x3x2_ne2_na64_nm16", 2, 3, 2, 2, 64, 16, ""),
]
SEED = 20240611


def main() -> None:
    oracle.build(with_reference=True)
    for name, nx, ny, nz, ne, na, nm, extra in CASES:
        args = f"--ncell_x {nx} --ncell_y {ny} --ncell_z {nz} --ne {ne} --na {na} {extra}".strip()
        if name.startswith("random"):
            a, m, vi = oracle.random_problem(nx, ny, nz, ne, nm, na, seed=SEED)
            vo, vi_out, s, d = oracle.ref_run(args, nx, ny, nz, ne, nm, a, m, vi)
        else:
            a, m = oracle.am_matrices(nm, na)
            vi = oracle.init_state(nx, ny, nz, ne, nm)
            vo, vi_out, s, d = oracle.ref_run(args, nx, ny, nz, ne, nm)
        assert np.array_equal(vi_out, vi)
        np.savez_compressed(os.path.join(HERE, name + ".npz"), dims=np.array([nx, ny, nz, ne, na, nm]),
                            a_from_m=a, m_from_a=m, vi=vi, vo=vo, normsq=s, normsqdiff=d,
                            flags=np.array(args))
        print(f"{name}: normsq {s:.8e} normsqdiff {d:.3e}")


if __name__ == "__main__":
    main()
