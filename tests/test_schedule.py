"""Host-side checks of the on-device sweep schedule (no GPU needed).

The schedule replaces the reference's StepScheduler (stepscheduler_kba.c) and
host step loop (sweeper_kba_c.h:588-845).  These tests check the properties
the kernel relies on: every (octant, group pair, cell) is swept exactly once,
every dependency precedes its dependant in launch order, the face producer of
every tile edge is the recorded dependency, and each tile's cells are visited
by the eight octants in phase order (the vo accumulation order).
"""
import numpy as np
import pytest

import minisweep_b200 as msb

(OCT, PHASE, GP, X0, X1, Y0, Y1, Z0, Z1, FLAGS, DX, DY, DZ, DVO, MODE, LEVEL) = range(16)
F_XIN, F_YIN, F_ZIN, F_XOUT, F_YOUT, F_ZOUT, F_FIRST = (1 << i for i in range(7))


def cell_owner(T, nx, ny, nz, ngp):
    """owner[o, gp, z, y, x] = task index."""
    own = -np.ones((8, ngp, nz, ny, nx), dtype=np.int64)
    for i, t in enumerate(T):
        blk = own[t[OCT], t[GP], t[Z0]:t[Z1], t[Y0]:t[Y1], t[X0]:t[X1]]
        assert (blk == -1).all(), "cell swept twice"
        blk[...] = i
    return own


SIZES = [(1, 1, 1, 1), (2, 1, 2, 3), (5, 4, 5, 3), (3, 4, 2, 5), (7, 5, 3, 2), (16, 16, 16, 4), (9, 10, 11, 6)]


@pytest.mark.parametrize("nx,ny,nz,ne", SIZES)
@pytest.mark.parametrize("tx,ty,gpb", [(4, 2, 1), (2, 2, 1), (4, 2, 2), (4, 2, 3)])
def test_schedule_properties(nx, ny, nz, ne, tx, ty, gpb):
    T = msb.schedule(nx, ny, nz, ne, tx, ty, gpb)
    ngp = (ne + 1) // 2
    own = cell_owner(T, nx, ny, nz, ngp)
    assert (own >= 0).all(), "cell not swept"
    n = len(T)
    for i, t in enumerate(T):
        o, p, gp = t[OCT], t[PHASE], t[GP]
        dx, dy, dz = (-1 if o & 1 else 1), (-1 if o & 2 else 1), (-1 if o & 4 else 1)
        for d in (DX, DY, DZ, DVO):
            assert t[d] < i, "dependency after dependant"
        assert 0 <= t[X1] - t[X0] <= tx and 0 < t[Y1] - t[Y0] <= ty
        # x-upwind producer: the owner of the neighbouring column
        xu = t[X0] - 1 if dx > 0 else t[X1]
        if 0 <= xu < nx:
            prod = set(own[o, gp, t[Z0]:t[Z1], t[Y0]:t[Y1], xu].ravel())
            assert prod == {t[DX]}, "x face producer mismatch"
            assert t[FLAGS] & F_XIN
            assert T[t[DX]][FLAGS] & F_XOUT
            same_phase = T[t[DX]][PHASE] == p
            assert bool(t[MODE] & 1) == same_phase
            if same_phase:
                assert T[t[DX]][Z0] == t[Z0] and T[t[DX]][Z1] == t[Z1]
        else:
            assert t[DX] == -1 and not (t[FLAGS] & F_XIN)
        yu = t[Y0] - 1 if dy > 0 else t[Y1]
        if 0 <= yu < ny:
            prod = set(own[o, gp, t[Z0]:t[Z1], yu, t[X0]:t[X1]].ravel())
            assert prod == {t[DY]}, "y face producer mismatch"
            assert t[FLAGS] & F_YIN and T[t[DY]][FLAGS] & F_YOUT
        else:
            assert t[DY] == -1 and not (t[FLAGS] & F_YIN)
        zu = t[Z0] - 1 if dz > 0 else t[Z1]
        if 0 <= zu < nz:
            prod = set(own[o, gp, zu, t[Y0]:t[Y1], t[X0]:t[X1]].ravel())
            assert prod == {t[DZ]}
            assert t[FLAGS] & F_ZIN and T[t[DZ]][FLAGS] & F_ZOUT
        else:
            assert t[DZ] == -1 and not (t[FLAGS] & F_ZIN)
        # downwind flags: set exactly when a consumer exists inside the grid
        xd = t[X1] if dx > 0 else t[X0] - 1
        assert bool(t[FLAGS] & F_XOUT) == (0 <= xd < nx)
        yd = t[Y1] if dy > 0 else t[Y0] - 1
        assert bool(t[FLAGS] & F_YOUT) == (0 <= yd < ny)
        zd = t[Z1] if dz > 0 else t[Z0] - 1
        assert bool(t[FLAGS] & F_ZOUT) == (0 <= zd < nz)
        # vo order: phase p-1 visited the same cells just before
        if p == 0:
            assert t[FLAGS] & F_FIRST and t[DVO] == -1
        else:
            pv = T[t[DVO]]
            assert pv[PHASE] == p - 1 and pv[GP] == gp
            assert tuple(pv[X0:Z1 + 1]) == tuple(t[X0:Z1 + 1])
    # phases of one region are distinct per octant: 8 octants x 8 phases
    for o in range(8):
        phases = set(T[T[:, OCT] == o][:, PHASE])
        assert phases <= set(range(8))
    # within one phase the octants occupy disjoint cells of one group pair
    for p in range(8):
        cover = np.zeros((ngp, nz, ny, nx), dtype=np.int64)
        for t in T[T[:, PHASE] == p]:
            cover[t[GP], t[Z0]:t[Z1], t[Y0]:t[Y1], t[X0]:t[X1]] += 1
        assert cover.max() <= 1


def test_schedule_counts_config2():
    T = msb.schedule(64, 64, 64, 64, 4, 2)
    # 8 phases x 8 octants x 32 group pairs x (32/4)*(32/2) tiles
    assert len(T) == 8 * 8 * 32 * 8 * 16
    assert (T[:, Z1] - T[:, Z0] == 32).all()
