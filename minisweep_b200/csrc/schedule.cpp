// schedule.cpp -- host-side construction of the on-device sweep schedule.
//
// Replaces the reference's host step loop (sweeper_kba_c.h:588-845) and its
// StepScheduler (stepscheduler_kba.c:80-372).  Instead of numbered KBA steps
// driven from the host, the sweep is a DAG of tasks that one persistent kernel
// executes in the order built here, each task waiting on per-task progress
// counters in global memory.
//
// Race freedom of the vo accumulation follows the reference's semiblock idea
// (sweeper_kba_c_kernels.h:1118-1159), applied to the whole grid: the grid is
// cut into 2x2x2 regions and in phase p octant o works in region o^p.  Bit b
// of p says whether the region lies on the downwind half along axis b for
// that octant, so each octant visits its regions in a valid upwind order, and
// within one phase the eight octants are in eight different regions.  The
// tiles of one region are visited by the octants in phase order, which is the
// order in which vo is accumulated (phase 0 writes, later phases add).
#include <algorithm>
#include <array>
#include <cstdint>

#include "internal.h"

namespace msb {

namespace {

struct Range {
  int lo, hi;  // [lo, hi)
  bool empty() const { return hi <= lo; }
};

Range half(int n, int bit) {
  const int h = (n + 1) / 2;
  return bit ? Range{h, n} : Range{0, h};
}

inline int ceil_div(int a, int b) { return (a + b - 1) / b; }

}  // namespace

int build_schedule(int nx, int ny, int nz, int ngp, int tx, int ty, int gp_block, Schedule& out) {
  if (nx <= 0 || ny <= 0 || nz <= 0 || ngp <= 0 || tx <= 0 || ty <= 0 || gp_block <= 0)
    return set_error(MSB_ERR_ARG, "schedule: invalid sizes");
  if (ngp >= (1 << 20) || nx >= (1 << 18) || ny >= (1 << 18))
    return set_error(MSB_ERR_ARG, "schedule: sizes too large");
  out = Schedule();
  out.nx = nx;
  out.ny = ny;
  out.nz = nz;
  out.ngp = ngp;
  out.tx = tx;
  out.ty = ty;

  // Tiles per region along x and y (the largest over the regions), and a
  // dense index (phase, octant, group pair, tile x, tile y) -> task.
  int ntxm = 0, ntym = 0;
  for (int reg = 0; reg < NOCTANT; ++reg) {
    ntxm = std::max(ntxm, ceil_div(half(nx, reg & 1).hi - half(nx, reg & 1).lo, tx));
    ntym = std::max(ntym, ceil_div(half(ny, (reg >> 1) & 1).hi - half(ny, (reg >> 1) & 1).lo, ty));
  }
  const size_t ndense = (size_t)NOCTANT * NOCTANT * ngp * ntxm * ntym;
  if (ndense >= (size_t)1 << 31) return set_error(MSB_ERR_ARG, "schedule: too many tasks");
  std::vector<int> index(ndense, -1);
  auto dense = [&](int p, int o, int gp, int itx, int ity) -> size_t {
    return ((((size_t)p * NOCTANT + o) * ngp + gp) * ntxm + itx) * ntym + ity;
  };
  auto find = [&](int p, int o, int gp, int itx, int ity) -> int { return index[dense(p, o, gp, itx, ity)]; };

  // Tasks in launch order: (phase, block of gp_block group pairs, level of
  // the tile along the octant's sweep direction, group pair, octant, tile row,
  // tile column) -- generated in that order directly.
  std::vector<int>& rec = out.rec;
  long long n = 0;
  for (int p = 0; p < NOCTANT; ++p)
    for (int gb = 0; gb * gp_block < ngp; ++gb) {
      int maxlevel = 0;
      for (int o = 0; o < NOCTANT; ++o) {
        const int reg = o ^ p;
        const int ntx = ceil_div(half(nx, reg & 1).hi - half(nx, reg & 1).lo, tx);
        const int nty = ceil_div(half(ny, (reg >> 1) & 1).hi - half(ny, (reg >> 1) & 1).lo, ty);
        maxlevel = std::max(maxlevel, ntx + nty - 1);
      }
      for (int level = 0; level < maxlevel; ++level)
        for (int gp = gb * gp_block; gp < std::min(ngp, (gb + 1) * gp_block); ++gp)
          for (int o = 0; o < NOCTANT; ++o) {
            const int reg = o ^ p;
            const Range rx = half(nx, reg & 1), ry = half(ny, (reg >> 1) & 1), rz = half(nz, (reg >> 2) & 1);
            if (rx.empty() || ry.empty() || rz.empty()) continue;
            const int dx = (o & 1) ? -1 : 1, dy = (o & 2) ? -1 : 1;
            const int ntx = ceil_div(rx.hi - rx.lo, tx), nty = ceil_div(ry.hi - ry.lo, ty);
            for (int ity = 0; ity < nty; ++ity) {
              const int ay = dy > 0 ? ity : nty - 1 - ity;
              const int ax = level - ay;
              if (ax < 0 || ax >= ntx) continue;
              const int itx = dx > 0 ? ax : ntx - 1 - ax;
              rec.resize(rec.size() + MSB_TASK_INTS, -1);
              int* r = &rec[(size_t)n * MSB_TASK_INTS];
              r[TK_OCT] = o;
              r[TK_PHASE] = p;
              r[TK_GP] = gp;
              r[TK_X0] = rx.lo + itx * tx;
              r[TK_X1] = std::min(rx.hi, rx.lo + (itx + 1) * tx);
              r[TK_Y0] = ry.lo + ity * ty;
              r[TK_Y1] = std::min(ry.hi, ry.lo + (ity + 1) * ty);
              r[TK_Z0] = rz.lo;
              r[TK_Z1] = rz.hi;
              r[TK_LEVEL] = level;
              index[dense(p, o, gp, itx, ity)] = (int)n;
              ++n;
            }
          }
    }

  // Dependencies; every one points to an earlier task.
  for (long long i = 0; i < n; ++i) {
    int* r = &rec[(size_t)i * MSB_TASK_INTS];
    const int o = r[TK_OCT], p = r[TK_PHASE], gp = r[TK_GP];
    const int reg = o ^ p;
    const int dx = (o & 1) ? -1 : 1, dy = (o & 2) ? -1 : 1;
    const Range rx = half(nx, reg & 1), ry = half(ny, (reg >> 1) & 1);
    const int ntx = ceil_div(rx.hi - rx.lo, tx), nty = ceil_div(ry.hi - ry.lo, ty);
    const int itx = (r[TK_X0] - rx.lo) / tx, ity = (r[TK_Y0] - ry.lo) / ty;
    int flags = 0, mode = 0;

    // ---- x: upwind neighbour tile, inside the region or across its boundary
    {
      const bool first_in_reg = dx > 0 ? itx == 0 : itx == ntx - 1;
      const bool last_in_reg = dx > 0 ? itx == ntx - 1 : itx == 0;
      if (!first_in_reg) {
        r[TK_DEP_X] = find(p, o, gp, itx - dx, ity);
        mode |= DM_X_PLANE;
      } else if ((p >> 0) & 1) {
        // the other x-half is upwind iff this region is on the downwind half
        const Range px = half(nx, (reg ^ 1) & 1);
        const int pntx = ceil_div(px.hi - px.lo, tx);
        if (!px.empty()) r[TK_DEP_X] = find(p ^ 1, o, gp, dx > 0 ? pntx - 1 : 0, ity);
      }
      if (r[TK_DEP_X] >= 0) flags |= TF_X_IN;
      const bool has_down = !last_in_reg || (((p >> 0) & 1) == 0 && !half(nx, (reg ^ 1) & 1).empty());
      if (has_down) flags |= TF_X_OUT;
    }
    // ---- y
    {
      const bool first_in_reg = dy > 0 ? ity == 0 : ity == nty - 1;
      const bool last_in_reg = dy > 0 ? ity == nty - 1 : ity == 0;
      if (!first_in_reg) {
        r[TK_DEP_Y] = find(p, o, gp, itx, ity - dy);
        mode |= DM_Y_PLANE;
      } else if ((p >> 1) & 1) {
        const Range py = half(ny, ((reg ^ 2) >> 1) & 1);
        const int pnty = ceil_div(py.hi - py.lo, ty);
        if (!py.empty()) r[TK_DEP_Y] = find(p ^ 2, o, gp, itx, dy > 0 ? pnty - 1 : 0);
      }
      if (r[TK_DEP_Y] >= 0) flags |= TF_Y_IN;
      const bool has_down = !last_in_reg || (((p >> 1) & 1) == 0 && !half(ny, ((reg ^ 2) >> 1) & 1).empty());
      if (has_down) flags |= TF_Y_OUT;
    }
    // ---- z: the task spans its region's z extent; the neighbour is the same
    // tile in the other z-half
    {
      const bool downwind_half = ((p >> 2) & 1) != 0;
      if (downwind_half) r[TK_DEP_Z] = find(p ^ 4, o, gp, itx, ity);
      if (r[TK_DEP_Z] >= 0) flags |= TF_Z_IN;
      if (!downwind_half && !half(nz, ((reg ^ 4) >> 2) & 1).empty()) flags |= TF_Z_OUT;
    }
    // ---- vo order: previous visitor of this tile (phase p-1, octant reg^(p-1))
    if (p == 0) {
      flags |= TF_FIRST;
    } else {
      r[TK_DEP_VO] = find(p - 1, reg ^ (p - 1), gp, itx, ity);
      if (r[TK_DEP_VO] < 0) return set_error(MSB_ERR_ARG, "schedule: missing vo predecessor");
    }
    r[TK_FLAGS] = flags;
    r[TK_DEP_MODE] = mode;
    for (int d = TK_DEP_X; d <= TK_DEP_VO; ++d)
      if (r[d] >= (int)i) return set_error(MSB_ERR_ARG, "schedule: dependency not topological");
  }
  return MSB_OK;
}

int build_slab_schedule(int nx, int ny, int z0, int z1, int ngp, int tx, int ty, int gp_block, int oct,
                        const SlabEdges& e, Schedule& out) {
  if (nx <= 0 || ny <= 0 || z1 <= z0 || z0 < 0 || ngp <= 0 || tx <= 0 || ty <= 0 || gp_block <= 0 || oct < 0 ||
      oct >= NOCTANT)
    return set_error(MSB_ERR_ARG, "slab schedule: invalid sizes");
  const int ntx = ceil_div(nx, tx), nty = ceil_div(ny, ty);
  if ((long long)ntx * nty * ngp >= (1LL << 30)) return set_error(MSB_ERR_ARG, "slab schedule: too many tasks");
  out = Schedule();
  out.nx = nx;
  out.ny = ny;
  out.nz = z1;
  out.ngp = ngp;
  out.tx = tx;
  out.ty = ty;
  const int dx = (oct & 1) ? -1 : 1, dy = (oct & 2) ? -1 : 1;
  std::vector<int> index((size_t)ngp * ntx * nty, -1);
  auto dense = [&](int gp, int itx, int ity) { return ((size_t)gp * ntx + itx) * nty + ity; };
  std::vector<int>& rec = out.rec;
  rec.reserve((size_t)ngp * ntx * nty * MSB_TASK_INTS);
  int n = 0;
  for (int gb = 0; gb * gp_block < ngp; ++gb)
    for (int level = 0; level < ntx + nty - 1; ++level)
      for (int gp = gb * gp_block; gp < std::min(ngp, (gb + 1) * gp_block); ++gp)
        for (int ity = 0; ity < nty; ++ity) {
          // ax, ay: the tile's position counted from the slab's upwind corner
          const int ay = dy > 0 ? ity : nty - 1 - ity;
          const int ax = level - ay;
          if (ax < 0 || ax >= ntx) continue;
          const int itx = dx > 0 ? ax : ntx - 1 - ax;
          rec.resize(rec.size() + MSB_TASK_INTS, -1);
          int* r = &rec[(size_t)n * MSB_TASK_INTS];
          r[TK_OCT] = oct;
          r[TK_PHASE] = 0;
          r[TK_GP] = gp;
          r[TK_X0] = itx * tx;
          r[TK_X1] = std::min(nx, (itx + 1) * tx);
          r[TK_Y0] = ity * ty;
          r[TK_Y1] = std::min(ny, (ity + 1) * ty);
          r[TK_Z0] = z0;
          r[TK_Z1] = z1;
          r[TK_LEVEL] = level;
          int flags = 0, mode = 0;
          if (ax > 0) {
            r[TK_DEP_X] = index[dense(gp, itx - dx, ity)];
            mode |= DM_X_PLANE;
          }
          if (ay > 0) {
            r[TK_DEP_Y] = index[dense(gp, itx, ity - dy)];
            mode |= DM_Y_PLANE;
          }
          if (ax > 0 || e.x_in) flags |= TF_X_IN;
          if (ax < ntx - 1 || e.x_out) flags |= TF_X_OUT;
          if (ay > 0 || e.y_in) flags |= TF_Y_IN;
          if (ay < nty - 1 || e.y_out) flags |= TF_Y_OUT;
          if (e.z_in) flags |= TF_Z_IN;
          if (e.z_out) flags |= TF_Z_OUT;
          if (e.first) flags |= TF_FIRST;
          r[TK_FLAGS] = flags;
          r[TK_DEP_MODE] = mode;
          index[dense(gp, itx, ity)] = n;
          if ((mode & DM_X_PLANE && r[TK_DEP_X] < 0) || (mode & DM_Y_PLANE && r[TK_DEP_Y] < 0))
            return set_error(MSB_ERR_ARG, "slab schedule: dependency not topological");
          ++n;
        }
  return MSB_OK;
}

int pick_gp_block_slab(int nx, int ny, int ngp, int tx, int ty, int window) {
  const int ntx = ceil_div(nx, tx), nty = ceil_div(ny, ty);
  const double per_level = (double)ntx * nty / (ntx + nty - 1);
  int b = (int)((window + per_level - 1) / per_level);
  return std::max(1, std::min(b, ngp));
}

int pick_gp_block(int nx, int ny, int ngp, int tx, int ty, int window) {
  // one region sweep: ntx x nty tiles over ntx + nty - 1 levels, 8 octants
  const int hx = (nx + 1) / 2, hy = (ny + 1) / 2;
  const int ntx = ceil_div(hx, tx), nty = ceil_div(hy, ty);
  const double per_level = 8.0 * ntx * nty / (ntx + nty - 1);
  int b = (int)((window + per_level - 1) / per_level);
  if (b < 1) b = 1;
  if (b > ngp) b = ngp;
  return b;
}

}  // namespace msb
