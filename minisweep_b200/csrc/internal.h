// internal.h -- declarations shared by the library's translation units.
#pragma once

#include <cstddef>
#include <vector>

#include "minisweep_b200.h"

#ifdef __CUDACC__
#include <cuda_runtime.h>
#endif

namespace msb {

// Time budget of one device-side wait (a dependency, a barrier phase) before
// the sweep gives up with MSB_ERR_TIMEOUT.
constexpr long long kDefaultTimeoutNs = 4000000000LL;  // 4 s

int set_error(int code, const char* fmt, ...);
#ifdef __CUDACC__
int cuda_check(cudaError_t e, const char* what);
#endif
void insist_status(int rc, const char* what);

int scale_space(int ix, int iy, int iz);
int scale_energy(int ie);
int scale_unknown(int iu);
int scale_angle(int ia);
void build_am_matrices(int nm, int na, double* a, double* m);

// State layout of the reference (array_accessors_kernels.h:64-89):
// im fastest, then iu, ix, iy, ie, and iz slowest.
inline size_t ind_state(const Dimensions& d, int nu, int ix, int iy, int iz, int ie, int im, int iu) {
  return im + (size_t)d.nm * (iu + (size_t)nu * (ix + (size_t)d.ncell_x *
              (iy + (size_t)d.ncell_y * (ie + (size_t)d.ne * (size_t)iz))));
}

// ------------------------------------------------------------------ schedule
// One task = one octant sweeping one xy tile (TX x TY cells, the full z extent
// of its region) of one region for one group pair.  Regions are the 2x2x2
// halves of the grid; in phase p octant o sweeps region (o ^ p), so the eight
// octants of a phase touch disjoint cells and every region is visited by the
// octants in phase order (which fixes the order of the vo accumulation).
enum TaskField {
  TK_OCT = 0, TK_PHASE, TK_GP, TK_X0, TK_X1, TK_Y0, TK_Y1, TK_Z0, TK_Z1,
  TK_FLAGS, TK_DEP_X, TK_DEP_Y, TK_DEP_Z, TK_DEP_VO, TK_DEP_MODE, TK_LEVEL
};
static_assert(TK_LEVEL + 1 == MSB_TASK_INTS, "task record size");

enum TaskFlags {
  TF_X_IN = 1 << 0,   // x-upwind face comes from the global face buffer
  TF_Y_IN = 1 << 1,   //   (otherwise: domain boundary value)
  TF_Z_IN = 1 << 2,
  TF_X_OUT = 1 << 3,  // x-downwind face goes to the global face buffer
  TF_Y_OUT = 1 << 4,  //   (otherwise: domain boundary, nobody reads it)
  TF_Z_OUT = 1 << 5,
  TF_FIRST = 1 << 6   // first visitor of its cells in this sweep: vo = ...
};
enum DepMode {
  DM_X_PLANE = 1 << 0,  // DEP_X is a same-phase neighbour: wait plane by plane
  DM_Y_PLANE = 1 << 1   //   (otherwise wait for completion before starting)
};

struct Schedule {
  int nx = 0, ny = 0, nz = 0, ngp = 0, tx = 0, ty = 0;
  std::vector<int> rec;  // ntask * MSB_TASK_INTS, topological launch order
  long long ntask() const { return (long long)rec.size() / MSB_TASK_INTS; }
};

// Builds the task DAG in a topological order: (phase, block of gp_block
// group pairs, level of the tile along the octant's sweep direction, group
// pair, octant, tile).  Interleaving gp_block group pairs at each level keeps
// enough independent tasks in the window of tasks the CTAs hold at once.
// Returns 0 or an error code.
int build_schedule(int nx, int ny, int nz, int ngp, int tx, int ty, int gp_block, Schedule& out);

// Number of group pairs to interleave so that one level of the schedule holds
// about `window` tasks.
int pick_gp_block(int nx, int ny, int ngp, int tx, int ty, int window);

// ------------------------------------------------------- KBA decomposition
// One slab of a decomposed sweep: one octant over the process's whole x-y
// extent and the z-planes [z0, z1).  The edge flags say where the slab's
// faces come from and go: *_in on an x/y edge = the neighbouring process's
// face, placed in the face plane before the launch; z_in = the previous
// z-block's face, left in the plane by an earlier launch; *_out = somebody
// reads the face leaving that side; first = the slab's cells get vo = (not +=).
struct SlabEdges {
  bool x_in = false, x_out = false, y_in = false, y_out = false, z_in = false, z_out = false, first = false;
};
// Tasks of one slab in launch order (block of group pairs, tile level, group
// pair, tile); dependencies only between tiles of the slab.
int build_slab_schedule(int nx, int ny, int z0, int z1, int ngp, int tx, int ty, int gp_block, int oct,
                        const SlabEdges& e, Schedule& out);
int pick_gp_block_slab(int nx, int ny, int ngp, int tx, int ty, int window);

// Steps of a decomposed sweep: unit k = (unit_oct[k], unit_zb[k]) is swept by
// process p = px + nproc_x * py at step start[p * nunit + k].
struct KbaPlan {
  int npx = 1, npy = 1, nblock = 1, nstep = 0;
  std::vector<int> unit_oct, unit_zb, start;
  int nunit() const { return (int)unit_oct.size(); }
  int at(int px, int py, int k) const { return start[(size_t)(px + npx * py) * nunit() + k]; }
};
// A face slab crossing between neighbours after a step: is_send 1 = this
// process sends unit `unit`'s leaving face to `peer`; 0 = it receives the
// face entering its own copy of that unit.  axis 0: x faces (yz planes),
// 1: y faces (xz planes).  side: the peer's position along the axis (0 the
// lower neighbour, 1 the higher).
struct KbaMsg {
  int peer, is_send, axis, side, unit;
};
int build_kba_plan(int npx, int npy, int nblock, KbaPlan& out);
int kba_unit_at(const KbaPlan& plan, int proc, int step);  // unit swept at the step, or -1
int kba_messages(const KbaPlan& plan, int proc, int step, std::vector<KbaMsg>& msgs);

// The node-local process group (node_comm.cpp): joined by Env_initialize when
// the launcher's MSB_NPROC / MSB_PROC / MSB_GROUP are set; left by
// Env_finalize.
int node_attach(Env* env);
void node_detach(Env* env);

}  // namespace msb
