// kba.cpp -- the KBA x/y process decomposition: which (octant, z-block) unit
// each process sweeps at each step of a sweep, and which faces cross between
// neighbouring processes after each step.
//
// The reference decomposes the x-y plane over an nproc_x x nproc_y process
// grid (runner.c:95-106), cuts z into nblock_z blocks and pipelines the blocks
// of every octant through the process grid (stepscheduler_kba.c:80-284), with
// the faces between neighbouring processes sent after every step
// (faces_kba.c:86-479).  Here every process sweeps one (octant, z-block) unit
// per step -- one launch of the persistent sweep kernel over the unit's slab,
// whose own task DAG carries the wavefront across the process's tiles -- and
// the steps are assigned by a small dynamic program instead of the
// reference's closed form:
//
//   start(p, k) = max(start(p, k-1), start(up_x(p), k), start(up_y(p), k)) + 1
//
// over the units k in one fixed order shared by all processes (octants in
// the sequence below, each octant's z-blocks in its upwind z order).  The
// octant sequence changes one direction bit at a time and the z bit every
// other time, so consecutive octants share their upwind corner in x and y
// four times out of seven and the pipeline refills only at the three x/y
// turns: 8 nblock_z + 2 (nproc_x - 1) + 3 (nproc_y - 1) steps, the
// reference's count for one octant per step.
#include <algorithm>
#include <vector>

#include "internal.h"

namespace msb {

namespace {
// Octant o sweeps +x if bit 0 is clear, +y if bit 1 is clear, +z if bit 2 is
// clear.  Neighbours in the sequence differ in one bit.
constexpr int kOctSeq[NOCTANT] = {0, 4, 6, 2, 3, 7, 5, 1};
}  // namespace

int build_kba_plan(int npx, int npy, int nblock, KbaPlan& out) {
  if (npx <= 0 || npy <= 0 || nblock <= 0) return set_error(MSB_ERR_ARG, "kba plan: invalid sizes");
  if ((long long)npx * npy * nblock > (1 << 24)) return set_error(MSB_ERR_ARG, "kba plan: too many units");
  out = KbaPlan();
  out.npx = npx;
  out.npy = npy;
  out.nblock = nblock;
  const int nunit = NOCTANT * nblock, nproc = npx * npy;
  out.unit_oct.resize(nunit);
  out.unit_zb.resize(nunit);
  for (int i = 0; i < NOCTANT; ++i) {
    const int oct = kOctSeq[i];
    for (int j = 0; j < nblock; ++j) {
      out.unit_oct[i * nblock + j] = oct;
      out.unit_zb[i * nblock + j] = (oct & 4) ? nblock - 1 - j : j;
    }
  }
  out.start.assign((size_t)nproc * nunit, -1);
  int last = -1;
  for (int k = 0; k < nunit; ++k) {
    const int oct = out.unit_oct[k];
    const int dx = (oct & 1) ? -1 : 1, dy = (oct & 2) ? -1 : 1;
    // processes in upwind-first order for this octant
    for (int a = 0; a < npy; ++a)
      for (int b = 0; b < npx; ++b) {
        const int py = dy > 0 ? a : npy - 1 - a, px = dx > 0 ? b : npx - 1 - b;
        int s = k > 0 ? out.at(px, py, k - 1) + 1 : 0;
        const int ux = px - dx, uy = py - dy;
        if (ux >= 0 && ux < npx) s = std::max(s, out.at(ux, py, k) + 1);
        if (uy >= 0 && uy < npy) s = std::max(s, out.at(px, uy, k) + 1);
        out.start[(size_t)(px + npx * py) * nunit + k] = s;
        last = std::max(last, s);
      }
  }
  out.nstep = last + 1;
  return MSB_OK;
}

int kba_unit_at(const KbaPlan& plan, int proc, int step) {
  const int nunit = plan.nunit();
  const int* st = &plan.start[(size_t)proc * nunit];
  // starts are strictly increasing along k for one process
  const int* it = std::lower_bound(st, st + nunit, step);
  return (it != st + nunit && *it == step) ? (int)(it - st) : -1;
}

int kba_messages(const KbaPlan& plan, int proc, int step, std::vector<KbaMsg>& msgs) {
  msgs.clear();
  const int npx = plan.npx, npy = plan.npy;
  const int px = proc % npx, py = proc / npx;
  // sends: the unit this process swept at this step, to its downwind neighbours
  const int k = kba_unit_at(plan, proc, step);
  if (k >= 0) {
    const int oct = plan.unit_oct[k];
    const int dx = (oct & 1) ? -1 : 1, dy = (oct & 2) ? -1 : 1;
    // side: where the receiver lies (1 = the higher neighbour)
    if (px + dx >= 0 && px + dx < npx) msgs.push_back(KbaMsg{px + dx + npx * py, 1, 0, dx > 0 ? 1 : 0, k});
    if (py + dy >= 0 && py + dy < npy) msgs.push_back(KbaMsg{px + npx * (py + dy), 1, 1, dy > 0 ? 1 : 0, k});
  }
  // receives: units the neighbours swept at this step whose downwind side is
  // this process (side 0: from the lower neighbour along the axis)
  for (int axis = 0; axis < 2; ++axis)
    for (int side = 0; side < 2; ++side) {
      const int qx = axis == 0 ? px + (side ? 1 : -1) : px, qy = axis == 1 ? py + (side ? 1 : -1) : py;
      if (qx < 0 || qx >= npx || qy < 0 || qy >= npy) continue;
      const int q = qx + npx * qy;
      const int kq = kba_unit_at(plan, q, step);
      if (kq < 0) continue;
      const int oct = plan.unit_oct[kq];
      const int d = axis == 0 ? ((oct & 1) ? -1 : 1) : ((oct & 2) ? -1 : 1);
      // the lower neighbour feeds this process when the octant sweeps upward
      if ((side == 0 && d > 0) || (side == 1 && d < 0)) msgs.push_back(KbaMsg{q, 0, axis, side, kq});
    }
  return (int)msgs.size();
}

}  // namespace msb

// ------------------------------------------------------------ host-only API
using msb::KbaPlan;

extern "C" int msb_kba_plan(int nproc_x, int nproc_y, int nblock_z, int* nstep, int* unit_oct, int* unit_zb,
                            int* start) {
  KbaPlan plan;
  const int rc = msb::build_kba_plan(nproc_x, nproc_y, nblock_z, plan);
  if (rc) return rc;
  if (nstep) *nstep = plan.nstep;
  if (unit_oct) std::copy(plan.unit_oct.begin(), plan.unit_oct.end(), unit_oct);
  if (unit_zb) std::copy(plan.unit_zb.begin(), plan.unit_zb.end(), unit_zb);
  if (start) std::copy(plan.start.begin(), plan.start.end(), start);
  return MSB_OK;
}

extern "C" int msb_kba_plan_messages(int nproc_x, int nproc_y, int nblock_z, int proc, int step, int* out,
                                     int max_msgs) {
  KbaPlan plan;
  int rc = msb::build_kba_plan(nproc_x, nproc_y, nblock_z, plan);
  if (rc) return rc;
  if (proc < 0 || proc >= nproc_x * nproc_y || step < 0 || step >= plan.nstep)
    return msb::set_error(MSB_ERR_ARG, "kba messages: proc or step out of range");
  std::vector<msb::KbaMsg> msgs;
  const int n = msb::kba_messages(plan, proc, step, msgs);
  for (int i = 0; i < n && i < max_msgs; ++i) {
    out[5 * i + 0] = msgs[i].peer;
    out[5 * i + 1] = msgs[i].is_send;
    out[5 * i + 2] = msgs[i].axis;
    out[5 * i + 3] = msgs[i].side;
    out[5 * i + 4] = msgs[i].unit;
  }
  return n;
}
