// sweep_fp64_chain.cuh -- the plain-FP64 sweep kernel for sm_100a with a
// chained wavefront.
//
// Replaces the reference's device path: Sweeper_sweep_block_impl_global and
// everything under it (sweeper_kba_c_kernels.h:30-1383) plus the host step
// loop that launched it once per KBA step (sweeper_kba_c.h:588-845).
//
// A CTA sweeps tasks (octant, group pair, TX x TY tile of cell columns, the
// z extent of a region; schedule.cpp) with TX*TY compute warps, warp (a, b)
// owning cell column (a, b) of the tile.  The warps step through a global
// step counter G; task k starts at step S_k, and at step G warp (a, b) solves
// plane G - S_k - a - b of it.  Consecutive tasks of a CTA are chained:
// S_{k+1} >= S_k + (planes of task k), so the first warps start the next task
// while the last ones finish the previous one and no step is spent filling or
// draining the diagonal wavefront.  A neighbour's x / y face of step G - 1 is
// always of the same task and plane, whichever tasks the warps are in.
//
// Per step a compute warp
//   * issues 16-byte cp.async copies of what it needs LA steps later: vi and
//     the previous vo of its cell, the face entering the tile at its x- or
//     y-upwind edge, the face entering at the task's first plane;
//   * waits for its own copies of this step, solves its cell (FP64
//     tensor-core transforms mma.sync m8n8k4 f64, Quantities_solve on
//     registers, z face carried in registers), writes its x / y faces into
//     parity-double-buffered shared slots (and to global memory at the
//     tile's downwind edges) and vo;
//   * meets the other compute warps at one named hardware barrier.
// Nothing else is on the step: the producer warps act once per task.
//   loader    grabs tasks from the topologically ordered table, waits -- with
//             a time budget -- until every task feeding it has completed,
//             and posts it into a ring of task slots (record + the octant's
//             matrices in fragment order).
//   leader    (lane 0 of compute warp 0) gives each newly posted task its
//             start step before the step barrier, so every warp learns it at
//             the same step, at least LA + 1 steps before it starts.
//   publisher waits for every compute warp to finish a task, fences and
//             publishes the task's completion, and frees its slot.
// (The producer warpgroup's other two warps only give up their registers.)
// Tasks only wait for whole tasks with smaller table indices; compute warps
// never wait for a task (they step idle until one is posted), so a CTA whose
// next task depends on its own current task drains that task first: the
// schedule cannot deadlock.
//
// Lane layout (lane l, q = l >> 2, r = l & 3), as in the transforms of
// sweep_fp64_ws.cuh:
//   column n = q        -> group 2*gp + (q >> 2), unknown q & 3
//   angles held         -> ia = 8*t + 2*r + i   (t < 4, i < 2)
//   vi fragment k       -> moment im = (NM/4)*r + k
//   vo fragment (mt, j) -> moment 8*mt + q, column 2*r + j
//
// Quantities_solve (quantities_testing_kernels.h:337-447) is evaluated in an
// exactly equivalent 7-operation form: every reassociated factor is a power of
// two, so each rounded result equals the reference's 12-operation expression.
#pragma once

#include "sweep_fp64_ws.cuh"

namespace msb {

// Task slot record written by the loader (start step by the leader).
struct ChainDesc {
  int rec[MSB_TASK_INTS];  // the task's record (TaskField order)
  int task, stop, prob, pad;
  long long start;
};

template <int NM_, int TX, int TY>
struct ChainCfg {
  static constexpr int KS = NM_ / 4;        // k-steps of the first product
  static constexpr int MT = (NM_ + 7) / 8;  // m-tiles of the second product
  static constexpr int NW = TX * TY;        // compute warps
  static constexpr int NT = (NW + 4) * 32;  // + one producer warpgroup (loader, publisher, two idle)
  // Registers: the launch gives every thread 65536 / 384 -> 168; the producer
  // warpgroup hands most of its share to the compute warps.  The split uses
  // exactly the launch's total: 8*32*216 + 4*32*72 = 384*168, and per SMSP
  // (two compute warps + one producer warp) 2*216 + 72 <= 512.
  static constexpr int REG_PRODUCER = 72;
  static constexpr int REG_COMPUTE = 216;
  static_assert(NW != 8 || NW * 32 * REG_COMPUTE + 4 * 32 * REG_PRODUCER <= (NW + 4) * 32 * 168, "register split");
  static constexpr int ENT = 256;           // doubles per face entry: 8 columns x 32 angles
  static constexpr int VSZ = 2 * NM_ * NU;  // doubles of vi (or vo) per warp-cell
  static constexpr int LA = 3;              // prefetch lookahead (steps)
  static constexpr int D = LA + 1;          // prefetch ring depth
  static constexpr int NSLOT = 3;           // task slots
  static constexpr int MIN_GAP = 6;         // steps between task starts at least (bounds tasks in flight)
  static constexpr int MAT = (KS * 4 + MT * 8) * 32;  // doubles per matrix buffer
  // shared memory layout, in doubles
  static constexpr int SM_XCH = 0;                          // [2 kinds][2 parity][NW][ENT]
  static constexpr int SM_V = SM_XCH + 4 * NW * ENT;        // [NW][D][2][VSZ]: vi, previous vo
  static constexpr int SM_YZ = SM_V + NW * D * 2 * VSZ;     // [TY][D][ENT]: x-upwind edge faces
  static constexpr int SM_XZ = SM_YZ + TY * D * ENT;        // [TX][D][ENT]: y-upwind edge faces
  static constexpr int SM_XY = SM_XZ + TX * D * ENT;        // [NW][ENT]: z face of a task's first plane
  static constexpr int SM_MAT = SM_XY + NW * ENT;           // [NSLOT][MAT]
  static constexpr int SM_DESC = SM_MAT + NSLOT * MAT;      // [NSLOT] ChainDesc
  static constexpr int DESC_D = (int)(sizeof(ChainDesc) / sizeof(double));
  static constexpr int SM_BAR = SM_DESC + NSLOT * DESC_D;   // full[NSLOT], done[NSLOT], free[NSLOT]
  static constexpr int SM_INT = SM_BAR + 3 * NSLOT;         // shared ints and the stop step (4 doubles)
  static constexpr int SM_END = SM_INT + 4;
  static constexpr size_t smem_bytes() { return sizeof(double) * (size_t)SM_END; }
  static_assert(sizeof(ChainDesc) % sizeof(double) == 0, "desc size");
};

// shared ints (SM_INT; the stop step, a long long, is its third double)
enum ChainInt {
  CI_NKNOWN = 0,  // tasks whose start step is assigned
  CI_FINAL = 1,   // loader: real tasks posted, once it stops (-1 before)
  CI_STOPSET = 2  // leader: the stop step is assigned
};
constexpr int kChainStopSlot = 2;  // double index of the stop step inside SM_INT

__device__ __forceinline__ void named_barrier_sync(int id, int nthreads) {
  asm volatile("bar.sync %0, %1;" ::"r"(id), "r"(nthreads) : "memory");
}

template <int NM_, int TX, int TY>
__global__ void __launch_bounds__((TX * TY + 4) * 32, 1) sweep_fp64_chain_kernel(const Fp64Params P) {
  using C = ChainCfg<NM_, TX, TY>;
  constexpr int KS = C::KS, MT = C::MT, NW = C::NW, ENT = C::ENT, VSZ = C::VSZ, LA = C::LA, D = C::D;
  constexpr int NSLOT = C::NSLOT;
  static_assert(NM_ % 4 == 0 && NM_ <= 16, "NM must be 4, 8 or 16");
  static_assert(NW == 8, "two compute warpgroups + one producer warpgroup");
  static_assert(C::smem_bytes() <= 227 * 1024, "shared memory budget");

  extern __shared__ __align__(128) double smem[];
  double* const xch = smem + C::SM_XCH;
  double* const ringv = smem + C::SM_V;
  double* const ringyz = smem + C::SM_YZ;
  double* const ringxz = smem + C::SM_XZ;
  double* const bufxy = smem + C::SM_XY;
  double* const mats = smem + C::SM_MAT;
  ChainDesc* const desc = reinterpret_cast<ChainDesc*>(smem + C::SM_DESC);
  uint64_t* const sfull = reinterpret_cast<uint64_t*>(smem + C::SM_BAR);
  uint64_t* const sdone = sfull + NSLOT;
  uint64_t* const sfree = sdone + NSLOT;
  volatile int* const si = reinterpret_cast<volatile int*>(smem + C::SM_INT);
  volatile long long* const s_stop = reinterpret_cast<volatile long long*>(smem + C::SM_INT + kChainStopSlot);

  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  int* const sync = P.sy.sync;
  int* const progress = sync + SY_PROGRESS;
  const Fp64Prob& Q = P.pr;

  if (threadIdx.x == 0) {
    for (int i = 0; i < NSLOT; ++i) {
      mbar_init(&sfull[i], 1);   // the loader's arrive after writing the slot
      mbar_init(&sdone[i], NW);  // every compute warp, after its last plane of the task
      mbar_init(&sfree[i], 1);   // the publisher, after publishing the task
    }
    si[CI_NKNOWN] = 0;
    si[CI_FINAL] = -1;
    si[CI_STOPSET] = 0;
    *s_stop = -1;
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  __syncthreads();

  if (warp >= NW) {
    asm volatile("setmaxnreg.dec.sync.aligned.u32 %0;" ::"n"(C::REG_PRODUCER));
    if (warp == NW) {
      // ============================================================== loader
      int n = 0;
      bool failed = false;
      // bounded wait for a task's completion; false if the budget ran out or
      // another CTA aborted (the error is then recorded)
      auto wait_complete = [&](int dep, int task) -> bool {
        const int* p = &progress[dep];
        if (ld_acquire(p) >= kComplete) return true;
        const long long t0 = global_ns();
        for (;;) {
          __nanosleep(128);
          if (ld_acquire(p) >= kComplete) return true;
          if (ld_relaxed(&sync[SY_ABORT]) != 0) return false;
          if (global_ns() - t0 > P.sy.timeout_ns) {
            if (lane == 0) raise_error(sync, MSB_ERR_TIMEOUT, task);
            return false;
          }
        }
      };
      auto wait_slot = [&](int m) -> bool {  // slot of task m free again (task m - NSLOT published)
        if (m < NSLOT) return true;
        return mbar_wait(&sfree[m % NSLOT], (uint32_t)(((m / NSLOT) - 1) & 1), P.sy, -1);
      };
      for (;;) {
        int t = -1;
        if (lane == 0 && ld_relaxed(&sync[SY_ABORT]) == 0) {
          const long long tt = atomicAdd(&sync[SY_COUNTER], 1);
          t = tt < P.ntask ? (int)tt : -1;
        }
        t = __shfl_sync(0xffffffffu, t, 0);
        if (t < 0) break;
        const int rec_lane = lane < MSB_TASK_INTS ? __ldg(&P.tasks[(size_t)t * MSB_TASK_INTS + lane]) : 0;
#pragma unroll 1
        for (int d = TK_DEP_X; d <= TK_DEP_VO && !failed; ++d) {
          const int dep = __shfl_sync(0xffffffffu, rec_lane, d);
          if (dep >= 0 && !wait_complete(dep, t)) failed = true;
        }
        if (failed || !wait_slot(n)) {
          failed = true;
          break;
        }
        const int q = n % NSLOT, oct = __shfl_sync(0xffffffffu, rec_lane, TK_OCT);
        double* mat = mats + q * C::MAT;
#pragma unroll 2
        for (int e = lane; e < KS * 4 * 32; e += 32) {
          const int ln = e & 31, tt = (e >> 5) & 3, k = e >> 7;
          const int ia = 8 * tt + (ln >> 2), im = KS * (ln & 3) + k;
          mat[e] = ia < Q.na ? __ldg(&Q.afm[ia + (size_t)Q.na * (im + (size_t)NM_ * oct)]) : 0.0;
        }
#pragma unroll 2
        for (int e = lane; e < MT * 8 * 32; e += 32) {
          const int ln = e & 31, i = (e >> 5) & 1, tt = (e >> 6) & 3, mt = e >> 8;
          const int ia = 8 * tt + 2 * (ln & 3) + i, im = 8 * mt + (ln >> 2);
          mat[KS * 4 * 32 + e] =
              (ia < Q.na && im < NM_) ? __ldg(&Q.mfa[im + (size_t)NM_ * (ia + (size_t)Q.na * oct)]) : 0.0;
        }
        ChainDesc& dd = desc[q];
        if (lane < MSB_TASK_INTS) dd.rec[lane] = rec_lane;
        if (lane == 0) {
          dd.task = t;
          dd.stop = 0;
          dd.prob = 0;
          dd.start = 0;
        }
        __syncwarp();
        if (lane == 0) mbar_arrive(&sfull[q]);
        ++n;
      }
      // stop record: tells the leader and the publisher how many tasks came
      if (lane == 0) si[CI_FINAL] = n;
      if (wait_slot(n)) {
        if (lane == 0) {
          desc[n % NSLOT].stop = 1;
          mbar_arrive(&sfull[n % NSLOT]);
        }
      }
      // (if the slot never frees, the publisher is stuck past its time
      // budget: the leader's idle budget then ends the compute warps)
      __syncwarp();
    } else if (warp == NW + 1) {
      // =========================================================== publisher
      for (int k = 0;; ++k) {
        const int q = k % NSLOT;
        bool ready = false, quit = false;
        const long long t0 = global_ns();
        for (;;) {
          const int fin = si[CI_FINAL];
          if (fin >= 0 && k >= fin) {
            quit = true;
            break;
          }
          if (mbar_try_wait(&sdone[q], (uint32_t)((k / NSLOT) & 1), 5000)) {
            ready = true;
            break;
          }
          if (global_ns() - t0 > P.sy.timeout_ns) {
            if (lane == 0) raise_error(sync, MSB_ERR_TIMEOUT, -1);
            quit = true;
            break;
          }
        }
        if (quit || !ready) break;
        const int task = desc[q].task;
        __threadfence();
        if (lane == 0) {
          st_release(&progress[task], kComplete);
          mbar_arrive(&sfree[q]);
        }
        __syncwarp();
      }
    }
  } else {
    asm volatile("setmaxnreg.inc.sync.aligned.u32 %0;" ::"n"(C::REG_COMPUTE));
    // =============================================================== compute
    const int q4 = lane >> 2, r = lane & 3;
    const int wa = warp % TX, wb = warp / TX;
    double wz[2];
#pragma unroll
    for (int i = 0; i < 2; ++i) wz[i] = 1.0 / 4.0 - 1.0 / (double)(1 << (2 * r + i));
    const int vi_lane = (q4 >> 2) * (VSZ / 2) + NM_ * (q4 & 3) + KS * r;  // vi fragment
    const int vo_lane = (r >> 1) * (VSZ / 2) + NM_ * 2 * (r & 1) + q4;    // vo value (mt = 0, j = 0)
    const size_t slab = (size_t)NM_ * NU * Q.nx * Q.ny;  // one (iz, ie) layer of the state
    const size_t zlayer = slab * Q.ne;
    const bool leader = warp == 0 && lane == 0;
    // L2 policies (with Q.l2_hints): faces leaving a tile are kept
    // (evict_last) until the downstream tile reads them; the state and the
    // faces read are streamed (evict_first)
    const bool hints = Q.l2_hints != 0;
    const uint64_t pol_first = l2_policy_evict_first(), pol_last = l2_policy_evict_last();
    auto cpa = [&](double* d, const double* src) {
      if (hints) cp_async16_hint(d, src, pol_first);
      else cp_async16(d, src);
    };

    // leader state: assignment of start steps
    long long last_start = 0, last_end_all = 0;  // last task's start; step after every warp finished it
    int last_gap = 0;
    int assigned = 0;
    long long idle_since = global_ns();

    int nknown = 0;  // tasks with an assigned start (from the shared counter)
    long long stop_step = -1;
    int kc = 0, kp = 0;  // compute / prefetch cursor (task index)

    // prefetch cursor: constants of task kp for this warp (valid when p_have)
    bool p_have = false, p_act = false, p_vo = false, p_g1 = false;
    long long p_lo = 0, p_hi = 0;  // the warp's first step of the task, first step after it
    long long p_off = 0, p_zs = 0;  // state offset (doubles) of plane 0 and per plane
    int p_dz = 1;
    const double* p_fyz = nullptr;  // faces entering at this warp's edges, plane 0
    const double* p_fxz = nullptr;
    const double* p_fxy = nullptr;
    auto load_prefetch = [&]() {
      mbar_test_wait(&sfull[kp % NSLOT], (uint32_t)((kp / NSLOT) & 1));  // acquire the loader's writes
      const ChainDesc& dd = desc[kp % NSLOT];
      const int oct = dd.rec[TK_OCT], gp = dd.rec[TK_GP], fl = dd.rec[TK_FLAGS];
      const int w = dd.rec[TK_X1] - dd.rec[TK_X0], h = dd.rec[TK_Y1] - dd.rec[TK_Y0];
      const int dx = (oct & 1) ? -1 : 1, dy = (oct & 2) ? -1 : 1;
      p_dz = (oct & 4) ? -1 : 1;
      p_lo = dd.start + wa + wb;
      p_hi = p_lo + (dd.rec[TK_Z1] - dd.rec[TK_Z0]);
      p_act = wa < w && wb < h;
      p_vo = !((fl & TF_FIRST) != 0 && !Q.vo_add);
      p_g1 = 2 * gp + 1 < Q.ne;
      const int pix = dx > 0 ? dd.rec[TK_X0] + wa : dd.rec[TK_X1] - 1 - wa;
      const int piy = dy > 0 ? dd.rec[TK_Y0] + wb : dd.rec[TK_Y1] - 1 - wb;
      const int piz0 = p_dz > 0 ? dd.rec[TK_Z0] : dd.rec[TK_Z1] - 1;
      p_off = (long long)((size_t)NM_ * NU * (pix + (size_t)Q.nx * piy) + slab * (size_t)(2 * gp) +
                          zlayer * (size_t)piz0);
      p_zs = p_dz * (long long)zlayer;
      const size_t eo = (size_t)(oct * Q.ngp + gp);
      p_fyz = (wa == 0 && (fl & TF_X_IN)) ? Q.fyz + ((eo * Q.nz + piz0) * Q.ny + piy) * (size_t)ENT : nullptr;
      p_fxz = (wb == 0 && (fl & TF_Y_IN)) ? Q.fxz + ((eo * Q.nz + piz0) * Q.nx + pix) * (size_t)ENT : nullptr;
      p_fxy = (fl & TF_Z_IN) ? Q.fxy + ((eo * Q.ny + piy) * Q.nx + pix) * (size_t)ENT : nullptr;
      p_have = true;
    };

    // compute cursor: constants of task kc (valid when have)
    bool have = false;
    long long c_lo = 0, c_hi = 0;  // the warp's first step of the task, first step after it
    int c_oct = 0, c_gp = 0, c_flags = 0, c_nzr = 0, c_dz = 1, c_iz0 = 0;
    bool c_act = false, c_first = false, c_gval = false, c_gvo = false;
    bool x_in = false, y_in = false, z_in = false, x_out = false, y_out = false, z_out = false;
    int ix = 0, iy = 0, sp_xy = 0, g_vo = 0, gx = 0, gy = 0, gz = 0;
    double so = 1.0, so_r = 1.0, face_k = 0.0;
    size_t col = 0, ent_z = 0, ent_y = 0;
    double b1r[KS][4];
    double a2r[MT][4][2];
    double carry[4][2];
    // task kc's constants and matrices into registers (the previous task of
    // this warp is finished, so its matrices are free)
    auto load_compute = [&]() {
      const int qs = kc % NSLOT;
      mbar_test_wait(&sfull[qs], (uint32_t)((kc / NSLOT) & 1));  // acquire the loader's writes
      const ChainDesc& dd = desc[qs];
      c_oct = dd.rec[TK_OCT];
      c_gp = dd.rec[TK_GP];
      c_flags = dd.rec[TK_FLAGS];
      c_nzr = dd.rec[TK_Z1] - dd.rec[TK_Z0];
      c_lo = dd.start + wa + wb;
      c_hi = c_lo + c_nzr;
      const int w = dd.rec[TK_X1] - dd.rec[TK_X0], h = dd.rec[TK_Y1] - dd.rec[TK_Y0];
      const int dx = (c_oct & 1) ? -1 : 1, dy = (c_oct & 2) ? -1 : 1;
      c_dz = (c_oct & 4) ? -1 : 1;
      c_act = wa < w && wb < h;
      c_first = (c_flags & TF_FIRST) != 0 && !Q.vo_add;
      ix = dx > 0 ? dd.rec[TK_X0] + wa : dd.rec[TK_X1] - 1 - wa;
      iy = dy > 0 ? dd.rec[TK_Y0] + wb : dd.rec[TK_Y1] - 1 - wb;
      c_iz0 = c_dz > 0 ? dd.rec[TK_Z0] : dd.rec[TK_Z1] - 1;
      const int g_col = 2 * c_gp + (q4 >> 2);
      c_gval = g_col < Q.ne;
      g_vo = 2 * c_gp + (r >> 1);
      c_gvo = g_vo < Q.ne;
      so = (double)(1 + c_oct);
      so_r = 1.0 / so;  // rounded, as the reference's 1/(1+octant)
      face_k = c_gval ? (double)d_scale_energy(Q.ie_base + g_col) * (double)d_scale_unknown(q4 & 3) * so : 0.0;
      sp_xy = ix + 3 * iy + 2;
      col = (size_t)NM_ * NU * (ix + (size_t)Q.nx * iy);
      ent_z = (size_t)(c_oct * Q.ngp + c_gp) * Q.nz;
      ent_y = (size_t)(c_oct * Q.ngp + c_gp) * Q.ny;
      x_in = wa == 0 && (c_flags & TF_X_IN);
      y_in = wb == 0 && (c_flags & TF_Y_IN);
      z_in = (c_flags & TF_Z_IN) != 0;
      x_out = wa == w - 1 && (c_flags & TF_X_OUT);
      y_out = wb == h - 1 && (c_flags & TF_Y_OUT);
      z_out = (c_flags & TF_Z_OUT) != 0;
      gx = dx > 0 ? -1 : Q.nx;
      gy = dy > 0 ? -1 : Q.ny;
      gz = c_dz > 0 ? -1 : Q.nz;
      const double* mat = mats + qs * C::MAT;
#pragma unroll
      for (int k = 0; k < KS; ++k)
#pragma unroll
        for (int t = 0; t < 4; ++t) b1r[k][t] = mat[(k * 4 + t) * 32 + lane];
#pragma unroll
      for (int mt = 0; mt < MT; ++mt)
#pragma unroll
        for (int t = 0; t < 4; ++t)
#pragma unroll
          for (int i = 0; i < 2; ++i) a2r[mt][t][i] = mat[KS * 4 * 32 + ((mt * 4 + t) * 2 + i) * 32 + lane];
      have = true;
    };

    long long G = 0;
    int rs = 0;  // G % D
    for (;; ++G, rs = rs + 1 == D ? 0 : rs + 1) {
      const int par = (int)(G & 1);
      // ---------------------------------------------------- prefetch G + LA
      {
        const long long G2 = G + LA;
        int rs2 = rs + LA;
        if (rs2 >= D) rs2 -= D;
        for (;;) {
          if (p_have && G2 >= p_hi) {
            ++kp;
            p_have = false;
          } else if (!p_have && kp < nknown) {
            load_prefetch();
          } else {
            break;
          }
        }
        if (p_have && p_act && G2 >= p_lo) {
          const int c2 = (int)(G2 - p_lo);
          const long long off0 = p_off + p_zs * c2;
          double* dst = ringv + (size_t)(warp * D + rs2) * 2 * VSZ;
#pragma unroll
          for (int g2 = 0; g2 < 2; ++g2) {
            if (g2 == 1 && !p_g1) continue;
#pragma unroll
            for (int o = lane * 2; o < VSZ / 2; o += 64) {
              cpa(dst + g2 * (VSZ / 2) + o, Q.vi + off0 + g2 * slab + o);
              if (p_vo) cpa(dst + VSZ + g2 * (VSZ / 2) + o, Q.vo + off0 + g2 * slab + o);
            }
          }
          if (p_fyz) {
            const double* src = p_fyz + (long long)p_dz * c2 * (long long)(Q.ny * ENT);
            double* d2 = ringyz + (size_t)(wb * D + rs2) * ENT;
#pragma unroll
            for (int o = lane * 2; o < ENT; o += 64) cpa(d2 + o, src + o);
          }
          if (p_fxz) {
            const double* src = p_fxz + (long long)p_dz * c2 * (long long)(Q.nx * ENT);
            double* d2 = ringxz + (size_t)(wa * D + rs2) * ENT;
#pragma unroll
            for (int o = lane * 2; o < ENT; o += 64) cpa(d2 + o, src + o);
          }
          if (c2 == 0 && p_fxy) {
            double* d2 = bufxy + (size_t)warp * ENT;
#pragma unroll
            for (int o = lane * 2; o < ENT; o += 64) cpa(d2 + o, p_fxy + o);
          }
        }
        cp_async_commit();
      }

      // ---------------------------------------------- finish / stop / start
      for (;;) {
        if (have && G >= c_hi) {
          // every write of task kc by this warp is issued: report it finished
          __syncwarp();
          if (lane == 0) mbar_arrive(&sdone[kc % NSLOT]);
          ++kc;
          have = false;
        } else if (!have && kc < nknown) {
          load_compute();
        } else {
          break;
        }
      }
      if (stop_step >= 0 && G >= stop_step) break;

      if (have && G >= c_lo) {
        const int c = (int)(G - c_lo);
        cp_async_wait<LA>();  // this thread's copies of step G have landed
        __syncwarp();         // ... and every lane's
        if (c_act) {
          const int iz = c_iz0 + c_dz * c;
          const int dx = (c_oct & 1) ? -1 : 1, dy = (c_oct & 2) ? -1 : 1, dz = c_dz;
          const double* const vst = ringv + (size_t)(warp * D + rs) * 2 * VSZ;
          // solve coefficients: powers of two except so_r
          const double cxy = d_pow2(-1 - ((sp_xy + 7 * (iz - dz)) & 3));
          const double cxz = d_pow2(-2 - ((sp_xy - 3 * dy + 7 * iz) & 3));
          const double sx_r = d_pow2(-((sp_xy - dx + 7 * iz) & 3));
          const double cyz[2] = {wz[0] * sx_r, wz[1] * sx_r};
          const double cc = so_r * d_pow2((sp_xy + 7 * iz) & 3);
          // where the three incoming faces come from
          const double* in_yz = wa > 0 ? xch + (size_t)((0 * 2 + (1 - par)) * NW + warp - 1) * ENT
                                : x_in ? ringyz + (size_t)(wb * D + rs) * ENT
                                       : nullptr;
          const double* in_xz = wb > 0 ? xch + (size_t)((1 * 2 + (1 - par)) * NW + warp - TX) * ENT
                                : y_in ? ringxz + (size_t)(wa * D + rs) * ENT
                                       : nullptr;
          const double* in_xy = (c == 0 && z_in) ? bufxy + (size_t)warp * ENT : nullptr;
          double* out_yz = xch + (size_t)((0 * 2 + par) * NW + warp) * ENT;
          double* out_xz = xch + (size_t)((1 * 2 + par) * NW + warp) * ENT;
          double* gout_yz = x_out ? Q.fyz + ((ent_z + iz) * Q.ny + iy) * (size_t)ENT : nullptr;
          double* gout_xz = y_out ? Q.fxz + ((ent_z + iz) * Q.nx + ix) * (size_t)ENT : nullptr;
          double* gout_xy = (c == c_nzr - 1 && z_out) ? Q.fxy + ((ent_y + iy) * Q.nx + ix) * (size_t)ENT : nullptr;

          // ---- moments -> angles (FP64 tensor-core products)
          double vf[KS];
          {
            const double* src = vst + vi_lane;
#pragma unroll
            for (int k = 0; k < KS; ++k) vf[k] = c_gval ? src[k] : 0.0;
          }
          double d1[4][2];
#pragma unroll
          for (int t = 0; t < 4; ++t) {
            d1[t][0] = d1[t][1] = 0.0;
#pragma unroll
            for (int k = 0; k < KS; ++k) dmma(d1[t], vf[k], b1r[k][t]);
          }
          double d2[MT][2][2];  // two accumulators per m-tile (even / odd t)
#pragma unroll
          for (int mt = 0; mt < MT; ++mt) d2[mt][0][0] = d2[mt][0][1] = d2[mt][1][0] = d2[mt][1][1] = 0.0;

#pragma unroll
          for (int t = 0; t < 4; ++t) {
            const int eo = (t * 32 + lane) * 2;
            double fyz[2], fxz[2], fxy[2];
            if (in_yz) {
              const double2 v = *reinterpret_cast<const double2*>(in_yz + eo);
              fyz[0] = v.x;
              fyz[1] = v.y;
            } else {
#pragma unroll
              for (int i = 0; i < 2; ++i) {
                const int ia = 8 * t + 2 * r + i, iag = Q.ia_base + ia;
                fyz[i] =
                    ia < Q.na ? (double)((1 + iag) << (iag & 7)) * d_pow2(d_log2_space(gx, iy, iz)) * face_k : 0.0;
              }
            }
            if (in_xz) {
              const double2 v = *reinterpret_cast<const double2*>(in_xz + eo);
              fxz[0] = v.x;
              fxz[1] = v.y;
            } else {
#pragma unroll
              for (int i = 0; i < 2; ++i) {
                const int ia = 8 * t + 2 * r + i, iag = Q.ia_base + ia;
                fxz[i] =
                    ia < Q.na ? (double)((1 + iag) << (iag & 7)) * d_pow2(d_log2_space(ix, gy, iz)) * face_k : 0.0;
              }
            }
            if (c > 0) {
              fxy[0] = carry[t][0];
              fxy[1] = carry[t][1];
            } else if (in_xy) {
              const double2 v = *reinterpret_cast<const double2*>(in_xy + eo);
              fxy[0] = v.x;
              fxy[1] = v.y;
            } else {
#pragma unroll
              for (int i = 0; i < 2; ++i) {
                const int ia = 8 * t + 2 * r + i, iag = Q.ia_base + ia;
                fxy[i] =
                    ia < Q.na ? (double)((1 + iag) << (iag & 7)) * d_pow2(d_log2_space(ix, iy, gz)) * face_k : 0.0;
              }
            }
            // ---- Quantities_solve, exact 7-operation form (no contraction)
            double out[2];
#pragma unroll
            for (int i = 0; i < 2; ++i) {
              const double bxz = __dmul_rn(fxz[i], cxz);
              const double sab = __fma_rn(fxy[i], cxy, bxz);  // fxy*cxy is exact
              const double cyzv = __dmul_rn(fyz[i], cyz[i]);
              const double sm = __dadd_rn(sab, cyzv);
              const double psi = __dadd_rn(d1[t][i], __dmul_rn(sm, cc));
              d1[t][i] = psi;
              out[i] = __dmul_rn(psi, so);
              carry[t][i] = out[i];
            }
            const double2 ov = make_double2(out[0], out[1]);
            *reinterpret_cast<double2*>(out_yz + eo) = ov;
            *reinterpret_cast<double2*>(out_xz + eo) = ov;
            if (hints) {
              if (gout_yz) st_v2_hint(gout_yz + eo, out[0], out[1], pol_last);
              if (gout_xz) st_v2_hint(gout_xz + eo, out[0], out[1], pol_last);
              if (gout_xy) st_v2_hint(gout_xy + eo, out[0], out[1], pol_last);
            } else {
              if (gout_yz) __stcg(reinterpret_cast<double2*>(gout_yz + eo), ov);
              if (gout_xz) __stcg(reinterpret_cast<double2*>(gout_xz + eo), ov);
              if (gout_xy) __stcg(reinterpret_cast<double2*>(gout_xy + eo), ov);
            }
            // ---- angles -> moments for this t (psi is the B operand as is)
#pragma unroll
            for (int i = 0; i < 2; ++i)
#pragma unroll
              for (int mt = 0; mt < MT; ++mt) dmma(d2[mt][t & 1], a2r[mt][t][i], d1[t][i]);
          }
          // ---- accumulate vo in the region's visiting order
          if (c_gvo) {
            double* vdst =
                Q.vo + col + slab * (size_t)g_vo + zlayer * (size_t)iz + (vo_lane - (r >> 1) * (VSZ / 2));
            const double* vold = vst + VSZ + vo_lane;
#pragma unroll
            for (int mt = 0; mt < MT; ++mt)
#pragma unroll
              for (int j = 0; j < 2; ++j) {
                if (8 * mt + q4 < NM_) {
                  const int o = NM_ * j + 8 * mt;
                  const double dsum = __dadd_rn(d2[mt][0][j], d2[mt][1][j]);
                  const double vnew = c_first ? dsum : __dadd_rn(vold[o], dsum);
                  if (hints) st_f64_hint(vdst + o, vnew, pol_first);
                  else vdst[o] = vnew;
                }
              }
          }
        }
      }

      // ------------------------------------------ leader: newly posted tasks
      if (leader) {
        bool progress_made = false;
        while (!si[CI_STOPSET]) {
          const int qs = assigned % NSLOT;
          if (!mbar_test_wait(&sfull[qs], (uint32_t)((assigned / NSLOT) & 1))) break;
          ChainDesc& dd = desc[qs];
          if (dd.stop) {
            // every warp has finished every task by this step
            stop_step = max(last_end_all, G + 1);
            *s_stop = stop_step;
            si[CI_STOPSET] = 1;
            break;
          }
          const long long s = max(assigned == 0 ? 0LL : last_start + last_gap, G + LA + 1);
          const int nzr = dd.rec[TK_Z1] - dd.rec[TK_Z0];
          dd.start = s;
          last_start = s;
          last_gap = max(nzr, C::MIN_GAP);
          last_end_all = s + (TX - 1) + (TY - 1) + nzr;
          ++assigned;
          si[CI_NKNOWN] = assigned;
          progress_made = true;
        }
        if (progress_made || have || kc < nknown) {
          idle_since = global_ns();
        } else if (!si[CI_STOPSET] && global_ns() - idle_since > P.sy.timeout_ns) {
          // nothing was posted within the budget (the loader could not post
          // the stop record): give up at the next step
          raise_error(sync, MSB_ERR_TIMEOUT, -1);
          stop_step = max(last_end_all, G + 1);
          *s_stop = stop_step;
          si[CI_STOPSET] = 1;
        }
      }
      // every compute warp: step G done
      named_barrier_sync(1, NW * 32);
      nknown = si[CI_NKNOWN];
      if (stop_step < 0 && si[CI_STOPSET]) stop_step = *s_stop;
      if (!have && !(kc < nknown)) __nanosleep(32);  // idle: nothing to compute yet
    }
    cp_async_wait<0>();  // no copy into shared memory outlives the CTA
  }
}

}  // namespace msb
