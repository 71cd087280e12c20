// sweep_fp64_ws.cuh -- the plain-FP64 sweep kernel for sm_100a, warp
// specialised.
//
// Replaces the reference's device path: Sweeper_sweep_block_impl_global and
// everything under it (sweeper_kba_c_kernels.h:30-1383) plus the host step
// loop that launched it once per KBA step (sweeper_kba_c.h:588-845).
//
// Roles inside one CTA (TX*TY compute warps + one producer warpgroup):
//   loader    grabs tasks (octant, group pair, region tile) from the
//             topologically ordered table, waits -- with a time budget -- on
//             the progress counters of the tasks that feed it, and stages the
//             inputs of every wavefront step into a ring of shared-memory
//             stages with asynchronous 16-byte copies (vi, the previous vo,
//             the faces entering the tile).
//   publisher follows the compute warps' done phases and publishes this
//             CTA's task progress to global memory, one fence per batch of
//             finished steps, so no fence sits on the loader's or the compute
//             warps' path.
//   compute   warp (a, b) owns cell column (a, b) of the tile and, at step s,
//             solves plane s - a - b: FP64 tensor-core transforms
//             (mma.sync m8n8k4 f64), Quantities_solve on registers, the z face
//             carried in registers, x/y faces passed to the neighbouring warp
//             through double-buffered shared memory.  They only touch global
//             memory to write vo and the faces leaving the tile.
//
// Stage protocol (global step G counts across tasks):
//   full[G % NS]  loader: cp.async copies + header; completes when every
//                 piece has landed; compute waits.
//   done[G % NS]  each compute warp arrives after its writes of step G and
//                 waits for the others (the step barrier); the publisher
//                 consumes the phase, fences, publishes progress, and lets
//                 the loader reuse the stage.
//
// Lane layout (lane l, q = l >> 2, r = l & 3):
//   column n = q        -> group 2*gp + (q >> 2), unknown q & 3
//   angles held         -> ia = 32*ch + 8*t + 2*r + i   (t < 4, i < 2)
//   vi fragment k       -> moment im = (NM/4)*r + k
//   vo fragment (mt, j) -> moment 8*mt + q, column 2*r + j
// The accumulator of the first product is the B operand of the second after
// relabelling the angle index, so psi never leaves registers.
//
// Quantities_solve (quantities_testing_kernels.h:337-447) is evaluated in an
// exactly equivalent 7-operation form: every reassociated factor is a power of
// two, so each rounded result equals the reference's 12-operation expression.
#pragma once

#include "sweep_async.cuh"

namespace msb {

// One sweep problem as the kernel sees it.
struct Fp64Prob {
  const double* vi;
  double* vo;
  const double* afm;  // a_from_m [oct][im][ia] (im stride nm)
  const double* mfa;  // m_from_a [oct][ia][im]
  double* fxy;        // face planes, one entry = one warp's 8 columns x angles
  double* fxz;
  double* fyz;
  int nx, ny, nz, ne, na, ngp;
  int ia_base;  // angle index of the first angle of afm / mfa (a multiple of 64: passes over na > 64)
  int ie_base;  // global index of group 0 (energy-group slices of a larger problem)
  signed char vo_add;    // nonzero: every phase adds to vo (the passes after the first)
  signed char l2_hints;  // nonzero: faces written evict_last, state and consumed faces evict_first (chained kernel)
  signed char sp_off;    // (ix_base + 3 iy_base) & 3 of a process's subdomain (KBA decomposition): the space
                         // factor (quantities_testing_kernels.h:97-126) takes global coordinates
  signed char pad_;
  int a_stride;  // angles per octant row of afm / mfa (0: na); afm and mfa then point at the pass's first
                 // angle of the caller's full matrices (a batch's angle passes read them in place)
};
static_assert(sizeof(Fp64Prob) == 96, "problem record size");

// One problem per launch.
struct Fp64Params {
  Fp64Prob pr;
  const int* tasks;
  long long ntask;
  SyncArgs sy;
};

// Many problems per launch.  Tasks of all problems share one table with
// global task ids; the problems are grouped in classes (moment count, angle
// chunks, tile shape), each class a contiguous range of the table that the
// CTAs work through in class order.  A problem whose face planes reuse the
// scratch of earlier problems waits until those have completed every task.
constexpr int kMaxBatchClasses = 16;
struct Fp64Batch {
  const int* tasks;       // MSB_TASK_INTS ints per task, dependencies as global ids
  const int* task_prob;   // problem of each task
  const Fp64Prob* probs;  // per problem, for direction 0 (vi -> vo)
  const int* pred_off;    // scratch predecessors of problem p: pred[pred_off[p] .. pred_off[p + 1])
  const int* pred;
  const int* prob_ntask;  // tasks per problem
  int* pdone;             // completed tasks per problem (zeroed before the launch)
  long long* ptime;       // %globaltimer when each problem completed; [nprob] = launch start
  long long cls_base[kMaxBatchClasses];
  long long cls_ntask[kMaxBatchClasses];
  int cls_kind[kMaxBatchClasses];
  int nclass, nprob;
  int dir;  // 1: every problem sweeps vo -> vi (the iteration loop's odd sweeps)
  SyncArgs sy;
};
// First sync slot of the per-class task counters of a batched launch.
constexpr int SY_CLASS0 = 4;
static_assert(SY_CLASS0 + kMaxBatchClasses <= SY_PROGRESS, "sync header");

__device__ __forceinline__ int atom_add_release(int* p, int v) {
  int old;
  asm volatile("atom.add.release.gpu.global.s32 %0, [%1], %2;" : "=r"(old) : "l"(p), "r"(v) : "memory");
  return old;
}

__device__ __forceinline__ void mbar_inval(uint64_t* b) {
  asm volatile("mbarrier.inval.shared::cta.b64 [%0];" ::"r"(smem_u32(b)) : "memory");
}

__device__ __forceinline__ void dmma(double (&d)[2], double a, double b) {
  asm volatile("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0,%1}, {%2}, {%3}, {%0,%1};"
               : "+d"(d[0]), "+d"(d[1])
               : "d"(a), "d"(b));
}


template <int NM_, int NCH, int TX, int TY, int NS>
struct Fp64Cfg {
  static constexpr int KS = NM_ / 4;        // k-steps of the first product
  static constexpr int MT = (NM_ + 7) / 8;  // m-tiles of the second product
  static constexpr int NW = TX * TY;        // compute warps
  static constexpr int NT = (NW + 4) * 32;  // threads: compute warps + one producer warpgroup
  // With 8 compute warps the launch gives every thread 65536 / 384 = 168
  // registers; the producer warpgroup hands most of its share to them.
  static constexpr bool REBALANCE = NW == 8;
  // measured at 64^3 x ne 64: 208 / 80 gives 118.0 ms per sweep, 200 / 96
  // 121.1 ms (the compute warps spill below ~200)
  static constexpr int REG_PRODUCER = 80;
  static constexpr int REG_COMPUTE = 208;  // 8*32*208 + 4*32*80 <= 384 * 168; per SMSP 2*208 + 80 <= 512
  static_assert(!REBALANCE || NW * 32 * REG_COMPUTE + 4 * 32 * REG_PRODUCER <= NT * 168, "register split");
  static constexpr int ENT = NCH * 256;     // doubles per face entry
  static constexpr bool FACE_PF = NCH == 1; // faces entering the tile staged by the producer
  static constexpr int NXY = TY;  // first-plane xy faces staged per step: one per row
  static constexpr int VSZ = 2 * NM_ * NU;  // doubles of vi (or vo) per warp-cell
  // stage layout in doubles
  static constexpr int ST_VI = 0;
  static constexpr int ST_VO = ST_VI + NW * VSZ;
  static constexpr int ST_YZ = ST_VO + NW * VSZ;
  static constexpr int ST_XZ = ST_YZ + (FACE_PF ? TY * ENT : 0);
  static constexpr int ST_XY = ST_XZ + (FACE_PF ? TX * ENT : 0);
  static constexpr int ST_HDR = ST_XY + (FACE_PF ? NXY * ENT : 0);
  static constexpr int STAGE = ST_HDR + (int)(sizeof(StepHdr) / sizeof(double));
  static constexpr int MAT = NCH * (KS * 4 + MT * 8) * 32;  // doubles per matrix buffer
  // smem layout in doubles
  static constexpr int SM_SLOT = 0;                   // [2 faces][2 parity][NW][ENT]
  static constexpr int SM_STAGE = 4 * NW * ENT;
  static constexpr int SM_MAT = SM_STAGE + NS * STAGE;  // [2][MAT]
  static constexpr int SM_BAR = SM_MAT + 2 * MAT;       // full[NS], done[NS], freed[NS]
  static constexpr int SM_FINAL = SM_BAR + 3 * NS;      // loader -> publisher: steps issued (int)
  static constexpr int SM_PROB = SM_FINAL + 1;          // batched: Fp64Prob of the task in each mat buffer
  static constexpr size_t smem_bytes() { return sizeof(double) * (size_t)SM_PROB; }
  // batched: two problem records, then the problem whose predecessors the loader last saw complete (int)
  static constexpr size_t smem_bytes_batch() { return sizeof(double) * (size_t)SM_PROB + 2 * sizeof(Fp64Prob) + 16; }
};

// Shared-memory barriers of one body: set up before its first stage, and
// invalidated before another body reuses the memory.
template <int NM_, int NCH, int TX, int TY, int NS>
__device__ __forceinline__ void fp64_barriers(bool init) {
  using C = Fp64Cfg<NM_, NCH, TX, TY, NS>;
  extern __shared__ __align__(128) double smem[];
  uint64_t* const bars = reinterpret_cast<uint64_t*>(smem + C::SM_BAR);
  if (init) {
    for (int i = 0; i < NS; ++i) {
      mbar_init(&bars[i], 1);            // full: the loader's arrive.expect_tx (header + face copies)
      mbar_init(&bars[NS + i], 1);       // done: compute warp 0, after the compute warps' step barrier
      mbar_init(&bars[2 * NS + i], 1);   // freed: the publisher
    }
    *reinterpret_cast<volatile int*>(smem + C::SM_FINAL) = -1;
    reinterpret_cast<volatile int*>(smem + C::SM_FINAL)[1] = 0;  // compute warps' quit flag
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  } else {
    for (int i = 0; i < 3 * NS; ++i) mbar_inval(&bars[i]);
  }
}

// The sweep of one class of tasks by one CTA.  ROLE 0: the whole CTA (sets
// up its barriers, then splits into the producer warpgroup and the compute
// warps, moving registers from the first to the second); ROLE 1: the
// producer warps only; ROLE 2: the compute warps only (a batched kernel
// splits the roles once and sets up the barriers of each class itself).
// BATCH: P is an Fp64Batch and `cls` the class whose table range this call
// works through; otherwise P is an Fp64Params.
template <int NM_, int NCH, int TX, int TY, int NS, bool PIPE_T1, bool BATCH, int ROLE, class PP>
__device__ __forceinline__ void fp64_body(const PP& P, int cls) {
  using C = Fp64Cfg<NM_, NCH, TX, TY, NS>;
  constexpr int KS = C::KS, MT = C::MT, NW = C::NW, ENT = C::ENT, VSZ = C::VSZ;
  static_assert(NM_ % 4 == 0 && NM_ <= 16, "NM must be 4, 8 or 16");

  extern __shared__ __align__(128) double smem[];
  double* const slots = smem + C::SM_SLOT;
  double* const stages = smem + C::SM_STAGE;
  double* const mats = smem + C::SM_MAT;
  uint64_t* const full = reinterpret_cast<uint64_t*>(smem + C::SM_BAR);
  uint64_t* const done = full + NS;
  uint64_t* const freed = done + NS;  // publisher consumed the step: loader may refill the stage

  Fp64Prob* const s_prob = reinterpret_cast<Fp64Prob*>(smem + C::SM_PROB);  // BATCH only
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  int* const sync = P.sy.sync;
  int* const progress = sync + SY_PROGRESS;
  // loader <-> publisher hand-off: total steps issued, once the loader stops (-1 before)
  volatile int& s_final = *reinterpret_cast<volatile int*>(smem + C::SM_FINAL);

  if constexpr (ROLE == 0) {
    if (threadIdx.x == 0) fp64_barriers<NM_, NCH, TX, TY, NS>(true);
    __syncthreads();
  }

  if (ROLE == 1 || (ROLE == 0 && warp >= NW)) {
    // ====================================================== producer warpgroup
    if constexpr (C::REBALANCE && ROLE == 0) asm volatile("setmaxnreg.dec.sync.aligned.u32 %0;" ::"n"(C::REG_PRODUCER));
    if (warp == NW) {
      // ------------------------------------------------------------ loader
      long long g_load = 0;
      long long last_step[2] = {-1, -1};  // last global step of the task using mat buffer 0/1
      int ntask_seen = 0;
      // BATCH: the problem whose predecessors were last seen complete (kept
      // in shared memory: the producer warps' registers are all in use)
      volatile int* const preds_done_for = reinterpret_cast<volatile int*>(s_prob + 2);
      if (BATCH && lane == 0) *preds_done_for = -1;
      __syncwarp();
      bool failed = false;

      // Steps up to freed_upto have been consumed by the publisher.  Waiting
      // for step g uses the phase of freed[g % NS] that step g completes;
      // it is always that barrier's latest phase, so parities never alias.
      long long freed_upto = -1;
      auto wait_freed = [&](long long g) -> bool {
        for (long long x = freed_upto + 1; x <= g; ++x) {
          if (!mbar_wait(&freed[x % NS], (uint32_t)((x / NS) & 1), P.sy, -1)) return false;
          freed_upto = x;
        }
        return true;
      };
      // bounded wait for *p >= target; returns the value seen (or -1)
      auto wait_dep = [&](const int* p, int target, int task) -> int {
        int v = ld_acquire(p);
        if (v >= target) return v;
        const long long t0 = global_ns();
        for (;;) {
          __nanosleep(64);
          v = ld_acquire(p);
          if (v >= target) return v;
          if (ld_relaxed(&sync[SY_ABORT]) != 0) return -1;
          if (global_ns() - t0 > P.sy.timeout_ns) {
            if (lane == 0) raise_error(sync, MSB_ERR_TIMEOUT, task);
            return -1;
          }
        }
      };
      auto grab = [&]() -> int {
        int t = -1;
        if (lane == 0 && ld_relaxed(&sync[SY_ABORT]) == 0) {
          if constexpr (BATCH) {
            const long long tt = atomicAdd(&sync[SY_CLASS0 + cls], 1);
            t = tt < P.cls_ntask[cls] ? (int)(P.cls_base[cls] + tt) : -1;
          } else {
            const long long tt = atomicAdd(&sync[SY_COUNTER], 1);
            t = tt < P.ntask ? (int)tt : -1;
          }
        }
        return __shfl_sync(0xffffffffu, t, 0);
      };

      // A task is grabbed only once the previous one is fully issued (the
      // compute warps still have NS steps of work in hand), so a reserved
      // task never waits behind another task of the same CTA.
      for (;;) {
        const int t = grab();
        if (t < 0) break;
        const int rec_lane = lane < MSB_TASK_INTS ? __ldg(&P.tasks[(size_t)t * MSB_TASK_INTS + lane]) : 0;
        int rec[MSB_TASK_INTS];
#pragma unroll
        for (int k = 0; k < MSB_TASK_INTS; ++k) rec[k] = __shfl_sync(0xffffffffu, rec_lane, k);

        const int oct = rec[TK_OCT], gp = rec[TK_GP], flags = rec[TK_FLAGS], mode = rec[TK_DEP_MODE];
        const int x0 = rec[TK_X0], x1 = rec[TK_X1], y0 = rec[TK_Y0], y1 = rec[TK_Y1];
        const int z0 = rec[TK_Z0], z1 = rec[TK_Z1];
        const int w = x1 - x0, h = y1 - y0, nzr = z1 - z0, nsteps = nzr + w + h - 2;
        const int dx = (oct & 1) ? -1 : 1, dy = (oct & 2) ? -1 : 1, dz = (oct & 4) ? -1 : 1;
        const int depx = (mode & DM_X_PLANE) ? rec[TK_DEP_X] : -1;
        const int depy = (mode & DM_Y_PLANE) ? rec[TK_DEP_Y] : -1;
        // the task's problem
        Fp64Prob Q;
        int prob = 0;
        if constexpr (BATCH) {
          prob = __ldg(&P.task_prob[t]);
          Q = P.probs[prob];
          if (P.dir) {
            const double* a = Q.vi;
            Q.vi = Q.vo;
            Q.vo = const_cast<double*>(a);
          }
          // the face scratch is free once its previous users completed
          // (completion is final: checked once per run of tasks of one problem)
          if (prob != *preds_done_for) {
            for (int k = __ldg(&P.pred_off[prob]), ke = __ldg(&P.pred_off[prob + 1]); k < ke && !failed; ++k) {
              const int q2 = __ldg(&P.pred[k]);
              if (wait_dep(&P.pdone[q2], __ldg(&P.prob_ntask[q2]), t) < 0) failed = true;
            }
            __syncwarp();
            if (!failed && lane == 0) *preds_done_for = prob;
            __syncwarp();
          }
        } else {
          Q = P.pr;
        }
        // cross-phase dependencies: whole task complete
        if (!failed && rec[TK_DEP_X] >= 0 && depx < 0 && wait_dep(&progress[rec[TK_DEP_X]], kComplete, t) < 0) failed = true;
        if (!failed && rec[TK_DEP_Y] >= 0 && depy < 0 && wait_dep(&progress[rec[TK_DEP_Y]], kComplete, t) < 0) failed = true;
        if (!failed && rec[TK_DEP_Z] >= 0 && wait_dep(&progress[rec[TK_DEP_Z]], kComplete, t) < 0) failed = true;
        if (!failed && rec[TK_DEP_VO] >= 0 && wait_dep(&progress[rec[TK_DEP_VO]], kComplete, t) < 0) failed = true;
        // octant matrices into the buffer the task before last used
        const int mb = ntask_seen & 1;
        if (!failed && !wait_freed(last_step[mb])) failed = true;
        if (failed) break;
        __threadfence_block();
        double* mat = mats + mb * C::MAT;
        const size_t as = Q.a_stride ? (size_t)Q.a_stride : (size_t)Q.na;
        for (int e = lane; e < NCH * KS * 4 * 32; e += 32) {
          const int ln = e & 31, tt = (e >> 5) & 3, k = (e >> 7) % KS, ch = (e >> 7) / KS;
          const int ia = 32 * ch + 8 * tt + (ln >> 2), im = KS * (ln & 3) + k;
          mat[e] = ia < Q.na ? __ldg(&Q.afm[ia + as * (im + (size_t)NM_ * oct)]) : 0.0;
        }
        for (int e = lane; e < NCH * MT * 8 * 32; e += 32) {
          const int ln = e & 31, i = (e >> 5) & 1, tt = (e >> 6) & 3, mt = (e >> 8) % MT, ch = (e >> 8) / MT;
          const int ia = 32 * ch + 8 * tt + 2 * (ln & 3) + i, im = 8 * mt + (ln >> 2);
          mat[NCH * KS * 4 * 32 + e] =
              (ia < Q.na && im < NM_) ? __ldg(&Q.mfa[im + (size_t)NM_ * (ia + as * oct)]) : 0.0;
        }
        if constexpr (BATCH) {
          if (lane == 0) s_prob[mb] = Q;  // published to the compute warps with the task's first stage
        }
        __syncwarp();
        ++ntask_seen;
        last_step[mb] = g_load + nsteps - 1;

        const size_t ent_z = (size_t)(oct * Q.ngp + gp) * Q.nz;
        const size_t ent_y = (size_t)(oct * Q.ngp + gp) * Q.ny;
        int seen_x = 0, seen_y = 0;  // progress of the upwind tiles already observed
        for (int s = 0; s < nsteps; ++s) {
          const int st = (int)(g_load % NS);
          // the stage was last used by step g_load - NS
          if (g_load >= NS && !wait_freed(g_load - NS)) { failed = true; break; }
          // faces of this plane from the upwind tiles of the same phase
          const int need = min(s + 1, nzr);
          if (depx >= 0 && seen_x < need && (seen_x = wait_dep(&progress[depx], need, t)) < 0) { failed = true; break; }
          if (depy >= 0 && seen_y < need && (seen_y = wait_dep(&progress[depy], need, t)) < 0) { failed = true; break; }
          fence_proxy_async();
          __threadfence_block();
          double* stg = stages + (size_t)st * C::STAGE;
          StepHdr* hdr = reinterpret_cast<StepHdr*>(stg + C::ST_HDR);
          // Faces entering the tile at this step, one bulk copy each: lane j
          // handles piece j = (kind, position) with kind 0 yz (x-upwind edge,
          // row b), 1 xz (y-upwind edge, column a), 2 xy (first plane of
          // column (a, b) with b = row of the anti-diagonal cell).
          uint32_t bytes = 0;
          if constexpr (C::FACE_PF) {
            for (int b = 0; b < h; ++b) {
              const int c = s - b;
              if ((flags & TF_X_IN) && c >= 0 && c < nzr) bytes += ENT * 8;
              const int a = s - b;
              if ((flags & TF_Z_IN) && a >= 0 && a < w) bytes += ENT * 8;
            }
            for (int a = 0; a < w; ++a) {
              const int c = s - a;
              if ((flags & TF_Y_IN) && c >= 0 && c < nzr) bytes += ENT * 8;
            }
          }
          if (lane == 0) {
            hdr->task = t; hdr->s = s; hdr->oct = oct; hdr->gp = gp;
            hdr->x0 = x0; hdr->x1 = x1; hdr->y0 = y0; hdr->y1 = y1; hdr->z0 = z0; hdr->z1 = z1;
            hdr->flags = flags; hdr->mat = mb; hdr->stop = 0; hdr->pad1 = prob;
            // progress this task reaches once step s is done (-2: nothing new)
            hdr->pad0 = s == nsteps - 1 ? kComplete : (s + 1 - (w + h - 2) > 0 ? s + 1 - (w + h - 2) : -2);
            mbar_arrive_expect_tx(&full[st], bytes);
          }
          __syncwarp();
          if constexpr (C::FACE_PF) {
            // lanes [0, TY): yz of row b; [8, 8+TX): xz of column a; [16, 16+TY): xy of row b
            const int kind = lane >> 3, pos = lane & 7;
            if (kind == 0 && pos < h && (flags & TF_X_IN)) {
              const int b = pos, c = s - b;
              if (c >= 0 && c < nzr) {
                const int iy = dy > 0 ? y0 + b : y1 - 1 - b, iz = dz > 0 ? z0 + c : z1 - 1 - c;
                bulk_g2s(stg + C::ST_YZ + b * ENT, Q.fyz + ((ent_z + iz) * Q.ny + iy) * (size_t)ENT, ENT * 8, &full[st]);
              }
            } else if (kind == 1 && pos < w && (flags & TF_Y_IN)) {
              const int a = pos, c = s - a;
              if (c >= 0 && c < nzr) {
                const int ix = dx > 0 ? x0 + a : x1 - 1 - a, iz = dz > 0 ? z0 + c : z1 - 1 - c;
                bulk_g2s(stg + C::ST_XZ + a * ENT, Q.fxz + ((ent_z + iz) * Q.nx + ix) * (size_t)ENT, ENT * 8, &full[st]);
              }
            } else if (kind == 2 && pos < h && (flags & TF_Z_IN)) {
              const int b = pos, a = s - b;
              if (a >= 0 && a < w) {
                const int ix = dx > 0 ? x0 + a : x1 - 1 - a, iy = dy > 0 ? y0 + b : y1 - 1 - b;
                bulk_g2s(stg + C::ST_XY + b * ENT, Q.fxy + ((ent_y + iy) * Q.nx + ix) * (size_t)ENT, ENT * 8, &full[st]);
              }
            }
          }
          ++g_load;
        }
        if (failed) break;
      }
      // Drain: every stage that was issued is consumed by the compute warps
      // (its copies always land); then a stop header ends their loop and the
      // publisher stops at the same step.  A failed wait (error already
      // recorded) ends the same way, so nothing in this CTA is left waiting.
      if (lane == 0) s_final = (int)g_load;
      if (wait_freed(g_load - 1)) {
        const int st = (int)(g_load % NS);  // last used by step g_load - NS, consumed
        __threadfence_block();
        if (lane == 0) {
          StepHdr* hdr = reinterpret_cast<StepHdr*>(stages + (size_t)st * C::STAGE + C::ST_HDR);
          hdr->stop = 1;
          mbar_arrive_expect_tx(&full[st], 0);
        }
      } else {
        // the compute warps stopped early (a wait ran out): let this warp's
        // copies into the stages land before the shared memory is reused or
        // released; a copy takes microseconds, the bound is 1 ms
        const long long t1 = global_ns();
        for (long long x = freed_upto + 1; x < g_load; ++x)
          while (!mbar_test_wait(&full[x % NS], (uint32_t)((x / NS) & 1)) && global_ns() - t1 < 1000000) {
          }
      }
      __syncwarp();
    } else if (warp == NW + 1) {
      // --------------------------------------------------------- publisher
      // Sleeps on the done phases in order, hands each stage back to the
      // loader and publishes this CTA's task progress, one fence per batch
      // of steps that finished together.
      long long G = 0;
      long long t0 = global_ns();
      bool quit = false;
      while (!quit) {
        // wait for step G (or for the loader to stop before it)
        const int st0 = (int)(G % NS);
        bool ready = false;
        for (;;) {
          const int fin = s_final;
          if (fin >= 0 && G >= fin) { quit = true; break; }
          if (mbar_try_wait(&done[st0], (uint32_t)((G / NS) & 1), 2000)) { ready = true; break; }
          if (global_ns() - t0 > P.sy.timeout_ns) {
            if (lane == 0) raise_error(sync, MSB_ERR_TIMEOUT, -1);
            quit = true;
            break;
          }
        }
        if (!ready) break;
        int pend_task[2] = {-1, -1}, pend_val[2] = {-2, -2}, pend_prob[2] = {0, 0};
        for (;;) {  // consume step G and any later steps already done
          const int st = (int)(G % NS);
          const StepHdr* hdr = reinterpret_cast<const StepHdr*>(stages + (size_t)st * C::STAGE + C::ST_HDR);
          const int task = hdr->task, val = hdr->pad0, hprob = hdr->pad1;
          __syncwarp();
          if (lane == 0) mbar_arrive(&freed[st]);
          if (val != -2) {
            if (pend_task[1] >= 0 && pend_task[1] != task) {
              pend_task[0] = pend_task[1];
              pend_val[0] = pend_val[1];
              pend_prob[0] = pend_prob[1];
            }
            pend_task[1] = task;
            pend_val[1] = val;
            pend_prob[1] = hprob;
          }
          ++G;
          // a task boundary ends a batch so older tasks are published first
          if (pend_task[0] >= 0) break;
          const int fin = s_final;
          if (fin >= 0 && G >= fin) break;
          if (!mbar_test(&done[G % NS], (uint32_t)((G / NS) & 1))) break;
        }
        if (pend_task[1] >= 0 || pend_task[0] >= 0) {
          __threadfence();
          if (lane == 0) {
            if (pend_task[0] >= 0) st_release(&progress[pend_task[0]], pend_val[0]);
            if (pend_task[1] >= 0) st_release(&progress[pend_task[1]], pend_val[1]);
            if constexpr (BATCH) {
              // a problem is complete once all its tasks are: the last one
              // stamps the time and releases its face scratch to later problems
              for (int k = 0; k < 2; ++k)
                if (pend_task[k] >= 0 && pend_val[k] == kComplete) {
                  const int pr2 = pend_prob[k];
                  if (atom_add_release(&P.pdone[pr2], 1) + 1 == __ldg(&P.prob_ntask[pr2])) P.ptime[pr2] = global_ns();
                }
            }
          }
        }
        t0 = global_ns();
      }
    }
  } else {
  if constexpr (C::REBALANCE && ROLE == 0) asm volatile("setmaxnreg.inc.sync.aligned.u32 %0;" ::"n"(C::REG_COMPUTE));

  // ================================================================ compute
  const int q = lane >> 2, r = lane & 3;
  const int wa = warp % TX, wb = warp / TX;
  double wz[2];
#pragma unroll
  for (int i = 0; i < 2; ++i) wz[i] = 1.0 / 4.0 - 1.0 / (double)(1 << (2 * r + i));
  double* const slot_yz = slots;                 // [2][NW][ENT]
  double* const slot_xz = slots + 2 * NW * ENT;  // [2][NW][ENT]
  // lane-constant offsets inside a warp's stage blocks and face entries
  const int vi_lane = (q >> 2) * (VSZ / 2) + NM_ * (q & 3) + KS * r;  // vi fragment
  const int vo_lane = (r >> 1) * (VSZ / 2) + NM_ * 2 * (r & 1) + q;   // vo value (mt = 0, j = 0)

  double b1r[NCH == 1 ? KS : 1][4];
  double a2r[NCH == 1 ? MT : 1][4][2];
  double carry[NCH][4][2];
  double d1n[NCH][4][2];  // angle values of the next plane (PIPE_T1)

  // The compute warps meet at a hardware barrier (bar.sync 1) once per step
  // and once per task start.  Every exit is decided uniformly: a warp whose
  // bounded wait ran out, or that finds the stop header, raises s_quit before
  // the barrier, and all warps leave after it; no warp leaves the others at a
  // barrier.
  volatile int& s_quit = reinterpret_cast<volatile int*>(smem + C::SM_FINAL)[1];
  long long G = 0;
  for (;;) {
    // ------------------------------------------------ one task per iteration
    {
      const bool ok = mbar_wait(&full[G % NS], (uint32_t)((G / NS) & 1), P.sy, -1);
      const StepHdr* h0 = reinterpret_cast<const StepHdr*>(stages + (size_t)(G % NS) * C::STAGE + C::ST_HDR);
      if (lane == 0 && (!ok || h0->stop)) s_quit = 1;
      asm volatile("bar.sync 1, %0;" ::"n"(NW * 32) : "memory");
      if (s_quit) break;
    }
    const StepHdr* hdr0 = reinterpret_cast<const StepHdr*>(stages + (size_t)(G % NS) * C::STAGE + C::ST_HDR);
    const int oct = hdr0->oct, gp = hdr0->gp, flags = hdr0->flags;
    const int x0 = hdr0->x0, x1 = hdr0->x1, y0 = hdr0->y0, y1 = hdr0->y1, z0 = hdr0->z0, z1 = hdr0->z1;
    const double* mat = mats + hdr0->mat * C::MAT;
    // the task's problem: the launch's own, or (batched) the loader's copy in
    // shared memory, read where used rather than held in registers
    Fp64Prob Qv;
    const Fp64Prob* qp = &Qv;
    if constexpr (BATCH) qp = s_prob + hdr0->mat; else Qv = P.pr;
    const Fp64Prob& Q = *qp;
    const size_t slab = (size_t)NM_ * NU * Q.nx * Q.ny;  // one (iz, ie) layer of the state
    const int w = x1 - x0, h = y1 - y0, nzr = z1 - z0, nsteps = nzr + w + h - 2;
    const int dx = (oct & 1) ? -1 : 1, dy = (oct & 2) ? -1 : 1, dz = (oct & 4) ? -1 : 1;
    const bool first = (flags & TF_FIRST) != 0 && !Q.vo_add;
    const bool act = wa < w && wb < h;
    const int ix = dx > 0 ? x0 + wa : x1 - 1 - wa;
    const int iy = dy > 0 ? y0 + wb : y1 - 1 - wb;
    const int iz0 = dz > 0 ? z0 : z1 - 1;  // z of plane 0; plane c is iz0 + dz * c
    const int cbeg = wa + wb;              // step of this warp's plane 0
    const int g_col = 2 * gp + (q >> 2);
    const bool gval = g_col < Q.ne;
    const int g_vo = 2 * gp + (r >> 1);
    const bool gvo = g_vo < Q.ne;
    const double so = (double)(1 + oct);
    const double so_r = 1.0 / so;  // rounded, as the reference's 1/(1+octant)
    // boundary flux = (1+ia) 2^(ia&7) s_space s_energy s_unknown (1+oct):
    // exact small integers, so the per-lane factor is formed once per task
    const double face_k =
        gval ? (double)d_scale_energy(Q.ie_base + g_col) * (double)d_scale_unknown(q & 3) * so : 0.0;
    const int sp_xy = ix + 3 * iy + 2 + Q.sp_off;  // log2 s_space(x, y, z) = (sp_xy + 7 z) & 3
    // state offsets (doubles) of this column: + zstep per plane
    const size_t col = (size_t)NM_ * NU * (ix + (size_t)Q.nx * iy);
    const long long zstep = (long long)slab * Q.ne * dz;
    const size_t ent_z = (size_t)(oct * Q.ngp + gp) * Q.nz;
    const size_t ent_y = (size_t)(oct * Q.ngp + gp) * Q.ny;
    // edges of the tile that read or write global faces
    const bool x_in = wa == 0 && (flags & TF_X_IN), y_in = wb == 0 && (flags & TF_Y_IN);
    const bool z_in = (flags & TF_Z_IN) != 0;
    const bool x_out = wa == w - 1 && (flags & TF_X_OUT), y_out = wb == h - 1 && (flags & TF_Y_OUT);
    const bool z_out = (flags & TF_Z_OUT) != 0;
    if constexpr (NCH == 1) {
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
    }

    // Each warp stages its own vi (and the previous vo) three steps ahead
    // with 16-byte cp.async copies into the stage of that step; one commit
    // group per step keeps the group count uniform.
    auto prefetch = [&](int s2, long long G2) {
      const int c2 = s2 - cbeg;
      if (act && s2 < nsteps && c2 >= 0 && c2 < nzr) {
        double* dst = stages + (size_t)(G2 % NS) * C::STAGE + warp * VSZ;
        const size_t off0 = col + slab * (size_t)(2 * gp) + (size_t)(slab * Q.ne) * (size_t)(iz0 + dz * c2);
#pragma unroll
        for (int g2 = 0; g2 < 2; ++g2) {
          if (2 * gp + g2 >= Q.ne) continue;
#pragma unroll
          for (int o = lane * 2; o < VSZ / 2; o += 64) {
            cp_async16(dst + C::ST_VI + g2 * (VSZ / 2) + o, Q.vi + off0 + g2 * slab + o);
            if (!first) cp_async16(dst + C::ST_VO + g2 * (VSZ / 2) + o, Q.vo + off0 + g2 * slab + o);
          }
        }
      }
      cp_async_commit();
    };
    auto load_vi = [&](const double* stage, double (&vf)[KS]) {
      const double* src = stage + C::ST_VI + warp * VSZ + vi_lane;
#pragma unroll
      for (int k = 0; k < KS; ++k) vf[k] = gval ? src[k] : 0.0;
    };
    // moments -> angles of one t-tile (FP64 tensor-core products)
    auto transform1 = [&](const double (&vf)[KS], int ch, int t, double (&d)[2]) {
      d[0] = d[1] = 0.0;
#pragma unroll
      for (int k = 0; k < KS; ++k) {
        const double b = NCH == 1 ? b1r[NCH == 1 ? k : 0][t] : mat[((ch * KS + k) * 4 + t) * 32 + lane];
        dmma(d, vf[k], b);
      }
    };
    prefetch(0, G);
    prefetch(1, G + 1);
    prefetch(2, G + 2);

    bool stop = false;
    for (int s = 0; s < nsteps; ++s, ++G) {
      const int st = (int)(G % NS);
      const double* stg = stages + (size_t)st * C::STAGE;
      bool go = true;  // this warp computes step G
      if (s > 0) {
        go = mbar_wait(&full[st], (uint32_t)((G / NS) & 1), P.sy, -1) &&
             !reinterpret_cast<const StepHdr*>(stg + C::ST_HDR)->stop;
        if (!go && lane == 0) s_quit = 1;
      }
      if (go) {
      prefetch(s + 3, G + 3);
      cp_async_wait<2>();  // the groups of steps s and s+1 have landed (this thread's copies)
      __syncwarp();        // ... and every lane's

      const int c = s - cbeg;
      if (act && c >= 0 && c < nzr) {
        const int iz = iz0 + dz * c;
        const int prev = (int)((G - 1) & 1), cur = (int)(G & 1);
        // solve coefficients: powers of two except so_r
        const double cxy = d_pow2(-1 - ((sp_xy + 7 * (iz - dz)) & 3));
        const double cxz = d_pow2(-2 - ((sp_xy - 3 * dy + 7 * iz) & 3));
        const double sx_r = d_pow2(-((sp_xy - dx + 7 * iz) & 3));
        const double cyz[2] = {wz[0] * sx_r, wz[1] * sx_r};
        const double cc = so_r * d_pow2((sp_xy + 7 * iz) & 3);

        // where the three incoming faces come from
        const double* in_yz = wa > 0 ? slot_yz + (size_t)(prev * NW + warp - 1) * ENT
                              : (x_in && C::FACE_PF) ? stg + C::ST_YZ + wb * ENT : nullptr;
        const double* gin_yz = (!C::FACE_PF && x_in) ? Q.fyz + ((ent_z + iz) * Q.ny + iy) * (size_t)ENT : nullptr;
        const double* in_xz = wb > 0 ? slot_xz + (size_t)(prev * NW + warp - TX) * ENT
                              : (y_in && C::FACE_PF) ? stg + C::ST_XZ + wa * ENT : nullptr;
        const double* gin_xz = (!C::FACE_PF && y_in) ? Q.fxz + ((ent_z + iz) * Q.nx + ix) * (size_t)ENT : nullptr;
        const double* in_xy = (c == 0 && z_in && C::FACE_PF) ? stg + C::ST_XY + wb * ENT : nullptr;
        const double* gin_xy = (c == 0 && z_in && !C::FACE_PF) ? Q.fxy + ((ent_y + iy) * Q.nx + ix) * (size_t)ENT : nullptr;
        double* out_yz = slot_yz + (size_t)(cur * NW + warp) * ENT;
        double* out_xz = slot_xz + (size_t)(cur * NW + warp) * ENT;
        double* gout_yz = x_out ? Q.fyz + ((ent_z + iz) * Q.ny + iy) * (size_t)ENT : nullptr;
        double* gout_xz = y_out ? Q.fxz + ((ent_z + iz) * Q.nx + ix) * (size_t)ENT : nullptr;
        double* gout_xy = (c == nzr - 1 && z_out) ? Q.fxy + ((ent_y + iy) * Q.nx + ix) * (size_t)ENT : nullptr;
        const int gx = dx > 0 ? -1 : Q.nx, gy = dy > 0 ? -1 : Q.ny, gz = dz > 0 ? -1 : Q.nz;  // ghost cells

        const bool has_next = PIPE_T1 && c + 1 < nzr;
        double vin[KS];
        if (has_next) load_vi(stages + (size_t)((G + 1) % NS) * C::STAGE, vin);
        if (!PIPE_T1 || c == 0) {
          double vif[KS];
          load_vi(stg, vif);
#pragma unroll
          for (int ch = 0; ch < NCH; ++ch)
#pragma unroll
            for (int t = 0; t < 4; ++t) transform1(vif, ch, t, d1n[ch][t]);
        }

        double d2[MT][2][2];  // two accumulators per m-tile (even / odd t)
#pragma unroll
        for (int mt = 0; mt < MT; ++mt) d2[mt][0][0] = d2[mt][0][1] = d2[mt][1][0] = d2[mt][1][1] = 0.0;

#pragma unroll
        for (int ch = 0; ch < NCH; ++ch) {
#pragma unroll
          for (int t = 0; t < 4; ++t) {
            double d1[2] = {d1n[ch][t][0], d1n[ch][t][1]};
            // the next plane's moments -> angles does not depend on this
            // plane's faces: interleave it with this plane's solve
            if (has_next) transform1(vin, ch, t, d1n[ch][t]);
            const int eo = ((ch * 4 + t) * 32 + lane) * 2;
            double fyz[2], fxz[2], fxy[2];
            if (in_yz) {
              const double2 v = *reinterpret_cast<const double2*>(in_yz + eo);
              fyz[0] = v.x; fyz[1] = v.y;
            } else if (gin_yz) {
              const double2 v = __ldcg(reinterpret_cast<const double2*>(gin_yz + eo));
              fyz[0] = v.x; fyz[1] = v.y;
            } else {
#pragma unroll
              for (int i = 0; i < 2; ++i) {
                const int ia = 32 * ch + 8 * t + 2 * r + i, iag = Q.ia_base + ia;
                fyz[i] = ia < Q.na ? (double)((1 + iag) << (iag & 7)) * d_pow2(d_log2_space(gx + Q.sp_off, iy, iz)) * face_k : 0.0;
              }
            }
            if (in_xz) {
              const double2 v = *reinterpret_cast<const double2*>(in_xz + eo);
              fxz[0] = v.x; fxz[1] = v.y;
            } else if (gin_xz) {
              const double2 v = __ldcg(reinterpret_cast<const double2*>(gin_xz + eo));
              fxz[0] = v.x; fxz[1] = v.y;
            } else {
#pragma unroll
              for (int i = 0; i < 2; ++i) {
                const int ia = 32 * ch + 8 * t + 2 * r + i, iag = Q.ia_base + ia;
                fxz[i] = ia < Q.na ? (double)((1 + iag) << (iag & 7)) * d_pow2(d_log2_space(ix + Q.sp_off, gy, iz)) * face_k : 0.0;
              }
            }
            if (c > 0) {
              fxy[0] = carry[ch][t][0]; fxy[1] = carry[ch][t][1];
            } else if (in_xy) {
              const double2 v = *reinterpret_cast<const double2*>(in_xy + eo);
              fxy[0] = v.x; fxy[1] = v.y;
            } else if (gin_xy) {
              const double2 v = __ldcg(reinterpret_cast<const double2*>(gin_xy + eo));
              fxy[0] = v.x; fxy[1] = v.y;
            } else {
#pragma unroll
              for (int i = 0; i < 2; ++i) {
                const int ia = 32 * ch + 8 * t + 2 * r + i, iag = Q.ia_base + ia;
                fxy[i] = ia < Q.na ? (double)((1 + iag) << (iag & 7)) * d_pow2(d_log2_space(ix + Q.sp_off, iy, gz)) * face_k : 0.0;
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
              const double psi = __dadd_rn(d1[i], __dmul_rn(sm, cc));
              d1[i] = psi;
              out[i] = __dmul_rn(psi, so);
              carry[ch][t][i] = out[i];
            }
            const double2 ov = make_double2(out[0], out[1]);
            *reinterpret_cast<double2*>(out_yz + eo) = ov;
            *reinterpret_cast<double2*>(out_xz + eo) = ov;
            if (gout_yz) __stcg(reinterpret_cast<double2*>(gout_yz + eo), ov);
            if (gout_xz) __stcg(reinterpret_cast<double2*>(gout_xz + eo), ov);
            if (gout_xy) __stcg(reinterpret_cast<double2*>(gout_xy + eo), ov);

            // ---- angles -> moments for this t (psi is the B operand as is)
#pragma unroll
            for (int i = 0; i < 2; ++i)
#pragma unroll
              for (int mt = 0; mt < MT; ++mt) {
                const double a = NCH == 1 ? a2r[NCH == 1 ? mt : 0][t][i]
                                          : mat[NCH * KS * 4 * 32 + ((((ch * MT + mt) * 4 + t) * 2 + i) * 32) + lane];
                dmma(d2[mt][t & 1], a, d1[i]);
              }
          }
        }

        // ---- accumulate vo in the region's visiting order
        if (gvo) {
          double* vdst = Q.vo + col + slab * (size_t)g_vo + (size_t)(slab * Q.ne) * (size_t)iz + (vo_lane - (r >> 1) * (VSZ / 2));
          const double* vold = stg + C::ST_VO + warp * VSZ + vo_lane;
#pragma unroll
          for (int mt = 0; mt < MT; ++mt)
#pragma unroll
            for (int j = 0; j < 2; ++j) {
              if (8 * mt + q < NM_) {
                const int o = NM_ * j + 8 * mt;
                const double dsum = __dadd_rn(d2[mt][0][j], d2[mt][1][j]);
                vdst[o] = first ? dsum : __dadd_rn(vold[o], dsum);
              }
            }
        }
      }
      }  // go
      // step G done by every compute warp: their writes are ordered before
      // the barrier, the neighbours' faces of step G are visible and step
      // G + 1 may start; warp 0 then tells the publisher
      __syncwarp();
      asm volatile("bar.sync 1, %0;" ::"n"(NW * 32) : "memory");
      if (s_quit) { stop = true; break; }
      if (warp == 0 && lane == 0) mbar_arrive(&done[st]);
    }
    if (stop) break;
  }
  cp_async_wait<0>();  // no copy into shared memory outlives the CTA
  }
}

template <int NM_, int NCH, int TX, int TY, int NS, bool PIPE_T1>
__global__ void __launch_bounds__((TX * TY + 4) * 32, 1) sweep_fp64_kernel(const Fp64Params P) {
  fp64_body<NM_, NCH, TX, TY, NS, PIPE_T1, false, 0>(P, 0);
}

// Batched FP64 sweep: one class kind per (NM, angle chunks, tile shape), all
// with 8 compute warps + the producer warpgroup (384 threads).  The CTAs work
// through the classes in order; a CTA moves on when its class's table is
// exhausted, so a task only ever waits on tasks that CTAs hold and advance.
enum Fp64BatchKind {
  BK_NM4_C1_42 = 0, BK_NM4_C1_24, BK_NM4_C2_42, BK_NM4_C2_24,
  BK_NM8_C1_42, BK_NM8_C1_24, BK_NM8_C2_42, BK_NM8_C2_24,
  BK_NM16_C1_42, BK_NM16_C1_24, BK_NM16_C2_42, BK_NM16_C2_24,
  BK_COUNT
};
constexpr int batch_kind(int nm, int nch, bool tile24) {
  return (nm == 4 ? 0 : nm == 8 ? 4 : 8) + (nch == 2 ? 2 : 0) + (tile24 ? 1 : 0);
}

// Every body kind of the batched kernel, in increasing kind order:
// F(kind, NM, NCH, TX, TY).  A batch sweeps its problems in 32-angle
// entries, so only the one-chunk bodies are compiled.
#define MSB_FP64_BATCH_KINDS(F)                                                                   \
  F(BK_NM4_C1_42, 4, 1, 4, 2) F(BK_NM4_C1_24, 4, 1, 2, 4) F(BK_NM8_C1_42, 8, 1, 4, 2)             \
  F(BK_NM8_C1_24, 8, 1, 2, 4) F(BK_NM16_C1_42, 16, 1, 4, 2) F(BK_NM16_C1_24, 16, 1, 2, 4)

// Between two classes: every warp of the CTA is done with the previous
// class's stages (a barrier that warps reach from their own role's code, so
// the non-aligned form), thread 0 swaps the barrier sets, and nobody starts
// the new class before that.
template <int NS>
__device__ __forceinline__ void fp64_batch_switch(const Fp64Batch& P, int c) {
  asm volatile("barrier.sync 0;" ::: "memory");
  if (threadIdx.x == 0) {
#define MSB_K(K, NM, NCH, TX, TY) \
  case K: fp64_barriers<NM, NCH, TX, TY, NS>(init); break;
    for (int k = 0; k < 2; ++k) {
      const bool init = k == 1;
      const int cc = init ? c : c - 1;
      if (cc < 0 || cc >= P.nclass) continue;
      switch (P.cls_kind[cc]) { MSB_FP64_BATCH_KINDS(MSB_K) default: break; }
    }
#undef MSB_K
  }
  asm volatile("barrier.sync 0;" ::: "memory");
}

// The classes of a launch come in increasing kind order (the host sorts
// them so), and the kernel visits the kinds in that order, one straight-line
// region per kind: compiled as separate regions (rather than the cases of a
// switch) the bodies keep their register allocations apart.
// Register split of the batched kernel (all class bodies in one kernel):
// 200 / 96 (its producer code spills with the single-problem kernel's 80).
constexpr int kBatchRegCompute = 200, kBatchRegProducer = 96;
static_assert(8 * 32 * kBatchRegCompute + 4 * 32 * kBatchRegProducer <= 12 * 32 * 168, "batch register split");

template <int NS>
__global__ void __launch_bounds__(12 * 32, 1) sweep_fp64_batch_kernel(const Fp64Batch P) {
  if (blockIdx.x == 0 && threadIdx.x == 0) P.ptime[P.nprob] = global_ns();
  // the register split of the 8-compute-warp bodies, once for all classes
  if ((threadIdx.x >> 5) >= 8) {
    asm volatile("setmaxnreg.dec.sync.aligned.u32 %0;" ::"n"(kBatchRegProducer));
    int c = 0;
#define MSB_K(K, NM, NCH, TX, TY)                                 \
  if (c < P.nclass && P.cls_kind[c] == K) {                       \
    fp64_batch_switch<NS>(P, c);                                  \
    fp64_body<NM, NCH, TX, TY, NS, false, true, 1>(P, c);         \
    ++c;                                                          \
  }
    MSB_FP64_BATCH_KINDS(MSB_K)
#undef MSB_K
  } else {
    asm volatile("setmaxnreg.inc.sync.aligned.u32 %0;" ::"n"(kBatchRegCompute));
    int c = 0;
#define MSB_K(K, NM, NCH, TX, TY)                                 \
  if (c < P.nclass && P.cls_kind[c] == K) {                       \
    fp64_batch_switch<NS>(P, c);                                  \
    fp64_body<NM, NCH, TX, TY, NS, false, true, 2>(P, c);         \
    ++c;                                                          \
  }
    MSB_FP64_BATCH_KINDS(MSB_K)
#undef MSB_K
  }
}

// Dynamic shared memory of the batched kernel: the largest class body.
template <int NS>
constexpr size_t fp64_batch_smem() {
  size_t m = 0;
  const size_t v[] = {Fp64Cfg<4, 1, 4, 2, NS>::smem_bytes_batch(),  Fp64Cfg<4, 1, 2, 4, NS>::smem_bytes_batch(),
                      Fp64Cfg<8, 1, 4, 2, NS>::smem_bytes_batch(),  Fp64Cfg<8, 1, 2, 4, NS>::smem_bytes_batch(),
                      Fp64Cfg<16, 1, 4, 2, NS>::smem_bytes_batch(), Fp64Cfg<16, 1, 2, 4, NS>::smem_bytes_batch()};
  for (size_t x : v) m = x > m ? x : m;
  return m;
}

}  // namespace msb
