// sweep_fp64.cuh -- the plain-FP64 sweep kernel for sm_100a.
//
// Replaces the reference's device path: Sweeper_sweep_block_impl_global and
// everything under it (sweeper_kba_c_kernels.h:30-1383) plus the host step
// loop that launched it once per KBA step (sweeper_kba_c.h:588-845).
//
// Structure
//   * One persistent launch per sweep.  Each CTA repeatedly grabs the next
//     task (octant, group pair, region tile) from a topologically ordered
//     table and waits -- with a time budget -- on the progress counters of the
//     tasks that feed it faces or precede it in the vo accumulation order.
//   * A CTA holds TX x TY warps, one per (x, y) cell column of its tile, and
//     sweeps the tile's z extent as a diagonal wavefront: at step s warp (a, b)
//     works on plane s - a - b.  The z face stays in registers; the x and y
//     faces pass to the neighbouring warp through double-buffered shared
//     memory, and across tiles through per-octant face planes in global memory.
//   * Each warp handles 8 columns = 2 energy groups x 4 unknowns of its cell.
//     The two moment/angle transforms are FP64 tensor-core products
//     (mma.sync m8n8k4 f64): vs^T(8 x na) = vi^T(8 x NM) . a_from_m^T and
//     vo(NM x 8) = m_from_a(NM x na) . psi(na x 8).  The accumulator layout of
//     the first product is used directly as the B operand of the second by
//     relabelling the angle index, so psi never leaves registers.
//   * Quantities_solve (quantities_testing_kernels.h:337-447) runs on the
//     same registers.  The reference's 12-operation expression is evaluated
//     as an exactly equivalent 7-operation form: every factor that is
//     reassociated is a power of two, so the rounded results are identical.
//
// Lane layout (lane l, q = l >> 2, r = l & 3):
//   column n = q        -> group 2*gp + (q >> 2), unknown q & 3
//   angles held         -> ia = 32*ch + 8*t + 2*r + i   (t < 4, i < 2)
//   vi fragment k       -> moment im = (NM/4)*r + k
//   vo fragment (mt, j) -> moment 8*mt + q, column 2*r + j
#pragma once

#include "sweep_common.cuh"

namespace msb {

struct Fp64Params {
  const double* vi;
  double* vo;
  const double* afm;  // a_from_m [oct][im][ia] (im stride nm)
  const double* mfa;  // m_from_a [oct][ia][im]
  double* fxy;        // face planes, one entry = one warp's 8 columns x angles
  double* fxz;
  double* fyz;
  const int* tasks;
  long long ntask;
  int nx, ny, nz, ne, na, ngp;
  SyncArgs sy;
};

__device__ __forceinline__ void dmma(double (&d)[2], double a, double b) {
  asm volatile("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0,%1}, {%2}, {%3}, {%0,%1};"
               : "+d"(d[0]), "+d"(d[1])
               : "d"(a), "d"(b));
}

template <int NM_, int NCH, int TX, int TY>
struct Fp64Cfg {
  static constexpr int KS = NM_ / 4;        // k-steps of the first product
  static constexpr int MT = (NM_ + 7) / 8;  // m-tiles of the second product
  static constexpr int NW = TX * TY;        // warps per CTA
  static constexpr int ENT = NCH * 256;     // doubles per face entry
  static constexpr size_t smem_bytes() {
    return sizeof(double) * (size_t)(4 * NW * ENT + (NCH > 1 ? NCH * (KS * 4 + MT * 8) * 32 : 0));
  }
};

template <int NM_, int NCH, int TX, int TY>
__global__ void __launch_bounds__(TX* TY * 32, 1) sweep_fp64_kernel(const Fp64Params P) {
  using C = Fp64Cfg<NM_, NCH, TX, TY>;
  constexpr int KS = C::KS, MT = C::MT, NW = C::NW, ENT = C::ENT;
  static_assert(NM_ % 4 == 0 && NM_ <= 16, "NM must be 4, 8 or 16");

  extern __shared__ __align__(16) double smem[];
  __shared__ int s_rec[MSB_TASK_INTS];
  __shared__ int s_cmd;
  __shared__ int s_stop[2];

  double* slot_yz = smem;                 // [2][NW][ENT]
  double* slot_xz = smem + 2 * NW * ENT;  // [2][NW][ENT]
  double* b1s = smem + 4 * NW * ENT;      // [NCH][KS][4][32]     (NCH > 1)
  double* a2s = b1s + NCH * KS * 4 * 32;  // [NCH][MT][4][2][32]  (NCH > 1)

  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int q = lane >> 2, r = lane & 3;
  const int wa = warp % TX, wb = warp / TX;
  int* const sync = P.sy.sync;
  int* const progress = sync + SY_PROGRESS;
  const size_t slab = (size_t)NM_ * NU * P.nx * P.ny;  // one (iz, ie) layer

  for (;;) {
    // ------------------------------------------------------ grab a task
    if (threadIdx.x == 0) {
      int t = -1;
      if (ld_relaxed(&sync[SY_ABORT]) == 0) {
        const long long tt = atomicAdd(&sync[SY_COUNTER], 1);
        t = tt < P.ntask ? (int)tt : -1;
      }
      if (t >= 0) {
        for (int k = 0; k < MSB_TASK_INTS; ++k) s_rec[k] = P.tasks[(size_t)t * MSB_TASK_INTS + k];
        const int mode = s_rec[TK_DEP_MODE];
        bool ok = true;
        if (ok && s_rec[TK_DEP_X] >= 0 && !(mode & DM_X_PLANE))
          ok = wait_geq(P.sy, &progress[s_rec[TK_DEP_X]], kComplete, t);
        if (ok && s_rec[TK_DEP_Y] >= 0 && !(mode & DM_Y_PLANE))
          ok = wait_geq(P.sy, &progress[s_rec[TK_DEP_Y]], kComplete, t);
        if (ok && s_rec[TK_DEP_Z] >= 0) ok = wait_geq(P.sy, &progress[s_rec[TK_DEP_Z]], kComplete, t);
        if (ok && s_rec[TK_DEP_VO] >= 0) ok = wait_geq(P.sy, &progress[s_rec[TK_DEP_VO]], kComplete, t);
        if (!ok) t = -1;
      }
      s_cmd = t;
    }
    __syncthreads();
    const int task = s_cmd;
    if (task < 0) break;

    const int oct = s_rec[TK_OCT], gp = s_rec[TK_GP];
    const int x0 = s_rec[TK_X0], x1 = s_rec[TK_X1], y0 = s_rec[TK_Y0], y1 = s_rec[TK_Y1];
    const int z0 = s_rec[TK_Z0], z1 = s_rec[TK_Z1];
    const int flags = s_rec[TK_FLAGS], mode = s_rec[TK_DEP_MODE];
    const int depx = (mode & DM_X_PLANE) ? s_rec[TK_DEP_X] : -1;
    const int depy = (mode & DM_Y_PLANE) ? s_rec[TK_DEP_Y] : -1;
    const int dx = (oct & 1) ? -1 : 1, dy = (oct & 2) ? -1 : 1, dz = (oct & 4) ? -1 : 1;
    const int w = x1 - x0, h = y1 - y0, nzr = z1 - z0;
    const int nsteps = nzr + w + h - 2;
    const bool wactive = wa < w && wb < h;
    const int ix = dx > 0 ? x0 + wa : x1 - 1 - wa;
    const int iy = dy > 0 ? y0 + wb : y1 - 1 - wb;
    const bool first = (flags & TF_FIRST) != 0;

    // ---------------------------------------- octant transform matrices
    // b1 (k, t): a_from_m[oct][im = KS*r + k][ia = 32ch + 8t + q]
    // a2 (mt, t, i): m_from_a[oct][ia = 32ch + 8t + 2r + i][im = 8mt + q]
    double b1r[NCH == 1 ? KS : 1][4];
    double a2r[NCH == 1 ? MT : 1][4][2];
    if constexpr (NCH == 1) {
#pragma unroll
      for (int k = 0; k < KS; ++k)
#pragma unroll
        for (int t = 0; t < 4; ++t) {
          const int ia = 8 * t + q, im = KS * r + k;
          b1r[k][t] = ia < P.na ? __ldg(&P.afm[ia + (size_t)P.na * (im + (size_t)NM_ * oct)]) : 0.0;
        }
#pragma unroll
      for (int mt = 0; mt < MT; ++mt)
#pragma unroll
        for (int t = 0; t < 4; ++t)
#pragma unroll
          for (int i = 0; i < 2; ++i) {
            const int ia = 8 * t + 2 * r + i, im = 8 * mt + q;
            a2r[mt][t][i] = (ia < P.na && im < NM_) ? __ldg(&P.mfa[im + (size_t)NM_ * (ia + (size_t)P.na * oct)]) : 0.0;
          }
    } else {
      for (int e = threadIdx.x; e < NCH * KS * 4 * 32; e += blockDim.x) {
        const int ln = e & 31, t = (e >> 5) & 3, k = (e >> 7) % KS, ch = (e >> 7) / KS;
        const int ia = 32 * ch + 8 * t + (ln >> 2), im = KS * (ln & 3) + k;
        b1s[e] = ia < P.na ? __ldg(&P.afm[ia + (size_t)P.na * (im + (size_t)NM_ * oct)]) : 0.0;
      }
      for (int e = threadIdx.x; e < NCH * MT * 8 * 32; e += blockDim.x) {
        const int ln = e & 31, i = (e >> 5) & 1, t = (e >> 6) & 3, mt = (e >> 8) % MT, ch = (e >> 8) / MT;
        const int ia = 32 * ch + 8 * t + 2 * (ln & 3) + i, im = 8 * mt + (ln >> 2);
        a2s[e] = (ia < P.na && im < NM_) ? __ldg(&P.mfa[im + (size_t)NM_ * (ia + (size_t)P.na * oct)]) : 0.0;
      }
    }

    // ------------------------------------------------- per-lane constants
    const int g_col = 2 * gp + (q >> 2);  // group of this lane's column
    const int u_col = q & 3;
    const bool gval = g_col < P.ne;
    const int g_vo = 2 * gp + (r >> 1);   // group of this lane's vo values
    const bool gvo = g_vo < P.ne;
    const double so = (double)(1 + oct);
    const double so_r = 1.0 / so;           // rounded, as the reference's 1/(1+octant)
    double wz[2];
#pragma unroll
    for (int i = 0; i < 2; ++i) wz[i] = 1.0 / 4.0 - 1.0 / (double)(1 << (2 * r + i));
    const size_t ent_yz_base = (size_t)(oct * P.ngp + gp) * P.nz;
    const size_t ent_xy_base = (size_t)(oct * P.ngp + gp) * P.ny;

    double carry[NCH][4][2];  // z face of this warp's column
    double vin[KS], von[MT][2];
    bool have_next = false;

    auto load_cell = [&](int c, double (&vi_f)[KS], double (&vo_f)[MT][2]) {
      const int iz = dz > 0 ? z0 + c : z1 - 1 - c;
      const size_t cbase = (size_t)NM_ * NU * (ix + (size_t)P.nx * iy);
      if (gval) {
        const double* src = P.vi + cbase + slab * (g_col + (size_t)P.ne * iz) + NM_ * u_col + KS * r;
        if constexpr (KS == 4) {
          const double2 v0 = __ldg(reinterpret_cast<const double2*>(src));
          const double2 v1 = __ldg(reinterpret_cast<const double2*>(src) + 1);
          vi_f[0] = v0.x; vi_f[1] = v0.y; vi_f[2] = v1.x; vi_f[3] = v1.y;
        } else if constexpr (KS == 2) {
          const double2 v0 = __ldg(reinterpret_cast<const double2*>(src));
          vi_f[0] = v0.x; vi_f[1] = v0.y;
        } else {
          vi_f[0] = __ldg(src);
        }
      } else {
#pragma unroll
        for (int k = 0; k < KS; ++k) vi_f[k] = 0.0;
      }
#pragma unroll
      for (int mt = 0; mt < MT; ++mt)
#pragma unroll
        for (int j = 0; j < 2; ++j) {
          const int im = 8 * mt + q;
          vo_f[mt][j] = 0.0;
          if (!first && gvo && im < NM_)
            vo_f[mt][j] = __ldcg(P.vo + cbase + slab * (g_vo + (size_t)P.ne * iz) + NM_ * (2 * (r & 1) + j) + im);
        }
    };

    // ------------------------------------------------ wavefront steps
    for (int s = 0; s <= nsteps; ++s) {
      // wait (one thread) until the upwind tiles of this plane are done ...
      if (threadIdx.x == 0) {
        int stop = 0;
        if (s < nsteps) {
          const int need = min(s + 1, nzr);
          if (depx >= 0 && !wait_geq(P.sy, &progress[depx], need, task)) stop = 1;
          if (!stop && depy >= 0 && !wait_geq(P.sy, &progress[depy], need, task)) stop = 1;
        }
        s_stop[s & 1] = stop;
      }
      __syncthreads();
      // ... then publish the planes that step s-1 completed (every warp's
      // writes of step s-1 happen before the barrier above)
      if (threadIdx.x == 0 && s > 0) {
        __threadfence();
        const int done = s == nsteps ? kComplete : max(0, s - (w + h - 2));
        st_release(&progress[task], done);
      }
      if (s == nsteps || s_stop[s & 1]) break;

      const int c = s - wa - wb;
      if (!wactive || c < 0 || c >= nzr) continue;

      const int iz = dz > 0 ? z0 + c : z1 - 1 - c;
      double vif[KS], vof[MT][2];
      if (!have_next) load_cell(c, vin, von);
#pragma unroll
      for (int k = 0; k < KS; ++k) vif[k] = vin[k];
#pragma unroll
      for (int mt = 0; mt < MT; ++mt) { vof[mt][0] = von[mt][0]; vof[mt][1] = von[mt][1]; }
      have_next = c + 1 < nzr;
      if (have_next) load_cell(c + 1, vin, von);

      // solve coefficients of this cell (all powers of two except so_r)
      const double s_sp = (double)d_scale_space(ix, iy, iz);
      const double cxy = 0.5 / (double)d_scale_space(ix, iy, iz - dz);
      const double cxz = 0.25 / (double)d_scale_space(ix, iy - dy, iz);
      const double sx_r = 1.0 / (double)d_scale_space(ix - dx, iy, iz);
      const double cyz[2] = {wz[0] * sx_r, wz[1] * sx_r};
      const double cc = so_r * s_sp;

      const int prev = (s - 1) & 1, cur = s & 1;
      const double* in_yz = nullptr;
      const double* in_xz = nullptr;
      const double* in_xy = nullptr;
      if (wa > 0) in_yz = slot_yz + (size_t)(prev * NW + warp - 1) * ENT;
      else if (flags & TF_X_IN) in_yz = P.fyz + ((ent_yz_base + iz) * P.ny + iy) * (size_t)ENT;
      if (wb > 0) in_xz = slot_xz + (size_t)(prev * NW + warp - TX) * ENT;
      else if (flags & TF_Y_IN) in_xz = P.fxz + ((ent_yz_base + iz) * P.nx + ix) * (size_t)ENT;
      if (c == 0 && (flags & TF_Z_IN)) in_xy = P.fxy + ((ent_xy_base + iy) * P.nx + ix) * (size_t)ENT;
      const bool glob_yz = wa == 0, glob_xz = wb == 0;
      double* out_yz = slot_yz + (size_t)(cur * NW + warp) * ENT;
      double* out_xz = slot_xz + (size_t)(cur * NW + warp) * ENT;
      double* gout_yz = (wa == w - 1 && (flags & TF_X_OUT)) ? P.fyz + ((ent_yz_base + iz) * P.ny + iy) * (size_t)ENT : nullptr;
      double* gout_xz = (wb == h - 1 && (flags & TF_Y_OUT)) ? P.fxz + ((ent_yz_base + iz) * P.nx + ix) * (size_t)ENT : nullptr;
      double* gout_xy = (c == nzr - 1 && (flags & TF_Z_OUT)) ? P.fxy + ((ent_xy_base + iy) * P.nx + ix) * (size_t)ENT : nullptr;

      double d2[MT][2];
#pragma unroll
      for (int mt = 0; mt < MT; ++mt) d2[mt][0] = d2[mt][1] = 0.0;

#pragma unroll
      for (int ch = 0; ch < NCH; ++ch) {
        // ---- moments -> angles
        double d1[4][2];
#pragma unroll
        for (int t = 0; t < 4; ++t) d1[t][0] = d1[t][1] = 0.0;
#pragma unroll
        for (int k = 0; k < KS; ++k)
#pragma unroll
          for (int t = 0; t < 4; ++t) {
            const double b = NCH == 1 ? b1r[NCH == 1 ? k : 0][t] : b1s[((ch * KS + k) * 4 + t) * 32 + lane];
            dmma(d1[t], vif[k], b);
          }

        // ---- incoming faces
#pragma unroll
        for (int t = 0; t < 4; ++t) {
          const size_t eo = (size_t)((ch * 4 + t) * 32 + lane) * 2;
          double fyz[2], fxz[2], fxy[2];
          if (in_yz) {
            const double2 v = glob_yz ? __ldcg(reinterpret_cast<const double2*>(in_yz + eo))
                                      : *reinterpret_cast<const double2*>(in_yz + eo);
            fyz[0] = v.x; fyz[1] = v.y;
          } else {
#pragma unroll
            for (int i = 0; i < 2; ++i) {
              const int ia = 32 * ch + 8 * t + 2 * r + i;
              fyz[i] = (gval && ia < P.na) ? d_init_face(ia, dx > 0 ? -1 : P.nx, iy, iz, g_col, u_col, oct) : 0.0;
            }
          }
          if (in_xz) {
            const double2 v = glob_xz ? __ldcg(reinterpret_cast<const double2*>(in_xz + eo))
                                      : *reinterpret_cast<const double2*>(in_xz + eo);
            fxz[0] = v.x; fxz[1] = v.y;
          } else {
#pragma unroll
            for (int i = 0; i < 2; ++i) {
              const int ia = 32 * ch + 8 * t + 2 * r + i;
              fxz[i] = (gval && ia < P.na) ? d_init_face(ia, ix, dy > 0 ? -1 : P.ny, iz, g_col, u_col, oct) : 0.0;
            }
          }
          if (c > 0) {
            fxy[0] = carry[ch][t][0]; fxy[1] = carry[ch][t][1];
          } else if (in_xy) {
            const double2 v = __ldcg(reinterpret_cast<const double2*>(in_xy + eo));
            fxy[0] = v.x; fxy[1] = v.y;
          } else {
#pragma unroll
            for (int i = 0; i < 2; ++i) {
              const int ia = 32 * ch + 8 * t + 2 * r + i;
              fxy[i] = (gval && ia < P.na) ? d_init_face(ia, ix, iy, dz > 0 ? -1 : P.nz, g_col, u_col, oct) : 0.0;
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
            carry[ch][t][i] = out[i];
          }
          const double2 ov = make_double2(out[0], out[1]);
          *reinterpret_cast<double2*>(out_yz + eo) = ov;
          *reinterpret_cast<double2*>(out_xz + eo) = ov;
          if (gout_yz) __stcg(reinterpret_cast<double2*>(gout_yz + eo), ov);
          if (gout_xz) __stcg(reinterpret_cast<double2*>(gout_xz + eo), ov);
          if (gout_xy) __stcg(reinterpret_cast<double2*>(gout_xy + eo), ov);
        }

        // ---- angles -> moments (psi is already in B-operand layout)
#pragma unroll
        for (int t = 0; t < 4; ++t)
#pragma unroll
          for (int i = 0; i < 2; ++i)
#pragma unroll
            for (int mt = 0; mt < MT; ++mt) {
              const double a = NCH == 1 ? a2r[NCH == 1 ? mt : 0][t][i]
                                        : a2s[((((ch * MT + mt) * 4 + t) * 2 + i) * 32) + lane];
              dmma(d2[mt], a, d1[t][i]);
            }
      }

      // ---- accumulate vo in the region's visiting order
      if (gvo) {
        const size_t vbase = (size_t)NM_ * NU * (ix + (size_t)P.nx * iy) + slab * (g_vo + (size_t)P.ne * iz);
#pragma unroll
        for (int mt = 0; mt < MT; ++mt)
#pragma unroll
          for (int j = 0; j < 2; ++j) {
            const int im = 8 * mt + q;
            if (im < NM_) {
              const double v = first ? d2[mt][j] : __dadd_rn(vof[mt][j], d2[mt][j]);
              P.vo[vbase + NM_ * (2 * (r & 1) + j) + im] = v;
            }
          }
      }
    }
    if (s_stop[0] | s_stop[1]) {
      // a wait gave up: leave the task loop (the error is recorded)
      __syncthreads();
      break;
    }
  }
}

}  // namespace msb
