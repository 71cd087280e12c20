// sweep_mixed_tc.cuh -- the mixed-precision sweep kernel for sm_100a: the two
// per-cell transforms on the 5th-generation tensor cores (tcgen05.mma,
// accumulators in tensor memory), the face recurrence in FP32, the octant
// accumulation into vo in FP64.
//
// Same work as the plain-FP64 kernel (the reference's
// Sweeper_sweep_block_impl_global and Sweeper_sweep_cell,
// sweeper_kba_c_kernels.h:30-1383, under the host step loop of
// sweeper_kba_c.h:588-845), same task schedule and inter-CTA protocol.
//
// Numerics
//   T1  vs[angle]  = sum_m a_from_m[oct][m][angle] * vi[m]      (K = moments)
//   T2  vo[m]     += sum_a m_from_a[oct][a][m] * psi[a]          (K = angles)
//   Each operand is split into two 16-bit halves, x ~ hi + lo with
//   hi = rn16(x * 2^k), lo = rn16(x * 2^k - hi), where 2^k brings the largest
//   entry of the operand's row (or of the octant's matrix) to [2^14, 2^15);
//   the product keeps hi*hi + hi*lo + lo*hi and accumulates in FP32.  With
//   FP16 halves that is a 22-bit significand per operand (errors near FP32
//   rounding); with BF16 halves 16 bits.  Quantities_solve
//   (quantities_testing_kernels.h:337-447) runs in FP32 with fused
//   multiply-adds except its last step, psi = sm * cc + vs, which carries
//   the FP64 reciprocal 1 / (1 + octant) as an FP32 pair and the product's
//   and the sum's rounding errors (fma, TwoSum) to one final rounding;
//   faces are stored in FP32.  vo is summed and written in FP64.
//
// Tile and roles (one CTA, 10 warps)
//   A task is a 4 x 4 tile of cell columns x one group pair.  MMA row
//   32b + l (l = 8a + 4g + u) is (cell (a, b), group 2*gp + g, unknown u); at
//   step s it holds plane s - a - b of its column.  The 128 rows are the
//   M = 128 dimension of both products:
//     T1  D1[row][angle]  (N = 32)  = A1[row][moment]  x B1[angle][moment]^T
//     T2  D2[row][moment] (N = 16)  = A2[row][angle]   x B2[moment][angle]^T
//   so each row's angles and moments are read (tcgen05.ld 32x32b) from the
//   TMEM lane of that row, and A1 / A2 rows are written by their own threads.
//   warps 0-7  compute: warps b and b + 4 share tile row b (TMEM lanes
//              32b..32b+31) and split its 32 angles; half 0 converts vi,
//              half 1 accumulates vo; one thread of warp 0 issues the MMAs
//              and owns the tensor memory
//   warp 8     loader: tasks, dependencies, faces and vi entering the tile
//              (bulk and TMA copies), the octant's matrices (split, scaled,
//              in the MMA operand layout)
//   warp 9     publisher: task progress to global memory
//
// Faces inside the tile: every thread writes its output of step G to a
// double-buffered shared-memory slot; at step G + 1 cell (a, b) reads its yz
// face from lane l-8 of its own tile row and its xz face from tile row b-1;
// the xy face is the thread's own register copy (`carry`).
//
// Pipelining per global step G (TMEM accumulators and A2 indexed by G % 2):
//   wait T1(G); read D1(G); convert vi(G+1) -> A1, barrier, T1(G+1) issued;
//   solve, write A2(G), faces out; wait T2(G-1), vo partial += D2(G-1);
//   barrier of all compute warps; T2(G) issued; stage G handed back
// so T1 has most of a step and T2 a whole step to finish before they are
// read, the vo update trails the solve by one step, and no step waits for
// the previous step's T2 before writing its own A2.
#pragma once

#include <cuda.h>
#include <cuda_bf16.h>
#include <cuda_fp16.h>

#include "sweep_async.cuh"

namespace msb {

// vi16 holds the sweep's input state converted once per sweep into the first
// transform's operand format (convert_vi16 below): one block of kViBlock
// bytes per (cell, group pair), copied whole into a stage by the loader.
// Each octant's contribution to vo is written to its own FP32 partial array
// (the state layout, `part + oct * state`); a second kernel sums the eight
// partials into vo in FP64.
struct MixParams {
  const unsigned char* vi16;
  float* part;
  size_t state;  // elements of one state array
  const double* afm;  // a_from_m [oct][im][ia]
  const double* mfa;  // m_from_a [oct][ia][im]
  float* fxy;         // face planes: one 1 KiB entry per (octant, group pair, position)
  float* fxz;
  float* fyz;
  const int* tasks;
  long long ntask;
  int nx, ny, nz, ne, na, ngp;
  int ia_base;     // angle index of the first angle of afm / mfa (32-angle passes over a larger na)
  int ie_base;     // global index of group 0 (energy-group slices of a larger problem)
  SyncArgs sy;
};

// One (cell, group pair) of vi in the first transform's operand format: the
// cell's 8 rows (group g, unknown u: row 4 g + u) of A1, hi halves then lo
// halves, each 256 bytes in the K-major core-matrix order of A1 ([moment
// chunk 8 m / 8][row][moment % 8], 2 bytes each), then the row scale 2^k1
// of each (moment chunk, row) as one signed byte.
constexpr int kViBlock = 2 * 256 + 16;

enum MixFormat { MIX_F16 = 0, MIX_BF16 = 1 };

// ------------------------------------------------------------- tcgen05 ops
// Shared-memory matrix descriptor, K-major, no swizzle: element (row i, k) of
// an operand lives at byte (i/8)*sbo + (k/8)*lbo + (i%8)*16 + (k%8)*2.
__device__ __forceinline__ uint64_t umma_sdesc(uint32_t addr, uint32_t lbo, uint32_t sbo) {
  return (uint64_t)((addr >> 4) & 0x3fff) | ((uint64_t)((lbo >> 4) & 0x3fff) << 16) |
         ((uint64_t)((sbo >> 4) & 0x3fff) << 32) | ((uint64_t)1 << 46);
}
__host__ __device__ constexpr int kmajor_off(int i, int k, int lbo, int sbo) {
  return (i >> 3) * sbo + (k >> 3) * lbo + (i & 7) * 16 + (k & 7) * 2;
}
// Instruction descriptor of kind::f16: FP32 accumulator, A and B of the same
// 16-bit format, both K-major, M x N.
__host__ __device__ constexpr uint32_t umma_idesc(int fmt, int M, int N) {
  return (1u << 4) | ((uint32_t)fmt << 7) | ((uint32_t)fmt << 10) | ((uint32_t)(N >> 3) << 17) |
         ((uint32_t)(M >> 4) << 24);
}
__device__ __forceinline__ void umma_f16(uint32_t d_tmem, uint64_t a, uint64_t b, uint32_t idesc, uint32_t acc) {
  asm volatile(
      "{\n .reg .pred p;\n setp.ne.b32 p, %4, 0;\n tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n}" ::"r"(
          d_tmem),
      "l"(a), "l"(b), "r"(idesc), "r"(acc)
      : "memory");
}
__device__ __forceinline__ void umma_commit(uint64_t* bar) {
  asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(smem_u32(bar))
               : "memory");
}
__device__ __forceinline__ void tc_fence_before() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void tc_fence_after() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void fence_async_smem() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }
// One 5-D TMA tile copy global -> shared, completion counted on an mbarrier.
__device__ __forceinline__ void tma_load_5d(void* dst, const CUtensorMap* map, int c0, int c1, int c2, int c3, int c4,
                                            uint64_t* bar) {
  asm volatile(
      "cp.async.bulk.tensor.5d.shared::cluster.global.tile.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3, %4, %5, %6}], "
      "[%7];" ::"r"(smem_u32(dst)),
      "l"(reinterpret_cast<uint64_t>(map)), "r"(c0), "r"(c1), "r"(c2), "r"(c3), "r"(c4), "r"(smem_u32(bar))
      : "memory");
}
__device__ __forceinline__ void tmem_wait_ld() { asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory"); }
__device__ __forceinline__ void tmem_ld8(uint32_t taddr, float (&v)[8]) {
  uint32_t r[8];
  asm volatile("tcgen05.ld.sync.aligned.32x32b.x8.b32 {%0,%1,%2,%3,%4,%5,%6,%7}, [%8];"
               : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7])
               : "r"(taddr));
#pragma unroll
  for (int i = 0; i < 8; ++i) v[i] = __uint_as_float(r[i]);
}
__device__ __forceinline__ void tmem_ld16(uint32_t taddr, float (&v)[16]) {
  uint32_t r[16];
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15}, [%16];"
      : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]), "=r"(r[8]),
        "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
      : "r"(taddr));
#pragma unroll
  for (int i = 0; i < 16; ++i) v[i] = __uint_as_float(r[i]);
}

// ------------------------------------------------------- 16-bit splitting
template <int FMT>
struct Half16;
template <>
struct Half16<MIX_F16> {
  static __device__ __forceinline__ uint16_t rn(double x) { return __half_as_ushort(__double2half(x)); }
  static __device__ __forceinline__ float val(uint16_t h) { return __half2float(__ushort_as_half(h)); }
  static __device__ __forceinline__ uint32_t pack(float x, float y) {
    const __half2 t = __floats2half2_rn(x, y);
    return *reinterpret_cast<const uint32_t*>(&t);
  }
  static __device__ __forceinline__ float2 unpack(uint32_t p) {
    return __half22float2(*reinterpret_cast<const __half2*>(&p));
  }
};
template <>
struct Half16<MIX_BF16> {
  static __device__ __forceinline__ uint16_t rn(double x) { return __bfloat16_as_ushort(__double2bfloat16(x)); }
  static __device__ __forceinline__ float val(uint16_t h) { return __bfloat162float(__ushort_as_bfloat16(h)); }
  static __device__ __forceinline__ uint32_t pack(float x, float y) {
    const __nv_bfloat162 t = __floats2bfloat162_rn(x, y);
    return *reinterpret_cast<const uint32_t*>(&t);
  }
  static __device__ __forceinline__ float2 unpack(uint32_t p) {
    return __bfloat1622float2(*reinterpret_cast<const __nv_bfloat162*>(&p));
  }
};

// The scale 2^k that brings m (> 0) to [2^14, 2^15); k is clamped so that
// 2^k and 2^-k stay normal floats.  m = 0 gives k = 0.
__device__ __forceinline__ int split_scale_d(double m) {
  if (!(m > 0.0)) return 0;
  const int be = (int)((__double_as_longlong(m) >> 52) & 0x7ff);
  const int e = be == 0 ? -1021 : be - 1022;  // m in [2^(e-1), 2^e)
  return max(-120, min(120, 15 - e));
}
__device__ __forceinline__ int split_scale_f(float m) {
  if (!(m > 0.0f)) return 0;
  const int be = (__float_as_int(m) >> 23) & 0xff;
  const int e = be == 0 ? -125 : be - 126;
  return max(-120, min(120, 15 - e));
}
__device__ __forceinline__ float f_pow2(int k) { return __int_as_float((127 + k) << 23); }

template <int NM_, int NS>
struct MixCfg {
  static constexpr int TX = 4, TY = 4;      // cell columns of a tile
  static constexpr int NW = 8;              // compute warps: tile row x angle half
  static constexpr int NT = (NW + 3) * 32;  // + loader, publisher, MMA issuer
  static constexpr int KP = 16;             // moments, padded to one MMA K-step
  static constexpr int NA = 32;             // angles per MMA: one pass (larger na: one pass per 32)
  static constexpr int EB = 1024;           // bytes per face entry: 8 rows x 32 floats
  // stage (bytes), filled by the loader with bulk copies: entering yz faces
  // (one per tile row), xz (one per column), xy of the first plane (one per
  // row), the vi16 block of every cell column at this step, then the step
  // header
  static constexpr int ST_YZ = 0;
  static constexpr int ST_XZ = ST_YZ + TY * EB;
  static constexpr int ST_XY = ST_XZ + TX * EB;
  static constexpr int ST_VI = ST_XY + TY * EB;
  static constexpr int ST_HDR = ST_VI + TX * TY * kViBlock;
  static constexpr int STAGE = (ST_HDR + 128 + 1023) / 1024 * 1024;
  // MMA operands (bytes); each comes as a hi and a lo matrix
  static constexpr int A1M = 128 * KP * 2;  // LBO 128, SBO 256
  static constexpr int A2M = 128 * NA * 2;  // LBO 128, SBO 512
  static constexpr int B1M = NA * KP * 2;   // [angle][moment], LBO 128, SBO 256
  static constexpr int B2M = 16 * NA * 2;   // [moment][angle], LBO 128, SBO 512
  // B1 comes twice, with moments 8-15 and with moments 0-7 zeroed (the two
  // halves of vi carry separate row scales: T1 is two products); then B2
  static constexpr bool SPLIT_K = NM_ > 8;
  static constexpr int MATBUF = 4 * B1M + 2 * B2M;
  static constexpr int SLOT = 32 * 16 * 4;  // one warp's outgoing faces (16 angles)
  // shared-memory layout (bytes)
  static constexpr int SM_STAGE = 0;
  static constexpr int SM_A1 = SM_STAGE + NS * STAGE;  // [hi, lo]
  static constexpr int SM_A2 = SM_A1 + 2 * A1M;       // [step parity][hi, lo]
  static constexpr int SM_MAT = SM_A2 + 4 * A2M;      // [2 buffers][B1 hi, B1 lo, B2 hi, B2 lo]
  static constexpr int SM_SLOT = SM_MAT + 2 * MATBUF;  // [2 parity][tile row][2 halves]
  static constexpr int SM_KS = SM_SLOT + 2 * TY * 2 * SLOT;  // row scales k1, k2: [2][2][128] ints
  static constexpr int SM_BAR = SM_KS + 2 * 2 * 2 * 128 * 4;
  // barriers: full, done, freed [NS]; d1, d2 [2]; fin
  static constexpr int NBAR = 3 * NS + 2 * 2 + 1;
  static constexpr int SM_MISC = SM_BAR + 8 * NBAR;  // tmem base, matrix scales [2][2]
  static constexpr size_t smem_bytes() { return (size_t)SM_MISC + 64; }
  // tensor memory columns: D1 [2 buffers][2 moment halves][32 angles],
  // D2 [2 buffers][2 angle halves][16 moments]
  static constexpr int TM_COLS = 256;
  static constexpr int TM_D1 = 0, TM_D2 = 128;
};

template <int NM_, int FMT, int NS>
__global__ void __launch_bounds__(MixCfg<NM_, NS>::NT, 1) sweep_mixed_kernel(const __grid_constant__ MixParams P) {
  using C = MixCfg<NM_, NS>;
  using H = Half16<FMT>;
  constexpr int NW = C::NW, TX = C::TX, TY = C::TY, EB = C::EB;
  constexpr int EF = EB / 4;   // floats per face entry
  constexpr int CH = NM_ / 2;  // 16-byte chunks per vi/vo row
  static_assert(NM_ == 4 || NM_ == 8 || NM_ == 16, "NM must be 4, 8 or 16");
  static_assert(TX * TY * 2 * NU == 128, "one MMA row per (cell, group, unknown)");
  static_assert(NW == 2 * TY, "two compute warps (angle halves) per tile row");

  extern __shared__ __align__(1024) unsigned char smem_mx[];
  unsigned char* const smem = smem_mx;
  unsigned char* const stages = smem + C::SM_STAGE;
  uint64_t* const full = reinterpret_cast<uint64_t*>(smem + C::SM_BAR);
  uint64_t* const done = full + NS;
  uint64_t* const freed = done + NS;
  uint64_t* const d1bar = freed + NS;  // T1 of step G done (tcgen05.commit)
  uint64_t* const d2bar = d1bar + 2;    // T2 of step G done
  uint64_t* const finbar = d2bar + 2;
  uint32_t* const tmem_base = reinterpret_cast<uint32_t*>(smem + C::SM_MISC);
  int* const mat_scale = reinterpret_cast<int*>(smem + C::SM_MISC + 16);  // [2][kb1, kb2]
  __shared__ volatile int s_final;
  __shared__ volatile int s_abort;  // a compute thread's bounded wait ran out

  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  int* const sync = P.sy.sync;
  int* const progress = sync + SY_PROGRESS;
  const size_t slab = (size_t)NM_ * NU * P.nx * P.ny;  // one (iz, ie) layer of the state

  if (threadIdx.x == 0) {
    for (int i = 0; i < NS; ++i) {
      mbar_init(&full[i], 1);
      mbar_init(&done[i], 1);
      mbar_init(&freed[i], 1);
    }
    for (int i = 0; i < 2; ++i) {
      mbar_init(&d1bar[i], 1);
      mbar_init(&d2bar[i], 1);
    }
    mbar_init(finbar, 1);
    s_final = -1;
    s_abort = 0;
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  if (warp == NW + 2) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(tmem_base)),
                 "r"(C::TM_COLS)
                 : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
  }
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tmem = *tmem_base;

  // Named barriers.  1: the eight compute warps and the MMA warp, once per
  // step (A2, slots and row scales of the step complete) and at task starts;
  // 2: the compute warps arrive, the MMA warp waits (A1 complete).  A
  // bounded mbarrier wait that runs out only raises s_abort; every warp reads
  // it after the next barrier 1 and they all leave together, so no warp is
  // ever left at a barrier.
  auto bar_step = []() { asm volatile("bar.sync 1, %0;" ::"n"((NW + 1) * 32) : "memory"); };
  auto arrive_a1 = []() { asm volatile("bar.arrive 2, %0;" ::"n"((NW + 1) * 32) : "memory"); };
  auto sync_a1 = []() { asm volatile("bar.sync 2, %0;" ::"n"((NW + 1) * 32) : "memory"); };
  auto wait = [&](uint64_t* bar, long long phase_index, int per) {
    if (!mbar_wait(bar, (uint32_t)((phase_index / per) & 1), P.sy, -1)) s_abort = 1;
  };

  if (warp == NW) {
    // ================================================================ loader
    long long g_load = 0;
    long long last_step[2] = {-1, -1};
    int ntask_seen = 0;
    bool failed = false;
    long long freed_upto = -1;
    auto wait_freed = [&](long long g) -> bool {
      for (long long x = freed_upto + 1; x <= g; ++x) {
        if (!mbar_wait(&freed[x % NS], (uint32_t)((x / NS) & 1), P.sy, -1)) return false;
        freed_upto = x;
      }
      return true;
    };
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
        const long long tt = atomicAdd(&sync[SY_COUNTER], 1);
        t = tt < P.ntask ? (int)tt : -1;
      }
      return __shfl_sync(0xffffffffu, t, 0);
    };
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
      if (rec[TK_DEP_X] >= 0 && depx < 0 && wait_dep(&progress[rec[TK_DEP_X]], kComplete, t) < 0) failed = true;
      if (!failed && rec[TK_DEP_Y] >= 0 && depy < 0 && wait_dep(&progress[rec[TK_DEP_Y]], kComplete, t) < 0) failed = true;
      if (!failed && rec[TK_DEP_Z] >= 0 && wait_dep(&progress[rec[TK_DEP_Z]], kComplete, t) < 0) failed = true;
      if (!failed && rec[TK_DEP_VO] >= 0 && wait_dep(&progress[rec[TK_DEP_VO]], kComplete, t) < 0) failed = true;
      const int mb = ntask_seen & 1;
      if (!failed && !wait_freed(last_step[mb])) failed = true;
      if (failed) break;
      __threadfence_block();
      // ---- the octant's matrices, split into scaled hi/lo operand matrices
      {
        unsigned char* mat = smem + C::SM_MAT + mb * C::MATBUF;
        double m1 = 0.0, m2 = 0.0;
        for (int e = lane; e < NM_ * P.na; e += 32) {
          m1 = fmax(m1, fabs(__ldg(&P.afm[(size_t)e + (size_t)NM_ * P.na * oct])));
          m2 = fmax(m2, fabs(__ldg(&P.mfa[(size_t)e + (size_t)NM_ * P.na * oct])));
        }
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) {
          m1 = fmax(m1, __shfl_xor_sync(0xffffffffu, m1, o));
          m2 = fmax(m2, __shfl_xor_sync(0xffffffffu, m2, o));
        }
        const int kb1 = split_scale_d(m1), kb2 = split_scale_d(m2);
        const double s1 = d_pow2(kb1), s2 = d_pow2(kb2);
        // B1[angle][moment] = a_from_m[oct][moment][angle]: B1a keeps moments
        // 0-7 (all of them when NM <= 8), B1b moments 8-15
        for (int e = lane; e < C::NA * C::KP; e += 32) {
          const int n = e / C::KP, k = e % C::KP;
          const double x = (n < P.na && k < NM_) ? __ldg(&P.afm[n + (size_t)P.na * (k + (size_t)NM_ * oct)]) * s1 : 0.0;
          const uint16_t hi = H::rn(x), lo = H::rn(x - (double)H::val(hi));
          const int off = kmajor_off(n, k, 128, 256);
          const bool in_a = k < 8 || !C::SPLIT_K;
          *reinterpret_cast<uint16_t*>(mat + off) = in_a ? hi : (uint16_t)0;
          *reinterpret_cast<uint16_t*>(mat + C::B1M + off) = in_a ? lo : (uint16_t)0;
          *reinterpret_cast<uint16_t*>(mat + 2 * C::B1M + off) = in_a ? (uint16_t)0 : hi;
          *reinterpret_cast<uint16_t*>(mat + 3 * C::B1M + off) = in_a ? (uint16_t)0 : lo;
        }
        // B2[moment][angle] = m_from_a[oct][angle][moment]
        for (int e = lane; e < 16 * C::NA; e += 32) {
          const int n = e / C::NA, k = e % C::NA;
          const double x = (n < NM_ && k < P.na) ? __ldg(&P.mfa[n + (size_t)NM_ * (k + (size_t)P.na * oct)]) * s2 : 0.0;
          const uint16_t hi = H::rn(x), lo = H::rn(x - (double)H::val(hi));
          const int off = kmajor_off(n, k, 128, 512);
          *reinterpret_cast<uint16_t*>(mat + 4 * C::B1M + off) = hi;
          *reinterpret_cast<uint16_t*>(mat + 4 * C::B1M + C::B2M + off) = lo;
        }
        if (lane == 0) {
          mat_scale[2 * mb] = kb1;
          mat_scale[2 * mb + 1] = kb2;
        }
        fence_async_smem();  // generic writes -> tensor-core reads
        __syncwarp();
      }
      ++ntask_seen;
      last_step[mb] = g_load + nsteps - 1;

      const size_t ent_z = (size_t)(oct * P.ngp + gp) * P.nz;
      const size_t ent_y = (size_t)(oct * P.ngp + gp) * P.ny;
      int seen_x = 0, seen_y = 0;
      for (int s = 0; s < nsteps; ++s) {
        const int st = (int)(g_load % NS);
        if (g_load >= NS && !wait_freed(g_load - NS)) { failed = true; break; }
        const int need = min(s + 1, nzr);
        if (depx >= 0 && seen_x < need && (seen_x = wait_dep(&progress[depx], need, t)) < 0) { failed = true; break; }
        if (depy >= 0 && seen_y < need && (seen_y = wait_dep(&progress[depy], need, t)) < 0) { failed = true; break; }
        fence_proxy_async();
        fence_async_smem();
        __threadfence_block();
        unsigned char* stg = stages + (size_t)st * C::STAGE;
        StepHdr* hdr = reinterpret_cast<StepHdr*>(stg + C::ST_HDR);
        // vi of cell (va, vb), both groups, at this step: lane 4*vb + va
        const int va = lane & 3, vb = lane >> 2, cvi = s - va - vb;
        const bool vi_ok = lane < TX * TY && va < w && vb < h && cvi >= 0 && cvi < nzr;
        uint32_t bytes = (uint32_t)__popc(__ballot_sync(0xffffffffu, vi_ok)) * (uint32_t)kViBlock;
        for (int b = 0; b < h; ++b) {
          const int c = s - b;
          if ((flags & TF_X_IN) && c >= 0 && c < nzr) bytes += EB;
          if ((flags & TF_Z_IN) && c >= 0 && c < w) bytes += EB;  // xy of cell (s - b, b), plane 0
        }
        for (int a = 0; a < w; ++a) {
          const int c = s - a;
          if ((flags & TF_Y_IN) && c >= 0 && c < nzr) bytes += EB;
        }
        if (lane == 0) {
          hdr->task = t; hdr->s = s; hdr->oct = oct; hdr->gp = gp;
          hdr->x0 = x0; hdr->x1 = x1; hdr->y0 = y0; hdr->y1 = y1; hdr->z0 = z0; hdr->z1 = z1;
          hdr->flags = flags; hdr->mat = mb; hdr->stop = 0;
          hdr->pad0 = s == nsteps - 1 ? kComplete : (s + 1 - (w + h - 2) > 0 ? s + 1 - (w + h - 2) : -2);
          mbar_arrive_expect_tx(&full[st], bytes);
        }
        __syncwarp();
        if (vi_ok) {
          const int ix = dx > 0 ? x0 + va : x1 - 1 - va, iy = dy > 0 ? y0 + vb : y1 - 1 - vb;
          const int iz = dz > 0 ? z0 + cvi : z1 - 1 - cvi;
          bulk_g2s(stg + C::ST_VI + (4 * vb + va) * kViBlock,
                   P.vi16 + (((size_t)iz * P.ngp + gp) * P.ny * P.nx + (size_t)iy * P.nx + ix) * kViBlock, kViBlock,
                   &full[st]);
        }
        // lanes [0, TY): yz of row b; [8, 8+TX): xz of column a; [16, 16+TY): xy of row b
        const int kind = lane >> 3, pos = lane & 7;
        if (kind == 0 && pos < h && (flags & TF_X_IN)) {
          const int b = pos, c = s - b;
          if (c >= 0 && c < nzr) {
            const int iy = dy > 0 ? y0 + b : y1 - 1 - b, iz = dz > 0 ? z0 + c : z1 - 1 - c;
            bulk_g2s(stg + C::ST_YZ + b * EB, P.fyz + ((ent_z + iz) * P.ny + iy) * (size_t)EF, EB, &full[st]);
          }
        } else if (kind == 1 && pos < w && (flags & TF_Y_IN)) {
          const int a = pos, c = s - a;
          if (c >= 0 && c < nzr) {
            const int ix = dx > 0 ? x0 + a : x1 - 1 - a, iz = dz > 0 ? z0 + c : z1 - 1 - c;
            bulk_g2s(stg + C::ST_XZ + a * EB, P.fxz + ((ent_z + iz) * P.nx + ix) * (size_t)EF, EB, &full[st]);
          }
        } else if (kind == 2 && pos < h && (flags & TF_Z_IN)) {
          const int b = pos, a = s - b;
          if (a >= 0 && a < w) {
            const int ix = dx > 0 ? x0 + a : x1 - 1 - a, iy = dy > 0 ? y0 + b : y1 - 1 - b;
            bulk_g2s(stg + C::ST_XY + b * EB, P.fxy + ((ent_y + iy) * P.nx + ix) * (size_t)EF, EB, &full[st]);
          }
        }
        ++g_load;
      }
      if (failed) break;
    }
    // Drain, then a stop header ends the other roles at the same step.
    if (lane == 0) s_final = (int)g_load;
    if (wait_freed(g_load - 1)) {
      const int st = (int)(g_load % NS);
      __threadfence_block();
      if (lane == 0) {
        StepHdr* hdr = reinterpret_cast<StepHdr*>(stages + (size_t)st * C::STAGE + C::ST_HDR);
        hdr->stop = 1;
        mbar_arrive_expect_tx(&full[st], 0);
      }
    }
    __syncwarp();
  } else if (warp == NW + 1) {
    // ============================================================= publisher
    long long G = 0;
    long long t0 = global_ns();
    bool quit = false;
    while (!quit) {
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
      int pend_task[2] = {-1, -1}, pend_val[2] = {-2, -2};
      for (;;) {
        const int st = (int)(G % NS);
        const StepHdr* hdr = reinterpret_cast<const StepHdr*>(stages + (size_t)st * C::STAGE + C::ST_HDR);
        const int task = hdr->task, val = hdr->pad0;
        __syncwarp();
        if (lane == 0) mbar_arrive(&freed[st]);
        if (val != -2) {
          if (pend_task[1] >= 0 && pend_task[1] != task) {
            pend_task[0] = pend_task[1];
            pend_val[0] = pend_val[1];
          }
          pend_task[1] = task;
          pend_val[1] = val;
        }
        ++G;
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
        }
      }
      t0 = global_ns();
    }
  } else if (warp == NW + 2) {
    // ============================================================ MMA issuer
    // Follows the compute warps' barriers: T1 of step G + 1 once the
    // converters have written A1, T2 of step G at the end of step G.
    constexpr uint32_t ID1 = umma_idesc(FMT, 128, C::NA), ID2 = umma_idesc(FMT, 128, 16);
    const uint32_t a1u = smem_u32(smem + C::SM_A1), a2u = smem_u32(smem + C::SM_A2);
    // the two moment halves of A1 carry separate row scales: one product and
    // one accumulator each (B1a / B1b zero the other half's moments)
    auto issue_t1 = [&](long long gg, uint32_t b1) {
      tc_fence_after();
      if (lane == 0) {
#pragma unroll
        for (int kh = 0; kh < (C::SPLIT_K ? 2 : 1); ++kh) {
          const uint32_t d = tmem + C::TM_D1 + (uint32_t)(gg & 1) * 64 + 32u * kh, bb = b1 + 2 * C::B1M * kh;
          umma_f16(d, umma_sdesc(a1u + C::A1M, 128, 256), umma_sdesc(bb, 128, 256), ID1, 0);  // lo x hi
          umma_f16(d, umma_sdesc(a1u, 128, 256), umma_sdesc(bb + C::B1M, 128, 256), ID1, 1);  // hi x lo
          umma_f16(d, umma_sdesc(a1u, 128, 256), umma_sdesc(bb, 128, 256), ID1, 1);           // hi x hi
        }
        umma_commit(&d1bar[gg & 1]);
      }
      __syncwarp();
    };
    // angles 0-15 and 16-31 carry separate row scales: one accumulator each
    auto issue_t2 = [&](long long gg, uint32_t b2) {
      tc_fence_after();
      if (lane == 0) {
#pragma unroll
        for (int kk = 0; kk < 2; ++kk) {
          // o: this angle half's K chunk in A2 and B2; A2 also by step parity
          const uint32_t o = 256u * kk, a2 = a2u + (uint32_t)(gg & 1) * 2 * C::A2M + o;
          const uint32_t d = tmem + C::TM_D2 + (uint32_t)(gg & 1) * 32 + 16u * kk;
          umma_f16(d, umma_sdesc(a2 + C::A2M, 128, 512), umma_sdesc(b2 + o, 128, 512), ID2, 0);
          umma_f16(d, umma_sdesc(a2, 128, 512), umma_sdesc(b2 + C::B2M + o, 128, 512), ID2, 1);
          umma_f16(d, umma_sdesc(a2, 128, 512), umma_sdesc(b2 + o, 128, 512), ID2, 1);
        }
        umma_commit(&d2bar[gg & 1]);
      }
      __syncwarp();
    };
    long long G = 0;
    for (;;) {
      wait(&full[G % NS], G, NS);
      bar_step();  // task start
      if (s_abort) break;
      const StepHdr* hdr = reinterpret_cast<const StepHdr*>(stages + (size_t)(G % NS) * C::STAGE + C::ST_HDR);
      if (hdr->stop) break;
      const int nsteps = (hdr->z1 - hdr->z0) + (hdr->x1 - hdr->x0) + (hdr->y1 - hdr->y0) - 2;
      const uint32_t b1u = smem_u32(smem + C::SM_MAT + hdr->mat * C::MATBUF), b2u = b1u + 4 * C::B1M;
      bar_step();  // A1 of the task's first step written
      if (s_abort) break;
      issue_t1(G, b1u);
      bool quit = false;
      for (int s = 0; s < nsteps; ++s, ++G) {
        if (s + 1 < nsteps) {
          sync_a1();
          issue_t1(G + 1, b1u);
        }
        bar_step();  // end of step G
        if (s_abort) { quit = true; break; }
        issue_t2(G, b2u);
        // step G's stage is consumed and its faces are written: the
        // publisher may publish its progress and hand the stage back (the vo
        // partials need no ordering: each octant writes its own array, read
        // only by the next kernel)
        if (lane == 0) mbar_arrive(&done[G % NS]);
        if (s == nsteps - 1) {
          bar_step();  // the task's last vo written
          if (s_abort) { quit = true; break; }
        }
      }
      if (quit) break;
    }
    // every product issued has completed before the tensor memory is released
    if (lane == 0) umma_commit(finbar);
    __syncwarp();
    mbar_wait(finbar, 0, P.sy, -1);
  } else {
    // =============================================================== compute
    // Warps b and b + 4 own the same 32 MMA rows (tile row b; TMEM lanes
    // 32b..32b+31) and split the angles: half 0 takes angles 0-15 and converts
    // vi, half 1 takes angles 16-31 and accumulates vo.
    const int half = warp >> 2, b = warp & 3;
    const int a = lane >> 3, g = (lane >> 2) & 1, u = lane & 3, j = lane & 7;
    const int row = 32 * b + lane;
    const int ia0 = 16 * half;
    const uint32_t trow = tmem + ((uint32_t)(32 * b) << 16);
    unsigned char* const a1s = smem + C::SM_A1;
    unsigned char* const a2s = smem + C::SM_A2;
    float* const slots = reinterpret_cast<float*>(smem + C::SM_SLOT);
    int* const k1s = reinterpret_cast<int*>(smem + C::SM_KS);  // [2][moment half][128] row scales of A1
    int* const k2s = k1s + 512;                                 // [2][angle half][128] row scales of A2
    const int sw = (lane >> 1) & 3;  // swizzle of the 64-byte slot rows
    float carry[16];
#pragma unroll
    for (int i = 0; i < 16; ++i) carry[i] = 0.0f;

    long long G = 0;
    bool stop = false;
    while (!stop) {
      // ------------------------------------------------ one task per iteration
      wait(&full[G % NS], G, NS);
      bar_step();  // task start
      if (s_abort) break;
      const StepHdr* hdr0 = reinterpret_cast<const StepHdr*>(stages + (size_t)(G % NS) * C::STAGE + C::ST_HDR);
      if (hdr0->stop) break;
      const int oct = hdr0->oct, gp = hdr0->gp, flags = hdr0->flags, mb = hdr0->mat;
      const int x0 = hdr0->x0, x1 = hdr0->x1, y0 = hdr0->y0, y1 = hdr0->y1, z0 = hdr0->z0, z1 = hdr0->z1;
      const int w = x1 - x0, h = y1 - y0, nzr = z1 - z0, nsteps = nzr + w + h - 2;
      const int dx = (oct & 1) ? -1 : 1, dy = (oct & 2) ? -1 : 1, dz = (oct & 4) ? -1 : 1;
      const int g_col = 2 * gp + g;
      const bool rowv = a < w && b < h && g_col < P.ne;  // this row exists in the task
      const int ix = dx > 0 ? x0 + a : x1 - 1 - a;
      const int iy = dy > 0 ? y0 + b : y1 - 1 - b;
      const int iz0 = dz > 0 ? z0 : z1 - 1;
      const int cbeg = a + b;
      const int kb1 = mat_scale[2 * mb], kb2 = mat_scale[2 * mb + 1];
      const float so = (float)(1 + oct);
      // 1 / (1 + octant) rounded in FP64, as the reference rounds it, carried
      // as an FP32 pair so_hi + so_lo (to 2^-48): the solve forms its product
      // with psi's other terms with one final rounding (see below)
      const double so_rd = 1.0 / (double)(1 + oct);
      const float so_hi = __double2float_rn(so_rd);
      const float so_lo = __double2float_rn(so_rd - (double)so_hi);
      const float face_k =
          rowv ? (float)d_scale_energy(P.ie_base + g_col) * (float)d_scale_unknown(u) * so : 0.0f;
      const int sp_xy = ix + 3 * iy + 2;
      const size_t ent_z = (size_t)(oct * P.ngp + gp) * P.nz;
      const size_t ent_y = (size_t)(oct * P.ngp + gp) * P.ny;
      const bool x_in = a == 0 && (flags & TF_X_IN), y_in = b == 0 && (flags & TF_Y_IN);
      const bool z_in = (flags & TF_Z_IN) != 0;
      const bool x_out = a == w - 1 && (flags & TF_X_OUT), y_out = b == h - 1 && (flags & TF_Y_OUT);
      const bool z_out = (flags & TF_Z_OUT) != 0;
      const int gx = dx > 0 ? -1 : P.nx, gy = dy > 0 ? -1 : P.ny, gz = dz > 0 ? -1 : P.nz;
      const long long G0 = G;
      // state offset (doubles) of this row at plane 0; + zstep per plane
      const size_t row0 = (size_t)NM_ * u + (size_t)NM_ * NU * (ix + (size_t)P.nx * iy) + slab * (size_t)g_col +
                          (size_t)(slab * P.ne) * (size_t)iz0;
      const long long zstep = (long long)(slab * P.ne) * dz;
      float* const part_oct = P.part + P.state * (size_t)oct;

      // vi of global step gg (its vi16 block landed in its stage) -> K-chunk
      // `half` of this row of A1, hi and lo, and the chunk's row scale
      auto convert_vi = [&](long long gg, bool act) {
        int k1 = 0;
        if (act) {
          const unsigned char* blk = stages + (size_t)(gg % NS) * C::STAGE + C::ST_VI + (row >> 3) * kViBlock;
          const int o = half * 128 + (row & 7) * 16;
          const int off = kmajor_off(row, 8 * half, 128, 256);
          *reinterpret_cast<uint4*>(a1s + off) = *reinterpret_cast<const uint4*>(blk + o);
          *reinterpret_cast<uint4*>(a1s + C::A1M + off) = *reinterpret_cast<const uint4*>(blk + 256 + o);
          k1 = (int)reinterpret_cast<const signed char*>(blk + 512)[half * 8 + (row & 7)];
        }
        k1s[(gg & 1) * 256 + half * 128 + row] = k1;
      };
      struct Pend {
        long long gg;
        float* dst;
        int k2;
        bool act;
      };
      // this octant's contribution D2(gg) to vo, this row's moments of this
      // half (8*half ..), into the octant's FP32 partial array (D2 complete:
      // waited by the caller; the A2 scales of both angle halves were written
      // before a barrier)
      auto epilogue = [&](const Pend& pe) {
        constexpr int MH = NM_ / 2;  // moments per half
        tc_fence_after();
        float d0[8], d1[8];
        tmem_ld8(trow + C::TM_D2 + (uint32_t)(pe.gg & 1) * 32 + MH * half, d0);
        tmem_ld8(trow + C::TM_D2 + (uint32_t)(pe.gg & 1) * 32 + 16 + MH * half, d1);
        tmem_wait_ld();
        if (pe.act) {
          // un-scale: each accumulator times 2^e with e = -k2 - kb2 (|e| <=
          // 240) in two exact power-of-two steps of e / 2 (an intermediate
          // lies between the accumulator and the result, so it stays normal
          // wherever both do), the two halves' terms added with one
          // rounding (fma)
          const int kx = (pe.gg & 1) * 256 + row;
          const int e0 = -k2s[kx] - kb2, e1 = -k2s[kx + 128] - kb2;
          const float f0a = f_pow2(e0 / 2), f0b = f_pow2(e0 - e0 / 2);
          const float f1a = f_pow2(e1 / 2), f1b = f_pow2(e1 - e1 / 2);
          float o[MH];
#pragma unroll
          for (int m = 0; m < MH; ++m)
            o[m] = __fmaf_rn(__fmul_rn(d0[m], f0a), f0b, __fmul_rn(__fmul_rn(d1[m], f1a), f1b));
          float* dst = pe.dst + MH * half;
          if constexpr (MH % 4 == 0) {
#pragma unroll
            for (int q = 0; q < MH / 4; ++q)
              reinterpret_cast<float4*>(dst)[q] = make_float4(o[4 * q], o[4 * q + 1], o[4 * q + 2], o[4 * q + 3]);
          } else {
#pragma unroll
            for (int q = 0; q < MH / 2; ++q) reinterpret_cast<float2*>(dst)[q] = make_float2(o[2 * q], o[2 * q + 1]);
          }
        }
      };
      // ---- prologue: vi of step 0 -> A1 (only cell (0, 0) is active), T1 of
      // step 0 issued; the previous vo of step 0 requested
      convert_vi(G0, rowv && cbeg == 0);
      fence_async_smem();
      tc_fence_before();
      bar_step();
      if (s_abort) break;

      Pend pend{0, nullptr, 0, false};
      bool has_pend = false;
      for (int s = 0; s < nsteps; ++s, ++G) {
        const int st = (int)(G % NS);
        const unsigned char* stg = stages + (size_t)st * C::STAGE;
        if (s > 0) wait(&full[st], G, NS);
        const int c = s - cbeg;
        const bool act = rowv && c >= 0 && c < nzr;
        // ---- this step's T1 is done: D1 readable, A1 free for the next step.
        // D1 is read before the next step's T1 is released: a TMEM load
        // issued while an MMA runs waits for it.
        wait(&d1bar[G & 1], G, 2);
        tc_fence_after();
        float v[16], vb[16];
        tmem_ld16(trow + C::TM_D1 + (uint32_t)(G & 1) * 64 + 16 * half, v);
        if constexpr (C::SPLIT_K) tmem_ld16(trow + C::TM_D1 + (uint32_t)(G & 1) * 64 + 32 + 16 * half, vb);
        tmem_wait_ld();
        if (s + 1 < nsteps) {
          // vi of the next step of this task: the loader's stage G + 1
          wait(&full[(G + 1) % NS], G + 1, NS);
          convert_vi(G + 1, rowv && c + 1 >= 0 && c + 1 < nzr);
          fence_async_smem();
          tc_fence_before();
          arrive_a1();
        }
        const int k1 = k1s[(G & 1) * 256 + row], k1b = k1s[(G & 1) * 256 + 128 + row];

        const int iz = iz0 + dz * c;
        const float cxy = f_pow2(-1 - ((sp_xy + 7 * (iz - dz)) & 3));
        const float cxz = f_pow2(-2 - ((sp_xy - 3 * dy + 7 * iz) & 3));
        const float sx_r = f_pow2(-((sp_xy - dx + 7 * iz) & 3));
        const float ccp = f_pow2((sp_xy + 7 * iz) & 3);  // exact scalings of so_hi / so_lo
        const float cch = __fmul_rn(so_hi, ccp), ccl = __fmul_rn(so_lo, ccp);
        // vs = D1a * 2^-(k1 + kb1) [+ D1b * 2^-(k1b + kb1)], each term in two
        // exact steps, the smaller factor first, so no intermediate leaves the
        // FP32 range unless the term itself does
        const float vsc1 = f_pow2(min(-k1, -kb1)), vsc2 = f_pow2(max(-k1, -kb1));
        const float vbs1 = f_pow2(min(-k1b, -kb1)), vbs2 = f_pow2(max(-k1b, -kb1));
        const int prev = (int)((G - 1) & 1), cur = (int)(G & 1);
        float* out_slot = slots + ((size_t)((cur * TY + b) * 2 + half) * 32 + lane) * 16;
        float* gout_yz = x_out ? P.fyz + ((ent_z + iz) * P.ny + iy) * (size_t)EF + j * 32 : nullptr;
        float* gout_xz = y_out ? P.fxz + ((ent_z + iz) * P.nx + ix) * (size_t)EF + j * 32 : nullptr;
        float* gout_xy = (c == nzr - 1 && z_out) ? P.fxy + ((ent_y + iy) * P.nx + ix) * (size_t)EF + j * 32 : nullptr;

        // ---- incoming faces (16 angles each)
        float fyz[16], fxz[16], fxy[16];
        // a slot row holds one lane's 16 angles of this half, chunk q at q ^ sw
        auto load_slot = [&](const float* e, float (&f)[16]) {
#pragma unroll
          for (int q4 = 0; q4 < 4; ++q4) {
            const float4 t4 = *reinterpret_cast<const float4*>(e + 4 * (q4 ^ sw));
            f[4 * q4] = t4.x; f[4 * q4 + 1] = t4.y; f[4 * q4 + 2] = t4.z; f[4 * q4 + 3] = t4.w;
          }
        };
        if (act) {
          // an entry row holds 32 angles in float4 chunks, chunk q at q ^ j
          auto load_entry = [&](const float* e, float (&f)[16]) {
#pragma unroll
            for (int q4 = 0; q4 < 4; ++q4) {
              const float4 t4 = *reinterpret_cast<const float4*>(e + 4 * ((4 * half + q4) ^ j));
              f[4 * q4] = t4.x; f[4 * q4 + 1] = t4.y; f[4 * q4 + 2] = t4.z; f[4 * q4 + 3] = t4.w;
            }
          };
          auto boundary = [&](float sg, float (&f)[16]) {
#pragma unroll
            for (int i = 0; i < 16; ++i) {
              const int ia = ia0 + i, iag = P.ia_base + ia;
              f[i] = ia < P.na ? (float)((1 + iag) << (iag & 7)) * sg * face_k : 0.0f;
            }
          };
          if (a > 0) {
            // cell (a-1, b) wrote its output of this plane last step: lane - 8
            load_slot(slots + ((size_t)((prev * TY + b) * 2 + half) * 32 + lane - 8) * 16, fyz);
          } else if (x_in) {
            load_entry(reinterpret_cast<const float*>(stg + C::ST_YZ + b * EB) + j * 32, fyz);
          } else {
            boundary((float)d_scale_space(gx, iy, iz), fyz);
          }
          if (b > 0) {
            load_slot(slots + ((size_t)((prev * TY + (b - 1)) * 2 + half) * 32 + lane) * 16, fxz);
          } else if (y_in) {
            load_entry(reinterpret_cast<const float*>(stg + C::ST_XZ + a * EB) + j * 32, fxz);
          } else {
            boundary((float)d_scale_space(ix, gy, iz), fxz);
          }
          if (c > 0) {
#pragma unroll
            for (int i = 0; i < 16; ++i) fxy[i] = carry[i];
          } else if (z_in) {
            load_entry(reinterpret_cast<const float*>(stg + C::ST_XY + b * EB) + j * 32, fxy);
          } else {
            boundary((float)d_scale_space(ix, iy, gz), fxy);
          }
        }
        // ---- Quantities_solve in FP32 (fused multiply-adds: fewer roundings)
        float pmax = 0.0f;
        if (act) {
#pragma unroll
          for (int i = 0; i < 16; ++i) {
            const int iag = P.ia_base + ia0 + i;
            const float wz = 0.25f - 1.0f / (float)(1 << (iag & 7));
            const float sab = __fmaf_rn(fxy[i], cxy, __fmul_rn(fxz[i], cxz));
            const float sm = __fmaf_rn(fyz[i], __fmul_rn(wz, sx_r), sab);
            float vs = __fmul_rn(__fmul_rn(v[i], vsc1), vsc2);
            if constexpr (C::SPLIT_K) vs = __fmaf_rn(__fmul_rn(vb[i], vbs1), vbs2, vs);
            // psi = sm * cc + vs rounded once to FP32, with cc the FP64
            // reciprocal of (1 + octant) as cch + ccl: the product's
            // rounding error (fma), the sum's (TwoSum) and the low part
            // are added back before the final rounding.  (With the FP32
            // reciprocal and a rounded product, the cancellation of the
            // large boundary fluxes in T2 amplified that rounding up to
            // 1e-4 relative in vo at na 64-128.)  FP32 operations only; the
            // same sum formed in FP64 and rounded took 1 % more time.
            const float pp = __fmul_rn(sm, cch);
            const float pl = __fmaf_rn(sm, ccl, __fmaf_rn(sm, cch, -pp));
            const float s2 = __fadd_rn(pp, vs);
            const float bb = __fsub_rn(s2, pp);
            const float er = __fadd_rn(__fsub_rn(pp, __fsub_rn(s2, bb)), __fsub_rn(vs, bb));
            const float psi = __fadd_rn(s2, __fadd_rn(er, pl));
            v[i] = psi;
            pmax = fmaxf(pmax, fabsf(psi));
            carry[i] = __fmul_rn(psi, so);
          }
        }
        // ---- psi (this half's 16 angles) -> scaled hi/lo, K-chunks 2*half,
        // 2*half+1 of A2 buffer G % 2, last read by T2(G - 2), whose completion
        // this thread saw before the vo update of step G - 2 (one step ago)
        unsigned char* const a2b = a2s + (size_t)(G & 1) * 2 * C::A2M;
        int k2 = 0;
        if (act) {
          k2 = split_scale_f(pmax);
          const float sc = f_pow2(k2);
#pragma unroll
          for (int kc = 0; kc < 2; ++kc) {
            uint32_t hi[4], lo[4];
#pragma unroll
            for (int p = 0; p < 4; ++p) {
              const float x0 = __fmul_rn(v[8 * kc + 2 * p], sc), x1 = __fmul_rn(v[8 * kc + 2 * p + 1], sc);
              hi[p] = H::pack(x0, x1);
              const float2 hv = H::unpack(hi[p]);
              lo[p] = H::pack(__fsub_rn(x0, hv.x), __fsub_rn(x1, hv.y));
            }
            const int off = kmajor_off(row, 16 * half + 8 * kc, 128, 512);
            *reinterpret_cast<uint4*>(a2b + off) = make_uint4(hi[0], hi[1], hi[2], hi[3]);
            *reinterpret_cast<uint4*>(a2b + C::A2M + off) = make_uint4(lo[0], lo[1], lo[2], lo[3]);
          }
        }
        k2s[(G & 1) * 256 + half * 128 + row] = k2;
        fence_async_smem();  // A2 rows before the MMA warp's T2 (issued after the step barrier)
        // ---- outgoing faces: the slot (next step's neighbours) and the tile's edges
        if (act) {
#pragma unroll
          for (int q4 = 0; q4 < 4; ++q4) {
            const float4 o4 = make_float4(carry[4 * q4], carry[4 * q4 + 1], carry[4 * q4 + 2], carry[4 * q4 + 3]);
            const int pos = 4 * ((4 * half + q4) ^ j);
            *reinterpret_cast<float4*>(out_slot + 4 * (q4 ^ sw)) = o4;
            if (gout_yz) __stcg(reinterpret_cast<float4*>(gout_yz + pos), o4);
            if (gout_xz) __stcg(reinterpret_cast<float4*>(gout_xz + pos), o4);
            if (gout_xy) __stcg(reinterpret_cast<float4*>(gout_xy + pos), o4);
          }
        }
        // ---- vo of the previous step (its products had this step to finish)
        if (has_pend) {
          wait(&d2bar[pend.gg & 1], pend.gg, 2);
          epilogue(pend);
        }
        pend = Pend{G, act ? part_oct + (size_t)((long long)row0 + zstep * c) : nullptr, k2, act};
        has_pend = true;
        // ---- step barrier: A2 rows, slots and row scales of step G complete
        tc_fence_before();
        bar_step();
        if (s_abort) { stop = true; break; }
        if (s == nsteps - 1) {
          // flush: the task's last vo before the task is reported complete
          wait(&d2bar[G & 1], G, 2);
          epilogue(pend);
          tc_fence_before();
          bar_step();
          if (s_abort) { stop = true; break; }
          has_pend = false;
        }
      }
      if (stop) break;
    }
  }

  // the issuer's final commit has completed: release the tensor memory
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  if (warp == NW + 2)
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(C::TM_COLS) : "memory");
}

// vi -> vi16, once per sweep, for the group pairs [gp0, gp1): thread t
// converts moment chunk `half` (moments 8 half .. 8 half + 7, zero padded) of
// row r8 = 4 g + u of the (t / 16)-th block of that range (cell (ix, iy, iz),
// group pair gp; group 2 gp + g, unknown u).  The chunk
// is scaled by 2^k1 so that its largest entry lies in [2^14, 2^15) (k1
// clamped to [-120, 120]), rounded to FP32 in FP64 and split into hi + lo
// 16-bit halves -- the operand every octant's first transform of that cell
// uses.  A group beyond ne (odd ne) and the chunks beyond NM are zeros.
template <int NM_, int FMT>
__global__ void __launch_bounds__(256) convert_vi16(const double* __restrict__ vi, unsigned char* __restrict__ out,
                                                    int nx, int ny, int nz, int ne, int ngp, int gp0, int gp1) {
  using H = Half16<FMT>;
  constexpr int NMC = NM_ < 8 ? NM_ : 8;  // moments of a chunk
  const int ngr = gp1 - gp0;  // the group pairs converted: [gp0, gp1)
  const long long nunit = (long long)nx * ny * nz * ngr * 16;
  for (long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x; t < nunit;
       t += (long long)gridDim.x * blockDim.x) {
    const int r8 = (int)(t & 7), half = (int)((t >> 3) & 1);
    long long q = t >> 4;
    const int ix = (int)(q % nx);
    q /= nx;
    const int iy = (int)(q % ny);
    q /= ny;
    const int gp = gp0 + (int)(q % ngr), iz = (int)(q / ngr);
    const long long blk = (((long long)iz * ngp + gp) * ny + iy) * nx + ix;
    const int g = r8 >> 2, u = r8 & 3, ie = 2 * gp + g;
    int k1 = 0;
    uint32_t hi[4] = {0u, 0u, 0u, 0u}, lo[4] = {0u, 0u, 0u, 0u};
    if (ie < ne && 8 * half < NM_) {
      const double* src =
          vi + (size_t)NM_ * (u + (size_t)NU * (ix + (size_t)nx * (iy + (size_t)ny * (ie + (size_t)ne * iz)))) +
          8 * half;
      double v[NMC];
#pragma unroll
      for (int k = 0; k < NMC; ++k) v[k] = __ldcs(src + k);
      int emax = 0;  // largest biased exponent of the chunk
#pragma unroll
      for (int k = 0; k < NMC; ++k) emax = max(emax, (int)((__double_as_longlong(v[k]) >> 52) & 0x7ff));
      k1 = emax == 0 ? 0 : max(-120, min(120, 15 - (emax - 1022)));
      const double sc = d_pow2(k1);
#pragma unroll
      for (int p = 0; p < 4; ++p) {
        const float x0 = 2 * p < NMC ? __double2float_rn(v[2 * p < NMC ? 2 * p : 0] * sc) : 0.0f;
        const float x1 = 2 * p + 1 < NMC ? __double2float_rn(v[2 * p + 1 < NMC ? 2 * p + 1 : 0] * sc) : 0.0f;
        hi[p] = H::pack(x0, x1);
        const float2 hv = H::unpack(hi[p]);
        lo[p] = H::pack(__fsub_rn(x0, hv.x), __fsub_rn(x1, hv.y));
      }
    }
    unsigned char* b = out + (size_t)blk * kViBlock;
    const int o = half * 128 + r8 * 16;
    *reinterpret_cast<uint4*>(b + o) = make_uint4(hi[0], hi[1], hi[2], hi[3]);
    *reinterpret_cast<uint4*>(b + 256 + o) = make_uint4(lo[0], lo[1], lo[2], lo[3]);
    reinterpret_cast<signed char*>(b + 512)[half * 8 + r8] = (signed char)k1;
  }
}

// vo = sum over the eight octants of their FP32 partials, in FP64 and in
// octant order (deterministic); with `accumulate` the sum is added to vo (the
// angle passes after the first of a larger na).  The elements summed are
// iz * zstride + off + [0, width) for iz in [0, nz): one contiguous run of
// groups per z-plane (the whole state: zstride = width, off = 0).  width,
// zstride and off are multiples of 4 (NM * NU elements per (cell, group)).
__global__ void __launch_bounds__(256) reduce_octant_partials(double* __restrict__ vo,
                                                              const float* __restrict__ part, size_t state,
                                                              int accumulate, size_t zstride, size_t off,
                                                              size_t width, int nz) {
  const size_t w4 = width / 4, n4 = w4 * (size_t)nz;
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n4; i += (size_t)gridDim.x * blockDim.x) {
    size_t e4 = off / 4 + i;  // in units of 4 elements; one run when the groups are all of them
    if (zstride != width) {
      const size_t iz = i / w4;
      e4 = (iz * zstride + off) / 4 + (i - iz * w4);
    }
    double a0 = 0.0, a1 = 0.0, a2 = 0.0, a3 = 0.0;
    if (accumulate) {
      const double2* d = reinterpret_cast<const double2*>(vo) + 2 * e4;
      const double2 p0 = __ldcs(d), p1 = __ldcs(d + 1);
      a0 = p0.x;
      a1 = p0.y;
      a2 = p1.x;
      a3 = p1.y;
    }
#pragma unroll
    for (int o = 0; o < NOCTANT; ++o) {
      const float4 q = __ldcs(reinterpret_cast<const float4*>(part + state * o) + e4);
      a0 = __dadd_rn(a0, (double)q.x);
      a1 = __dadd_rn(a1, (double)q.y);
      a2 = __dadd_rn(a2, (double)q.z);
      a3 = __dadd_rn(a3, (double)q.w);
    }
    double2* d = reinterpret_cast<double2*>(vo) + 2 * e4;
    __stcs(d, make_double2(a0, a1));
    __stcs(d + 1, make_double2(a2, a3));
  }
}

}  // namespace msb
