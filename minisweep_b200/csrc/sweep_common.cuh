// sweep_common.cuh -- device helpers shared by the sweep kernels:
// inter-CTA synchronisation (bounded waits), the built-in problem's scale
// factors, and the task record.
#pragma once

#include <cstdint>

#include "internal.h"

namespace msb {

// Layout of the per-sweep synchronisation block in global memory.
enum SyncSlot {
  SY_COUNTER = 0,   // next task index to grab
  SY_ERROR = 1,     // first error code (0 = ok)
  SY_ABORT = 2,     // set when any CTA gives up; makes every wait return
  SY_ERRTASK = 3,   // task that reported the error
  SY_PROGRESS = 32  // per-task progress counters start here
};
// progress value meaning "task complete" (larger than any plane count)
constexpr int kComplete = 1 << 30;

struct SyncArgs {
  int* sync;
  long long timeout_ns;
};

__device__ __forceinline__ long long global_ns() {
  long long t;
  asm volatile("mov.u64 %0, %globaltimer;" : "=l"(t));
  return t;
}

__device__ __forceinline__ int ld_acquire(const int* p) {
  int v;
  asm volatile("ld.acquire.gpu.global.s32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
  return v;
}

__device__ __forceinline__ void st_release(int* p, int v) {
  asm volatile("st.release.gpu.global.s32 [%0], %1;" ::"l"(p), "r"(v) : "memory");
}

__device__ __forceinline__ int ld_relaxed(const int* p) {
  int v;
  asm volatile("ld.relaxed.gpu.global.s32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
  return v;
}

// Record an error (first one wins) and raise the abort flag.
__device__ __forceinline__ void raise_error(int* sync, int code, int task) {
  if (atomicCAS(&sync[SY_ERROR], 0, code) == 0) sync[SY_ERRTASK] = task;
  st_release(&sync[SY_ABORT], 1);
}

// Bounded wait, executed by one thread: returns true once *p >= target,
// false if the time budget ran out or another CTA aborted (then the error
// is already recorded).
static __device__ __noinline__ bool wait_geq(const SyncArgs& s, const int* p, int target, int task) {
  if (ld_acquire(p) >= target) return true;
  const long long t0 = global_ns();
  unsigned ns = 32;
  for (;;) {
    __nanosleep(ns);
    if (ns < 256) ns <<= 1;
    if (ld_acquire(p) >= target) return true;
    if (ld_relaxed(&s.sync[SY_ABORT]) != 0) return false;
    if (global_ns() - t0 > s.timeout_ns) {
      raise_error(s.sync, MSB_ERR_TIMEOUT, task);
      return false;
    }
  }
}

// ---- built-in problem (quantities_testing_kernels.h:52-214)
__device__ __forceinline__ int d_scale_space(int ix, int iy, int iz) {
  return 1 << ((ix + 3 * iy + 7 * iz + 2) & 3);
}
// log2 of the space scale factor, and 2^k / 2^-k built from exponent bits
// (exact; used instead of FP64 divisions by the power-of-two factors).
__device__ __forceinline__ int d_log2_space(int ix, int iy, int iz) { return (ix + 3 * iy + 7 * iz + 2) & 3; }
__device__ __forceinline__ double d_pow2(int k) { return __longlong_as_double((long long)(1023 + k) << 52); }
__device__ __forceinline__ int d_scale_energy(int ie) { return 1 << (((ie * 1366 + 150889) % 714025) & 3); }
__device__ __forceinline__ int d_scale_unknown(int iu) { return 1 << (((iu * 741 + 66037) % 312500) & 3); }

// Boundary flux one cell outside the grid (Quantities_init_facexy/xz/yz,
// quantities_testing_kernels.h:219-332; all three use the same formula with
// the ghost coordinate on the face axis).  Exact small integers in FP64.
__device__ __forceinline__ double d_init_face(int ia, int ix, int iy, int iz, int ie, int iu, int oct) {
  return (double)(1 + ia) * (double)(1 << (ia & 7)) * (double)d_scale_space(ix, iy, iz) *
         (double)d_scale_energy(ie) * (double)d_scale_unknown(iu) * (double)(1 + oct);
}

}  // namespace msb
