// noalloc.cu -- one FP64 sweep that allocates nothing.
//
// Some callers cannot allocate device memory at the time they sweep: code that
// runs inside a memory pool or arena that owns every device byte, callers that
// must not synchronise the device (cudaMalloc/cudaFree can), and embedding
// hosts whose allocator forbids foreign allocations.  msb_sweep_noalloc gives
// them the plain-FP64 sweep with every scratch buffer the kernel needs -- the
// task table, the progress counters and the face planes -- carved out of one
// file-scope device array of a fixed size, and with the schedule built on the
// host into file-scope static arrays (no heap).
//
// Properties a caller must know:
//   * The scratch array (MSB_NOALLOC_SCRATCH_BYTES, 32 MiB) is part of the
//     library image: every GPU that loads the library holds it until exit.
//     Under CUDA's default lazy module loading the array is committed on a
//     device when this file's module is first used there, i.e. by the first
//     call on that device (at load time with CUDA_MODULE_LOADING=EAGER), so a
//     caller whose pool takes every free byte makes one call first.
//   * Problems whose scratch does not fit are rejected with MSB_ERR_ARG and a
//     message giving the bytes needed.  Supported: NM 4 or 16, na <= 32.
//   * The first call on each device does the set-up: it takes the device
//     address of the scratch array (cudaGetSymbolAddress, with that device
//     current), sets the kernel's shared-memory limit and reads the SM count.
//   * Every call shares the scratch array and the host-side schedule buffers,
//     and the array keeps the last call's contents.  The progress counters are
//     cleared at every call; the face planes need no clearing (every entry is
//     written before it is read).  Calls that overlap -- on the GPU (different
//     streams) or on the host (different threads) -- race: serialise them.
//   * The call returns after the sweep has finished (it reads the kernel's
//     status word back and synchronises the stream), so its result is ready
//     in vo_d.  That read-back cannot be captured in a CUDA graph: a call on
//     a stream that is capturing is refused with MSB_ERR_UNSUPPORTED before
//     anything is enqueued.
#include <cuda_runtime.h>

#include <algorithm>
#include <cstdint>

#include "internal.h"
#include "sweep_fp64_ws.cuh"

namespace msb {
namespace {

constexpr size_t kScratchBytes = MSB_NOALLOC_SCRATCH_BYTES;
constexpr int kTx = 4, kTy = 2;           // the tile of the NCH = 1 kernel variant
constexpr int kMaxTasks = 16384;          // host schedule capacity
constexpr int kMaxIndex = 4 * kMaxTasks;  // dense (phase, octant, group pair, tile) index
constexpr int kMaxDevices = 64;

// The scratch: task table, progress counters and face planes of one sweep.
static __device__ __align__(256) unsigned char g_scratch[kScratchBytes];

// Host-side schedule buffers (static: no heap).
int g_rec[kMaxTasks * MSB_TASK_INTS];
int g_idx[kMaxIndex];

struct DeviceState {
  bool ready = false;
  unsigned char* scratch = nullptr;  // device address of g_scratch on this device
  int nsm = 0;
  int occ[2] = {0, 0};  // blocks per SM of the NM 4 / NM 16 kernels
  // problem whose task table is in the scratch
  int key[5] = {-1, -1, -1, -1, -1};
};
DeviceState g_dev[kMaxDevices];
int g_status[4];

using Kernel = void (*)(const Fp64Params);
template <int NM_>
Kernel kernel_for() {
  return sweep_fp64_kernel<NM_, 1, kTx, kTy, 4, false>;
}
template <int NM_>
size_t smem_for() {
  return Fp64Cfg<NM_, 1, kTx, kTy, 4>::smem_bytes();
}

inline int ceil_div(int a, int b) { return (a + b - 1) / b; }
inline size_t align256(size_t x) { return (x + 255) & ~(size_t)255; }
struct Range {
  int lo, hi;
  bool empty() const { return hi <= lo; }
};
inline Range half(int n, int bit) {
  const int h = (n + 1) / 2;
  return bit ? Range{h, n} : Range{0, h};
}

// The schedule of build_schedule (schedule.cpp) with one group pair per
// block, generated directly in its launch order (phase, group pair, level,
// octant, tile row, tile column) into the static buffers.  Returns the task
// count, or -1 when it does not fit.
long long build_static_schedule(int nx, int ny, int nz, int ngp) {
  int ntxm = 0, ntym = 0;
  for (int reg = 0; reg < NOCTANT; ++reg) {
    ntxm = std::max(ntxm, ceil_div(half(nx, reg & 1).hi - half(nx, reg & 1).lo, kTx));
    ntym = std::max(ntym, ceil_div(half(ny, (reg >> 1) & 1).hi - half(ny, (reg >> 1) & 1).lo, kTy));
  }
  if ((long long)NOCTANT * NOCTANT * ngp * ntxm * ntym > kMaxIndex) return -1;
  auto dense = [&](int p, int o, int gp, int itx, int ity) {
    return (((p * NOCTANT + o) * ngp + gp) * ntxm + itx) * ntym + ity;
  };
  std::fill(g_idx, g_idx + (size_t)NOCTANT * NOCTANT * ngp * ntxm * ntym, -1);

  long long n = 0;
  for (int p = 0; p < NOCTANT; ++p)
    for (int gp = 0; gp < ngp; ++gp)
      for (int level = 0; level < ntxm + ntym - 1; ++level)
        for (int o = 0; o < NOCTANT; ++o) {
          const int reg = o ^ p;
          const Range rx = half(nx, reg & 1), ry = half(ny, (reg >> 1) & 1), rz = half(nz, (reg >> 2) & 1);
          if (rx.empty() || ry.empty() || rz.empty()) continue;
          const int dx = (o & 1) ? -1 : 1, dy = (o & 2) ? -1 : 1;
          const int ntx = ceil_div(rx.hi - rx.lo, kTx), nty = ceil_div(ry.hi - ry.lo, kTy);
          for (int ity = 0; ity < nty; ++ity)
            for (int itx = 0; itx < ntx; ++itx) {
              const int ax = dx > 0 ? itx : ntx - 1 - itx;
              const int ay = dy > 0 ? ity : nty - 1 - ity;
              if (ax + ay != level) continue;
              if (n >= kMaxTasks) return -1;
              int* r = &g_rec[n * MSB_TASK_INTS];
              std::fill(r, r + MSB_TASK_INTS, -1);
              r[TK_OCT] = o;
              r[TK_PHASE] = p;
              r[TK_GP] = gp;
              r[TK_X0] = rx.lo + itx * kTx;
              r[TK_X1] = std::min(rx.hi, rx.lo + (itx + 1) * kTx);
              r[TK_Y0] = ry.lo + ity * kTy;
              r[TK_Y1] = std::min(ry.hi, ry.lo + (ity + 1) * kTy);
              r[TK_Z0] = rz.lo;
              r[TK_Z1] = rz.hi;
              r[TK_LEVEL] = level;
              g_idx[dense(p, o, gp, itx, ity)] = (int)n;
              ++n;
            }
        }
  // dependencies (the rules of build_schedule; every one points to an
  // earlier task, found through the dense index)
  for (long long i = 0; i < n; ++i) {
    int* r = &g_rec[i * MSB_TASK_INTS];
    const int o = r[TK_OCT], p = r[TK_PHASE], gp = r[TK_GP];
    const int reg = o ^ p;
    const int dx = (o & 1) ? -1 : 1, dy = (o & 2) ? -1 : 1;
    const Range rx = half(nx, reg & 1), ry = half(ny, (reg >> 1) & 1);
    const int ntx = ceil_div(rx.hi - rx.lo, kTx), nty = ceil_div(ry.hi - ry.lo, kTy);
    const int itx = (r[TK_X0] - rx.lo) / kTx, ity = (r[TK_Y0] - ry.lo) / kTy;
    int flags = 0, mode = 0;
    {
      const bool first_in = dx > 0 ? itx == 0 : itx == ntx - 1;
      const bool last_in = dx > 0 ? itx == ntx - 1 : itx == 0;
      if (!first_in) {
        r[TK_DEP_X] = g_idx[dense(p, o, gp, itx - dx, ity)];
        mode |= DM_X_PLANE;
      } else if (p & 1) {
        const Range px = half(nx, (reg ^ 1) & 1);
        const int pntx = ceil_div(px.hi - px.lo, kTx);
        if (!px.empty()) r[TK_DEP_X] = g_idx[dense(p ^ 1, o, gp, dx > 0 ? pntx - 1 : 0, ity)];
      }
      if (r[TK_DEP_X] >= 0) flags |= TF_X_IN;
      if (!last_in || (!(p & 1) && !half(nx, (reg ^ 1) & 1).empty())) flags |= TF_X_OUT;
    }
    {
      const bool first_in = dy > 0 ? ity == 0 : ity == nty - 1;
      const bool last_in = dy > 0 ? ity == nty - 1 : ity == 0;
      if (!first_in) {
        r[TK_DEP_Y] = g_idx[dense(p, o, gp, itx, ity - dy)];
        mode |= DM_Y_PLANE;
      } else if (p & 2) {
        const Range py = half(ny, ((reg ^ 2) >> 1) & 1);
        const int pnty = ceil_div(py.hi - py.lo, kTy);
        if (!py.empty()) r[TK_DEP_Y] = g_idx[dense(p ^ 2, o, gp, itx, dy > 0 ? pnty - 1 : 0)];
      }
      if (r[TK_DEP_Y] >= 0) flags |= TF_Y_IN;
      if (!last_in || (!(p & 2) && !half(ny, ((reg ^ 2) >> 1) & 1).empty())) flags |= TF_Y_OUT;
    }
    if (p & 4) {
      if (!half(nz, ((reg ^ 4) >> 2) & 1).empty()) r[TK_DEP_Z] = g_idx[dense(p ^ 4, o, gp, itx, ity)];
      if (r[TK_DEP_Z] >= 0) flags |= TF_Z_IN;
    } else if (!half(nz, ((reg ^ 4) >> 2) & 1).empty()) {
      flags |= TF_Z_OUT;
    }
    if (p == 0) flags |= TF_FIRST;
    else r[TK_DEP_VO] = g_idx[dense(p - 1, reg ^ (p - 1), gp, itx, ity)];
    r[TK_FLAGS] = flags;
    r[TK_DEP_MODE] = mode;
    for (int d = TK_DEP_X; d <= TK_DEP_VO; ++d)
      if (r[d] >= i) return -1;  // not topological: cannot happen by construction
  }
  return n;
}

int setup_device(int dev, DeviceState& D) {
  int rc;
  void* p = nullptr;
  if ((rc = cuda_check(cudaGetSymbolAddress(&p, g_scratch), "cudaGetSymbolAddress(scratch)"))) return rc;
  D.scratch = static_cast<unsigned char*>(p);
  if ((rc = cuda_check(cudaDeviceGetAttribute(&D.nsm, cudaDevAttrMultiProcessorCount, dev), "SM count"))) return rc;
  const Kernel k[2] = {kernel_for<4>(), kernel_for<16>()};
  const size_t sm[2] = {smem_for<4>(), smem_for<16>()};
  for (int i = 0; i < 2; ++i) {
    if ((rc = cuda_check(cudaFuncSetAttribute(k[i], cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm[i]),
                         "cudaFuncSetAttribute")))
      return rc;
    if ((rc = cuda_check(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&D.occ[i], k[i],
                                                                       Fp64Cfg<16, 1, kTx, kTy, 4>::NT, sm[i]),
                         "occupancy")))
      return rc;
    if (D.occ[i] < 1) return set_error(MSB_ERR_UNSUPPORTED, "sweep kernel does not fit on an SM");
  }
  D.ready = true;
  return MSB_OK;
}

}  // namespace
}  // namespace msb

extern "C" int msb_sweep_noalloc(double* vo_d, const double* vi_d, const double* a_from_m_d,
                                 const double* m_from_a_d, int ncell_x, int ncell_y, int ncell_z, int ne, int nm,
                                 int na, void* stream) {
  using namespace msb;
  if (!vo_d || !vi_d || !a_from_m_d || !m_from_a_d) return set_error(MSB_ERR_ARG, "noalloc sweep: null pointer");
  if (ncell_x <= 0 || ncell_y <= 0 || ncell_z <= 0 || ne <= 0 || na <= 0)
    return set_error(MSB_ERR_ARG, "noalloc sweep: invalid dimensions");
  if (!(nm == 4 || nm == 16) || na > 32)
    return set_error(MSB_ERR_UNSUPPORTED, "noalloc sweep: supports NM 4 or 16 and na <= 32 (got NM %d, na %d)",
                     nm, na);
  int dev = 0, rc;
  cudaStreamCaptureStatus cap = cudaStreamCaptureStatusNone;
  if ((rc = cuda_check(cudaStreamIsCapturing(static_cast<cudaStream_t>(stream), &cap), "cudaStreamIsCapturing")))
    return rc;
  if (cap != cudaStreamCaptureStatusNone)
    return set_error(MSB_ERR_UNSUPPORTED, "noalloc sweep: the stream is capturing; this call synchronises and "
                                          "cannot be captured");
  if ((rc = cuda_check(cudaGetDevice(&dev), "cudaGetDevice"))) return rc;
  if (dev < 0 || dev >= kMaxDevices) return set_error(MSB_ERR_UNSUPPORTED, "noalloc sweep: device index %d", dev);
  DeviceState& D = g_dev[dev];
  if (!D.ready && (rc = setup_device(dev, D))) return rc;

  // scratch layout: sync words + progress | task table | face planes xy, xz, yz
  const int ngp = (ne + 1) / 2;
  const int key[4] = {ncell_x, ncell_y, ncell_z, ngp};
  const bool same = std::equal(key, key + 4, D.key);
  long long ntask = 0;
  if (!same) {
    ntask = build_static_schedule(ncell_x, ncell_y, ncell_z, ngp);
    if (ntask < 0)
      return set_error(MSB_ERR_ARG, "noalloc sweep: %dx%dx%d cells x %d group pairs exceed the %d-task schedule",
                       ncell_x, ncell_y, ncell_z, ngp, kMaxTasks);
  } else {
    ntask = D.key[4];
  }
  const size_t ent = 256;  // doubles per face entry (32 angles)
  const size_t per = (size_t)NOCTANT * ngp * ent * sizeof(double);
  const size_t sync_b = align256(sizeof(int) * (SY_PROGRESS + (size_t)ntask));
  const size_t task_b = align256(sizeof(int) * MSB_TASK_INTS * (size_t)ntask);
  const size_t fxy_b = align256(per * ncell_y * ncell_x);
  const size_t fxz_b = align256(per * ncell_z * ncell_x);
  const size_t fyz_b = align256(per * ncell_z * ncell_y);
  const size_t need = sync_b + task_b + fxy_b + fxz_b + fyz_b;
  if (need > kScratchBytes)
    return set_error(MSB_ERR_ARG, "noalloc sweep: needs %zu bytes of scratch, the fixed array holds %zu (%dx%dx%d, ne %d)",
                     need, kScratchBytes, ncell_x, ncell_y, ncell_z, ne);
  unsigned char* base = D.scratch;
  int* sync = reinterpret_cast<int*>(base);
  int* tasks = reinterpret_cast<int*>(base + sync_b);
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  if (!same) {
    // the previous call's kernel may still read the table: order on the stream
    if ((rc = cuda_check(cudaMemcpyAsync(tasks, g_rec, sizeof(int) * MSB_TASK_INTS * (size_t)ntask,
                                         cudaMemcpyHostToDevice, st),
                         "copy schedule")))
      return rc;
    if ((rc = cuda_check(cudaStreamSynchronize(st), "copy schedule"))) return rc;
    std::copy(key, key + 4, D.key);
    D.key[4] = (int)ntask;
  }
  if ((rc = cuda_check(cudaMemsetAsync(sync, 0, sync_b, st), "clear progress"))) return rc;

  Fp64Params P{};
  P.pr.vi = vi_d;
  P.pr.vo = vo_d;
  P.pr.afm = a_from_m_d;
  P.pr.mfa = m_from_a_d;
  P.pr.fxy = reinterpret_cast<double*>(base + sync_b + task_b);
  P.pr.fxz = reinterpret_cast<double*>(base + sync_b + task_b + fxy_b);
  P.pr.fyz = reinterpret_cast<double*>(base + sync_b + task_b + fxy_b + fxz_b);
  P.tasks = tasks;
  P.ntask = ntask;
  P.pr.nx = ncell_x;
  P.pr.ny = ncell_y;
  P.pr.nz = ncell_z;
  P.pr.ne = ne;
  P.pr.na = na;
  P.pr.ngp = ngp;
  P.pr.ia_base = 0;
  P.pr.vo_add = 0;
  P.pr.ie_base = 0;
  P.sy.sync = sync;
  P.sy.timeout_ns = kDefaultTimeoutNs;
  const int v = nm == 16 ? 1 : 0;
  const int grid = (int)std::min<long long>(ntask, (long long)D.nsm * D.occ[v]);
  const Kernel k = v ? kernel_for<16>() : kernel_for<4>();
  const size_t smem = v ? smem_for<16>() : smem_for<4>();
  k<<<grid, Fp64Cfg<16, 1, kTx, kTy, 4>::NT, smem, st>>>(P);
  if ((rc = cuda_check(cudaGetLastError(), "noalloc sweep launch"))) return rc;
  if ((rc = cuda_check(cudaMemcpyAsync(g_status, sync, sizeof g_status, cudaMemcpyDeviceToHost, st), "status")))
    return rc;
  if ((rc = cuda_check(cudaStreamSynchronize(st), "noalloc sweep"))) return rc;
  if (g_status[SY_ERROR] == MSB_ERR_TIMEOUT)
    return set_error(MSB_ERR_TIMEOUT, "noalloc sweep: a device wait ran out of time (task %d)", g_status[SY_ERRTASK]);
  if (g_status[SY_ERROR]) return set_error(g_status[SY_ERROR], "noalloc sweep: device error %d", g_status[SY_ERROR]);
  return MSB_OK;
}
