// sweeper.cu -- the Sweeper C API on one B200.
//
// Sweeper_create (sweeper_kba_c.h:44-287) consumes and validates the same
// flags as the reference, then builds the task schedule and the device
// buffers (face planes per octant, schedule, progress counters).
// Sweeper_sweep (sweeper_kba_c.h:588-845) is one persistent kernel launch.
#include <cuda.h>
#include <cudaTypedefs.h>
#include <cuda_runtime.h>

#include <algorithm>
#include <climits>
#include <cstdint>
#include <memory>
#include <new>
#include <type_traits>
#include <vector>

#include "internal.h"
#include "sweep_fp64_chain.cuh"
#include "sweep_fp64_ws.cuh"
#include "sweep_mixed_tc.cuh"

namespace msb {

namespace {

using KernelFn = void (*)(const Fp64Params);
using MixKernelFn = void (*)(const MixParams);
using MixConvFn = void (*)(const double*, unsigned char*, int, int, int, int, int, int, int);

// One compiled kernel: the FP64 kernel (fn) or a mixed-precision one (mix).
struct Variant {
  KernelFn fn = nullptr;
  MixKernelFn mix = nullptr;
  MixConvFn conv = nullptr;  // mixed precision: vi into the first transform's operand format
  size_t smem = 0;
  size_t entry_bytes = 0;  // one face entry (octant, group pair, position)
  int tx = 0, ty = 0, nch = 0, threads = 0;
  int pass = 64;  // angles swept per launch (na above it is swept in passes)
  int kernel = 0; // FP64: 0 staged, 1 chained wavefront
  bool valid() const { return fn || mix; }
  const void* func() const { return fn ? (const void*)fn : (const void*)mix; }
};

constexpr int kStages = 4;
#ifndef MSB_PIPE_T1
#define MSB_PIPE_T1 false
#endif
constexpr bool kPipeT1 = MSB_PIPE_T1;

template <int NM_, int NCH, int TX, int TY>
Variant make_variant() {
  using C = Fp64Cfg<NM_, NCH, TX, TY, kStages>;
  static_assert(C::smem_bytes() <= 227 * 1024, "shared memory budget");
  Variant v;
  v.fn = sweep_fp64_kernel<NM_, NCH, TX, TY, kStages, kPipeT1>;
  v.smem = C::smem_bytes();
  v.entry_bytes = (size_t)NCH * 256 * sizeof(double);
  v.tx = TX;
  v.ty = TY;
  v.nch = NCH;
  v.threads = C::NT;
  v.pass = 32 * NCH;
  return v;
}

// The chained-wavefront FP64 kernel (sweep_fp64_chain.cuh): one 32-angle
// chunk per pass.
template <int NM_, int TX, int TY>
Variant make_chain_variant() {
  using C = ChainCfg<NM_, TX, TY>;
  Variant v;
  v.fn = sweep_fp64_chain_kernel<NM_, TX, TY>;
  v.smem = C::smem_bytes();
  v.entry_bytes = (size_t)C::ENT * sizeof(double);
  v.tx = TX;
  v.ty = TY;
  v.nch = 1;
  v.threads = C::NT;
  v.pass = 32;
  v.kernel = 1;
  return v;
}

// FP64 tile shapes: 4 x 2 (tile 42, the default) or 2 x 4 (tile 24) cell
// columns, for one or two 32-angle chunks per pass (na > 64 is swept in
// passes of 64 angles).
template <int NM_>
Variant pick_nch(int nch, int tile) {
  const bool t24 = tile == 24;
  switch (nch) {
    case 1: return t24 ? make_variant<NM_, 1, 2, 4>() : make_variant<NM_, 1, 4, 2>();
    case 2: return t24 ? make_variant<NM_, 2, 2, 4>() : make_variant<NM_, 2, 4, 2>();
    default: return Variant();
  }
}

constexpr int kMixStages = 4;

template <int NM_, int FMT>
Variant make_mixed() {
  using C = MixCfg<NM_, kMixStages>;
  static_assert(C::smem_bytes() + 128 <= 227 * 1024, "shared memory budget (dynamic + static)");
  Variant v;
  v.mix = sweep_mixed_kernel<NM_, FMT, kMixStages>;
  v.conv = convert_vi16<NM_, FMT>;
  v.smem = C::smem_bytes();
  v.entry_bytes = C::EB;
  v.tx = C::TX;
  v.ty = C::TY;
  v.nch = 1;
  v.threads = C::NT;
  v.pass = 32;
  return v;
}

template <int FMT>
Variant pick_mixed(int nm) {
  switch (nm) {
    case 4: return make_mixed<4, FMT>();
    case 8: return make_mixed<8, FMT>();
    case 16: return make_mixed<16, FMT>();
    default: return Variant();
  }
}

template <int NM_>
Variant pick_chain(int tile) {
  return tile == 24 ? make_chain_variant<NM_, 2, 4>() : make_chain_variant<NM_, 4, 2>();
}

// precision 0: FP64; 1: mixed with FP16 halves; 2: mixed with BF16 halves.
// tile: 0 = the default shape, 42 or 24 (FP64 only).  kernel (FP64 only):
// 0 = the staged kernel, 32 or 64 angles per pass; 1 = the chained-wavefront
// kernel, 32 angles per pass.  angle_pass (staged kernel): 0 or 32 = 32
// angles per pass (the transform matrices stay in registers), 64 = two
// 32-angle chunks per pass (matrices read from shared memory; slower per
// angle).  na <= 128; the mixed kernels sweep 32 angles per pass.
Variant pick_variant(int nm, int na, int precision, int tile = 0, int kernel = 0, int angle_pass = 0) {
  if (na > 128) return Variant();
  if (precision == 1 || precision == 2) {
    if (tile != 0) return Variant();
    return precision == 1 ? pick_mixed<MIX_F16>(nm) : pick_mixed<MIX_BF16>(nm);
  }
  if (precision != 0) return Variant();
  if (kernel == 1) {
    switch (nm) {
      case 4: return pick_chain<4>(tile);
      case 8: return pick_chain<8>(tile);
      case 16: return pick_chain<16>(tile);
      default: return Variant();
    }
  }
  const int nch = angle_pass == 64 ? 2 : 1;
  switch (nm) {
    case 4: return pick_nch<4>(nch, tile);
    case 8: return pick_nch<8>(nch, tile);
    case 16: return pick_nch<16>(nch, tile);
    default: return Variant();
  }
}

}  // namespace

// One way to sweep an FP64 problem that --autotune 1 tries: a compiled kernel
// (tile shape), the schedule built for a task window, and the L2 policy.
struct AltPlan {
  Variant var;
  Schedule sched;
  int gp_block = 1;
  int* d_tasks = nullptr;
  int grid = 0;
  int window = 4;
  int l2_hints = 0;
  float ms = 0.f;  // its autotuning sweep
};

// A decomposed sweep (--nproc_x * --nproc_y > 1): this process's units, one
// slab schedule each, and the message buffers.  Unit k's tasks are
// d_tasks[off[k] .. off[k] + cnt[k]) with slab-local dependencies.
struct KbaState {
  KbaPlan plan;
  int proc = 0, px = 0, py = 0, nzb = 0, npass = 1, pa = 64;
  std::vector<long long> off, cnt;
  std::vector<int> grid;
  int* d_tasks = nullptr;
  long long ntask_max = 0;
  size_t plane_pass[3] = {0, 0, 0};  // bytes of one angle pass's plane: xy, xz, yz
  size_t slab_bytes[2] = {0, 0};     // one pass's face slab of a unit: x faces, y faces
  // message buffers: send x, send y, receive x from lower / higher, y lower / higher
  void* buf[6] = {nullptr, nullptr, nullptr, nullptr, nullptr, nullptr};
  void* own[6] = {nullptr, nullptr, nullptr, nullptr, nullptr, nullptr};
  double* vo_d = nullptr;
  const double* vi_d = nullptr;
  int rc = 0;  // first error of the sweep in progress (later steps still exchange)
  size_t msg_bytes(int axis) const { return (size_t)npass * slab_bytes[axis]; }
  ~KbaState() {
    cudaFree(d_tasks);
    for (void* p : own) cudaFree(p);
  }
};

// Task tables of a run split into slices of group pairs (see
// sweep_iterations_sliced): slice k holds the plan's tasks of group pairs
// [gp0[k], gp0[k + 1]) in the plan's order, dependencies renumbered.
struct SliceTables {
  const int* for_tasks = nullptr;  // the plan's table they were cut from
  std::vector<int> gp0;
  std::vector<int*> d_tasks;
  std::vector<long long> ntask;
  ~SliceTables() {
    for (int* p : d_tasks) cudaFree(p);
  }
};

struct SweeperImpl {
  Dimensions dims{};
  int precision = 0;
  int ngp = 0;
  int gp_block = 1;
  Variant var;
  Schedule sched;
  int grid = 0;
  int* d_tasks = nullptr;
  int* d_sync = nullptr;
  size_t sync_ints = 0;
  void* d_face[3] = {nullptr, nullptr, nullptr};  // xy, xz, yz
  size_t face_bytes[3] = {0, 0, 0};
  double* d_afm = nullptr;
  double* d_mfa = nullptr;
  float* d_part = nullptr;  // mixed precision: FP32 partial vo per octant
  unsigned char* d_vi16 = nullptr;  // mixed precision: vi in the first transform's operand format
  size_t part_elems = 0;
  double* d_afm_c = nullptr;  // na above one pass: the pass's angle range of each matrix
  double* d_mfa_c = nullptr;
  double* d_vi = nullptr;  // staging for host-only Pointers
  double* d_vo = nullptr;
  long long timeout_ns = kDefaultTimeoutNs;
  int nlaunch = 0;
  int nsm = 0;
  int* h_status = nullptr;  // pinned copy of the status words
  // --autotune 1: the first sweep runs with every candidate plan (tile shape
  // x task window x L2 policy) and keeps the fastest
  bool autotune = false;
  bool tuned = false;
  std::vector<AltPlan> alts;
  float tune_ms[2] = {0.f, 0.f};  // first sweep: the chosen plan, the fastest of the other tile shape
  int ie_base = 0;                // --ie_base: global index of this sweeper's group 0
  int window = 4;                 // --task_window: tasks between a tile and its downwind neighbour, x SMs
  int l2_hints = 0;               // --l2_hints: L2 eviction policies in the chained FP64 kernel
  int sp_off = 0;                 // (ix_base + 3 iy_base) & 3 of a decomposed process's subdomain
  std::unique_ptr<KbaState> kba;  // set: the sweep is decomposed over a process grid
  std::unique_ptr<SliceTables> slices;  // Sweeper_sweep_iterations in group-pair slices
  int run_slices = 0;                   // slices of the last host-buffer sweep call (1: whole)

  ~SweeperImpl() {
    cudaFree(d_tasks);
    for (auto& a : alts) cudaFree(a.d_tasks);
    cudaFree(d_sync);
    for (auto& f : d_face) cudaFree(f);
    cudaFree(d_afm);
    cudaFree(d_mfa);
    cudaFree(d_part);
    cudaFree(d_vi16);
    cudaFree(d_afm_c);
    cudaFree(d_mfa_c);
    cudaFree(d_vi);
    cudaFree(d_vo);
    if (h_status) cudaFreeHost(h_status);
  }
};

// Angles per pass: the FP64 kernels sweep up to 64 (two 32-angle chunks) at
// once, the mixed ones 32.  Angles are independent in the sweep (each has its
// own faces), so a larger na is swept in passes over consecutive angle
// ranges whose contributions add up in vo.
static int pass_angles(const SweeperImpl& S) { return S.var.pass; }

// Schedule, device task table and grid of one compiled tile shape, with a
// window of `window` x SMs consecutive tasks between a tile and its downwind
// neighbour in the table.
static int setup_plan(const SweeperImpl& S, const Variant& var, int window, Schedule& sched, int& gp_block,
                      int*& d_tasks, int& grid) {
  const Dimensions& dims = S.dims;
  int rc, occ = 0;
  gp_block = pick_gp_block(dims.ncell_x, dims.ncell_y, S.ngp, var.tx, var.ty, window * S.nsm);
  if ((rc = build_schedule(dims.ncell_x, dims.ncell_y, dims.ncell_z, S.ngp, var.tx, var.ty, gp_block, sched)))
    return rc;
  const long long ntask = sched.ntask();
  if (ntask >= (1LL << 31) - SY_PROGRESS) return set_error(MSB_ERR_ARG, "too many tasks");
  if ((rc = cuda_check(cudaMalloc(&d_tasks, sched.rec.size() * sizeof(int)), "cudaMalloc tasks"))) return rc;
  if ((rc = cuda_check(cudaMemcpy(d_tasks, sched.rec.data(), sched.rec.size() * sizeof(int), cudaMemcpyHostToDevice),
                       "copy tasks")))
    return rc;
  if ((rc = cuda_check(cudaFuncSetAttribute(var.func(), cudaFuncAttributeMaxDynamicSharedMemorySize, (int)var.smem),
                       "cudaFuncSetAttribute")))
    return rc;
  if ((rc = cuda_check(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, var.func(), var.threads, var.smem),
                       "occupancy")))
    return rc;
  if (occ < 1) return set_error(MSB_ERR_UNSUPPORTED, "sweep kernel does not fit on an SM");
  grid = (int)std::min<long long>(ntask, (long long)S.nsm * occ);
  return MSB_OK;
}

static int impl_create(SweeperImpl& S, const Dimensions& dims, int precision, int tile = 0, bool autotune = false,
                       int kernel = 0, int angle_pass = 0) {
  S.dims = dims;
  S.precision = precision;
  if (dims.ncell_x <= 0 || dims.ncell_y <= 0 || dims.ncell_z <= 0 || dims.ne <= 0 || dims.na <= 0)
    return set_error(MSB_ERR_ARG, "invalid dimensions");
  S.var = pick_variant(dims.nm, dims.na, precision, tile, kernel, angle_pass);
  if (!S.var.valid())
    return set_error(MSB_ERR_UNSUPPORTED,
                     "no kernel variant for nm=%d na=%d precision=%d tile=%d (nm in {4,8,16}; na <= 128; "
                     "--tile 42 / 24 only for the FP64 sweep)",
                     dims.nm, dims.na, precision, tile);
  if (autotune && precision != 0)
    return set_error(MSB_ERR_UNSUPPORTED, "--autotune 1 needs the FP64 sweep (the mixed sweep has one tile shape)");
  S.ngp = (dims.ne + 1) / 2;
  int rc, dev = 0, nsm = 0;
  if ((rc = cuda_check(cudaGetDevice(&dev), "cudaGetDevice"))) return rc;
  if ((rc = cuda_check(cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev), "SM count"))) return rc;
  S.nsm = nsm;
  if ((rc = setup_plan(S, S.var, S.window, S.sched, S.gp_block, S.d_tasks, S.grid))) return rc;
  long long ntask = S.sched.ntask();
  if (autotune) {
    // candidates: both FP64 kernels (the staged one with 32- and 64-angle
    // passes when na > 32) x both tile shapes x task windows of 4, 8 and 16
    // x SMs, besides the sweeper's own plan
    S.autotune = true;
    const int windows[3] = {4, 8, 16};
    for (int k = 0; k < 3; ++k)
      for (int t = 0; t < 2; ++t)
        for (int w : windows) {
          if (k == 2 && dims.na <= 32) continue;  // the staged kernel's passes differ only above 32 angles
          const int tile_c = t == 0 ? 42 : 24, kern = k == 2 ? 0 : k, pass_c = k == 2 ? 64 : 0;
          Variant v = pick_variant(dims.nm, dims.na, precision, tile_c, kern, pass_c);
          const bool is_main =
              v.kernel == S.var.kernel && v.pass == S.var.pass && v.tx == S.var.tx && w == S.window;
          if (is_main) continue;
          AltPlan a;
          a.var = v;
          a.window = w;
          a.l2_hints = S.l2_hints;
          if ((rc = setup_plan(S, a.var, a.window, a.sched, a.gp_block, a.d_tasks, a.grid))) {
            cudaFree(a.d_tasks);
            return rc;
          }
          ntask = std::max(ntask, a.sched.ntask());
          S.alts.push_back(std::move(a));
        }
  }
  // face entries and angle passes of every plan the sweeper may run
  size_t entry_bytes = S.var.entry_bytes;
  int pass_min = S.var.pass, pass_max = S.var.pass;
  for (const auto& a : S.alts) {
    entry_bytes = std::max(entry_bytes, a.var.entry_bytes);
    pass_min = std::min(pass_min, a.var.pass);
    pass_max = std::max(pass_max, a.var.pass);
  }
  S.sync_ints = SY_PROGRESS + (size_t)ntask;
  if ((rc = cuda_check(cudaMalloc(&S.d_sync, S.sync_ints * sizeof(int)), "cudaMalloc sync"))) return rc;
  if ((rc = cuda_check(cudaMallocHost(&S.h_status, 8 * sizeof(int)), "cudaMallocHost status"))) return rc;

  const size_t per = (size_t)NOCTANT * S.ngp * entry_bytes;
  S.face_bytes[0] = per * dims.ncell_y * dims.ncell_x;
  S.face_bytes[1] = per * dims.ncell_z * dims.ncell_x;
  S.face_bytes[2] = per * dims.ncell_z * dims.ncell_y;
  for (int f = 0; f < 3; ++f)
    if ((rc = cuda_check(cudaMalloc(&S.d_face[f], S.face_bytes[f]), "cudaMalloc faces"))) return rc;
  if (S.var.mix) {
    S.part_elems = (size_t)NOCTANT * Dimensions_size_state(dims, NU);
    if ((rc = cuda_check(cudaMalloc(&S.d_part, S.part_elems * sizeof(float)), "cudaMalloc octant partials")))
      return rc;
    const size_t nvi16 = (size_t)dims.ncell_x * dims.ncell_y * dims.ncell_z * S.ngp * kViBlock;
    if ((rc = cuda_check(cudaMalloc(&S.d_vi16, nvi16), "cudaMalloc converted vi"))) return rc;
  }
  const size_t nmat = (size_t)dims.nm * dims.na * NOCTANT;
  if ((rc = cuda_check(cudaMalloc(&S.d_afm, nmat * sizeof(double)), "cudaMalloc a_from_m"))) return rc;
  if ((rc = cuda_check(cudaMalloc(&S.d_mfa, nmat * sizeof(double)), "cudaMalloc m_from_a"))) return rc;
  if (dims.na > pass_min) {
    const size_t npass_mat = (size_t)dims.nm * pass_max * NOCTANT;
    if ((rc = cuda_check(cudaMalloc(&S.d_afm_c, npass_mat * sizeof(double)), "cudaMalloc a_from_m pass"))) return rc;
    if ((rc = cuda_check(cudaMalloc(&S.d_mfa_c, npass_mat * sizeof(double)), "cudaMalloc m_from_a pass"))) return rc;
  }
  return MSB_OK;
}

// The columns a0 .. a0 + nac of a_from_m[oct][im][ia] and the rows of
// m_from_a[oct][ia][im] into the pass buffers (layouts of an na = nac problem).
static int copy_pass_matrices(SweeperImpl& S, int a0, int nac, cudaStream_t stream, double* dst_a = nullptr,
                              double* dst_m = nullptr) {
  const int na = S.dims.na, nm = S.dims.nm;
  if (!dst_a) dst_a = S.d_afm_c;
  if (!dst_m) dst_m = S.d_mfa_c;
  int rc = cuda_check(cudaMemcpy2DAsync(dst_a, nac * sizeof(double), S.d_afm + a0, na * sizeof(double),
                                        nac * sizeof(double), (size_t)nm * NOCTANT, cudaMemcpyDeviceToDevice, stream),
                      "a_from_m pass");
  if (rc) return rc;
  return cuda_check(cudaMemcpy2DAsync(dst_m, (size_t)nac * nm * sizeof(double), S.d_mfa + (size_t)a0 * nm,
                                      (size_t)na * nm * sizeof(double), (size_t)nac * nm * sizeof(double), NOCTANT,
                                      cudaMemcpyDeviceToDevice, stream),
                    "m_from_a pass");
}

// Before a pass after the first: the task counter and the progress start
// over; an error (and the abort flag) of an earlier pass stays, so the later
// passes end at once and the host sees the first error.
static int reset_pass(SweeperImpl& S, cudaStream_t stream) {
  int rc = cuda_check(cudaMemsetAsync(S.d_sync + SY_COUNTER, 0, sizeof(int), stream), "reset sync");
  if (rc) return rc;
  return cuda_check(cudaMemsetAsync(S.d_sync + SY_PROGRESS, 0, (S.sync_ints - SY_PROGRESS) * sizeof(int), stream),
                    "reset sync");
}

// Problem fields (X) and schedule fields (P) of a launch; F is the face type.
template <class F, class X, class PP>
static void fill_params(const SweeperImpl& S, X& x, PP& P, const double* vi_d, const int* d_tasks, long long ntask) {
  if constexpr (std::is_same<X, Fp64Prob>::value) x.vi = vi_d;  // the mixed sweep reads vi16 instead
  else (void)vi_d;
  x.afm = S.d_afm;
  x.mfa = S.d_mfa;
  x.fxy = static_cast<F*>(S.d_face[0]);
  x.fxz = static_cast<F*>(S.d_face[1]);
  x.fyz = static_cast<F*>(S.d_face[2]);
  x.nx = S.dims.ncell_x;
  x.ny = S.dims.ncell_y;
  x.nz = S.dims.ncell_z;
  x.ne = S.dims.ne;
  x.na = S.dims.na;
  x.ngp = S.ngp;
  x.ia_base = 0;
  x.ie_base = S.ie_base;
  if constexpr (std::is_same<X, Fp64Prob>::value) {
    x.l2_hints = S.l2_hints;
    x.sp_off = S.sp_off;
  }
  P.tasks = d_tasks;
  P.ntask = ntask;
  P.sy.sync = S.d_sync;
  P.sy.timeout_ns = S.timeout_ns;
}

// Every pass of one FP64 sweep with the given compiled tile shape.
static int launch_fp64(SweeperImpl& S, const Variant& var, const int* d_tasks, long long ntask, int grid,
                       double* vo_d, const double* vi_d, cudaStream_t stream) {
  const int na = S.dims.na, pa = pass_angles(S), npass = (na + pa - 1) / pa;
  int rc;
  for (int c = 0; c < npass; ++c) {
    Fp64Params P{};
    fill_params<double>(S, P.pr, P, vi_d, d_tasks, ntask);
    P.pr.vo = vo_d;
    P.pr.vo_add = c > 0 ? 1 : 0;  // later passes add to vo in every phase
    if (npass > 1) {
      const int a0 = pa * c, nac = std::min(pa, na - a0);
      if ((rc = copy_pass_matrices(S, a0, nac, stream))) return rc;
      if (c > 0 && (rc = reset_pass(S, stream))) return rc;
      P.pr.afm = S.d_afm_c;
      P.pr.mfa = S.d_mfa_c;
      P.pr.na = nac;
      P.pr.ia_base = a0;
    }
    var.fn<<<grid, var.threads, var.smem, stream>>>(P);
    if ((rc = cuda_check(cudaGetLastError(), "sweep kernel launch"))) return rc;
  }
  return MSB_OK;
}

// Every pass of one mixed-precision sweep: per pass the sweep kernel writes
// each octant's FP32 contribution, and the partial sum adds them up in vo.
// The tasks given may be those of the group pairs [gp0, gp1) only (a slice of
// a host-buffer run); the conversion and the sum then cover those groups.
static int launch_mixed(SweeperImpl& S, double* vo_d, const double* vi_d, cudaStream_t stream,
                        const int* d_tasks, long long ntask, int gp0, int gp1) {
  const int na = S.dims.na, pa = pass_angles(S), npass = (na + pa - 1) / pa;
  const Dimensions& d = S.dims;
  MixParams P;
  fill_params<float>(S, P, P, vi_d, d_tasks, ntask);
  P.part = S.d_part;
  P.state = S.part_elems / NOCTANT;
  int rc;
  // vi in the first transform's operand format, once for every octant and pass
  S.var.conv<<<S.nsm * 8, 256, 0, stream>>>(vi_d, S.d_vi16, d.ncell_x, d.ncell_y, d.ncell_z, d.ne, S.ngp, gp0,
                                            gp1);
  if ((rc = cuda_check(cudaGetLastError(), "vi conversion launch"))) return rc;
  P.vi16 = S.d_vi16;
  for (int c = 0; c < npass; ++c) {
    if (npass > 1) {
      const int a0 = pa * c, nac = std::min(pa, na - a0);
      if ((rc = copy_pass_matrices(S, a0, nac, stream))) return rc;
      if (c > 0 && (rc = reset_pass(S, stream))) return rc;
      P.afm = S.d_afm_c;
      P.mfa = S.d_mfa_c;
      P.na = nac;
      P.ia_base = a0;
    }
    S.var.mix<<<S.grid, S.var.threads, S.var.smem, stream>>>(P);
    if ((rc = cuda_check(cudaGetLastError(), "sweep kernel launch"))) return rc;
    const size_t layer = (size_t)d.nm * NU * d.ncell_x * d.ncell_y;  // one (iz, ie) slab
    const int e0 = 2 * gp0, e1 = std::min(2 * gp1, d.ne);
    reduce_octant_partials<<<S.nsm * 8, 256, 0, stream>>>(vo_d, S.d_part, P.state, c > 0 ? 1 : 0, layer * d.ne,
                                                          layer * e0, layer * (e1 - e0), d.ncell_z);
    if ((rc = cuda_check(cudaGetLastError(), "partial sum launch"))) return rc;
  }
  return MSB_OK;
}

// Exchanges the sweeper's plan with a candidate.
static void swap_plan(SweeperImpl& S, AltPlan& a) {
  std::swap(S.var, a.var);
  std::swap(S.sched, a.sched);
  std::swap(S.gp_block, a.gp_block);
  std::swap(S.d_tasks, a.d_tasks);
  std::swap(S.grid, a.grid);
  std::swap(S.window, a.window);
  std::swap(S.l2_hints, a.l2_hints);
}

static int impl_sync(SweeperImpl& S, cudaStream_t stream);

// The sweep's transform matrices into the sweeper's device buffers, from the
// device copies when there are some, else from the host.
static int load_matrices(SweeperImpl& S, const double* afm_h, const double* mfa_h, const double* afm_d,
                         const double* mfa_d, cudaStream_t stream) {
  int rc;
  const size_t nmat = (size_t)S.dims.nm * S.dims.na * NOCTANT;
  if (afm_d && mfa_d) {
    if ((rc = cuda_check(cudaMemcpyAsync(S.d_afm, afm_d, nmat * sizeof(double), cudaMemcpyDeviceToDevice, stream),
                         "copy a_from_m")))
      return rc;
    if ((rc = cuda_check(cudaMemcpyAsync(S.d_mfa, mfa_d, nmat * sizeof(double), cudaMemcpyDeviceToDevice, stream),
                         "copy m_from_a")))
      return rc;
  } else {
    if ((rc = cuda_check(cudaMemcpyAsync(S.d_afm, afm_h, nmat * sizeof(double), cudaMemcpyHostToDevice, stream),
                         "copy a_from_m")))
      return rc;
    if ((rc = cuda_check(cudaMemcpyAsync(S.d_mfa, mfa_h, nmat * sizeof(double), cudaMemcpyHostToDevice, stream),
                         "copy m_from_a")))
      return rc;
  }
  return MSB_OK;
}

// Launches one sweep: vo_d = sweep(vi_d), asynchronously on `stream` (the
// first sweep of an autotuning sweeper waits for the stream).
static int impl_sweep(SweeperImpl& S, double* vo_d, const double* vi_d, const double* afm_h, const double* mfa_h,
                      const double* afm_d, const double* mfa_d, cudaStream_t stream) {
  int rc;
  if ((rc = load_matrices(S, afm_h, mfa_h, afm_d, mfa_d, stream))) return rc;
  if ((rc = cuda_check(cudaMemsetAsync(S.d_sync, 0, S.sync_ints * sizeof(int), stream), "reset sync"))) return rc;
  if (S.var.fn && S.autotune && !S.tuned) {
    // First sweep of an autotuning sweeper: the same sweep with the sweeper's
    // own plan and with every candidate (each writes all of vo), timed on the
    // stream; the fastest plan is kept for every later sweep.
    S.tuned = true;
    cudaEvent_t e0 = nullptr, e1 = nullptr;
    if ((rc = cuda_check(cudaEventCreate(&e0), "autotune event"))) return rc;
    if ((rc = cuda_check(cudaEventCreate(&e1), "autotune event"))) {
      cudaEventDestroy(e0);
      return rc;
    }
    float main_ms = 0.f;
    // i = -1: the sweeper's own plan; i >= 0: candidate i (swapped in)
    for (int i = -1; i < (int)S.alts.size() && !rc; ++i) {
      if (i >= 0) swap_plan(S, S.alts[i]);
      rc = cuda_check(cudaMemsetAsync(S.d_sync, 0, S.sync_ints * sizeof(int), stream), "reset sync");
      if (!rc) rc = cuda_check(cudaEventRecord(e0, stream), "autotune event");
      if (!rc) rc = launch_fp64(S, S.var, S.d_tasks, S.sched.ntask(), S.grid, vo_d, vi_d, stream);
      if (!rc) rc = cuda_check(cudaEventRecord(e1, stream), "autotune event");
      if (!rc) rc = cuda_check(cudaMemcpyAsync(S.h_status, S.d_sync, 4 * sizeof(int), cudaMemcpyDeviceToHost, stream),
                               "status copy");
      if (!rc) rc = cuda_check(cudaStreamSynchronize(stream), "autotune sweep");
      float ms = 0.f;
      if (!rc) cudaEventElapsedTime(&ms, e0, e1);
      if (!rc && S.h_status[SY_ERROR] != 0) rc = impl_sync(S, stream);  // reports the device error
      if (i >= 0) {
        swap_plan(S, S.alts[i]);
        S.alts[i].ms = ms;
      } else {
        main_ms = ms;
      }
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    if (rc) return rc;
    int best = -1;
    float best_ms = main_ms;
    for (int i = 0; i < (int)S.alts.size(); ++i)
      if (S.alts[i].ms < best_ms) {
        best = i;
        best_ms = S.alts[i].ms;
      }
    if (best >= 0) {
      swap_plan(S, S.alts[best]);
      S.alts[best].ms = main_ms;  // the slot now holds the former main plan
    }
    S.tune_ms[0] = best_ms;
    S.tune_ms[1] = 0.f;
    for (const auto& a : S.alts)
      if (a.var.tx != S.var.tx && (S.tune_ms[1] == 0.f || a.ms < S.tune_ms[1])) S.tune_ms[1] = a.ms;
    // the sync words hold the last trial's status, which was clean
  } else if (S.var.fn) {
    if ((rc = launch_fp64(S, S.var, S.d_tasks, S.sched.ntask(), S.grid, vo_d, vi_d, stream))) return rc;
  } else {
    if ((rc = launch_mixed(S, vo_d, vi_d, stream, S.d_tasks, S.sched.ntask(), 0, S.ngp))) return rc;
  }
  if ((rc = cuda_check(cudaMemcpyAsync(S.h_status, S.d_sync, 4 * sizeof(int), cudaMemcpyDeviceToHost, stream),
                       "status copy")))
    return rc;
  const int npass = (S.dims.na + pass_angles(S) - 1) / pass_angles(S);
  // mixed: the vi conversion, then the sweep kernel and the partial sum per pass
  S.nlaunch = S.var.mix ? 1 + 2 * npass : npass;
  return MSB_OK;
}

static int impl_sync(SweeperImpl& S, cudaStream_t stream) {
  int rc;
  if ((rc = cuda_check(cudaStreamSynchronize(stream), "sweep"))) return rc;
  const int err = S.h_status[SY_ERROR];
  if (err == MSB_ERR_TIMEOUT)
    return set_error(MSB_ERR_TIMEOUT, "a device wait ran out of time (task %d); sweep aborted", S.h_status[SY_ERRTASK]);
  if (err) return set_error(err, "device error %d", err);
  return MSB_OK;
}

// ------------------------------------------- host-buffer runs in group slices
// The energy groups are independent in the sweep (no face, dependency or sum
// crosses them), so a run of Sweeper_sweep_iterations on a large problem
// (FP64, or mixed precision: the vi conversion and the partial sum then cover
// the slice's groups) is split into slices of group pairs, each swept through every iteration
// with its own task table: the host->device copy of slice k + 1 then runs
// while slice k is swept, and the device->host copy of slice k while slice
// k + 1 is.  Every value is the one the unsliced run computes.  Slices are
// used only where they stay efficient (64^3 cells x na 32, one B200: 115.9 ms
// per sweep with 64 groups, 58.2 with 32, 29.8 with 16, 16.4 with 8).
static int slice_count(const SweeperImpl& S) {
  if (S.kba || !S.var.valid() || (S.autotune && !S.tuned)) return 1;
  const size_t bytes = Dimensions_size_state(S.dims, NU) * sizeof(double);
  if (bytes < ((size_t)256 << 20)) return 1;  // copies too short to be worth hiding
  return std::max(1, std::min(4, S.ngp / 8));
}

static int build_slices(SweeperImpl& S, int nslice) {
  if (S.slices && S.slices->for_tasks == S.d_tasks && (int)S.slices->d_tasks.size() == nslice) return MSB_OK;
  S.slices.reset();
  auto T = std::make_unique<SliceTables>();
  T->for_tasks = S.d_tasks;
  const long long n = S.sched.ntask();
  const int* rec = S.sched.rec.data();
  std::vector<long long> index(n, -1);  // task -> its index in its slice
  for (int k = 0; k <= nslice; ++k) T->gp0.push_back((int)((long long)S.ngp * k / nslice));
  for (int k = 0; k < nslice; ++k) {
    const int g0 = T->gp0[k], g1 = T->gp0[k + 1];
    std::vector<int> out;
    long long m = 0;
    for (long long t = 0; t < n; ++t) {
      const int* r = rec + (size_t)t * MSB_TASK_INTS;
      if (r[TK_GP] < g0 || r[TK_GP] >= g1) continue;
      index[t] = m++;
      out.insert(out.end(), r, r + MSB_TASK_INTS);
      int* q = out.data() + out.size() - MSB_TASK_INTS;
      for (int f : {TK_DEP_X, TK_DEP_Y, TK_DEP_Z, TK_DEP_VO}) {
        if (q[f] < 0) continue;
        const int gd = rec[(size_t)q[f] * MSB_TASK_INTS + TK_GP];
        if (q[f] >= t || gd < g0 || gd >= g1)
          return set_error(MSB_ERR_ARG, "schedule: task %lld depends on task %d outside its slice", t, q[f]);
        q[f] = (int)index[q[f]];
      }
    }
    int* d = nullptr;
    int rc = cuda_check(cudaMalloc(&d, std::max<size_t>(out.size(), 1) * sizeof(int)), "cudaMalloc slice tasks");
    if (rc) return rc;
    T->d_tasks.push_back(d);
    if ((rc = cuda_check(cudaMemcpy(d, out.data(), out.size() * sizeof(int), cudaMemcpyHostToDevice),
                         "upload slice tasks")))
      return rc;
    T->ntask.push_back(m);
  }
  S.slices = std::move(T);
  return MSB_OK;
}

// Groups [e0, e1) of a state array: one contiguous run per z-plane.
static int copy_groups(double* dst, const double* src, const Dimensions& d, int e0, int e1, cudaMemcpyKind kind,
                       cudaStream_t st) {
  const size_t slab = (size_t)d.nm * NU * d.ncell_x * d.ncell_y;
  const size_t pitch = (size_t)d.ne * slab * sizeof(double), width = (size_t)(e1 - e0) * slab * sizeof(double);
  const size_t off = (size_t)e0 * slab;
  if (width == pitch) return cuda_check(cudaMemcpyAsync(dst, src, pitch * d.ncell_z, kind, st), "state copy");
  if (pitch <= (size_t)INT_MAX)
    return cuda_check(cudaMemcpy2DAsync(dst + off, pitch, src + off, pitch, width, d.ncell_z, kind, st),
                      "state copy");
  for (int iz = 0; iz < d.ncell_z; ++iz) {
    const size_t o = off + (size_t)iz * d.ne * slab;
    int rc = cuda_check(cudaMemcpyAsync(dst + o, src + o, width, kind, st), "state copy");
    if (rc) return rc;
  }
  return MSB_OK;
}

// in_h -> (niterations sweeps) -> out_h in nslice group slices on three
// streams: copies in (sh), the sweeps (st, the Env's stream), copies out
// (sd).  in_h lands in the device array d_a; the sweeps alternate between
// d_a and d_b (the vi/vo swap).  The task counter and progress words start over before every sweep
// but the error words do not, so a failed sweep makes the later ones end at
// once and the final status reports it.
static int sweep_iterations_sliced(SweeperImpl& S, int nslice, double* out_h, const double* in_h, int niterations,
                                   double* d_a, double* d_b, const double* afm_h, const double* mfa_h,
                                   const double* afm_d, const double* mfa_d, cudaStream_t st) {
  int rc = build_slices(S, nslice);
  if (rc) return rc;
  const SliceTables& T = *S.slices;
  const Dimensions& d = S.dims;
  cudaStream_t sh = nullptr, sd = nullptr;
  std::vector<cudaEvent_t> ev(2 * nslice + 2, nullptr);  // [0] start, [1 + k] slice k in, [1 + nslice + k] swept, end
  bool enqueued = false;
  rc = cuda_check(cudaStreamCreateWithFlags(&sh, cudaStreamNonBlocking), "copy stream");
  if (!rc) rc = cuda_check(cudaStreamCreateWithFlags(&sd, cudaStreamNonBlocking), "copy stream");
  for (auto& e : ev)
    if (!rc) rc = cuda_check(cudaEventCreateWithFlags(&e, cudaEventDisableTiming), "slice event");
  // the copies wait for the work already on the Env's stream
  if (!rc) rc = cuda_check(cudaEventRecord(ev[0], st), "slice event");
  if (!rc) rc = cuda_check(cudaStreamWaitEvent(sh, ev[0], 0), "slice wait");
  if (!rc) rc = cuda_check(cudaStreamWaitEvent(sd, ev[0], 0), "slice wait");
  if (!rc) rc = load_matrices(S, afm_h, mfa_h, afm_d, mfa_d, st);
  if (!rc) rc = cuda_check(cudaMemsetAsync(S.d_sync, 0, S.sync_ints * sizeof(int), st), "reset sync");
  auto groups = [&](int k, int& e0, int& e1) {
    e0 = 2 * T.gp0[k];
    e1 = std::min(2 * T.gp0[k + 1], d.ne);
  };
  // Host order: copy in k + 1 and copy out k - 1 are issued after slice k's
  // sweeps, so that with pageable host buffers (whose copies return only
  // once done) the GPU is sweeping while the host thread copies.
  auto copy_in = [&](int k) {
    int e0, e1;
    groups(k, e0, e1);
    enqueued = true;
    int r = copy_groups(d_a, in_h, d, e0, e1, cudaMemcpyHostToDevice, sh);
    if (!r) r = cuda_check(cudaEventRecord(ev[1 + k], sh), "slice event");
    return r;
  };
  double* last = (niterations % 2) ? d_b : d_a;  // where the last sweep writes
  auto copy_out = [&](int k) {
    int e0, e1;
    groups(k, e0, e1);
    int r = cuda_check(cudaStreamWaitEvent(sd, ev[1 + nslice + k], 0), "slice wait");
    if (!r) r = copy_groups(out_h, last, d, e0, e1, cudaMemcpyDeviceToHost, sd);
    return r;
  };
  if (!rc) rc = copy_in(0);
  for (int k = 0; k < nslice && !rc; ++k) {
    rc = cuda_check(cudaStreamWaitEvent(st, ev[1 + k], 0), "slice wait");
    double* a = d_a;
    double* b = d_b;
    for (int it = 0; it < niterations && !rc; ++it) {
      if (k > 0 || it > 0) rc = reset_pass(S, st);
      if (!rc)
        rc = S.var.fn ? launch_fp64(S, S.var, T.d_tasks[k], T.ntask[k], S.grid, b, a, st)
                      : launch_mixed(S, b, a, st, T.d_tasks[k], T.ntask[k], T.gp0[k], T.gp0[k + 1]);
      std::swap(a, b);
    }
    if (!rc) rc = cuda_check(cudaEventRecord(ev[1 + nslice + k], st), "slice event");
    if (!rc && k + 1 < nslice) rc = copy_in(k + 1);
    if (!rc && k > 0) rc = copy_out(k - 1);
  }
  if (!rc) rc = copy_out(nslice - 1);
  // the Env's stream ends after the last copy out: its sync covers the run
  if (!rc) rc = cuda_check(cudaEventRecord(ev.back(), sd), "slice event");
  if (!rc) rc = cuda_check(cudaStreamWaitEvent(st, ev.back(), 0), "slice wait");
  if (!rc)
    rc = cuda_check(cudaMemcpyAsync(S.h_status, S.d_sync, 4 * sizeof(int), cudaMemcpyDeviceToHost, st),
                    "status copy");
  if (!rc) rc = impl_sync(S, st);
  if (rc && enqueued) {
    // nothing may still write the caller's buffer after the error is returned
    cudaStreamSynchronize(sh);
    cudaStreamSynchronize(st);
    cudaStreamSynchronize(sd);
  }
  for (auto& e : ev)
    if (e) cudaEventDestroy(e);
  if (sh) cudaStreamDestroy(sh);
  if (sd) cudaStreamDestroy(sd);
  if (!rc) {
    const int npass = (d.na + pass_angles(S) - 1) / pass_angles(S);
    S.nlaunch = S.var.mix ? 1 + 2 * npass : npass;  // of the last sweep
  }
  return rc;
}

// ------------------------------------------------------- KBA decomposition
// Process `proc` of an npx x npy grid sweeps its subdomain with the staged
// FP64 kernel, one launch per (octant, z-block) unit.  The face planes hold
// one region per angle pass so that a unit's passes leave each other's
// faces intact until they are sent.
static int impl_create_kba(SweeperImpl& S, const Dimensions& dims, int tile, int nblock, int npx, int npy, int proc,
                           int sp_off) {
  S.dims = dims;
  S.precision = 0;
  S.sp_off = sp_off & 3;
  S.var = pick_variant(dims.nm, dims.na, 0, tile, 0);
  if (!S.var.valid())
    return set_error(MSB_ERR_UNSUPPORTED, "no kernel variant for nm=%d na=%d (nm in {4,8,16}; na <= 128)", dims.nm,
                     dims.na);
  S.ngp = (dims.ne + 1) / 2;
  const Variant& var = S.var;
  int rc, dev = 0, nsm = 0, occ = 0;
  if ((rc = cuda_check(cudaGetDevice(&dev), "cudaGetDevice"))) return rc;
  if ((rc = cuda_check(cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev), "SM count"))) return rc;
  S.nsm = nsm;
  if ((rc = cuda_check(cudaFuncSetAttribute(var.func(), cudaFuncAttributeMaxDynamicSharedMemorySize, (int)var.smem),
                       "cudaFuncSetAttribute")))
    return rc;
  if ((rc = cuda_check(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, var.func(), var.threads, var.smem),
                       "occupancy")))
    return rc;
  if (occ < 1) return set_error(MSB_ERR_UNSUPPORTED, "sweep kernel does not fit on an SM");

  std::unique_ptr<KbaState> K(new (std::nothrow) KbaState());
  if (!K) return set_error(MSB_ERR_ARG, "out of host memory");
  if ((rc = build_kba_plan(npx, npy, nblock, K->plan))) return rc;
  K->proc = proc;
  K->px = proc % npx;
  K->py = proc / npx;
  K->nzb = dims.ncell_z / nblock;
  K->pa = var.pass;
  K->npass = (dims.na + var.pass - 1) / var.pass;
  const int nunit = K->plan.nunit(), nx = dims.ncell_x, ny = dims.ncell_y, nz = dims.ncell_z;
  S.gp_block = pick_gp_block_slab(nx, ny, S.ngp, var.tx, var.ty, S.window * nsm);
  K->off.resize(nunit);
  K->cnt.resize(nunit);
  K->grid.resize(nunit);
  std::vector<int>& all = S.sched.rec;  // every unit's tasks, for Sweeper_debug_tasks
  all.clear();
  for (int k = 0; k < nunit; ++k) {
    const int oct = K->plan.unit_oct[k], zb = K->plan.unit_zb[k];
    const int dx = (oct & 1) ? -1 : 1, dy = (oct & 2) ? -1 : 1, dz = (oct & 4) ? -1 : 1;
    SlabEdges e;
    e.x_in = K->px - dx >= 0 && K->px - dx < npx;
    e.x_out = K->px + dx >= 0 && K->px + dx < npx;
    e.y_in = K->py - dy >= 0 && K->py - dy < npy;
    e.y_out = K->py + dy >= 0 && K->py + dy < npy;
    e.z_in = dz > 0 ? zb > 0 : zb < nblock - 1;
    e.z_out = dz > 0 ? zb < nblock - 1 : zb > 0;
    e.first = k < nblock;  // the first octant of the sequence visits every z-block first
    Schedule sch;
    if ((rc = build_slab_schedule(nx, ny, zb * K->nzb, (zb + 1) * K->nzb, S.ngp, var.tx, var.ty, S.gp_block, oct, e,
                                  sch)))
      return rc;
    K->off[k] = (long long)(all.size() / MSB_TASK_INTS);
    K->cnt[k] = sch.ntask();
    K->grid[k] = (int)std::min<long long>(sch.ntask(), (long long)nsm * occ);
    K->ntask_max = std::max(K->ntask_max, sch.ntask());
    all.insert(all.end(), sch.rec.begin(), sch.rec.end());
  }
  S.sched.nx = nx;
  S.sched.ny = ny;
  S.sched.nz = nz;
  S.sched.ngp = S.ngp;
  S.sched.tx = var.tx;
  S.sched.ty = var.ty;
  if (K->ntask_max >= (1LL << 31) - SY_PROGRESS) return set_error(MSB_ERR_ARG, "too many tasks");
  if ((rc = cuda_check(cudaMalloc(&K->d_tasks, all.size() * sizeof(int)), "cudaMalloc tasks"))) return rc;
  if ((rc = cuda_check(cudaMemcpy(K->d_tasks, all.data(), all.size() * sizeof(int), cudaMemcpyHostToDevice),
                       "copy tasks")))
    return rc;
  S.sync_ints = SY_PROGRESS + (size_t)K->ntask_max;
  if ((rc = cuda_check(cudaMalloc(&S.d_sync, S.sync_ints * sizeof(int)), "cudaMalloc sync"))) return rc;
  if ((rc = cuda_check(cudaMallocHost(&S.h_status, 8 * sizeof(int)), "cudaMallocHost status"))) return rc;
  const size_t E = var.entry_bytes, per = (size_t)NOCTANT * S.ngp * E;
  K->plane_pass[0] = per * ny * nx;
  K->plane_pass[1] = per * nz * nx;
  K->plane_pass[2] = per * nz * ny;
  for (int f = 0; f < 3; ++f) {
    S.face_bytes[f] = K->plane_pass[f] * K->npass;
    if ((rc = cuda_check(cudaMalloc(&S.d_face[f], S.face_bytes[f]), "cudaMalloc faces"))) return rc;
  }
  K->slab_bytes[0] = (size_t)S.ngp * K->nzb * ny * E;
  K->slab_bytes[1] = (size_t)S.ngp * K->nzb * nx * E;
  const size_t nmat = (size_t)dims.nm * dims.na * NOCTANT;
  if ((rc = cuda_check(cudaMalloc(&S.d_afm, nmat * sizeof(double)), "cudaMalloc a_from_m"))) return rc;
  if ((rc = cuda_check(cudaMalloc(&S.d_mfa, nmat * sizeof(double)), "cudaMalloc m_from_a"))) return rc;
  if (K->npass > 1) {
    const size_t blk = (size_t)dims.nm * K->pa * NOCTANT * K->npass;
    if ((rc = cuda_check(cudaMalloc(&S.d_afm_c, blk * sizeof(double)), "cudaMalloc a_from_m passes"))) return rc;
    if ((rc = cuda_check(cudaMalloc(&S.d_mfa_c, blk * sizeof(double)), "cudaMalloc m_from_a passes"))) return rc;
  }
  S.kba = std::move(K);
  return MSB_OK;
}

// Face rows of one unit's slab in one pass's plane: x faces (axis 0) are the
// yz plane's rows [oct][gp][z-block][all y], y faces the xz plane's
// [oct][gp][z-block][all x]; one row run per group pair, `pitch` apart.
static char* kba_rows(const SweeperImpl& S, int axis, int pass, int unit, size_t& pitch, size_t& width) {
  const KbaState& K = *S.kba;
  const size_t E = S.var.entry_bytes;
  const int n_in = axis == 0 ? S.dims.ncell_y : S.dims.ncell_x, f = axis == 0 ? 2 : 1;
  pitch = (size_t)S.dims.ncell_z * n_in * E;
  width = (size_t)K.nzb * n_in * E;
  const int oct = K.plan.unit_oct[unit], zb = K.plan.unit_zb[unit];
  return static_cast<char*>(S.d_face[f]) + pass * K.plane_pass[f] +
         ((size_t)oct * S.ngp * S.dims.ncell_z + (size_t)zb * K.nzb) * n_in * E;
}

// Matrices of the sweep (and every pass's share of them) in place, progress
// cleared; the steps follow.
static int kba_begin(SweeperImpl& S, double* vo_d, const double* vi_d, const double* afm_h, const double* mfa_h,
                     const double* afm_d, const double* mfa_d, cudaStream_t stream) {
  KbaState& K = *S.kba;
  int rc;
  if ((rc = load_matrices(S, afm_h, mfa_h, afm_d, mfa_d, stream))) return rc;
  if (K.npass > 1) {
    const size_t blk = (size_t)S.dims.nm * K.pa * NOCTANT;
    for (int c = 0; c < K.npass; ++c) {
      const int a0 = K.pa * c, nac = std::min(K.pa, S.dims.na - a0);
      if ((rc = copy_pass_matrices(S, a0, nac, stream, S.d_afm_c + c * blk, S.d_mfa_c + c * blk))) return rc;
    }
  }
  if ((rc = cuda_check(cudaMemsetAsync(S.d_sync, 0, S.sync_ints * sizeof(int), stream), "reset sync"))) return rc;
  K.vo_d = vo_d;
  K.vi_d = vi_d;
  K.rc = MSB_OK;
  S.nlaunch = 0;
  return MSB_OK;
}

// This process's unit of `step` (every pass), then its leaving faces into the
// send buffers; returns with the stream drained (the previous step's
// unpacking included), so the receive buffers are free again.  After an
// error the later steps launch nothing, so that the process still takes part
// in every exchange.
static int kba_step(SweeperImpl& S, int step, cudaStream_t stream) {
  KbaState& K = *S.kba;
  if (K.rc) return K.rc;
  const int k = kba_unit_at(K.plan, K.proc, step);
  if (k < 0) return K.rc = cuda_check(cudaStreamSynchronize(stream), "sweep");
  const int oct = K.plan.unit_oct[k];
  int rc = MSB_OK;
  for (int c = 0; c < K.npass && !rc; ++c) {
    rc = cuda_check(cudaMemsetAsync(S.d_sync + SY_COUNTER, 0, sizeof(int), stream), "reset sync");
    if (!rc)
      rc = cuda_check(cudaMemsetAsync(S.d_sync + SY_PROGRESS, 0, (size_t)K.cnt[k] * sizeof(int), stream),
                      "reset sync");
    if (rc) break;
    Fp64Params P{};
    fill_params<double>(S, P.pr, P, K.vi_d, K.d_tasks + K.off[k] * MSB_TASK_INTS, K.cnt[k]);
    P.pr.vo = K.vo_d;
    P.pr.vo_add = c > 0 ? 1 : 0;
    P.pr.fxy = reinterpret_cast<double*>(static_cast<char*>(S.d_face[0]) + c * K.plane_pass[0]);
    P.pr.fxz = reinterpret_cast<double*>(static_cast<char*>(S.d_face[1]) + c * K.plane_pass[1]);
    P.pr.fyz = reinterpret_cast<double*>(static_cast<char*>(S.d_face[2]) + c * K.plane_pass[2]);
    if (K.npass > 1) {
      const size_t blk = (size_t)S.dims.nm * K.pa * NOCTANT;
      P.pr.afm = S.d_afm_c + c * blk;
      P.pr.mfa = S.d_mfa_c + c * blk;
      P.pr.na = std::min(K.pa, S.dims.na - K.pa * c);
      P.pr.ia_base = K.pa * c;
    }
    S.var.fn<<<K.grid[k], S.var.threads, S.var.smem, stream>>>(P);
    rc = cuda_check(cudaGetLastError(), "sweep kernel launch");
    ++S.nlaunch;
  }
  // leaving faces of the unit for the downwind neighbours
  const int dx = (oct & 1) ? -1 : 1, dy = (oct & 2) ? -1 : 1;
  const bool down[2] = {K.px + dx >= 0 && K.px + dx < K.plan.npx, K.py + dy >= 0 && K.py + dy < K.plan.npy};
  for (int axis = 0; axis < 2 && !rc; ++axis) {
    if (!down[axis]) continue;
    for (int c = 0; c < K.npass && !rc; ++c) {
      size_t pitch, width;
      const char* src = kba_rows(S, axis, c, k, pitch, width);
      rc = cuda_check(cudaMemcpy2DAsync(static_cast<char*>(K.buf[axis]) + c * K.slab_bytes[axis], width, src, pitch,
                                        width, S.ngp, cudaMemcpyDeviceToDevice, stream),
                      "pack faces");
    }
  }
  if (!rc)
    rc = cuda_check(cudaMemcpyAsync(S.h_status, S.d_sync, 4 * sizeof(int), cudaMemcpyDeviceToHost, stream),
                    "status copy");
  if (!rc) rc = impl_sync(S, stream);
  K.rc = rc;
  return rc;
}

// The step's messages with this process's buffers.
static int kba_message_list(const SweeperImpl& S, int step, std::vector<msb_kba_msg>& out) {
  const KbaState& K = *S.kba;
  std::vector<KbaMsg> msgs;
  kba_messages(K.plan, K.proc, step, msgs);
  out.clear();
  for (const KbaMsg& m : msgs) {
    msb_kba_msg r;
    r.peer = m.peer;
    r.is_send = m.is_send;
    r.axis = m.axis;
    r.side = m.side;
    r.bytes = K.msg_bytes(m.axis);
    r.buf = m.is_send ? K.buf[m.axis] : K.buf[2 + 2 * m.axis + m.side];
    out.push_back(r);
  }
  return (int)out.size();
}

// Faces received after `step` into this process's planes (asynchronous: the
// next step's launch follows on the same stream).
static int kba_unpack(SweeperImpl& S, int step, cudaStream_t stream) {
  KbaState& K = *S.kba;
  if (K.rc) return K.rc;
  std::vector<KbaMsg> msgs;
  kba_messages(K.plan, K.proc, step, msgs);
  int rc = MSB_OK;
  for (const KbaMsg& m : msgs) {
    if (m.is_send) continue;
    const char* src = static_cast<const char*>(K.buf[2 + 2 * m.axis + m.side]);
    for (int c = 0; c < K.npass && !rc; ++c) {
      size_t pitch, width;
      char* dst = kba_rows(S, m.axis, c, m.unit, pitch, width);
      rc = cuda_check(cudaMemcpy2DAsync(dst, pitch, src + c * K.slab_bytes[m.axis], width, width, S.ngp,
                                        cudaMemcpyDeviceToDevice, stream),
                      "unpack faces");
    }
  }
  K.rc = rc;
  return rc;
}

// Message buffers the sweeper owns, for the ones the host did not provide.
static int kba_own_buffers(SweeperImpl& S) {
  KbaState& K = *S.kba;
  for (int i = 0; i < 6; ++i) {
    if (K.buf[i]) continue;
    const size_t b = K.msg_bytes(i == 0 ? 0 : i == 1 ? 1 : (i - 2) / 2);
    if (!K.own[i]) {
      int rc = cuda_check(cudaMalloc(&K.own[i], b ? b : 16), "cudaMalloc message buffer");
      if (rc) return rc;
    }
    K.buf[i] = K.own[i];
  }
  return MSB_OK;
}

// A whole decomposed sweep with the transport of the Env's process group.
// When processes of the group share a GPU, their slabs of a step run one
// process after the other (a barrier between turns): no two processes' sweep
// kernels are on one GPU at once.
static int kba_sweep(SweeperImpl& S, double* vo_d, const double* vi_d, const double* afm_h, const double* mfa_h,
                     const double* afm_d, const double* mfa_d, const Env* env, cudaStream_t stream) {
  KbaState& K = *S.kba;
  const msb_comm* comm = env ? env->comm_ : nullptr;
  if (!comm) return set_error(MSB_ERR_ARG, "a decomposed sweep needs the Env's process group (msb_env_set_comm)");
  const int nactive = K.plan.npx * K.plan.npy;
  const bool turns = (env->flags_ & MSB_ENV_SHARED_GPU) != 0;
  int rc = kba_own_buffers(S);
  if (!rc) rc = kba_begin(S, vo_d, vi_d, afm_h, mfa_h, afm_d, mfa_d, stream);
  if (rc) K.rc = rc;
  std::vector<msb_kba_msg> msgs;
  // every process takes every step's barriers and exchange, errors or not
  for (int step = 0; step < K.plan.nstep; ++step) {
    if (turns) {
      for (int q = 0; q < nactive; ++q) {
        if (q == K.proc) kba_step(S, step, stream);
        if (comm->barrier(comm->ctx, nactive) != 0 && !K.rc)
          K.rc = set_error(MSB_ERR_ARG, "process group barrier failed at step %d", step);
      }
    } else {
      kba_step(S, step, stream);
    }
    const int n = kba_message_list(S, step, msgs);
    if (comm->exchange(comm->ctx, nactive, msgs.data(), n) != 0 && !K.rc)
      K.rc = set_error(MSB_ERR_ARG, "face exchange failed at step %d", step);
    kba_unpack(S, step, stream);
    if (turns && !K.rc) K.rc = cuda_check(cudaStreamSynchronize(stream), "unpack faces");
  }
  if (!K.rc) K.rc = cuda_check(cudaStreamSynchronize(stream), "sweep");
  return K.rc;
}

}  // namespace msb

using msb::SweeperImpl;

static SweeperImpl* impl_of(const Sweeper* s) { return static_cast<SweeperImpl*>(s->impl_); }
static cudaStream_t stream_of(Env* env) { return env ? (cudaStream_t)env->stream_kernel_faces_ : nullptr; }

extern "C" Sweeper Sweeper_null(void) {
  Sweeper s;
  memset(&s, 0, sizeof s);
  return s;
}

extern "C" int Sweeper_noctant_per_block(const Sweeper* sweeper) { return sweeper->noctant_per_block; }

// Flag handling follows sweeper_kba_c.h:44-233 (names, defaults, checks).
// Threading flags describe the reference's CPU/GPU thread decomposition; they
// are validated and recorded but the B200 schedule does not depend on them.
extern "C" int Sweeper_create_status(Sweeper* sweeper, Dimensions dims, const Quantities* quan, Env* env,
                                     Arguments* args) {
  *sweeper = Sweeper_null();
  auto bad = [](const char* m) { return msb::set_error(MSB_ERR_ARG, "%s", m); };
  sweeper->is_face_comm_async = Arguments_consume_int_or_default(args, "--is_face_comm_async", Bool_true);
  if (dims.ncell_x <= 0 || dims.ncell_y <= 0 || dims.ncell_z <= 0)
    return bad("Currently required that all spatial blocks be nonempty");
  sweeper->nblock_z = Arguments_consume_int_or_default(args, "--nblock_z", 1);
  if (sweeper->nblock_z <= 0) return bad("Invalid z blocking factor supplied");
  if (dims.ncell_z % sweeper->nblock_z != 0) return bad("Currently require all blocks have same z dimension");
  const int dims_b_ncell_z = dims.ncell_z / sweeper->nblock_z;
  sweeper->nthread_octant = Arguments_consume_int_or_default(args, "--nthread_octant", 1);
  const int nto = sweeper->nthread_octant;
  if (!(nto > 0 && nto <= NOCTANT && (nto & (nto - 1)) == 0)) return bad("Invalid thread count supplied");
  sweeper->noctant_per_block = nto;
  sweeper->nblock_octant = NOCTANT / nto;
  const int nsb_default = nto == 8 && sweeper->nblock_z % 2 == 0 ? 4 : nto;
  sweeper->nsemiblock = Arguments_consume_int_or_default(args, "--nsemiblock", nsb_default);
  const int nsb = sweeper->nsemiblock;
  if (!(nsb > 0 && nsb <= NOCTANT && (nsb & (nsb - 1)) == 0)) return bad("Invalid semiblock count supplied");
  if (!(nsb >= nto || (nto == 8 && sweeper->nblock_z % 2 == 0 && nsb == 4)))
    return bad("Incomplete set of semiblock steps requires atomic vo update");
  sweeper->ncell_x_per_subblock = Arguments_consume_int_or_default(
      args, "--ncell_x_per_subblock", nsb >= 2 ? (dims.ncell_x + 1) / 2 : dims.ncell_x);
  if (sweeper->ncell_x_per_subblock <= 0) return bad("Invalid subblock size supplied");
  sweeper->ncell_y_per_subblock = Arguments_consume_int_or_default(
      args, "--ncell_y_per_subblock", nsb >= 4 ? (dims.ncell_y + 1) / 2 : dims.ncell_y);
  if (sweeper->ncell_y_per_subblock <= 0) return bad("Invalid subblock size supplied");
  sweeper->ncell_z_per_subblock = Arguments_consume_int_or_default(
      args, "--ncell_z_per_subblock", nsb >= 8 ? (dims_b_ncell_z + 1) / 2 : dims_b_ncell_z);
  if (sweeper->ncell_z_per_subblock <= 0) return bad("Invalid subblock size supplied");
  sweeper->dims = dims;
  sweeper->dims_b = dims;
  sweeper->dims_b.ncell_z = dims_b_ncell_z;
  sweeper->dims_g = dims;
  if (quan) {
    sweeper->dims_g.ncell_x = quan->ncell_x_g;
    sweeper->dims_g.ncell_y = quan->ncell_y_g;
  }
  sweeper->nthread_e = Arguments_consume_int_or_default(args, "--nthread_e", 1);
  if (sweeper->nthread_e <= 0) return bad("Invalid thread count supplied.");
  sweeper->nthread_x = 1;
  sweeper->nthread_y = Arguments_consume_int_or_default(args, "--nthread_y", 1);
  if (sweeper->nthread_y <= 0) return bad("Invalid thread count supplied.");
  sweeper->nthread_z = Arguments_consume_int_or_default(args, "--nthread_z", 1);
  if (sweeper->nthread_z <= 0) return bad("Invalid thread count supplied.");
  sweeper->precision = Arguments_consume_int_or_default(args, "--precision", 0);
  if (sweeper->precision < 0 || sweeper->precision > 2)
    return msb::set_error(MSB_ERR_ARG, "--precision must be 0 (FP64), 1 (mixed, FP16 halves) or 2 (mixed, BF16 halves)");
  // tile shape of the FP64 sweep (cell columns per CTA): 0 = default, 42 = 4 x 2, 24 = 2 x 4
  const int tile = Arguments_consume_int_or_default(args, "--tile", 0);
  if (tile != 0 && tile != 42 && tile != 24) return msb::set_error(MSB_ERR_ARG, "--tile must be 0, 42 or 24");
  // 1: the first sweep times both FP64 tile shapes and keeps the faster
  const int autotune = Arguments_consume_int_or_default(args, "--autotune", 0);
  if (autotune != 0 && autotune != 1) return msb::set_error(MSB_ERR_ARG, "--autotune must be 0 or 1");
  // FP64 sweep kernel: 0 = the staged kernel (default), 1 = the chained wavefront
  const int fp64_kernel = Arguments_consume_int_or_default(args, "--fp64_kernel", 0);
  if (fp64_kernel != 0 && fp64_kernel != 1) return msb::set_error(MSB_ERR_ARG, "--fp64_kernel must be 0 or 1");
  // angles per pass of the staged FP64 kernel: 0 or 32 = 32, 64 = two chunks per pass
  const int angle_pass = Arguments_consume_int_or_default(args, "--angle_pass", 0);
  if (angle_pass != 0 && angle_pass != 32 && angle_pass != 64)
    return msb::set_error(MSB_ERR_ARG, "--angle_pass must be 0, 32 or 64");
  if (angle_pass != 0 && (fp64_kernel != 0 || sweeper->precision != 0))
    return msb::set_error(MSB_ERR_ARG, "--angle_pass applies to the staged FP64 kernel (--fp64_kernel 0, --precision 0)");
  // tasks between a tile and its downwind neighbour in the schedule, in
  // multiples of the SM count
  const int task_window = Arguments_consume_int_or_default(args, "--task_window", 4);
  if (task_window < 1 || task_window > 64) return msb::set_error(MSB_ERR_ARG, "--task_window must be in [1, 64]");
  // L2 eviction policies in the chained FP64 kernel: 1 = keep faces, stream the state
  const int l2_hints = Arguments_consume_int_or_default(args, "--l2_hints", 0);
  if (l2_hints != 0 && l2_hints != 1) return msb::set_error(MSB_ERR_ARG, "--l2_hints must be 0 or 1");
  // energy-group slice of a larger problem: group ie of the arrays is global
  // group ie_base + ie (one process per GPU, each sweeping its own groups)
  const int ie_base = Arguments_consume_int_or_default(args, "--ie_base", 0);
  if (ie_base < 0) return msb::set_error(MSB_ERR_ARG, "--ie_base must be >= 0");

  std::unique_ptr<SweeperImpl> S(new (std::nothrow) SweeperImpl());
  if (!S) return msb::set_error(MSB_ERR_ARG, "out of host memory");
  S->ie_base = ie_base;
  S->window = task_window;
  S->l2_hints = l2_hints;
  int rc;
  if (env && Env_nproc(env) > 1) {
    // KBA decomposition over the Env's process grid (sweeper_kba_c.h:44-287
    // with nproc_x * nproc_y > 1): this process's subdomain, offsets from the
    // Quantities (quantities_testing_c.h:206-333)
    if (!quan) return msb::set_error(MSB_ERR_ARG, "a decomposed sweep needs the Quantities (subdomain offsets)");
    if (sweeper->precision != 0 || fp64_kernel != 0 || autotune != 0)
      return msb::set_error(MSB_ERR_UNSUPPORTED,
                            "a decomposed sweep (--nproc_x * --nproc_y > 1) runs the staged FP64 kernel: "
                            "--precision 0 --fp64_kernel 0 --autotune 0");
    if (!Env_is_proc_active(env)) return msb::set_error(MSB_ERR_ARG, "this process is not in the process grid");
    rc = msb::impl_create_kba(*S, dims, tile, sweeper->nblock_z, Env_nproc_x(env), Env_nproc_y(env),
                              Env_proc_this(env), quan->ix_base + 3 * quan->iy_base);
  } else {
    rc = msb::impl_create(*S, dims, sweeper->precision, tile, autotune != 0, fp64_kernel, angle_pass);
  }
  if (rc) return rc;
  sweeper->impl_ = S.release();
  return MSB_OK;
}

extern "C" void Sweeper_create(Sweeper* sweeper, Dimensions dims, const Quantities* quan, Env* env, Arguments* args) {
  msb::insist_status(Sweeper_create_status(sweeper, dims, quan, env, args), "Sweeper_create");
}

extern "C" void Sweeper_destroy(Sweeper* sweeper, Env* env) {
  (void)env;
  delete impl_of(sweeper);
  sweeper->impl_ = nullptr;
}

extern "C" int Sweeper_sweep_device(Sweeper* sweeper, double* vo_d, const double* vi_d, const Quantities* quan,
                                    Env* env) {
  SweeperImpl* S = impl_of(sweeper);
  if (!S) return msb::set_error(MSB_ERR_ARG, "Sweeper not created");
  if (!vo_d || !vi_d || !quan) return msb::set_error(MSB_ERR_ARG, "null argument");
  const bool mats_on_dev = quan->a_from_m.d_ && quan->m_from_a.d_;
  if (S->kba)
    return msb::kba_sweep(*S, vo_d, vi_d, quan->a_from_m.h_, quan->m_from_a.h_,
                          mats_on_dev ? quan->a_from_m.d_ : nullptr, mats_on_dev ? quan->m_from_a.d_ : nullptr,
                          env, stream_of(env));
  return msb::impl_sweep(*S, vo_d, vi_d, quan->a_from_m.h_, quan->m_from_a.h_,
                         mats_on_dev ? quan->a_from_m.d_ : nullptr, mats_on_dev ? quan->m_from_a.d_ : nullptr,
                         stream_of(env));
}

extern "C" int Sweeper_sync_status(Sweeper* sweeper, Env* env) {
  SweeperImpl* S = impl_of(sweeper);
  if (!S) return msb::set_error(MSB_ERR_ARG, "Sweeper not created");
  return msb::impl_sync(*S, stream_of(env));
}

// Reference semantics: the sweep reads the host copy of vi and leaves the
// host copy of vo complete (sweeper_kba_c.h:719-781 stages every z-block).
extern "C" int Sweeper_sweep_status(Sweeper* sweeper, Pointer* vo, Pointer* vi, const Quantities* quan, Env* env) {
  SweeperImpl* S = impl_of(sweeper);
  if (!S) return msb::set_error(MSB_ERR_ARG, "Sweeper not created");
  const size_t n = Dimensions_size_state(S->dims, NU);
  if (vi->n_ < n || vo->n_ < n || !vi->h_ || !vo->h_) return msb::set_error(MSB_ERR_ARG, "state arrays too small");
  cudaStream_t st = stream_of(env);
  int rc;
  double* vi_d = vi->d_;
  double* vo_d = vo->d_;
  if (!vi_d || !vo_d) {
    if (!S->d_vi && (rc = msb::cuda_check(cudaMalloc(&S->d_vi, n * sizeof(double)), "cudaMalloc vi"))) return rc;
    if (!S->d_vo && (rc = msb::cuda_check(cudaMalloc(&S->d_vo, n * sizeof(double)), "cudaMalloc vo"))) return rc;
    if (!vi_d) vi_d = S->d_vi;
    if (!vo_d) vo_d = S->d_vo;
  }
  // a large FP64 problem: the copies overlap the sweep, slice by slice
  const int nslice = quan && vi_d != vo_d ? msb::slice_count(*S) : 1;
  S->run_slices = nslice;
  if (nslice > 1) {
    const bool mats_on_dev = quan->a_from_m.d_ && quan->m_from_a.d_;
    return msb::sweep_iterations_sliced(*S, nslice, vo->h_, vi->h_, 1, vi_d, vo_d, quan->a_from_m.h_,
                                        quan->m_from_a.h_, mats_on_dev ? quan->a_from_m.d_ : nullptr,
                                        mats_on_dev ? quan->m_from_a.d_ : nullptr, st);
  }
  if ((rc = msb::cuda_check(cudaMemcpyAsync(vi_d, vi->h_, n * sizeof(double), cudaMemcpyHostToDevice, st), "vi H2D")))
    return rc;
  if ((rc = Sweeper_sweep_device(sweeper, vo_d, vi_d, quan, env))) return rc;
  if ((rc = msb::cuda_check(cudaMemcpyAsync(vo->h_, vo_d, n * sizeof(double), cudaMemcpyDeviceToHost, st), "vo D2H")))
    return rc;
  return msb::impl_sync(*S, st);
}

extern "C" void Sweeper_sweep(Sweeper* sweeper, Pointer* vo, Pointer* vi, const Quantities* quan, Env* env) {
  msb::insist_status(Sweeper_sweep_status(sweeper, vo, vi, quan, env), "Sweeper_sweep");
}

extern "C" int Sweeper_last_stats(const Sweeper* sweeper, long long* ntask, int* nlaunch) {
  const SweeperImpl* S = impl_of(sweeper);
  if (!S) return msb::set_error(MSB_ERR_ARG, "Sweeper not created");
  if (ntask) *ntask = S->sched.ntask();
  if (nlaunch) *nlaunch = S->nlaunch;
  return MSB_OK;
}

extern "C" int Sweeper_tile(const Sweeper* sweeper, int* tx, int* ty, float* ms_chosen, float* ms_other) {
  const SweeperImpl* S = impl_of(sweeper);
  if (!S) return msb::set_error(MSB_ERR_ARG, "Sweeper not created");
  if (tx) *tx = S->var.tx;
  if (ty) *ty = S->var.ty;
  if (ms_chosen) *ms_chosen = S->tuned ? S->tune_ms[0] : 0.f;
  if (ms_other) *ms_other = S->tuned ? S->tune_ms[1] : 0.f;
  return MSB_OK;
}

extern "C" int Sweeper_plan(const Sweeper* sweeper, int* fp64_kernel, int* task_window, int* l2_hints,
                            int* ncandidates, int* angle_pass) {
  const SweeperImpl* S = impl_of(sweeper);
  if (!S) return msb::set_error(MSB_ERR_ARG, "Sweeper not created");
  if (fp64_kernel) *fp64_kernel = S->var.kernel;
  if (task_window) *task_window = S->window;
  if (l2_hints) *l2_hints = S->l2_hints;
  if (ncandidates) *ncandidates = S->autotune ? 1 + (int)S->alts.size() : 1;
  if (angle_pass) *angle_pass = S->var.pass;
  return MSB_OK;
}

extern "C" long long Sweeper_debug_tasks(const Sweeper* sweeper, int* out, long long max_tasks) {
  const SweeperImpl* S = impl_of(sweeper);
  if (!S) return msb::set_error(MSB_ERR_ARG, "Sweeper not created");
  const long long n = S->sched.ntask();
  if (out) {
    const long long m = std::min(n, max_tasks);
    memcpy(out, S->sched.rec.data(), (size_t)m * MSB_TASK_INTS * sizeof(int));
  }
  return n;
}

extern "C" int msb_iterations_slices(const Sweeper* sweeper) {
  const SweeperImpl* S = impl_of(sweeper);
  if (!S) return msb::set_error(MSB_ERR_ARG, "Sweeper not created");
  return S->run_slices;
}

extern "C" int Sweeper_set_spin_limit(Sweeper* sweeper, long long limit) {
  SweeperImpl* S = impl_of(sweeper);
  if (!S) return msb::set_error(MSB_ERR_ARG, "Sweeper not created");
  S->timeout_ns = limit > 0 ? limit : msb::kDefaultTimeoutNs;
  return MSB_OK;
}

// A whole run of the reference driver's iteration loop (runner.c:148-155) on
// the device: v_in_h (host) is copied in once, niterations sweeps ping-pong
// between two device arrays (the vi/vo swap), and the last sweep's output is
// copied to v_out_h.  Pinned host buffers make the copies asynchronous; on a
// large problem the run goes in group-pair slices whose copies overlap
// the other slices' sweeps (sweep_iterations_sliced).
extern "C" int Sweeper_sweep_iterations(Sweeper* sweeper, double* v_out_h, const double* v_in_h, int niterations,
                                        const Quantities* quan, Env* env) {
  SweeperImpl* S = impl_of(sweeper);
  if (!S) return msb::set_error(MSB_ERR_ARG, "Sweeper not created");
  if (!v_out_h || !v_in_h || niterations < 0) return msb::set_error(MSB_ERR_ARG, "invalid argument");
  const size_t n = Dimensions_size_state(S->dims, NU);
  cudaStream_t st = stream_of(env);
  int rc;
  if (!S->d_vi && (rc = msb::cuda_check(cudaMalloc(&S->d_vi, n * sizeof(double)), "cudaMalloc vi"))) return rc;
  if (!S->d_vo && (rc = msb::cuda_check(cudaMalloc(&S->d_vo, n * sizeof(double)), "cudaMalloc vo"))) return rc;
  const int nslice = niterations > 0 && quan ? msb::slice_count(*S) : 1;
  S->run_slices = nslice;
  if (nslice > 1) {
    const bool mats_on_dev = quan->a_from_m.d_ && quan->m_from_a.d_;
    return msb::sweep_iterations_sliced(*S, nslice, v_out_h, v_in_h, niterations, S->d_vi, S->d_vo,
                                        quan->a_from_m.h_, quan->m_from_a.h_,
                                        mats_on_dev ? quan->a_from_m.d_ : nullptr,
                                        mats_on_dev ? quan->m_from_a.d_ : nullptr, st);
  }
  if ((rc = msb::cuda_check(cudaMemcpyAsync(S->d_vi, v_in_h, n * sizeof(double), cudaMemcpyHostToDevice, st), "H2D")))
    return rc;
  double* a = S->d_vi;
  double* b = S->d_vo;
  for (int it = 0; it < niterations; ++it) {
    if ((rc = Sweeper_sweep_device(sweeper, b, a, quan, env))) return rc;
    double* tmp = a;
    a = b;
    b = tmp;
  }
  if ((rc = msb::cuda_check(cudaMemcpyAsync(v_out_h, a, n * sizeof(double), cudaMemcpyDeviceToHost, st), "D2H")))
    return rc;
  return msb::impl_sync(*S, st);
}

// ------------------------------------------------ decomposed sweep by steps
static SweeperImpl* kba_impl(const Sweeper* sweeper) {
  SweeperImpl* S = impl_of(sweeper);
  if (!S) {
    msb::set_error(MSB_ERR_ARG, "Sweeper not created");
    return nullptr;
  }
  if (!S->kba) {
    msb::set_error(MSB_ERR_ARG, "the Sweeper is not decomposed (nproc_x * nproc_y == 1)");
    return nullptr;
  }
  return S;
}

extern "C" int msb_kba_info(const Sweeper* sweeper, int* nstep, size_t* bytes_x, size_t* bytes_y) {
  const SweeperImpl* S = kba_impl(sweeper);
  if (!S) return MSB_ERR_ARG;
  if (nstep) *nstep = S->kba->plan.nstep;
  if (bytes_x) *bytes_x = S->kba->msg_bytes(0);
  if (bytes_y) *bytes_y = S->kba->msg_bytes(1);
  return MSB_OK;
}

extern "C" int msb_kba_set_buffers(Sweeper* sweeper, void* send_x, void* send_y, void* recv_x_lo, void* recv_x_hi,
                                   void* recv_y_lo, void* recv_y_hi) {
  SweeperImpl* S = kba_impl(sweeper);
  if (!S) return MSB_ERR_ARG;
  void* b[6] = {send_x, send_y, recv_x_lo, recv_x_hi, recv_y_lo, recv_y_hi};
  for (int i = 0; i < 6; ++i) S->kba->buf[i] = b[i];
  return MSB_OK;
}

extern "C" int msb_kba_begin(Sweeper* sweeper, double* vo_d, const double* vi_d, const Quantities* quan, Env* env) {
  SweeperImpl* S = kba_impl(sweeper);
  if (!S) return MSB_ERR_ARG;
  if (!vo_d || !vi_d || !quan) return msb::set_error(MSB_ERR_ARG, "null argument");
  int rc = msb::kba_own_buffers(*S);
  if (rc) return rc;
  const bool mats_on_dev = quan->a_from_m.d_ && quan->m_from_a.d_;
  return msb::kba_begin(*S, vo_d, vi_d, quan->a_from_m.h_, quan->m_from_a.h_,
                        mats_on_dev ? quan->a_from_m.d_ : nullptr, mats_on_dev ? quan->m_from_a.d_ : nullptr,
                        stream_of(env));
}

extern "C" int msb_kba_step(Sweeper* sweeper, int step, Env* env) {
  SweeperImpl* S = kba_impl(sweeper);
  if (!S) return MSB_ERR_ARG;
  if (step < 0 || step >= S->kba->plan.nstep) return msb::set_error(MSB_ERR_ARG, "step %d out of range", step);
  return msb::kba_step(*S, step, stream_of(env));
}

extern "C" int msb_kba_messages(const Sweeper* sweeper, int step, msb_kba_msg* msgs, int max_msgs) {
  const SweeperImpl* S = kba_impl(sweeper);
  if (!S) return MSB_ERR_ARG;
  if (step < 0 || step >= S->kba->plan.nstep) return msb::set_error(MSB_ERR_ARG, "step %d out of range", step);
  std::vector<msb_kba_msg> v;
  const int n = msb::kba_message_list(*S, step, v);
  for (int i = 0; i < n && i < max_msgs; ++i) msgs[i] = v[i];
  return n;
}

extern "C" int msb_kba_unpack(Sweeper* sweeper, int step, Env* env) {
  SweeperImpl* S = kba_impl(sweeper);
  if (!S) return MSB_ERR_ARG;
  if (step < 0 || step >= S->kba->plan.nstep) return msb::set_error(MSB_ERR_ARG, "step %d out of range", step);
  return msb::kba_unpack(*S, step, stream_of(env));
}

extern "C" int msb_kba_end(Sweeper* sweeper, Env* env) {
  SweeperImpl* S = kba_impl(sweeper);
  if (!S) return MSB_ERR_ARG;
  int rc = msb::cuda_check(cudaStreamSynchronize(stream_of(env)), "sweep");
  return S->kba->rc ? S->kba->rc : rc;
}
