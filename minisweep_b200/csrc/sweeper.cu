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
#include <cstdint>
#include <memory>
#include <new>
#include <type_traits>

#include "internal.h"
#include "sweep_fp64_ws.cuh"
#include "sweep_mixed_tc.cuh"

namespace msb {

namespace {

using KernelFn = void (*)(const Fp64Params);
using MixKernelFn = void (*)(const MixParams);

// One compiled kernel: the FP64 kernel (fn) or a mixed-precision one (mix).
struct Variant {
  KernelFn fn = nullptr;
  MixKernelFn mix = nullptr;
  size_t smem = 0;
  size_t entry_bytes = 0;  // one face entry (octant, group pair, position)
  int tx = 0, ty = 0, nch = 0, threads = 0;
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
  return v;
}

template <int NM_>
Variant pick_nch(int nch) {
  switch (nch) {
    case 1: return make_variant<NM_, 1, 4, 2>();
    case 2: return make_variant<NM_, 2, 4, 2>();
    case 3:
    case 4: return make_variant<NM_, 4, 2, 2>();
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
  v.smem = C::smem_bytes();
  v.entry_bytes = C::EB;
  v.tx = C::TX;
  v.ty = C::TY;
  v.nch = 1;
  v.threads = C::NT;
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

// precision 0: FP64; 1: mixed with FP16 halves; 2: mixed with BF16 halves
// (the mixed kernels take na <= 32).
Variant pick_variant(int nm, int na, int precision) {
  if (precision == 1 || precision == 2) {
    if (na > 32) return Variant();
    return precision == 1 ? pick_mixed<MIX_F16>(nm) : pick_mixed<MIX_BF16>(nm);
  }
  if (precision != 0) return Variant();
  const int nch = (na + 31) / 32;
  switch (nm) {
    case 4: return pick_nch<4>(nch);
    case 8: return pick_nch<8>(nch);
    case 16: return pick_nch<16>(nch);
    default: return Variant();
  }
}

constexpr long long kDefaultTimeoutNs = 4000000000LL;  // 4 s per wait

// cuTensorMapEncodeTiled from the driver, through the runtime (no -lcuda).
PFN_cuTensorMapEncodeTiled_v12000 tensor_map_encoder() {
  static PFN_cuTensorMapEncodeTiled_v12000 fn = nullptr;
  static bool tried = false;
  if (!tried) {
    tried = true;
    void* p = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) == cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      fn = reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(p);
  }
  return fn;
}

// The state array (im fastest, then iu, ix, iy, ie, iz) as a 5-D tensor
// (moment, unknown * x, y, group, z) whose box is one cell: NM moments x 4
// unknowns x 1 x (2 groups, 1 when ne == 1) x 1, copied with the swizzle the
// mixed kernel reads with.
int encode_state_map(CUtensorMap* map, const double* ptr, const Dimensions& d, int* box_bytes) {
  PFN_cuTensorMapEncodeTiled_v12000 enc = tensor_map_encoder();
  if (!enc) return set_error(MSB_ERR_CUDA, "cuTensorMapEncodeTiled is not available from the driver");
  if (reinterpret_cast<uintptr_t>(ptr) % 16 != 0)
    return set_error(MSB_ERR_ARG, "the mixed-precision sweep needs 16-byte aligned state arrays");
  const cuuint64_t row = (cuuint64_t)d.nm * sizeof(double);
  const cuuint64_t dims[5] = {(cuuint64_t)d.nm, (cuuint64_t)NU * d.ncell_x, (cuuint64_t)d.ncell_y, (cuuint64_t)d.ne,
                              (cuuint64_t)d.ncell_z};
  const cuuint64_t strides[4] = {row, row * NU * d.ncell_x, row * NU * d.ncell_x * d.ncell_y,
                                 row * NU * d.ncell_x * d.ncell_y * d.ne};
  const cuuint32_t ng = d.ne >= 2 ? 2 : 1;
  const cuuint32_t box[5] = {(cuuint32_t)d.nm, (cuuint32_t)NU, 1, ng, 1};
  const cuuint32_t estr[5] = {1, 1, 1, 1, 1};
  const CUtensorMapSwizzle swz = d.nm == 16 ? CU_TENSOR_MAP_SWIZZLE_128B
                                 : d.nm == 8 ? CU_TENSOR_MAP_SWIZZLE_64B
                                             : CU_TENSOR_MAP_SWIZZLE_32B;
  const CUresult r = enc(map, CU_TENSOR_MAP_DATA_TYPE_FLOAT64, 5, const_cast<double*>(ptr), dims, strides, box, estr,
                         CU_TENSOR_MAP_INTERLEAVE_NONE, swz, CU_TENSOR_MAP_L2_PROMOTION_L2_128B,
                         CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  if (r != CUDA_SUCCESS) return set_error(MSB_ERR_CUDA, "cuTensorMapEncodeTiled failed (%d)", (int)r);
  *box_bytes = (int)(d.nm * sizeof(double) * NU * ng);
  return MSB_OK;
}

}  // namespace

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
  size_t part_elems = 0;
  double* d_vi = nullptr;  // staging for host-only Pointers
  double* d_vo = nullptr;
  long long timeout_ns = kDefaultTimeoutNs;
  int nlaunch = 0;
  int nsm = 0;
  int* h_status = nullptr;  // pinned copy of the status words

  ~SweeperImpl() {
    cudaFree(d_tasks);
    cudaFree(d_sync);
    for (auto& f : d_face) cudaFree(f);
    cudaFree(d_afm);
    cudaFree(d_mfa);
    cudaFree(d_part);
    cudaFree(d_vi);
    cudaFree(d_vo);
    if (h_status) cudaFreeHost(h_status);
  }
};

static int impl_create(SweeperImpl& S, const Dimensions& dims, int precision) {
  S.dims = dims;
  S.precision = precision;
  if (dims.ncell_x <= 0 || dims.ncell_y <= 0 || dims.ncell_z <= 0 || dims.ne <= 0 || dims.na <= 0)
    return set_error(MSB_ERR_ARG, "invalid dimensions");
  S.var = pick_variant(dims.nm, dims.na, precision);
  if (!S.var.valid())
    return set_error(MSB_ERR_UNSUPPORTED,
                     "no kernel variant for nm=%d na=%d precision=%d (nm in {4,8,16}; na <= 128 for FP64, "
                     "na <= 32 for the mixed kernels)",
                     dims.nm, dims.na, precision);
  S.ngp = (dims.ne + 1) / 2;
  int rc, dev = 0, nsm = 0, occ = 0;
  if ((rc = cuda_check(cudaGetDevice(&dev), "cudaGetDevice"))) return rc;
  if ((rc = cuda_check(cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev), "SM count"))) return rc;
  S.gp_block = pick_gp_block(dims.ncell_x, dims.ncell_y, S.ngp, S.var.tx, S.var.ty, 2 * nsm);
  rc = build_schedule(dims.ncell_x, dims.ncell_y, dims.ncell_z, S.ngp, S.var.tx, S.var.ty, S.gp_block, S.sched);
  if (rc) return rc;
  const long long ntask = S.sched.ntask();
  if (ntask >= (1LL << 31) - SY_PROGRESS) return set_error(MSB_ERR_ARG, "too many tasks");

  if ((rc = cuda_check(cudaMalloc(&S.d_tasks, S.sched.rec.size() * sizeof(int)), "cudaMalloc tasks"))) return rc;
  if ((rc = cuda_check(cudaMemcpy(S.d_tasks, S.sched.rec.data(), S.sched.rec.size() * sizeof(int),
                                  cudaMemcpyHostToDevice), "copy tasks")))
    return rc;
  S.sync_ints = SY_PROGRESS + (size_t)ntask;
  if ((rc = cuda_check(cudaMalloc(&S.d_sync, S.sync_ints * sizeof(int)), "cudaMalloc sync"))) return rc;
  if ((rc = cuda_check(cudaMallocHost(&S.h_status, 8 * sizeof(int)), "cudaMallocHost status"))) return rc;

  const size_t per = (size_t)NOCTANT * S.ngp * S.var.entry_bytes;
  S.face_bytes[0] = per * dims.ncell_y * dims.ncell_x;
  S.face_bytes[1] = per * dims.ncell_z * dims.ncell_x;
  S.face_bytes[2] = per * dims.ncell_z * dims.ncell_y;
  for (int f = 0; f < 3; ++f)
    if ((rc = cuda_check(cudaMalloc(&S.d_face[f], S.face_bytes[f]), "cudaMalloc faces"))) return rc;
  if (S.var.mix) {
    S.part_elems = (size_t)NOCTANT * Dimensions_size_state(dims, NU);
    if ((rc = cuda_check(cudaMalloc(&S.d_part, S.part_elems * sizeof(float)), "cudaMalloc octant partials")))
      return rc;
  }
  const size_t nmat = (size_t)dims.nm * dims.na * NOCTANT;
  if ((rc = cuda_check(cudaMalloc(&S.d_afm, nmat * sizeof(double)), "cudaMalloc a_from_m"))) return rc;
  if ((rc = cuda_check(cudaMalloc(&S.d_mfa, nmat * sizeof(double)), "cudaMalloc m_from_a"))) return rc;

  if ((rc = cuda_check(cudaFuncSetAttribute(S.var.func(), cudaFuncAttributeMaxDynamicSharedMemorySize,
                                            (int)S.var.smem),
                       "cudaFuncSetAttribute")))
    return rc;
  if ((rc = cuda_check(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, S.var.func(), S.var.threads,
                                                                     S.var.smem),
                       "occupancy")))
    return rc;
  if (occ < 1) return set_error(MSB_ERR_UNSUPPORTED, "sweep kernel does not fit on an SM");
  S.grid = (int)std::min<long long>(ntask, (long long)nsm * occ);
  S.nsm = nsm;
  return MSB_OK;
}

// Launches one sweep: vo_d = sweep(vi_d), asynchronously on `stream`.
static int impl_sweep(SweeperImpl& S, double* vo_d, const double* vi_d, const double* afm_h, const double* mfa_h,
                      const double* afm_d, const double* mfa_d, cudaStream_t stream) {
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
  if ((rc = cuda_check(cudaMemsetAsync(S.d_sync, 0, S.sync_ints * sizeof(int), stream), "reset sync"))) return rc;
  // problem fields (X) and schedule fields (P)
  auto fill = [&](auto& X, auto& P, auto* face) {
    using F = std::remove_pointer_t<decltype(face)>;
    X.vi = vi_d;
    X.afm = S.d_afm;
    X.mfa = S.d_mfa;
    X.fxy = static_cast<F*>(S.d_face[0]);
    X.fxz = static_cast<F*>(S.d_face[1]);
    X.fyz = static_cast<F*>(S.d_face[2]);
    X.nx = S.dims.ncell_x;
    X.ny = S.dims.ncell_y;
    X.nz = S.dims.ncell_z;
    X.ne = S.dims.ne;
    X.na = S.dims.na;
    X.ngp = S.ngp;
    P.tasks = S.d_tasks;
    P.ntask = S.sched.ntask();
    P.sy.sync = S.d_sync;
    P.sy.timeout_ns = S.timeout_ns;
  };
  if (S.var.fn) {
    Fp64Params P;
    fill(P.pr, P, (double*)nullptr);
    P.pr.vo = vo_d;
    S.var.fn<<<S.grid, S.var.threads, S.var.smem, stream>>>(P);
  } else {
    MixParams P;
    fill(P, P, (float*)nullptr);
    P.part = S.d_part;
    P.state = S.part_elems / NOCTANT;
    if ((rc = encode_state_map(&P.tm_vi, vi_d, S.dims, &P.vbox_bytes))) return rc;
    S.var.mix<<<S.grid, S.var.threads, S.var.smem, stream>>>(P);
    if ((rc = cuda_check(cudaGetLastError(), "sweep kernel launch"))) return rc;
    reduce_octant_partials<<<S.nsm * 8, 256, 0, stream>>>(vo_d, S.d_part, P.state);
  }
  if ((rc = cuda_check(cudaGetLastError(), "sweep kernel launch"))) return rc;
  if ((rc = cuda_check(cudaMemcpyAsync(S.h_status, S.d_sync, 4 * sizeof(int), cudaMemcpyDeviceToHost, stream),
                       "status copy")))
    return rc;
  S.nlaunch = S.var.mix ? 2 : 1;
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
  (void)env;

  std::unique_ptr<SweeperImpl> S(new (std::nothrow) SweeperImpl());
  if (!S) return msb::set_error(MSB_ERR_ARG, "out of host memory");
  const int rc = msb::impl_create(*S, dims, sweeper->precision);
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

extern "C" int Sweeper_set_spin_limit(Sweeper* sweeper, long long limit) {
  SweeperImpl* S = impl_of(sweeper);
  if (!S) return msb::set_error(MSB_ERR_ARG, "Sweeper not created");
  S->timeout_ns = limit > 0 ? limit : msb::kDefaultTimeoutNs;
  return MSB_OK;
}

// A whole run of the reference driver's iteration loop (runner.c:148-155) on
// the device: v_in_h (host) is copied in once, niterations sweeps ping-pong
// between two device arrays (the vi/vo swap), and the last sweep's output is
// copied to v_out_h.  Pinned host buffers make the copies asynchronous.
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
