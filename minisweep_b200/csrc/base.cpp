// base.cpp -- host runtime behind the reference-compatible C API:
// Insist, Arguments (read-once flags), Env (one process, one GPU), Pointer
// (host array + device mirror), Dimensions sizes, the built-in Quantities and
// the host array operations.
//
// Reference behaviour followed (file:line in olcf/minisweep):
//   Insist message/exit           src/1_base/env_assert.c:27-32
//   Arguments parsing             src/1_base/arguments.c:37-198
//   Env (process grid, group)     src/1_base/env_mpi.c:100-480
//   --is_using_device             src/1_base/env_cuda.c:84-92
//   Pointer                       src/1_base/pointer.c:36-267
//   Dimensions sizes              src/2_sweeper_base/dimensions.c:36-101
//   built-in Quantities           src/3_sweeper/quantities_testing_c.h:28-359,
//                                 quantities_testing.h:60-90
//   initialize_state / norms      src/2_sweeper_base/array_operations.c:26-110
#include "minisweep_b200.h"

#include <cuda_runtime.h>
#include <sys/time.h>

#include <cstdarg>
#include <cstdint>
#include <string>
#include <vector>

#include "internal.h"

// ------------------------------------------------------------------ errors
namespace msb {
static thread_local std::string g_last_error;

int set_error(int code, const char* fmt, ...) {
  char buf[1024];
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(buf, sizeof buf, fmt, ap);
  va_end(ap);
  g_last_error = buf;
  return code;
}

int cuda_check(cudaError_t e, const char* what) {
  if (e == cudaSuccess) return MSB_OK;
  return set_error(MSB_ERR_CUDA, "CUDA error in %s: %s", what, cudaGetErrorString(e));
}

void insist_status(int rc, const char* what) {
  if (rc != MSB_OK) {
    fprintf(stderr, "Insist error: \"%s\": %s\n", what, g_last_error.c_str());
    exit(EXIT_FAILURE);
  }
}
}  // namespace msb

extern "C" const char* msb_last_error(void) { return msb::g_last_error.c_str(); }

extern "C" void insist_(const char* condition_string, const char* file, int line) {
  fprintf(stderr, "Insist error: \"%s\". At file %s, line %i.\n", condition_string, file, line);
  exit(EXIT_FAILURE);
}

// --------------------------------------------------------------- arguments
extern "C" Arguments Arguments_null(void) {
  Arguments a;
  memset(&a, 0, sizeof a);
  return a;
}

extern "C" void Arguments_create(Arguments* args, int argc, char** argv) {
  args->argc = argc;
  args->argv_unconsumed = (char**)malloc((argc > 0 ? argc : 1) * sizeof(char*));
  args->argstring = nullptr;
  for (int i = 0; i < argc; ++i) args->argv_unconsumed[i] = argv[i];
}

extern "C" void Arguments_create_from_string(Arguments* args, const char* argstring) {
  const size_t len = strlen(argstring);
  args->argstring = (char*)malloc(len + 1);
  memcpy(args->argstring, argstring, len + 1);
  // argv[0] is an empty program name, as in the reference (arguments.c:68-72)
  args->argv_unconsumed = (char**)malloc((len + 2) * sizeof(char*));
  args->argv_unconsumed[0] = &args->argstring[len];
  args->argc = 1;
  bool prev_delim = true;
  for (size_t i = 0; i < len; ++i) {
    if (args->argstring[i] == ' ' || args->argstring[i] == '\t') args->argstring[i] = 0;
    const bool delim = args->argstring[i] == 0;
    if (prev_delim && !delim) args->argv_unconsumed[args->argc++] = &args->argstring[i];
    prev_delim = delim;
  }
}

extern "C" void Arguments_destroy(Arguments* args) {
  free(args->argv_unconsumed);
  if (args->argstring) free(args->argstring);
  args->argv_unconsumed = nullptr;
  args->argstring = nullptr;
}

extern "C" Bool_t Arguments_exists(const Arguments* args, const char* arg_name) {
  for (int i = 0; i < args->argc; ++i)
    if (args->argv_unconsumed[i] && strcmp(args->argv_unconsumed[i], arg_name) == 0)
      return Bool_true;
  return Bool_false;
}

extern "C" int Arguments_consume_int_(Arguments* args, const char* arg_name) {
  int result = 0;
  bool found = false;
  for (int i = 0; i < args->argc; ++i) {
    if (!args->argv_unconsumed[i]) continue;
    if (strcmp(args->argv_unconsumed[i], arg_name) == 0) {
      found = true;
      args->argv_unconsumed[i] = nullptr;
      ++i;
      Insist(i < args->argc);
      result = atoi(args->argv_unconsumed[i]);
      args->argv_unconsumed[i] = nullptr;
    }
  }
  Insist(found ? "Invalid use of argument." : 0);
  return result;
}

extern "C" int Arguments_consume_int_or_default(Arguments* args, const char* arg_name,
                                                int default_value) {
  return Arguments_exists(args, arg_name) ? Arguments_consume_int_(args, arg_name)
                                          : default_value;
}

extern "C" Bool_t Arguments_are_all_consumed(const Arguments* args) {
  for (int i = 1; i < args->argc; ++i)
    if (args->argv_unconsumed[i] != nullptr) return Bool_false;
  return Bool_true;
}

// --------------------------------------------------------------------- env
extern "C" Env Env_null(void) {
  Env e;
  memset(&e, 0, sizeof e);
  return e;
}

extern "C" void Env_initialize(Env* env, int argc, char** argv) {
  (void)argc;
  (void)argv;
  env->nproc_x_ = 1;
  env->nproc_y_ = 1;
  env->is_proc_active_ = Bool_true;
  // env_mpi.c:75-95 joins MPI_COMM_WORLD here: a process started by the
  // node launcher joins its group (and takes its GPU) the same way
  msb::insist_status(msb::node_attach(env), "Env_initialize: process group");
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess) dev = 0;
  env->device_ = dev;
  cudaStream_t s = nullptr;
  if (cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking) != cudaSuccess) {
    cudaGetLastError();
    s = nullptr;
  }
  env->stream_kernel_faces_ = (Stream_t)s;
}

extern "C" int msb_env_set_comm(Env* env, int proc, int nproc, const msb_comm* comm) {
  if (!env || nproc < 1 || proc < 0 || proc >= nproc)
    return msb::set_error(MSB_ERR_ARG, "msb_env_set_comm: proc %d of %d", proc, nproc);
  if (nproc > 1 && (!comm || !comm->exchange || !comm->sum_double || !comm->allgather_int || !comm->barrier))
    return msb::set_error(MSB_ERR_ARG, "msb_env_set_comm: a group of %d processes needs every callback", nproc);
  env->proc_ = proc;
  env->nproc_world_ = nproc;
  env->comm_ = nproc > 1 ? comm : nullptr;
  return MSB_OK;
}

static int nproc_world(const Env* env) { return env->nproc_world_ > 0 ? env->nproc_world_ : 1; }

extern "C" void Env_set_values(Env* env, Arguments* args) {
  // env_mpi.c:114-135: the requested grid must fit the processes there are;
  // process numbers beyond it are inactive.
  const int npx = Arguments_consume_int_or_default(args, "--nproc_x", 1);
  const int npy = Arguments_consume_int_or_default(args, "--nproc_y", 1);
  Insist(npx > 0 ? "Invalid nproc_x supplied." : 0);
  Insist(npy > 0 ? "Invalid nproc_y supplied." : 0);
  const int requested = npx * npy, world = nproc_world(env);
  Insist(requested <= world ? "Not enough processors available." : 0);
  env->nproc_x_ = npx;
  env->nproc_y_ = npy;
  env->is_proc_active_ = env->proc_ < requested ? Bool_true : Bool_false;
  env->tag_ = 0;
  // env_cuda.c:87-92
  env->is_using_device_ = Arguments_consume_int_or_default(args, "--is_using_device", 0);
  Insist(env->is_using_device_ == 0 || env->is_using_device_ == 1
             ? "Invalid setting for is_using_device."
             : 0);
}

// The group's callbacks serve a decomposed grid only: a 1 x 1 run is process
// 0 alone and talks to nobody.
static const msb_comm* grid_comm(const Env* env) {
  return env && env->comm_ && env->nproc_x_ * env->nproc_y_ > 1 ? env->comm_ : nullptr;
}

extern "C" void Env_finalize(Env* env) {
  if (env->stream_kernel_faces_) cudaStreamDestroy((cudaStream_t)env->stream_kernel_faces_);
  env->stream_kernel_faces_ = nullptr;
  msb::node_detach(env);
}

extern "C" Bool_t Env_is_proc_master(Env* env) { return Env_is_proc_active(env) && Env_proc_this(env) == 0; }

extern "C" Timer Env_get_time(Env* env) {
  (void)env;
  struct timeval tv;
  gettimeofday(&tv, nullptr);
  return (Timer)tv.tv_sec + (Timer)tv.tv_usec * 1.e-6;
}

extern "C" Timer Env_get_synced_time(Env* env) {
  // The reference barriers its ranks here (env.c:81-85): drain the device
  // work queued on the Env's stream, then the group's barrier.
  if (env && env->stream_kernel_faces_) cudaStreamSynchronize((cudaStream_t)env->stream_kernel_faces_);
  Env_mpi_barrier(env);
  return Env_get_time(env);
}

extern "C" int Env_nproc_x(const Env* env) { return env->nproc_x_ > 0 ? env->nproc_x_ : 1; }
extern "C" int Env_nproc_y(const Env* env) { return env->nproc_y_ > 0 ? env->nproc_y_ : 1; }
extern "C" int Env_nproc(const Env* env) { return Env_nproc_x(env) * Env_nproc_y(env); }
extern "C" Bool_t Env_is_proc_active(const Env* env) { return env->is_proc_active_ ? Bool_true : Bool_false; }
extern "C" int Env_tag(const Env* env) { return env->tag_; }
extern "C" void Env_increment_tag(Env* env, int value) { env->tag_ += value; }
extern "C" int Env_proc(const Env* env, int proc_x, int proc_y) { return proc_x + Env_nproc_x(env) * proc_y; }
extern "C" int Env_proc_x(const Env* env, int proc) { return proc % Env_nproc_x(env); }
extern "C" int Env_proc_y(const Env* env, int proc) { return proc / Env_nproc_x(env); }
extern "C" int Env_proc_this(const Env* env) { return env->proc_; }
extern "C" int Env_proc_x_this(const Env* env) { return Env_proc_x(env, Env_proc_this(env)); }
extern "C" int Env_proc_y_this(const Env* env) { return Env_proc_y(env, Env_proc_this(env)); }
extern "C" void Env_mpi_barrier(Env* env) {
  const msb_comm* c = grid_comm(env);
  if (c) Insist(c->barrier(c->ctx, Env_nproc(env)) == 0 ? "barrier failed." : 0);
}
extern "C" double Env_sum_d(Env* env, double value) {
  // env_mpi.c:309-323: a sum over the active processes
  const msb_comm* c = grid_comm(env);
  if (c) Insist(c->sum_double(c->ctx, Env_nproc(env), &value) == 0 ? "sum over processes failed." : 0);
  return value;
}
extern "C" P Env_sum_P(Env* env, P value) { return Env_sum_d(env, value); }
extern "C" Bool_t Env_cuda_is_using_device(const Env* const env) { return env->is_using_device_; }
extern "C" Bool_t Env_cuda_last_call_succeeded(void) { return cudaPeekAtLastError() == cudaSuccess; }
extern "C" Stream_t Env_cuda_stream_kernel_faces(Env* env) { return env->stream_kernel_faces_; }
extern "C" void Env_cuda_stream_wait(Env* env, Stream_t stream) {
  (void)env;
  cudaStreamSynchronize((cudaStream_t)stream);
}

// ------------------------------------------------------------ memory helpers
extern "C" int* malloc_host_int(size_t n) { return (int*)malloc((n ? n : 1) * sizeof(int)); }
extern "C" P* malloc_host_P(size_t n) { return (P*)malloc((n ? n : 1) * sizeof(P)); }
extern "C" P* malloc_host_pinned_P(size_t n) {
  P* p = nullptr;
  msb::insist_status(msb::cuda_check(cudaMallocHost((void**)&p, (n ? n : 1) * sizeof(P)), "cudaMallocHost"),
                     "pinned host allocation");
  return p;
}
extern "C" P* malloc_device_P(size_t n) {
  P* p = nullptr;
  msb::insist_status(msb::cuda_check(cudaMalloc((void**)&p, (n ? n : 1) * sizeof(P)), "cudaMalloc"),
                     "device allocation");
  return p;
}
extern "C" void free_host_int(int* p) { free(p); }
extern "C" void free_host_P(P* p) { free(p); }
extern "C" void free_host_pinned_P(P* p) { cudaFreeHost(p); }
extern "C" void free_device_P(P* p) { cudaFree(p); }
extern "C" void cuda_copy_host_to_device_P(P* p_d, P* p_h, size_t n) {
  msb::insist_status(msb::cuda_check(cudaMemcpy(p_d, p_h, n * sizeof(P), cudaMemcpyHostToDevice), "cudaMemcpy H2D"),
                     "host to device copy");
}
extern "C" void cuda_copy_device_to_host_P(P* p_h, P* p_d, size_t n) {
  msb::insist_status(msb::cuda_check(cudaMemcpy(p_h, p_d, n * sizeof(P), cudaMemcpyDeviceToHost), "cudaMemcpy D2H"),
                     "device to host copy");
}

// ----------------------------------------------------------------- pointer
extern "C" Pointer Pointer_null(void) {
  Pointer p;
  memset(&p, 0, sizeof p);
  return p;
}
extern "C" void Pointer_create(Pointer* p, size_t n, Bool_t is_using_device) {
  *p = Pointer_null();
  p->n_ = n;
  p->is_using_device_ = is_using_device;
}
extern "C" void Pointer_create_alias(Pointer* p, Pointer* source, size_t base, size_t n) {
  *p = Pointer_null();
  p->n_ = n;
  p->is_using_device_ = source->is_using_device_;
  p->is_pinned_ = source->is_pinned_;
  p->is_alias_ = Bool_true;
  p->h_ = source->h_ ? source->h_ + base : nullptr;
  p->d_ = source->d_ ? source->d_ + base : nullptr;
}
extern "C" void Pointer_set_pinned(Pointer* p, Bool_t is_pinned) { p->is_pinned_ = is_pinned; }
extern "C" void Pointer_allocate_h_(Pointer* p) {
  p->h_ = p->is_pinned_ ? malloc_host_pinned_P(p->n_) : malloc_host_P(p->n_);
}
extern "C" void Pointer_allocate_d_(Pointer* p) {
  if (p->is_using_device_) p->d_ = malloc_device_P(p->n_);
}
extern "C" void Pointer_allocate(Pointer* p) {
  Insist(!p->is_alias_ ? "Cannot allocate an alias." : 0);
  Pointer_allocate_h_(p);
  Pointer_allocate_d_(p);
}
extern "C" void Pointer_deallocate_h_(Pointer* p) {
  if (p->h_ && !p->is_alias_) {
    if (p->is_pinned_) free_host_pinned_P(p->h_);
    else free_host_P(p->h_);
  }
  p->h_ = nullptr;
}
extern "C" void Pointer_deallocate_d_(Pointer* p) {
  if (p->d_ && !p->is_alias_) free_device_P(p->d_);
  p->d_ = nullptr;
}
extern "C" void Pointer_deallocate(Pointer* p) {
  Pointer_deallocate_h_(p);
  Pointer_deallocate_d_(p);
}
extern "C" void Pointer_destroy(Pointer* p) {
  Pointer_deallocate(p);
  *p = Pointer_null();
}
extern "C" void Pointer_update_h(Pointer* p) {
  if (p->is_using_device_ && p->d_ && p->h_) cuda_copy_device_to_host_P(p->h_, p->d_, p->n_);
}
extern "C" void Pointer_update_d(Pointer* p) {
  if (p->is_using_device_ && p->d_ && p->h_) cuda_copy_host_to_device_P(p->d_, p->h_, p->n_);
}
extern "C" void Pointer_update_h_stream(Pointer* p, Stream_t stream) {
  if (p->is_using_device_ && p->d_ && p->h_)
    msb::insist_status(msb::cuda_check(cudaMemcpyAsync(p->h_, p->d_, p->n_ * sizeof(P), cudaMemcpyDeviceToHost,
                                                       (cudaStream_t)stream),
                                       "cudaMemcpyAsync D2H"),
                       "device to host copy");
}
extern "C" void Pointer_update_d_stream(Pointer* p, Stream_t stream) {
  if (p->is_using_device_ && p->d_ && p->h_)
    msb::insist_status(msb::cuda_check(cudaMemcpyAsync(p->d_, p->h_, p->n_ * sizeof(P), cudaMemcpyHostToDevice,
                                                       (cudaStream_t)stream),
                                       "cudaMemcpyAsync H2D"),
                       "host to device copy");
}

// -------------------------------------------------------------- dimensions
extern "C" Dimensions Dimensions_null(void) {
  Dimensions d;
  memset(&d, 0, sizeof d);
  return d;
}
extern "C" size_t Dimensions_size_state(const Dimensions dims, int nu) {
  return (size_t)dims.ncell_x * dims.ncell_y * dims.ncell_z * dims.ne * dims.nm * nu;
}
extern "C" size_t Dimensions_size_state_angles(const Dimensions dims, int nu) {
  return (size_t)dims.ncell_x * dims.ncell_y * dims.ncell_z * dims.ne * dims.na * nu * NOCTANT;
}
extern "C" size_t Dimensions_size_facexy(const Dimensions dims, int nu, int noctant_per_block) {
  return (size_t)dims.ncell_x * dims.ncell_y * dims.ne * dims.na * nu * noctant_per_block;
}
extern "C" size_t Dimensions_size_facexz(const Dimensions dims, int nu, int noctant_per_block) {
  return (size_t)dims.ncell_x * dims.ncell_z * dims.ne * dims.na * nu * noctant_per_block;
}
extern "C" size_t Dimensions_size_faceyz(const Dimensions dims, int nu, int noctant_per_block) {
  return (size_t)dims.ncell_y * dims.ncell_z * dims.ne * dims.na * nu * noctant_per_block;
}

// -------------------------------------------------------------- quantities
namespace msb {
// Index-derived power-of-two scale factors of the built-in problem
// (quantities_testing_kernels.h:52-141, 203-214).
int scale_space(int ix, int iy, int iz) { return 1 << ((ix + 3 * iy + 7 * iz + 2) & 3); }
int scale_energy(int ie) { return 1 << (((ie * 1366 + 150889) % 714025) & 3); }
int scale_unknown(int iu) { return 1 << (((iu * 741 + 66037) % 312500) & 3); }
int scale_angle(int ia) { return 1 << (ia & 7); }

// The built-in transform matrices (quantities_testing_c.h:40-201): a_from_m
// maps affine moment vectors to affine angle vectors and adds a second-
// difference null-space fill; m_from_a maps back, divided by the octant count
// and the angle scale factor.  Entries are small integers / powers of two.
void build_am_matrices(int nm, int na, double* a, double* m) {
  const size_t n = (size_t)nm * na * NOCTANT;
  for (size_t i = 0; i < n; ++i) a[i] = m[i] = 0.0;
  auto A = [&](int im, int ia, int o) -> double& { return a[ia + (size_t)na * (im + (size_t)nm * o)]; };
  auto M = [&](int im, int ia, int o) -> double& { return m[im + (size_t)nm * (ia + (size_t)na * o)]; };
  for (int o = 0; o < NOCTANT; ++o) {
    for (int i = 0; i < na; ++i) {
      const int q = (i + 1) / nm, r = (i + 1) % nm;
      A(nm - 1, i, o) += q;
      if (r) {
        A(0, i, o) += -1.0;
        A(r, i, o) += 1.0;
      }
    }
    for (int im = 0; im + 2 < nm; ++im)
      for (int ia = 0; ia < na; ++ia) {
        const int w = 21 + (im + nm * ia) % 17;
        A(im, ia, o) += -1.0 * w;
        A(im + 1, ia, o) += 2.0 * w;
        A(im + 2, ia, o) += -1.0 * w;
      }
    for (int i = 0; i < nm; ++i) {
      const int q = (i + 1) / na, r = (i + 1) % na;
      M(i, na - 1, o) += q;
      if (r) {
        M(i, 0, o) += -1.0;
        M(i, r, o) += 1.0;
      }
    }
    for (int im = 0; im < nm; ++im)
      for (int ia = 0; ia + 2 < na; ++ia) {
        const int w = 37 + (im + nm * ia) % 19;
        M(im, ia, o) += -1.0 * w;
        M(im, ia + 1, o) += 2.0 * w;
        M(im, ia + 2, o) += -1.0 * w;
      }
    for (int im = 0; im < nm; ++im)
      for (int ia = 0; ia < na; ++ia) {
        M(im, ia, o) /= NOCTANT;
        M(im, ia, o) /= scale_angle(ia);
      }
  }
}
}  // namespace msb

extern "C" void Quantities_init_am_matrices_(Quantities* quan, const Dimensions dims, Env* env) {
  Insist(dims.nm == NM || dims.nm > 0 ? "Invalid nm." : 0);
  const size_t n = (size_t)dims.nm * dims.na * NOCTANT;
  Pointer_create(&quan->a_from_m, n, Env_cuda_is_using_device(env));
  Pointer_create(&quan->m_from_a, n, Env_cuda_is_using_device(env));
  Pointer_allocate(&quan->a_from_m);
  Pointer_allocate(&quan->m_from_a);
  msb::build_am_matrices(dims.nm, dims.na, quan->a_from_m.h_, quan->m_from_a.h_);
  Pointer_update_d(&quan->a_from_m);
  Pointer_update_d(&quan->m_from_a);
}

extern "C" void Quantities_init_decomp_(Quantities* quan, const Dimensions dims, Env* env) {
  // quantities_testing_c.h:206-333: the offsets of this process's subdomain
  // from the local x (y) sizes of the processes in its row (column).  The
  // reference gathers them with point-to-point messages; here one allgather.
  const int npx = Env_nproc_x(env), npy = Env_nproc_y(env), nproc = npx * npy;
  const int px = Env_proc_x_this(env), py = Env_proc_y_this(env);
  quan->ncell_z_g = dims.ncell_z;
  quan->ix_base_vals = malloc_host_int(npx + 1);
  quan->iy_base_vals = malloc_host_int(npy + 1);
  quan->ix_base_vals[0] = 0;
  quan->iy_base_vals[0] = 0;
  if (nproc == 1) {
    quan->ix_base_vals[1] = dims.ncell_x;
    quan->iy_base_vals[1] = dims.ncell_y;
  } else {
    const msb_comm* c = grid_comm(env);
    Insist(c ? "A decomposed grid needs the Env's process group (msb_env_set_comm)." : 0);
    std::vector<int> nx(nproc), ny(nproc);
    Insist(c->allgather_int(c->ctx, nproc, dims.ncell_x, nx.data()) == 0 ? "allgather failed." : 0);
    Insist(c->allgather_int(c->ctx, nproc, dims.ncell_y, ny.data()) == 0 ? "allgather failed." : 0);
    for (int i = 0; i < npx; ++i) quan->ix_base_vals[1 + i] = quan->ix_base_vals[i] + nx[Env_proc(env, i, py)];
    for (int i = 0; i < npy; ++i) quan->iy_base_vals[1 + i] = quan->iy_base_vals[i] + ny[Env_proc(env, px, i)];
  }
  quan->ix_base = quan->ix_base_vals[px];
  quan->iy_base = quan->iy_base_vals[py];
  quan->ncell_x_g = quan->ix_base_vals[npx];
  quan->ncell_y_g = quan->iy_base_vals[npy];
}

extern "C" void Quantities_create(Quantities* quan, const Dimensions dims, Env* env) {
  Quantities_init_am_matrices_(quan, dims, env);
  Quantities_init_decomp_(quan, dims, env);
}

extern "C" void Quantities_destroy(Quantities* quan) {
  Pointer_destroy(&quan->a_from_m);
  Pointer_destroy(&quan->m_from_a);
  free_host_int(quan->ix_base_vals);
  free_host_int(quan->iy_base_vals);
  quan->ix_base_vals = nullptr;
  quan->iy_base_vals = nullptr;
}

extern "C" double Quantities_flops_per_solve(const Dimensions dims) {
  (void)dims;
  return 3. + 3. * NDIM;  // quantities_testing_c.h:356-359
}

extern "C" P Quantities_init_state(const Quantities* quan, int ix, int iy, int iz, int ie, int im, int iu,
                                   const Dimensions dims) {
  (void)dims;
  return ((P)(1 + im)) * ((P)msb::scale_space(ix + quan->ix_base, iy + quan->iy_base, iz)) *
         ((P)msb::scale_energy(ie)) * ((P)msb::scale_unknown(iu));
}

// -------------------------------------------------------- array operations
extern "C" void initialize_state(P* const v, const Dimensions dims, const int nu, const Quantities* const quan) {
  for (int iz = 0; iz < dims.ncell_z; ++iz)
    for (int ie = 0; ie < dims.ne; ++ie)
      for (int iy = 0; iy < dims.ncell_y; ++iy)
        for (int ix = 0; ix < dims.ncell_x; ++ix)
          for (int iu = 0; iu < nu; ++iu)
            for (int im = 0; im < dims.nm; ++im)
              v[msb::ind_state(dims, nu, ix, iy, iz, ie, im, iu)] =
                  Quantities_init_state(quan, ix, iy, iz, ie, im, iu, dims);
}

extern "C" void initialize_state_zero(P* const v, const Dimensions dims, const int nu) {
  const size_t n = Dimensions_size_state(dims, nu);
  memset(v, 0, n * sizeof(P));
}

extern "C" void get_state_norms(const P* const vi, const P* const vo, const Dimensions dims, const int nu,
                                P* const normsqp, P* const normsqdiffp, Env* const env) {
  // array_operations.c:69-110, same loop order (iz, iy, ix, ie, im, iu).
  P normsq = 0, normsqdiff = 0;
  for (int iz = 0; iz < dims.ncell_z; ++iz)
    for (int iy = 0; iy < dims.ncell_y; ++iy)
      for (int ix = 0; ix < dims.ncell_x; ++ix)
        for (int ie = 0; ie < dims.ne; ++ie)
          for (int im = 0; im < dims.nm; ++im)
            for (int iu = 0; iu < nu; ++iu) {
              const size_t i = msb::ind_state(dims, nu, ix, iy, iz, ie, im, iu);
              const P d = vi[i] - vo[i];
              normsq += vo[i] * vo[i];
              normsqdiff += d * d;
            }
  *normsqp = Env_sum_P(env, normsq);
  *normsqdiffp = Env_sum_P(env, normsqdiff);
}

extern "C" void copy_vector(P* const vo, const P* const vi, const size_t n) { memcpy(vo, vi, n * sizeof(P)); }
