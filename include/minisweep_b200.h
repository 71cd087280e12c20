/*
 * minisweep_b200.h -- C ABI of the B200-native KBA sweep library
 * (libminisweep_b200.so).
 *
 * The library is a drop-in for the sweep path of olcf/minisweep: it exports the
 * reference's Env / Arguments / Dimensions / Pointer / Quantities / Sweeper C
 * API with the same names, argument meaning and error behaviour (Insist ->
 * message on stderr + exit(EXIT_FAILURE)), so the reference's own driver
 * sources (src/4_driver/runner.c, sweep.c, tester.c) compile against these
 * headers unchanged and link against this library instead of libsweeper.
 * The mirror headers in this directory (env.h, sweeper.h, ...) all include
 * this file, so the reference's #include lines resolve here.
 *
 * Every sweep runs on one B200 (sm_100a): there is no CPU path.  Functions
 * whose name ends in _status return an error code instead of exiting; they
 * and the *_device entry points have no counterpart in the reference.
 *
 * Compile-time sizes follow the reference: NM (moments) defaults to 16 and is
 * set with -DNM_VALUE=...; NU (unknowns) is fixed at 4 by this library.
 * The library itself handles NM in {4, 8, 16} at run time (Dimensions.nm).
 *
 * Reference interfaces are cited as file:line within olcf/minisweep.
 */
#ifndef MINISWEEP_B200_H
#define MINISWEEP_B200_H

#include <stddef.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#ifdef __cplusplus
extern "C" {
#endif

/*====================================================================== types
 * src/1_base/types_kernels.h:17-53 */
typedef double P;
typedef int Bool_t;
enum { Bool_true = (1 == 1), Bool_false = (0 == 1) };
static inline P P_zero(void) { return (P)0; }
static inline P P_one(void) { return (P)1; }

#ifndef TARGET_HD
#define TARGET_HD
#endif
#ifndef TARGET_G
#define TARGET_G
#endif

/* src/1_base/env_assert.h:19-40: Insist always checks (message + exit),
 * Assert is assert() unless NDEBUG. */
void insist_(const char* condition_string, const char* file, int line);
#define Insist(condition) \
  (void)((condition) || (insist_(#condition, __FILE__, __LINE__), 0))
#ifndef NDEBUG
#include <assert.h>
#define Assert(v) assert(v)
#else
#define Assert(v)
#endif
#define Static_Assert(condition) { int a[(condition) ? 1 : -1]; (void)a; }

/*=============================================================== definitions
 * src/2_sweeper_base/definitions_kernels.h:21-64 */
enum { NDIM = 3 };
enum { DIM_X = 0 };
enum { DIM_Y = 1 };
enum { DIM_Z = 2 };
enum { NOCTANT = 8 };
enum { DIR_UP = +1 };
enum { DIR_DN = -1 };
enum { DIR_HI = +1 };
enum { DIR_LO = -1 };
static inline int Dir_x(int octant) { return octant & (1 << 0) ? (int)DIR_DN : (int)DIR_UP; }
static inline int Dir_y(int octant) { return octant & (1 << 1) ? (int)DIR_DN : (int)DIR_UP; }
static inline int Dir_z(int octant) { return octant & (1 << 2) ? (int)DIR_DN : (int)DIR_UP; }
static inline int Dir_inc(int dir) { return dir; }
static inline int imin(const int i, const int j) { return i < j ? i : j; }
static inline int imax(const int i, const int j) { return i > j ? i : j; }

/*================================================================ dimensions
 * src/2_sweeper_base/dimensions_kernels.h:24-56 */
#ifdef NU_VALUE
#if NU_VALUE != 4
#error "libminisweep_b200 is built for NU = 4 unknowns per cell/moment/group"
#endif
#endif
enum { NU = 4 };
#ifdef NM_VALUE
enum { NM = NM_VALUE };
#else
enum { NM = 16 };
#endif

typedef struct {
  int ncell_x;
  int ncell_y;
  int ncell_z;
  int ne;
  int nm;
  int na;
} Dimensions;

/* src/2_sweeper_base/dimensions.h:28-57 */
Dimensions Dimensions_null(void);
size_t Dimensions_size_state(const Dimensions dims, int nu);
size_t Dimensions_size_state_angles(const Dimensions dims, int nu);
size_t Dimensions_size_facexy(const Dimensions dims, int nu, int noctant_per_block);
size_t Dimensions_size_facexz(const Dimensions dims, int nu, int noctant_per_block);
size_t Dimensions_size_faceyz(const Dimensions dims, int nu, int noctant_per_block);

/*================================================================= arguments
 * src/1_base/arguments.h:33-88 -- read-once integer flags */
typedef struct {
  int argc;
  char** argv_unconsumed;
  char* argstring;
} Arguments;

Arguments Arguments_null(void);
void Arguments_create(Arguments* args, int argc, char** argv);
void Arguments_create_from_string(Arguments* args, const char* argstring);
void Arguments_destroy(Arguments* args);
Bool_t Arguments_exists(const Arguments* args, const char* arg_name);
int Arguments_consume_int_(Arguments* args, const char* arg_name);
int Arguments_consume_int_or_default(Arguments* args, const char* arg_name,
                                     int default_value);
Bool_t Arguments_are_all_consumed(const Arguments* args);

/*======================================================================= env
 * src/1_base/env_types.h:54-70, env.h:46-80, env_mpi.h, env_cuda.h.
 * One process drives one GPU.  The process grid is 1 x 1 unless the host
 * program gave the Env a process group (msb_env_set_comm, below), the
 * counterpart of the reference's MPI_COMM_WORLD (env_mpi.c:100-141). */
typedef int Comm_t;
typedef int Request_t;
typedef void* Stream_t; /* a cudaStream_t */
typedef double Timer;

typedef struct msb_comm msb_comm;
/* Env.flags_: several processes of the group drive the same GPU; their
 * sweep kernels then take turns instead of sharing the GPU at once. */
enum { MSB_ENV_SHARED_GPU = 1 };

typedef struct {
  int nproc_x_;
  int nproc_y_;
  int tag_;
  Bool_t is_proc_active_;
  Bool_t is_using_device_;
  Stream_t stream_kernel_faces_;
  int device_;
  int proc_;         /* this process's number in its group (0 without one) */
  int nproc_world_;  /* processes in the group (1 without one)             */
  int flags_;        /* MSB_ENV_SHARED_GPU: processes of the group share GPUs */
  const msb_comm* comm_;
} Env;

Env Env_null(void);
void Env_initialize(Env* env, int argc, char** argv);
void Env_set_values(Env* env, Arguments* args);
void Env_finalize(Env* env);
Bool_t Env_is_proc_master(Env* env);
Timer Env_get_time(Env* env);
Timer Env_get_synced_time(Env* env);
int Env_nproc_x(const Env* env);
int Env_nproc_y(const Env* env);
int Env_nproc(const Env* env);
Bool_t Env_is_proc_active(const Env* env);
int Env_tag(const Env* env);
void Env_increment_tag(Env* env, int value);
int Env_proc(const Env* env, int proc_x, int proc_y);
int Env_proc_x(const Env* env, int proc);
int Env_proc_y(const Env* env, int proc);
int Env_proc_this(const Env* env);
int Env_proc_x_this(const Env* env);
int Env_proc_y_this(const Env* env);
void Env_mpi_barrier(Env* env);
double Env_sum_d(Env* env, double value);
P Env_sum_P(Env* env, P value);
Bool_t Env_cuda_is_using_device(const Env* const env);
Bool_t Env_cuda_last_call_succeeded(void);
Stream_t Env_cuda_stream_kernel_faces(Env* env);
void Env_cuda_stream_wait(Env* env, Stream_t stream);

/* src/1_base/env_cuda.h host/device memory helpers */
int* malloc_host_int(size_t n);
P* malloc_host_P(size_t n);
P* malloc_host_pinned_P(size_t n);
P* malloc_device_P(size_t n);
void free_host_int(int* p);
void free_host_P(P* p);
void free_host_pinned_P(P* p);
void free_device_P(P* p);
void cuda_copy_host_to_device_P(P* p_d, P* p_h, size_t n);
void cuda_copy_device_to_host_P(P* p_h, P* p_d, size_t n);

/*=================================================================== pointer
 * src/1_base/pointer_kernels.h:33-41, pointer.h:28-112: a host array with an
 * optional device mirror. */
enum { IS_USING_DEVICE = Bool_true, IS_NOT_USING_DEVICE = Bool_false };
enum { IS_PINNED = Bool_true, IS_NOT_PINNED = Bool_false };

typedef struct {
  size_t n_;
  P* h_;
  P* d_;
  Bool_t is_using_device_;
  Bool_t is_pinned_;
  Bool_t is_alias_;
} Pointer;

static inline P* Pointer_h(Pointer* p) { return p->h_; }
static inline const P* Pointer_const_h(const Pointer* p) { return p->h_; }
static inline P* Pointer_d(Pointer* p) { return p->d_; }
static inline const P* Pointer_const_d(const Pointer* p) { return p->d_; }
static inline P* Pointer_active(Pointer* p) { return p->is_using_device_ ? p->d_ : p->h_; }
static inline P* Pointer_const_active(const Pointer* p) { return p->is_using_device_ ? p->d_ : p->h_; }

Pointer Pointer_null(void);
void Pointer_create(Pointer* p, size_t n, Bool_t is_using_device);
void Pointer_create_alias(Pointer* p, Pointer* source, size_t base, size_t n);
void Pointer_set_pinned(Pointer* p, Bool_t is_pinned);
void Pointer_destroy(Pointer* p);
void Pointer_allocate_h_(Pointer* p);
void Pointer_allocate_d_(Pointer* p);
void Pointer_allocate(Pointer* p);
void Pointer_deallocate_h_(Pointer* p);
void Pointer_deallocate_d_(Pointer* p);
void Pointer_deallocate(Pointer* p);
void Pointer_update_h(Pointer* p);
void Pointer_update_d(Pointer* p);
void Pointer_update_h_stream(Pointer* p, Stream_t stream);
void Pointer_update_d_stream(Pointer* p, Stream_t stream);

/*================================================================ quantities
 * src/3_sweeper/quantities_testing_kernels.h:35-46 (struct),
 * quantities_testing.h:27-90 (API): the built-in deterministic problem. */
typedef struct {
  Pointer a_from_m; /* [octant][im][ia], im stride NM  */
  Pointer m_from_a; /* [octant][ia][im]                */
  int* ix_base_vals;
  int* iy_base_vals;
  int ix_base;
  int iy_base;
  int ncell_x_g;
  int ncell_y_g;
  int ncell_z_g;
} Quantities;

void Quantities_create(Quantities* quan, const Dimensions dims, Env* env);
void Quantities_destroy(Quantities* quan);
void Quantities_init_am_matrices_(Quantities* quan, const Dimensions dims, Env* env);
void Quantities_init_decomp_(Quantities* quan, const Dimensions dims, Env* env);
double Quantities_flops_per_solve(const Dimensions dims);
P Quantities_init_state(const Quantities* quan, int ix, int iy, int iz, int ie,
                        int im, int iu, const Dimensions dims);

/*========================================================== array operations
 * src/2_sweeper_base/array_operations.h:27-55 (host arrays, FP64). */
void initialize_state(P* const v, const Dimensions dims, const int nu,
                      const Quantities* const quan);
void initialize_state_zero(P* const v, const Dimensions dims, const int nu);
void get_state_norms(const P* const vi, const P* const vo, const Dimensions dims,
                     const int nu, P* const normsqp, P* const normsqdiffp,
                     Env* const env);
void copy_vector(P* const vo, const P* const vi, const size_t n);

/*=================================================================== sweeper
 * src/3_sweeper/sweeper_kba.h:34-257.  The struct keeps the reference's
 * flag-derived fields (all accepted and validated as the reference does,
 * sweeper_kba_c.h:44-287); the device state lives behind impl_. */
typedef struct {
  Dimensions dims;
  Dimensions dims_b;
  Dimensions dims_g;
  int nblock_z;
  int nblock_octant;
  int noctant_per_block;
  int nsemiblock;
  int ncell_x_per_subblock;
  int ncell_y_per_subblock;
  int ncell_z_per_subblock;
  int nthread_e;
  int nthread_octant;
  int nthread_x;
  int nthread_y;
  int nthread_z;
  Bool_t is_face_comm_async;
  int precision;    /* 0: FP64 plain; 1: mixed precision (--precision 1) */
  void* impl_;
} Sweeper;

/* sweeper_kba.h:66-70 */
Sweeper Sweeper_null(void);
/* sweeper_kba.h:74-80 / sweeper_kba_c.h:44-287: consumes the sweeper flags */
void Sweeper_create(Sweeper* sweeper, Dimensions dims, const Quantities* quan,
                    Env* env, Arguments* args);
/* sweeper_kba.h:84-87 / sweeper_kba_c.h:292-329 */
void Sweeper_destroy(Sweeper* sweeper, Env* env);
/* sweeper_kba.h:243-249 / sweeper_kba_c.h:588-845: vo = sweep(vi).  Reads vi
 * from its host copy and leaves vo's host copy complete on return, as the
 * reference does (its step loop copies every z-block back). */
void Sweeper_sweep(Sweeper* sweeper, Pointer* vo, Pointer* vi,
                   const Quantities* quan, Env* env);
/* sweeper_kba.h:253-257 */
int Sweeper_noctant_per_block(const Sweeper* sweeper);

/*------------------------------------------------ extensions (no reference
 * counterpart).  Status codes: 0 ok, <0 error; the message is available from
 * msb_last_error().  These never exit the process. */
enum {
  MSB_OK = 0,
  MSB_ERR_ARG = -1,        /* invalid flag / size                          */
  MSB_ERR_CUDA = -2,       /* CUDA runtime error                           */
  MSB_ERR_TIMEOUT = -3,    /* a bounded device spin-wait gave up           */
  MSB_ERR_UNSUPPORTED = -4 /* size outside the compiled kernel variants    */
};
const char* msb_last_error(void);
int Sweeper_create_status(Sweeper* sweeper, Dimensions dims, const Quantities* quan,
                          Env* env, Arguments* args);
int Sweeper_sweep_status(Sweeper* sweeper, Pointer* vo, Pointer* vi,
                         const Quantities* quan, Env* env);
/* vo_d/vi_d: device arrays in the reference state layout.  Asynchronous on the
 * Env's stream; the status of the device work is checked by
 * Sweeper_sync_status. */
int Sweeper_sweep_device(Sweeper* sweeper, double* vo_d, const double* vi_d,
                         const Quantities* quan, Env* env);
int Sweeper_sync_status(Sweeper* sweeper, Env* env);
/* The reference driver's iteration loop (runner.c:148-155) in one call:
 * v_in_h (host) is copied to the device once, niterations sweeps alternate
 * between two device arrays, and the last sweep's output is copied to v_out_h
 * (host).  Synchronous; returns the status of the device work. */
int Sweeper_sweep_iterations(Sweeper* sweeper, double* v_out_h, const double* v_in_h, int niterations,
                             const Quantities* quan, Env* env);
/* Group-pair slices the last host-buffer call (Sweeper_sweep[_status] or
 * Sweeper_sweep_iterations) ran in (1: the whole problem at once; 0: no call
 * yet).  On a large problem (FP64 or mixed precision; state of 256 MiB or
 * more, 16 or more group pairs) those calls sweep the groups in up to 4 slices, each through every
 * iteration, so that a slice's host copies overlap the other slices' sweeps;
 * the results are the same.  No reference counterpart. */
int msb_iterations_slices(const Sweeper* sweeper);
/* Device-side FP64 checksums of two device state arrays (same sums as
 * get_state_norms). */
int msb_state_norms_device(const double* vi_d, const double* vo_d, size_t n,
                           double* normsq, double* normsqdiff, Env* env);
/* Device-side built-in initial state (same values as initialize_state). */
int msb_initialize_state_device(double* v_d, Dimensions dims, Env* env);
/* The same for an energy-group slice: the array's group ie is global group
 * ie_base + ie (no reference counterpart; the reference never splits the
 * groups across processes, Quantities_init_state at quantities_testing.h:60-90
 * is its per-element formula). */
int msb_initialize_state_slice_device(double* v_d, Dimensions dims, int ie_base, Env* env);
/* Kernel statistics of the last sweep: number of tasks, kernel launches. */
int Sweeper_last_stats(const Sweeper* sweeper, long long* ntask, int* nlaunch);
/* Tile shape (cell columns per CTA) the sweeper uses and, with --autotune 1,
 * the first sweep's times (ms) of the chosen plan and of the fastest plan
 * with the other tile shape (0 before that sweep, or without autotuning).
 * No reference counterpart: the reference's --ncell_{x,y}_per_subblock size
 * its CPU/GPU thread blocks. */
int Sweeper_tile(const Sweeper* sweeper, int* tx, int* ty, float* ms_chosen, float* ms_other);
/* The rest of the FP64 plan in use: the kernel (0 staged, 1 chained
 * wavefront), the task window (x SMs) of its schedule, the L2 policy flag,
 * how many plans --autotune 1 timed (1 without it), and the angles per pass
 * (--angle_pass; na above it is swept in passes).  With --autotune 1 the
 * first sweep runs every candidate -- both kernels (the staged one with 64-
 * and with 32-angle passes when na > 32) x both tile shapes x task windows 4,
 * 8 and 16 -- and keeps the fastest.  No reference counterpart (the
 * reference's tuning flags, sweeper_kba_c.h:54-233, are set by hand). */
int Sweeper_plan(const Sweeper* sweeper, int* fp64_kernel, int* task_window, int* l2_hints, int* ncandidates,
                 int* angle_pass);
/* Copy of the schedule (one record of MSB_TASK_INTS ints per task, in launch
 * order) for host-side checks; returns the task count, or <0. */
enum { MSB_TASK_INTS = 16 };
long long Sweeper_debug_tasks(const Sweeper* sweeper, int* out, long long max_tasks);
/* Test hook: time budget (ns) of every device wait in the next sweeps;
 * 0 = default (4 s). */
int Sweeper_set_spin_limit(Sweeper* sweeper, long long limit);
/* The schedule the sweeper would build for these sizes, tile shape and
 * group-pair interleave, without touching a GPU (host-side checks). */
long long msb_schedule_tasks(int nx, int ny, int nz, int ne, int tx, int ty, int gp_block, int* out,
                             long long max_tasks);
/* Measured FP64 throughput of this GPU in TFLOP/s: tensor-core products
 * (mma.sync f64) and FMA pipe; best of `reps` launches.  The roofline
 * denominator of the FP64 sweep. */
int msb_measure_fp64_peak(double* tflops_dmma, double* tflops_dfma, int reps);

/* One FP64 sweep that allocates nothing.  No counterpart in the reference.
 * For callers that cannot allocate device memory when they sweep (their
 * device memory is owned by a pool or arena, or they must not trigger the
 * device synchronisation cudaMalloc/cudaFree can cause): every scratch buffer
 * of the sweep (task table, progress counters, face planes) lives in one
 * file-scope device array of MSB_NOALLOC_SCRATCH_BYTES that every GPU loading
 * the library holds until exit, and the schedule is built in static host
 * arrays.  vo_d = sweep(vi_d) with the caller's device arrays (reference state
 * and matrix layouts) on `stream`; returns after the sweep finished.
 * Limits: NM 4 or 16, na <= 32, and the problem's scratch must fit the array
 * (about 10^3 cells x 8 groups); larger problems return MSB_ERR_ARG with the
 * bytes needed.  The first call on each device sets up (takes the array's
 * device address with that device current).  Under CUDA's default lazy module
 * loading the array's 32 MiB are committed on a device by that first call
 * (at load time with CUDA_MODULE_LOADING=EAGER): a caller whose pool takes
 * every free byte makes one call before creating the pool.  Every call reads
 * the kernel's status back and synchronises `stream`, so no call may be made
 * while `stream` is capturing a graph (refused with MSB_ERR_UNSUPPORTED).
 * All calls share the array, which keeps the last call's contents; calls that
 * overlap, on the GPU or on the host, race. */
#define MSB_NOALLOC_SCRATCH_BYTES (32u << 20)
int msb_sweep_noalloc(double* vo_d, const double* vi_d, const double* a_from_m_d, const double* m_from_a_d,
                      int ncell_x, int ncell_y, int ncell_z, int ne, int nm, int na, void* stream);

/*---------------------------------------------------------------- batches
 * Many independent sweep problems in one persistent kernel launch.  No
 * counterpart in the reference, which sweeps one problem per Sweeper
 * (Sweeper_create, sweeper_kba_c.h:44-287; Sweeper_sweep, :588-845); a batch
 * sweeps every problem exactly as that problem's own Sweeper would (FP64, the
 * built-in or the caller's transform matrices), with results identical bit
 * for bit.
 *
 * Each problem has its own sizes (nm 4, 8 or 16; na <= 128) and its own device
 * arrays in the reference layouts: vi/vo the state (16-byte aligned),
 * a_from_m [octant][im][ia] and m_from_a [octant][ia][im].  The face planes
 * are scratch from one device arena of scratch_bytes (0: what all problems
 * need at once, capped at 80 % of the free device memory); problems that do
 * not fit at once reuse the bytes of problems that completed earlier in the
 * same launch.  autotune != 0 times the two tile shapes (4 x 2 and 2 x 4
 * cells) on the median problem of each nm group at creation;
 * those trial sweeps write that problem's vo.  Asynchronous calls run on the
 * given stream (a cudaStream_t, NULL = the legacy default stream); their
 * device status is checked by msb_batch_sync. */
typedef struct {
  int ncell_x, ncell_y, ncell_z, ne, na, nm;
  double* vi;               /* input of even sweeps (dir 0) */
  double* vo;               /* output of even sweeps        */
  const double* a_from_m;
  const double* m_from_a;
} msb_problem;
typedef struct msb_batch msb_batch;
enum { MSB_BATCH_MAX_CLASSES = 16 };
typedef struct {
  int nproblem, nclass, npred, nsm;
  long long ntask;
  size_t scratch_bytes;       /* arena size                              */
  size_t scratch_needed_all;  /* face scratch of all problems at once    */
  double sim_makespan;        /* planner's simulated time (relative units) */
  double sim_busy;            /* planner's simulated SM utilisation (0-1)  */
  double tune_ms;             /* time spent in autotuning trial sweeps   */
  int class_nm[MSB_BATCH_MAX_CLASSES], class_nch[MSB_BATCH_MAX_CLASSES];
  int class_tx[MSB_BATCH_MAX_CLASSES], class_ty[MSB_BATCH_MAX_CLASSES];
  long long class_ntask[MSB_BATCH_MAX_CLASSES];
} msb_batch_info_t;
/* precision must be 0 (FP64). */
int msb_batch_create(msb_batch** out, const msb_problem* problems, int nproblem, int precision,
                     size_t scratch_bytes, int autotune);
void msb_batch_destroy(msb_batch* b);
/* One launch: every problem sweeps vo = sweep(vi) (dir 0) or vi = sweep(vo)
 * (dir 1). */
int msb_batch_sweep(msb_batch* b, int dir, void* stream);
/* The reference driver's iteration loop (runner.c:148-155) for every problem:
 * niterations sweeps alternating dir 0 and 1 (the result of the last sweep is
 * in vo for an odd count, in vi for an even one), launched as one CUDA graph
 * captured on the first call with this count. */
int msb_batch_run(msb_batch* b, int niterations, void* stream);
int msb_batch_sync(msb_batch* b, void* stream);
/* Per problem: ms from the start of the last launch to the completion of the
 * problem's last task (device clock).  After msb_batch_sync. */
int msb_batch_problem_ms(const msb_batch* b, double* ms, int n);
int msb_batch_info(const msb_batch* b, msb_batch_info_t* info);
/* Host-only planning of the same batch for nsm SMs (no device, pointers may
 * be NULL) for host-side checks; bit k of tile24_mask, k = 0, 1, 2 for nm 4,
 * 8, 16, selects the 2 x 4 tile for that group. */
int msb_batch_plan(msb_batch** out, const msb_problem* problems, int nproblem, int nsm,
                   size_t scratch_bytes, int tile24_mask);
/* A batch sweeps every problem in entries of 32 angles, as a Sweeper sweeps
 * them in passes: entry e is problem problem[e]'s angles [angle0[e],
 * angle0[e] + 32); later entries of a problem add to vo after the entry
 * before them completed.  Returns the entry count. */
int msb_batch_entries(const msb_batch* b, int* problem, int* angle0, int max_entries);
/* The planned task table (global ids, MSB_TASK_INTS ints per task) and the
 * entry of each task; returns the task count. */
long long msb_batch_tasks(const msb_batch* b, int* rec, int* prob, long long max_tasks);
/* Arena placement per entry (offset, bytes) and the entries each one waits
 * for (pred[pred_off[e] .. pred_off[e + 1])); returns the predecessor count. */
int msb_batch_scratch(const msb_batch* b, long long* offset, long long* bytes, int* pred_off, int* pred,
                      int max_pred);
/* Test hook: time budget (ns) of every device wait; 0 = default (4 s). */
int msb_batch_set_spin_limit(msb_batch* b, long long limit);
/* The built-in transform matrices (Quantities_init_am_matrices_,
 * quantities_testing_c.h:40-201) for nm moments and na angles, 8 octants. */
int msb_builtin_matrices(int nm, int na, double* a_from_m, double* m_from_a);

/*------------------------------------------------------- KBA decomposition
 * --nproc_x / --nproc_y > 1: the x-y plane is split over a process grid, one
 * process (one GPU) per subdomain, as the reference's MPI build does
 * (runner.c:95-106 sizes, quantities_testing_c.h:206-333 offsets,
 * stepscheduler_kba.c:80-284 steps, faces_kba.c:86-479 face exchange).  A
 * sweep is a sequence of steps; at each step every process sweeps one
 * (octant, z-block) slab of its subdomain with one kernel launch, then the
 * faces leaving the slab cross to the downwind neighbours.  The transport is
 * the host program's: it hands the Env a table of callbacks (MPI, NCCL
 * through torch.distributed, ...), the counterpart of the reference's
 * Env_send / Env_recv / Env_sum_d over MPI_COMM_WORLD (env_mpi.c:309-480). */
typedef struct {
  int peer;      /* process number of the other side                         */
  int is_send;   /* 1: send `bytes` of buf to peer; 0: receive them into buf */
  int axis;      /* 0: x faces (yz planes), 1: y faces (xz planes)           */
  int side;      /* the peer's position along the axis: 0 lower, 1 higher    */
  size_t bytes;
  void* buf;     /* device memory of this process                            */
} msb_kba_msg;

struct msb_comm {
  void* ctx;
  /* Every active process calls this after each step with the messages of
   * that step (possibly none) and returns 0 once its sends and receives have
   * completed in device memory.  The device work that filled the send
   * buffers, and the unpacking of the previous step's receives, has
   * finished. */
  int (*exchange)(void* ctx, int nactive, const msb_kba_msg* msgs, int nmsg);
  /* The collectives run over the active processes 0 .. nactive - 1 (the
   * reference's active communicator, env_mpi.c:128-135), called by each of
   * them.  sum_double: *value = the sum of their *value (Env_sum_d).
   * allgather_int: values[p] = the value of process p.  A transport that
   * serves only the whole group returns nonzero for nactive < nproc. */
  int (*sum_double)(void* ctx, int nactive, double* value);
  int (*allgather_int)(void* ctx, int nactive, int value, int* values);
  int (*barrier)(void* ctx, int nactive);
};

/* Before Env_set_values: this process is number `proc` of `nproc`, reached
 * through `comm` (which must outlive the Env).  Env_set_values then accepts
 * any grid of up to nproc processes; processes numbered beyond it are
 * inactive (env_mpi.c:119-135). */
int msb_env_set_comm(Env* env, int proc, int nproc, const msb_comm* comm);

/* Host-only: the step plan of a decomposed sweep.  Unit k (0 <= k <
 * 8 * nblock_z) is octant unit_oct[k] on z-block unit_zb[k]; process p sweeps
 * it at step start[p * 8 * nblock_z + k]; nstep steps in all.  Arrays may be
 * NULL. */
int msb_kba_plan(int nproc_x, int nproc_y, int nblock_z, int* nstep, int* unit_oct, int* unit_zb, int* start);
/* Host-only: the messages of process `proc` after step `step`, 5 ints each
 * (peer, is_send, axis, side, unit); returns their count. */
int msb_kba_plan_messages(int nproc_x, int nproc_y, int nblock_z, int proc, int step, int* out, int max_msgs);

/* A decomposed sweep driven step by step, for hosts that run the exchange
 * themselves (Sweeper_sweep does all of it through the Env's callbacks).
 * Sweeper created with an Env whose grid is nproc_x x nproc_y > 1.
 *   msb_kba_info: steps per sweep; bytes of the largest message per axis.
 *   msb_kba_set_buffers: device buffers for the messages (send x, send y,
 *     then receives x from the lower / higher neighbour, y lower / higher),
 *     each at least the axis's bytes; NULL = buffers the sweeper allocates.
 *   msb_kba_begin: starts vo_d = sweep(vi_d) on the Env's stream.
 *   msb_kba_step: launches this process's slab of `step` (if any), copies
 *     its leaving faces into the send buffers and waits for the Env's stream
 *     (so the previous step's unpacking has finished too).
 *   msb_kba_messages: the step's messages with their buffers.
 *   msb_kba_unpack: after the receives of `step` landed: the entering faces
 *     into this process's face planes.
 *   msb_kba_end: waits for the device work; the sweep's status. */
int msb_kba_info(const Sweeper* sweeper, int* nstep, size_t* bytes_x, size_t* bytes_y);
int msb_kba_set_buffers(Sweeper* sweeper, void* send_x, void* send_y, void* recv_x_lo, void* recv_x_hi,
                        void* recv_y_lo, void* recv_y_hi);
int msb_kba_begin(Sweeper* sweeper, double* vo_d, const double* vi_d, const Quantities* quan, Env* env);
int msb_kba_step(Sweeper* sweeper, int step, Env* env);
int msb_kba_messages(const Sweeper* sweeper, int step, msb_kba_msg* msgs, int max_msgs);
int msb_kba_unpack(Sweeper* sweeper, int step, Env* env);
int msb_kba_end(Sweeper* sweeper, Env* env);

#ifdef __cplusplus
}
#endif
#endif /* MINISWEEP_B200_H */
