/*
 * ref_dump.c -- TEST INFRASTRUCTURE ONLY (never linked into the product).
 *
 * A small driver owned by this repository that runs the reference
 * implementation's own serial KBA sweeper through its public C API and hands
 * the result back to the caller, so the repository's CPU restatement
 * (oracle/sweep_oracle.c) and golden fixtures can be pinned element-wise to
 * the reference.  It follows the reference driver's flow
 * (src/4_driver/runner.c:51-182): dimensions from flags, Quantities_create,
 * initialize_state, Sweeper_create (which consumes the sweeper flags),
 * niterations sweeps with the vi/vo swap, get_state_norms.
 *
 * The reference has no hook for user inputs, so this driver optionally
 * overwrites, after Quantities_create/initialize_state, the host copies of
 * a_from_m, m_from_a and vi with caller-supplied arrays (same layouts as the
 * reference: a_from_m[oct][im][ia], m_from_a[oct][ia][im],
 * state[iz][ie][iy][ix][iu][im]).  Quantities_solve and the boundary faces
 * are untouched (they are index-derived in the reference).
 *
 * Built only by oracle/Makefile's `ref` target, into oracle/_ref/.
 */
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include "arguments.h"
#include "env.h"
#include "definitions.h"
#include "dimensions.h"
#include "pointer.h"
#include "quantities.h"
#include "array_operations.h"
#include "sweeper.h"

int ref_nm(void) { return NM; }
int ref_nu(void) { return NU; }

/*
 * Run the reference sweeper.  argstring uses the reference flag syntax
 * ("--ncell_x 5 --ne 3 ...").  Inputs may be NULL (keep the reference's
 * built-in values).  vo_out / vi_out (may be NULL) receive the final state
 * arrays as the reference's runner leaves them (runner.c:148-155 swaps vi and
 * vo every iteration).  Returns 0, or -1 if a flag was not consumed.
 */
int ref_run(const char* argstring,
            const double* a_from_m_in, const double* m_from_a_in,
            const double* vi_in,
            double* vo_out, double* vi_out,
            double* normsq, double* normsqdiff)
{
  Env env = Env_null();
  Arguments args = Arguments_null();
  Dimensions dims;
  Quantities quan;
  Sweeper sweeper = Sweeper_null();
  Pointer vi = Pointer_null();
  Pointer vo = Pointer_null();
  int iteration = 0, niterations = 0;
  size_t n = 0;
  P nsq = 0, nsqd = 0;

  Env_initialize(&env, 0, NULL);
  Arguments_create_from_string(&args, argstring);
  Env_set_values(&env, &args);

  dims.ncell_x = Arguments_consume_int_or_default(&args, "--ncell_x", 5);
  dims.ncell_y = Arguments_consume_int_or_default(&args, "--ncell_y", 5);
  dims.ncell_z = Arguments_consume_int_or_default(&args, "--ncell_z", 5);
  dims.ne      = Arguments_consume_int_or_default(&args, "--ne", 30);
  dims.na      = Arguments_consume_int_or_default(&args, "--na", 33);
  niterations  = Arguments_consume_int_or_default(&args, "--niterations", 1);
  dims.nm      = NM;

  Quantities_create(&quan, dims, &env);
  if (a_from_m_in) {
    memcpy(Pointer_h(&quan.a_from_m), a_from_m_in,
           sizeof(double) * (size_t)dims.nm * dims.na * NOCTANT);
    Pointer_update_d(&quan.a_from_m);
  }
  if (m_from_a_in) {
    memcpy(Pointer_h(&quan.m_from_a), m_from_a_in,
           sizeof(double) * (size_t)dims.nm * dims.na * NOCTANT);
    Pointer_update_d(&quan.m_from_a);
  }

  n = Dimensions_size_state(dims, NU);
  Pointer_create(&vi, n, Env_cuda_is_using_device(&env));
  Pointer_allocate(&vi);
  Pointer_create(&vo, n, Env_cuda_is_using_device(&env));
  Pointer_allocate(&vo);
  initialize_state(Pointer_h(&vi), dims, NU, &quan);
  if (vi_in) memcpy(Pointer_h(&vi), vi_in, sizeof(double) * n);
  initialize_state_zero(Pointer_h(&vo), dims, NU);

  Sweeper_create(&sweeper, dims, &quan, &env, &args);
  if (!Arguments_are_all_consumed(&args)) {
    Sweeper_destroy(&sweeper, &env);
    Pointer_destroy(&vi);
    Pointer_destroy(&vo);
    Quantities_destroy(&quan);
    Arguments_destroy(&args);
    return -1;
  }

  for (iteration = 0; iteration < niterations; ++iteration) {
    Sweeper_sweep(&sweeper,
                  iteration % 2 == 0 ? &vo : &vi,
                  iteration % 2 == 0 ? &vi : &vo,
                  &quan, &env);
  }

  get_state_norms(Pointer_h(&vi), Pointer_h(&vo), dims, NU, &nsq, &nsqd, &env);
  if (normsq) *normsq = nsq;
  if (normsqdiff) *normsqdiff = nsqd;
  if (vo_out) memcpy(vo_out, Pointer_h(&vo), sizeof(double) * n);
  if (vi_out) memcpy(vi_out, Pointer_h(&vi), sizeof(double) * n);

  Sweeper_destroy(&sweeper, &env);
  Pointer_destroy(&vi);
  Pointer_destroy(&vo);
  Quantities_destroy(&quan);
  Arguments_destroy(&args);
  Env_finalize(&env);
  return 0;
}
