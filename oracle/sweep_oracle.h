/*
 * sweep_oracle.h -- TEST INFRASTRUCTURE ONLY.
 *
 * CPU restatement of the reference minisweep sweep, used as the checker by
 * tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg.  It is never
 * linked into, or called by, the product library.
 *
 * Array layouts are the reference's:
 *   state    v[iz][ie][iy][ix][iu][im]          (array_accessors_kernels.h:64-89)
 *   a_from_m a[oct][im][ia]   stride NM=nm       (array_accessors_kernels.h:334-350)
 *   m_from_a m[oct][ia][im]                      (array_accessors_kernels.h:398-414)
 */
#ifndef SWEEP_ORACLE_H
#define SWEEP_ORACLE_H

#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

/* Built-in (index-derived) problem definition. */
void oracle_init_am_matrices(int nm, int na, double* a_from_m, double* m_from_a);
void oracle_init_state(int nx, int ny, int nz, int ne, int nm, int nu, double* v);

/* One sweep, vo = sum over octants (simple sweeper order). */
void oracle_sweep(int nx, int ny, int nz, int ne, int nm, int nu, int na,
                  const double* a_from_m, const double* m_from_a,
                  const double* vi, double* vo);

/* Same, restricted to groups [ie0, ie1) of a state with ne groups. */
void oracle_sweep_groups(int nx, int ny, int nz, int ne, int nm, int nu, int na,
                         int ie0, int ie1,
                         const double* a_from_m, const double* m_from_a,
                         const double* vi, double* vo);

void oracle_state_norms(size_t n, const double* vi, const double* vo,
                        double* normsq, double* normsqdiff);

/* normsq of the built-in initial state in closed form (independent of na and
 * of every sweep parameter when vo == vi). */
double oracle_normsq_closed_form(int nx, int ny, int nz, int ne, int nm, int nu);

/* Individual pieces, exported for unit tests. */
int    oracle_scalefactor_space(int ix, int iy, int iz);
int    oracle_scalefactor_energy(int ie);
int    oracle_scalefactor_unknown(int iu);
double oracle_init_face(int ia, int ix, int iy, int iz, int ie, int iu, int octant);

#ifdef __cplusplus
}
#endif
#endif
