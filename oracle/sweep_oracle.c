/*
 * sweep_oracle.c -- TEST INFRASTRUCTURE ONLY (the checker, never the product).
 *
 * Plain-C FP64 restatement of the reference minisweep sweep, written from the
 * reference's "simple" sweeper (src/3_sweeper/sweeper_simple_c.h:83-277) and its
 * built-in testing Quantities (src/3_sweeper/quantities_testing_kernels.h,
 * quantities_testing_c.h, quantities_testing.h).  Every floating-point
 * expression keeps the reference's C evaluation order; the file is compiled with
 * -ffp-contract=off so no multiply-add is fused, which keeps it bit-identical to
 * the reference's non-FMA x86 build.
 *
 * Parity pin: tests/test_oracle.py checks this file against the reference's own
 * serial sweeper (oracle/_ref, driven by oracle/ref_dump.c) and against the
 * committed golden fixtures under tests/golden/.
 */
#include "sweep_oracle.h"

#include <stdlib.h>
#include <string.h>

enum { NOCT = 8 };

/* Dir_x/y/z: bit b of the octant set means the DOWN direction
 * (definitions_kernels.h:46-64). */
static int dir_x(int o) { return (o & 1) ? -1 : +1; }
static int dir_y(int o) { return (o & 2) ? -1 : +1; }
static int dir_z(int o) { return (o & 4) ? -1 : +1; }

/* quantities_testing_kernels.h:97-141 -- the hash lines before the final
 * assignment are dead in the reference; the value is 2^((x+3y+7z+2)&3). */
int oracle_scalefactor_space(int ix, int iy, int iz)
{
  int r = ix + 3 * iy + 7 * iz + 2;
  r = r & 3;
  return 1 << r;
}

/* quantities_testing_kernels.h:52-72 */
int oracle_scalefactor_energy(int ie)
{
  int r = (ie * 1366 + 150889) % 714025;
  r = r & 3;
  return 1 << r;
}

/* quantities_testing_kernels.h:77-95 */
int oracle_scalefactor_unknown(int iu)
{
  int r = (iu * 741 + 66037) % 312500;
  r = r & 3;
  return 1 << r;
}

/* quantities_testing_kernels.h:146-157 */
static int scalefactor_angle(int ia) { return 1 << (ia & 7); }

/* quantities_testing_kernels.h:219-332: the three face initialisers share one
 * formula; the caller passes the ghost coordinate (-1 or n) on the face axis. */
double oracle_init_face(int ia, int ix, int iy, int iz, int ie, int iu, int octant)
{
  return   ((double)(1 + ia))
         * ((double)scalefactor_angle(ia))
         * ((double)oracle_scalefactor_space(ix, iy, iz))
         * ((double)oracle_scalefactor_energy(ie))
         * ((double)oracle_scalefactor_unknown(iu))
         * ((double)(1 + octant));
}

/* quantities_testing_c.h:40-201 */
void oracle_init_am_matrices(int nm, int na, double* a, double* m)
{
  int o, im, ia, i;
  const size_t n = (size_t)nm * na * NOCT;
#define A_(im_, ia_, o_) a[(ia_) + (size_t)na * ((im_) + (size_t)nm * (o_))]
#define M_(im_, ia_, o_) m[(im_) + (size_t)nm * ((ia_) + (size_t)na * (o_))]
  for (i = 0; i < (int)n; ++i) { a[i] = 0.0; m[i] = 0.0; }

  for (o = 0; o < NOCT; ++o)
    for (i = 0; i < na; ++i) {
      const int quot = (i + 1) / nm;
      const int rem = (i + 1) % nm;
      A_(nm - 1, i, o) += quot;
      if (rem != 0) {
        A_(0, i, o) += -1.0;
        A_(rem, i, o) += 1.0;
      }
    }
  for (o = 0; o < NOCT; ++o)
    for (im = 0; im < nm - 2; ++im)
      for (ia = 0; ia < na; ++ia) {
        const int rv = 21 + (im + nm * ia) % 17;
        A_(im + 0, ia, o) += -1.0 * rv;
        A_(im + 1, ia, o) += 2.0 * rv;
        A_(im + 2, ia, o) += -1.0 * rv;
      }

  for (o = 0; o < NOCT; ++o)
    for (i = 0; i < nm; ++i) {
      const int quot = (i + 1) / na;
      const int rem = (i + 1) % na;
      M_(i, na - 1, o) += quot;
      if (rem != 0) {
        M_(i, 0, o) += -1.0;
        M_(i, rem, o) += 1.0;
      }
    }
  for (o = 0; o < NOCT; ++o)
    for (im = 0; im < nm; ++im)
      for (ia = 0; ia < na - 2; ++ia) {
        const int rv = 37 + (im + nm * ia) % 19;
        M_(im, ia + 0, o) += -1.0 * rv;
        M_(im, ia + 1, o) += 2.0 * rv;
        M_(im, ia + 2, o) += -1.0 * rv;
      }
  for (o = 0; o < NOCT; ++o)
    for (im = 0; im < nm; ++im)
      for (ia = 0; ia < na; ++ia) {
        M_(im, ia, o) /= NOCT;
        M_(im, ia, o) /= scalefactor_angle(ia);
      }
#undef A_
#undef M_
}

static size_t ind_state(int nx, int ny, int ne, int nm, int nu,
                        int ix, int iy, int iz, int ie, int im, int iu)
{
  return im + (size_t)nm * (iu + (size_t)nu * (ix + (size_t)nx *
              (iy + (size_t)ny * (ie + (size_t)ne * (size_t)iz))));
}

/* array_operations.c:26-48 with quantities_testing.h:60-90 (one proc, so the
 * x/y base offsets are 0). */
void oracle_init_state(int nx, int ny, int nz, int ne, int nm, int nu, double* v)
{
  int ix, iy, iz, ie, im, iu;
  for (iz = 0; iz < nz; ++iz)
    for (iy = 0; iy < ny; ++iy)
      for (ix = 0; ix < nx; ++ix)
        for (ie = 0; ie < ne; ++ie)
          for (im = 0; im < nm; ++im)
            for (iu = 0; iu < nu; ++iu)
              v[ind_state(nx, ny, ne, nm, nu, ix, iy, iz, ie, im, iu)] =
                    ((double)(1 + im))
                  * ((double)oracle_scalefactor_space(ix, iy, iz))
                  * ((double)oracle_scalefactor_energy(ie))
                  * ((double)oracle_scalefactor_unknown(iu));
}

/* The simple sweeper (sweeper_simple_c.h:83-277) for groups [ie0, ie1). */
void oracle_sweep_groups(int nx, int ny, int nz, int ne, int nm, int nu, int na,
                         int ie0, int ie1,
                         const double* a_from_m, const double* m_from_a,
                         const double* vi, double* vo)
{
  const size_t nfxy = (size_t)nx * ny * ne * na * nu;
  const size_t nfxz = (size_t)nx * nz * ne * na * nu;
  const size_t nfyz = (size_t)ny * nz * ne * na * nu;
  double* fxy = (double*)malloc(sizeof(double) * nfxy);
  double* fxz = (double*)malloc(sizeof(double) * nfxz);
  double* fyz = (double*)malloc(sizeof(double) * nfyz);
  double* vs = (double*)malloc(sizeof(double) * (size_t)na * nu);
  int o, ix, iy, iz, ie, im, ia, iu;

  /* face layouts (array_accessors_kernels.h:460-647), one octant per block:
   * facexy[ie][iy][ix][iu][ia], facexz[ie][iz][ix][iu][ia],
   * faceyz[ie][iz][iy][iu][ia] */
#define FXY(ix_, iy_, ie_, ia_, iu_) fxy[(ia_) + (size_t)na * ((iu_) + (size_t)nu * ((ix_) + (size_t)nx * ((iy_) + (size_t)ny * (ie_))))]
#define FXZ(ix_, iz_, ie_, ia_, iu_) fxz[(ia_) + (size_t)na * ((iu_) + (size_t)nu * ((ix_) + (size_t)nx * ((iz_) + (size_t)nz * (ie_))))]
#define FYZ(iy_, iz_, ie_, ia_, iu_) fyz[(ia_) + (size_t)na * ((iu_) + (size_t)nu * ((iy_) + (size_t)ny * ((iz_) + (size_t)nz * (ie_))))]
#define AFM(im_, ia_, o_) a_from_m[(ia_) + (size_t)na * ((im_) + (size_t)nm * (o_))]
#define MFA(im_, ia_, o_) m_from_a[(im_) + (size_t)nm * ((ia_) + (size_t)na * (o_))]
#define ST(v_, ix_, iy_, iz_, ie_, im_, iu_) v_[ind_state(nx, ny, ne, nm, nu, ix_, iy_, iz_, ie_, im_, iu_)]

  for (iz = 0; iz < nz; ++iz)
    for (iy = 0; iy < ny; ++iy)
      for (ix = 0; ix < nx; ++ix)
        for (ie = ie0; ie < ie1; ++ie)
          for (im = 0; im < nm; ++im)
            for (iu = 0; iu < nu; ++iu)
              ST(vo, ix, iy, iz, ie, im, iu) = 0.0;

  for (o = 0; o < NOCT; ++o) {
    const int dx = dir_x(o), dy = dir_y(o), dz = dir_z(o);

    /* boundary faces one cell outside the domain (sweeper_simple_c.h:140-186) */
    iz = dz == +1 ? -1 : nz;
    for (iu = 0; iu < nu; ++iu)
      for (iy = 0; iy < ny; ++iy)
        for (ix = 0; ix < nx; ++ix)
          for (ie = ie0; ie < ie1; ++ie)
            for (ia = 0; ia < na; ++ia)
              FXY(ix, iy, ie, ia, iu) = oracle_init_face(ia, ix, iy, iz, ie, iu, o);
    iy = dy == +1 ? -1 : ny;
    for (iu = 0; iu < nu; ++iu)
      for (iz = 0; iz < nz; ++iz)
        for (ix = 0; ix < nx; ++ix)
          for (ie = ie0; ie < ie1; ++ie)
            for (ia = 0; ia < na; ++ia)
              FXZ(ix, iz, ie, ia, iu) = oracle_init_face(ia, ix, iy, iz, ie, iu, o);
    ix = dx == +1 ? -1 : nx;
    for (iu = 0; iu < nu; ++iu)
      for (iz = 0; iz < nz; ++iz)
        for (iy = 0; iy < ny; ++iy)
          for (ie = ie0; ie < ie1; ++ie)
            for (ia = 0; ia < na; ++ia)
              FYZ(iy, iz, ie, ia, iu) = oracle_init_face(ia, ix, iy, iz, ie, iu, o);

    for (ie = ie0; ie < ie1; ++ie) {
      const int ixb = dx == +1 ? 0 : nx - 1, ixe = dx == +1 ? nx : -1;
      const int iyb = dy == +1 ? 0 : ny - 1, iye = dy == +1 ? ny : -1;
      const int izb = dz == +1 ? 0 : nz - 1, ize = dz == +1 ? nz : -1;
      for (iz = izb; iz != ize; iz += dz)
        for (iy = iyb; iy != iye; iy += dy)
          for (ix = ixb; ix != ixe; ix += dx) {
            /* moments -> angles (sweeper_simple_c.h:219-232) */
            for (iu = 0; iu < nu; ++iu)
              for (ia = 0; ia < na; ++ia) {
                double r = 0.0;
                for (im = 0; im < nm; ++im)
                  r += AFM(im, ia, o) * ST(vi, ix, iy, iz, ie, im, iu);
                vs[ia + (size_t)na * iu] = r;
              }

            /* Quantities_solve per angle (quantities_testing_kernels.h:337-447) */
            {
              const double s_oct = (double)(1 + o);
              const double s_oct_r = 1.0 / s_oct;
              const double s_sp = (double)oracle_scalefactor_space(ix, iy, iz);
              const double s_sp_r = 1.0 / s_sp;
              const double s_x_r = 1.0 / (double)oracle_scalefactor_space(ix - dx, iy, iz);
              const double s_y_r = 1.0 / (double)oracle_scalefactor_space(ix, iy - dy, iz);
              const double s_z_r = 1.0 / (double)oracle_scalefactor_space(ix, iy, iz - dz);
              for (ia = 0; ia < na; ++ia) {
                const double wx = 1.0 / 2.0;
                const double wy = 1.0 / 4.0;
                const double wz = 1.0 / 4.0 - 1.0 / (double)scalefactor_angle(ia);
                for (iu = 0; iu < nu; ++iu) {
                  double* vsp = &vs[ia + (size_t)na * iu];
                  const double result =
                      (*vsp * s_sp_r + (
                          FXY(ix, iy, ie, ia, iu) * wx * s_z_r
                        + FXZ(ix, iz, ie, ia, iu) * wy * s_y_r
                        + FYZ(iy, iz, ie, ia, iu) * wz * s_x_r
                      ) * s_oct_r) * s_sp;
                  const double scaled = result * s_oct;
                  *vsp = result;
                  FXY(ix, iy, ie, ia, iu) = scaled;
                  FXZ(ix, iz, ie, ia, iu) = scaled;
                  FYZ(iy, iz, ie, ia, iu) = scaled;
                }
              }
            }

            /* angles -> moments, accumulate (sweeper_simple_c.h:256-269) */
            for (iu = 0; iu < nu; ++iu)
              for (im = 0; im < nm; ++im) {
                double r = 0.0;
                for (ia = 0; ia < na; ++ia)
                  r += MFA(im, ia, o) * vs[ia + (size_t)na * iu];
                ST(vo, ix, iy, iz, ie, im, iu) += r;
              }
          }
    }
  }
#undef FXY
#undef FXZ
#undef FYZ
#undef AFM
#undef MFA
#undef ST
  free(fxy);
  free(fxz);
  free(fyz);
  free(vs);
}

void oracle_sweep(int nx, int ny, int nz, int ne, int nm, int nu, int na,
                  const double* a_from_m, const double* m_from_a,
                  const double* vi, double* vo)
{
  oracle_sweep_groups(nx, ny, nz, ne, nm, nu, na, 0, ne, a_from_m, m_from_a, vi, vo);
}

/* array_operations.c:69-110.  The reference sums in (iz, iy, ix, ie, im, iu)
 * loop order; the flat order below differs only in the order of the additions,
 * which is exact whenever all terms are integers below 2^53 (the built-in
 * Quantities). */
void oracle_state_norms(size_t n, const double* vi, const double* vo,
                        double* normsq, double* normsqdiff)
{
  size_t i;
  double s = 0.0, d = 0.0;
  for (i = 0; i < n; ++i) {
    const double diff = vi[i] - vo[i];
    s += vo[i] * vo[i];
    d += diff * diff;
  }
  *normsq = s;
  *normsqdiff = d;
}

double oracle_normsq_closed_form(int nx, int ny, int nz, int ne, int nm, int nu)
{
  double sp = 0.0, se = 0.0, sm = 0.0, su = 0.0;
  int ix, iy, iz, i;
  for (iz = 0; iz < nz; ++iz)
    for (iy = 0; iy < ny; ++iy)
      for (ix = 0; ix < nx; ++ix) {
        const double s = (double)oracle_scalefactor_space(ix, iy, iz);
        sp += s * s;
      }
  for (i = 0; i < ne; ++i) {
    const double s = (double)oracle_scalefactor_energy(i);
    se += s * s;
  }
  for (i = 0; i < nm; ++i) sm += (double)(1 + i) * (double)(1 + i);
  for (i = 0; i < nu; ++i) {
    const double s = (double)oracle_scalefactor_unknown(i);
    su += s * s;
  }
  return sp * se * sm * su;
}
