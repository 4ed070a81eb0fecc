/*
 * CPU oracle kernels -- TEST INFRASTRUCTURE ONLY (see clover_oracle.h).
 *
 * Loop-for-loop restatement of the reference kernels. Citations are
 * file:line in UK-MAC/CloverLeaf3D_ref. Fortran evaluates a+b+c as (a+b)+c and
 * a*b/c as (a*b)/c; every expression below is written with that association.
 * Compile with -ffp-contract=off so no multiply-add is fused.
 */
#include "clover_oracle.h"

#include <math.h>
#include <stddef.h>
#include <stdlib.h>

/* Reference layout: column major, lower bound min-2 in every axis. */
#define DECL_EXTENTS                                  \
  const long xlo = *x_min - 2, ylo = *y_min - 2, zlo = *z_min - 2; \
  const long nxc = *x_max - *x_min + 5, nyc = *y_max - *y_min + 5;  \
  const long nxv = *x_max - *x_min + 6, nyv = *y_max - *y_min + 6;  \
  (void)xlo; (void)ylo; (void)zlo; (void)nxc; (void)nyc; (void)nxv; (void)nyv

#define AT(a, nx, ny, j, k, l) \
  (a)[((long)(j) - xlo) + ((long)(k) - ylo) * (nx) + ((long)(l) - zlo) * (nx) * (ny)]
/* cell-centred (x_min-2:x_max+2, y_min-2:y_max+2, ...) */
#define C3(a, j, k, l) AT(a, nxc, nyc, j, k, l)
/* vertex / work (x_min-2:x_max+3, y_min-2:y_max+3, ...) */
#define V3(a, j, k, l) AT(a, nxv, nyv, j, k, l)
/* x-face (x_min-2:x_max+3, y_min-2:y_max+2, ...) */
#define X3(a, j, k, l) AT(a, nxv, nyc, j, k, l)
/* y-face (x_min-2:x_max+2, y_min-2:y_max+3, ...) */
#define Y3(a, j, k, l) AT(a, nxc, nyv, j, k, l)
/* z-face (x_min-2:x_max+2, y_min-2:y_max+2, z_min-2:z_max+3) */
#define Z3(a, j, k, l) AT(a, nxc, nyc, j, k, l)
#define DX(a, j) (a)[(long)(j) - xlo]
#define DY(a, k) (a)[(long)(k) - ylo]
#define DZ(a, l) (a)[(long)(l) - zlo]

static inline double fmin2(double a, double b) { return b < a ? b : a; }
static inline double fmax2(double a, double b) { return b > a ? b : a; }
/* Fortran SIGN(a,b): |a| with the sign of b (gfortran honours -0.0). */
static inline double fsign(double a, double b) { return copysign(fabs(a), b); }

/* ideal_gas_kernel.f90:47-58 */
void oracle_ideal_gas_kernel(const int *x_min, const int *x_max, const int *y_min,
                             const int *y_max, const int *z_min, const int *z_max,
                             double *density, double *energy, double *pressure,
                             double *soundspeed) {
  DECL_EXTENTS;
#pragma omp parallel for
  for (int l = *z_min; l <= *z_max; l++)
    for (int k = *y_min; k <= *y_max; k++)
      for (int j = *x_min; j <= *x_max; j++) {
        double d = C3(density, j, k, l);
        double v = 1.0 / d;
        double p = (1.4 - 1.0) * d * C3(energy, j, k, l);
        C3(pressure, j, k, l) = p;
        double pressurebyenergy = (1.4 - 1.0) * d;
        double pressurebyvolume = -d * p;
        double ss2 = v * v * (p * pressurebyenergy - pressurebyvolume);
        C3(soundspeed, j, k, l) = sqrt(ss2);
      }
}

/* viscosity_kernel.f90:71-134 */
void oracle_viscosity_kernel(const int *x_min, const int *x_max, const int *y_min,
                             const int *y_max, const int *z_min, const int *z_max,
                             const double *xarea, const double *yarea, const double *zarea,
                             const double *celldx, const double *celldy, const double *celldz,
                             const double *density0, const double *pressure,
                             double *viscosity, const double *xvel0, const double *yvel0,
                             const double *zvel0) {
  DECL_EXTENTS;
#pragma omp parallel for
  for (int l = *z_min; l <= *z_max; l++)
    for (int k = *y_min; k <= *y_max; k++)
      for (int j = *x_min; j <= *x_max; j++) {
#define U(a, b, c) V3(xvel0, j + (a), k + (b), l + (c))
#define VV(a, b, c) V3(yvel0, j + (a), k + (b), l + (c))
#define W(a, b, c) V3(zvel0, j + (a), k + (b), l + (c))
        double ugradx1 = U(0, 0, 0) + U(0, 1, 0) + U(0, 0, 1) + U(0, 1, 1);
        double ugradx2 = U(1, 0, 0) + U(1, 1, 0) + U(1, 0, 1) + U(1, 1, 1);
        double ugrady1 = U(0, 0, 0) + U(1, 0, 0) + U(0, 0, 1) + U(1, 0, 1);
        double ugrady2 = U(0, 1, 0) + U(1, 1, 0) + U(0, 1, 1) + U(1, 1, 1);
        double ugradz1 = U(0, 0, 0) + U(1, 0, 0) + U(0, 1, 0) + U(1, 1, 0);
        double ugradz2 = U(0, 0, 1) + U(1, 0, 1) + U(0, 1, 1) + U(1, 1, 1);

        double vgradx1 = VV(0, 0, 0) + VV(0, 1, 0) + VV(0, 0, 1) + VV(0, 1, 1);
        double vgradx2 = VV(1, 0, 0) + VV(1, 1, 0) + VV(1, 0, 1) + VV(1, 1, 1);
        double vgrady1 = VV(0, 0, 0) + VV(1, 0, 0) + VV(0, 0, 1) + VV(1, 0, 1);
        double vgrady2 = VV(0, 1, 0) + VV(1, 1, 0) + VV(0, 1, 1) + VV(1, 1, 1);
        double vgradz1 = VV(0, 0, 0) + VV(1, 0, 0) + VV(0, 1, 0) + VV(1, 1, 0);
        double vgradz2 = VV(0, 0, 1) + VV(1, 0, 1) + VV(0, 1, 1) + VV(1, 1, 1);

        double wgradx1 = W(0, 0, 0) + W(0, 1, 0) + W(0, 0, 1) + W(0, 1, 1);
        double wgradx2 = W(1, 0, 0) + W(1, 1, 0) + W(1, 0, 1) + W(1, 1, 1);
        double wgrady1 = W(0, 0, 0) + W(1, 0, 0) + W(0, 0, 1) + W(1, 0, 1);
        double wgrady2 = W(0, 1, 0) + W(1, 1, 0) + W(0, 1, 1) + W(1, 1, 1);
        double wgradz1 = W(0, 0, 0) + W(1, 0, 0) + W(0, 1, 0) + W(1, 1, 0);
        double wgradz2 = W(0, 0, 1) + W(1, 0, 1) + W(0, 1, 1) + W(1, 1, 1);
#undef U
#undef VV
#undef W
        double cdx = DX(celldx, j), cdy = DY(celldy, k), cdz = DZ(celldz, l);
        double div = (X3(xarea, j, k, l) * (ugradx2 - ugradx1) +
                      Y3(yarea, j, k, l) * (vgrady2 - vgrady1)) +
                     Z3(zarea, j, k, l) * (wgradz2 - wgradz1);

        double xx = 0.25 * (ugradx2 - ugradx1) / cdx;
        double yy = 0.25 * (vgrady2 - vgrady1) / cdy;
        double zz = 0.25 * (wgradz2 - wgradz1) / cdz;
        double xy = 0.25 * (ugrady2 - ugrady1) / cdy + 0.25 * (vgradx2 - vgradx1) / cdx;
        double xz = 0.25 * (ugradz2 - ugradz1) / cdz + 0.25 * (wgradx2 - wgradx1) / cdx;
        double yz = 0.25 * (vgradz2 - vgradz1) / cdz + 0.25 * (wgrady2 - wgrady1) / cdy;

        double pgradx = (C3(pressure, j + 1, k, l) - C3(pressure, j - 1, k, l)) /
                        (cdx + DX(celldx, j + 1));
        double pgrady = (C3(pressure, j, k + 1, l) - C3(pressure, j, k - 1, l)) /
                        (cdy + DY(celldy, k + 1));
        double pgradz = (C3(pressure, j, k, l + 1) - C3(pressure, j, k, l - 1)) /
                        (cdz + DZ(celldz, l + 1));

        double pgradx2 = pgradx * pgradx;
        double pgrady2 = pgrady * pgrady;
        double pgradz2 = pgradz * pgradz;

        double limiter = (xx * pgradx2 + yy * pgrady2 + zz * pgradz2 + xy * pgradx * pgrady +
                          xz * pgradx * pgradz + yz * pgrady * pgradz) /
                         fmax2(pgradx2 + pgrady2 + pgradz2, 1.0e-16);

        if ((limiter > 0.0) || (div >= 0.0)) {
          C3(viscosity, j, k, l) = 0.0;
        } else {
          pgradx = fsign(fmax2(1.0e-16, fabs(pgradx)), pgradx);
          pgrady = fsign(fmax2(1.0e-16, fabs(pgrady)), pgrady);
          pgradz = fsign(fmax2(1.0e-16, fabs(pgradz)), pgradz);
          double pgrad = sqrt(pgradx * pgradx + pgrady * pgrady + pgradz * pgradz);
          double xgrad = fabs(cdx * pgrad / pgradx);
          double ygrad = fabs(cdy * pgrad / pgrady);
          double zgrad = fabs(cdz * pgrad / pgradz);
          double grad = fmin2(fmin2(xgrad, ygrad), zgrad);
          double grad2 = grad * grad;
          C3(viscosity, j, k, l) = 2.0 * C3(density0, j, k, l) * grad2 * limiter * limiter;
        }
      }
}

/* calc_dt_kernel.f90:94-181 */
void oracle_calc_dt_kernel(const int *x_min, const int *x_max, const int *y_min,
                           const int *y_max, const int *z_min, const int *z_max,
                           const double *g_small, const double *g_big, const double *dtmin,
                           const double *dtc_safe, const double *dtu_safe,
                           const double *dtv_safe, const double *dtw_safe,
                           const double *dtdiv_safe, const double *xarea,
                           const double *yarea, const double *zarea, const double *cellx,
                           const double *celly, const double *cellz, const double *celldx,
                           const double *celldy, const double *celldz, const double *volume,
                           const double *density0, const double *energy0,
                           const double *pressure, const double *viscosity_a,
                           const double *soundspeed, const double *xvel0,
                           const double *yvel0, const double *zvel0, double *dt_min,
                           double *dt_min_val, int *dtl_control, double *xl_pos,
                           double *yl_pos, double *zl_pos, int *jldt, int *kldt, int *lldt,
                           int *small) {
  DECL_EXTENTS;
  (void)energy0;
  (void)pressure;
  *small = 0;
  *dt_min_val = *g_big;
  /* jkl_control=1.1 assigns a default-REAL literal to a REAL(8) (:97) */
  double jkl_control = (double)1.1f;

#pragma omp parallel for
  for (int l = *z_min; l <= *z_max; l++)
    for (int k = *y_min; k <= *y_max; k++)
      for (int j = *x_min; j <= *x_max; j++) {
        double m = fmin2(fmin2(DX(celldx, j), DY(celldy, k)), DZ(celldz, l));
        double ds = 1.0 / (m * m);

        double cc = C3(soundspeed, j, k, l) * C3(soundspeed, j, k, l);
        cc = cc + 2.0 * C3(viscosity_a, j, k, l) / C3(density0, j, k, l);

        double dtct = ds * cc;
        dtct = *dtc_safe * 1.0 / fmax2(sqrt(dtct), *g_small);

        double vol = C3(volume, j, k, l);
        double xa = X3(xarea, j, k, l);
        double du1 = (V3(xvel0, j, k, l) + V3(xvel0, j, k + 1, l) + V3(xvel0, j, k, l + 1) +
                      V3(xvel0, j, k + 1, l + 1)) * xa;
        double du2 = (V3(xvel0, j + 1, k, l) + V3(xvel0, j + 1, k + 1, l) +
                      V3(xvel0, j + 1, k, l + 1) + V3(xvel0, j + 1, k + 1, l + 1)) * xa;
        double dtut = *dtu_safe * 4.0 * vol / fmax2(fmax2(fabs(du1), fabs(du2)), 1.0e-5 * vol);

        double ya = Y3(yarea, j, k, l);
        double dv1 = (V3(yvel0, j, k, l) + V3(yvel0, j + 1, k, l) + V3(yvel0, j, k, l + 1) +
                      V3(yvel0, j + 1, k, l + 1)) * ya;
        double dv2 = (V3(yvel0, j, k + 1, l) + V3(yvel0, j + 1, k + 1, l) +
                      V3(yvel0, j, k + 1, l + 1) + V3(yvel0, j + 1, k + 1, l + 1)) * ya;
        double dtvt = *dtv_safe * 4.0 * vol / fmax2(fmax2(fabs(dv1), fabs(dv2)), 1.0e-5 * vol);

        /* both faces use zarea(j,k,l) (:124-125) */
        double za = Z3(zarea, j, k, l);
        double dw1 = (V3(zvel0, j, k, l) + V3(zvel0, j, k + 1, l) + V3(zvel0, j + 1, k, l) +
                      V3(zvel0, j + 1, k + 1, l)) * za;
        double dw2 = (V3(zvel0, j, k, l + 1) + V3(zvel0, j, k + 1, l + 1) +
                      V3(zvel0, j + 1, k, l + 1) + V3(zvel0, j + 1, k + 1, l + 1)) * za;
        double dtwt = *dtw_safe * 4.0 * vol / fmax2(fmax2(fabs(dw1), fabs(dw2)), 1.0e-5 * vol);

        double div = du2 - du1 + dv2 - dv1 + dw2 - dw1;
        double dtdivt = *dtdiv_safe * 4.0 * vol / fmax2(vol * 1.0e-05, fabs(div));

        double mn = fmin2(fmin2(fmin2(fmin2(dtct, dtut), dtvt), dtwt), dtdivt);
        V3(dt_min, j, k, l) = mn;
      }

  double best = *dt_min_val;
  for (int l = *z_min; l <= *z_max; l++)
    for (int k = *y_min; k <= *y_max; k++)
      for (int j = *x_min; j <= *x_max; j++)
        if (V3(dt_min, j, k, l) < best) best = V3(dt_min, j, k, l);
  *dt_min_val = best;

  /* :154-161 (jkl_control is never updated, so these are constant) */
  *dtl_control = (int)((double)10.01f * (jkl_control - (double)(int)jkl_control));
  jkl_control = jkl_control - (jkl_control - (double)(int)jkl_control);
  *jldt = ((int)jkl_control) % (*x_max);
  *kldt = (int)(1.0 + (jkl_control / (double)(*x_max)));
  *lldt = (int)(1.0 + (jkl_control / (double)(*x_max)));
  *xl_pos = DX(cellx, *jldt);
  *yl_pos = DY(celly, *kldt);
  *zl_pos = DZ(cellz, *lldt);

  if (*dt_min_val < *dtmin) *small = 1;
}

/* PdV_kernel.f90:72-166 */
void oracle_pdv_kernel(const int *predict, const int *x_min, const int *x_max,
                       const int *y_min, const int *y_max, const int *z_min,
                       const int *z_max, const double *dt, const double *xarea,
                       const double *yarea, const double *zarea, const double *volume,
                       const double *density0, double *density1, const double *energy0,
                       double *energy1, const double *pressure, const double *viscosity,
                       const double *xvel0, const double *xvel1, const double *yvel0,
                       const double *yvel1, const double *zvel0, const double *zvel1) {
  DECL_EXTENTS;
  const int pred = *predict != 0;
  /* predictor: both velocity sets are vel0 and the flux carries an extra *0.5 */
  const double *xb = pred ? xvel0 : xvel1;
  const double *yb = pred ? yvel0 : yvel1;
  const double *zb = pred ? zvel0 : zvel1;
  const double dtv = *dt;
#pragma omp parallel for
  for (int l = *z_min; l <= *z_max; l++)
    for (int k = *y_min; k <= *y_max; k++)
      for (int j = *x_min; j <= *x_max; j++) {
#define XF(jj)                                                                        \
  (X3(xarea, jj, k, l) *                                                              \
   (V3(xvel0, jj, k, l) + V3(xvel0, jj, k + 1, l) + V3(xvel0, jj, k, l + 1) +         \
    V3(xvel0, jj, k + 1, l + 1) + V3(xb, jj, k, l) + V3(xb, jj, k + 1, l) +            \
    V3(xb, jj, k, l + 1) + V3(xb, jj, k + 1, l + 1)))
#define YF(kk)                                                                        \
  (Y3(yarea, j, kk, l) *                                                              \
   (V3(yvel0, j, kk, l) + V3(yvel0, j + 1, kk, l) + V3(yvel0, j, kk, l + 1) +         \
    V3(yvel0, j + 1, kk, l + 1) + V3(yb, j, kk, l) + V3(yb, j + 1, kk, l) +            \
    V3(yb, j, kk, l + 1) + V3(yb, j + 1, kk, l + 1)))
#define ZF(ll)                                                                        \
  (Z3(zarea, j, k, ll) *                                                              \
   (V3(zvel0, j, k, ll) + V3(zvel0, j + 1, k, ll) + V3(zvel0, j, k + 1, ll) +         \
    V3(zvel0, j + 1, k + 1, ll) + V3(zb, j, k, ll) + V3(zb, j + 1, k, ll) +            \
    V3(zb, j, k + 1, ll) + V3(zb, j + 1, k + 1, ll)))
        double left_flux, right_flux, bottom_flux, top_flux, back_flux, front_flux;
        if (pred) {
          left_flux = XF(j) * 0.125 * dtv * 0.5;
          right_flux = XF(j + 1) * 0.125 * dtv * 0.5;
          bottom_flux = YF(k) * 0.125 * dtv * 0.5;
          top_flux = YF(k + 1) * 0.125 * dtv * 0.5;
          back_flux = ZF(l) * 0.125 * dtv * 0.5;
          front_flux = ZF(l + 1) * 0.125 * dtv * 0.5;
        } else {
          left_flux = XF(j) * 0.125 * dtv;
          right_flux = XF(j + 1) * 0.125 * dtv;
          bottom_flux = YF(k) * 0.125 * dtv;
          top_flux = YF(k + 1) * 0.125 * dtv;
          back_flux = ZF(l) * 0.125 * dtv;
          front_flux = ZF(l + 1) * 0.125 * dtv;
        }
#undef XF
#undef YF
#undef ZF
        double total_flux =
            right_flux - left_flux + top_flux - bottom_flux + front_flux - back_flux;
        double vol = C3(volume, j, k, l);
        double vol_change_s = vol / (vol + total_flux);
        /* min_cell_volume (:102-105) is computed and never used */
        double recip_volume = 1.0 / vol;
        double d0 = C3(density0, j, k, l);
        double energy_change =
            (C3(pressure, j, k, l) / d0 + C3(viscosity, j, k, l) / d0) * total_flux *
            recip_volume;
        C3(energy1, j, k, l) = C3(energy0, j, k, l) - energy_change;
        C3(density1, j, k, l) = d0 * vol_change_s;
      }
}

/* revert_kernel.f90:41-61 */
void oracle_revert_kernel(const int *x_min, const int *x_max, const int *y_min,
                          const int *y_max, const int *z_min, const int *z_max,
                          const double *density0, double *density1,
                          const double *energy0, double *energy1) {
  DECL_EXTENTS;
#pragma omp parallel for
  for (int l = *z_min; l <= *z_max; l++)
    for (int k = *y_min; k <= *y_max; k++)
      for (int j = *x_min; j <= *x_max; j++) {
        C3(density1, j, k, l) = C3(density0, j, k, l);
        C3(energy1, j, k, l) = C3(energy0, j, k, l);
      }
}

/* accelerate_kernel.f90:61-109 */
void oracle_accelerate_kernel(const int *x_min, const int *x_max, const int *y_min,
                              const int *y_max, const int *z_min, const int *z_max,
                              const double *dt, const double *xarea, const double *yarea,
                              const double *zarea, const double *volume,
                              const double *density0, const double *pressure,
                              const double *viscosity, const double *xvel0,
                              const double *yvel0, const double *zvel0, double *xvel1,
                              double *yvel1, double *zvel1) {
  DECL_EXTENTS;
  const double dtv = *dt;
#pragma omp parallel for
  for (int l = *z_min; l <= *z_max + 1; l++)
    for (int k = *y_min; k <= *y_max + 1; k++)
      for (int j = *x_min; j <= *x_max + 1; j++) {
#define DV(a, b, c) (C3(density0, j + (a), k + (b), l + (c)) * C3(volume, j + (a), k + (b), l + (c)))
        double nodal_mass = (DV(-1, -1, 0) + DV(0, -1, 0) + DV(0, 0, 0) + DV(-1, 0, 0) +
                             DV(-1, -1, -1) + DV(0, -1, -1) + DV(0, 0, -1) + DV(-1, 0, -1)) *
                            0.125;
#undef DV
        double stepbymass_s = 0.25 * dtv / nodal_mass;
#define P(a, b, c) C3(pressure, j + (a), k + (b), l + (c))
#define Q(a, b, c) C3(viscosity, j + (a), k + (b), l + (c))
#define XA(a, b, c) X3(xarea, j + (a), k + (b), l + (c))
#define YA(a, b, c) Y3(yarea, j + (a), k + (b), l + (c))
#define ZA(a, b, c) Z3(zarea, j + (a), k + (b), l + (c))
        double xvel1_s =
            V3(xvel0, j, k, l) -
            stepbymass_s * (XA(0, 0, 0) * (P(0, 0, 0) - P(-1, 0, 0)) +
                            XA(0, -1, 0) * (P(0, -1, 0) - P(-1, -1, 0)) +
                            XA(0, 0, -1) * (P(0, 0, -1) - P(-1, 0, -1)) +
                            XA(0, -1, -1) * (P(0, -1, -1) - P(-1, -1, -1)));
        double yvel1_s =
            V3(yvel0, j, k, l) -
            stepbymass_s * (YA(0, 0, 0) * (P(0, 0, 0) - P(0, -1, 0)) +
                            YA(-1, 0, 0) * (P(-1, 0, 0) - P(-1, -1, 0)) +
                            YA(0, 0, -1) * (P(0, 0, -1) - P(0, -1, -1)) +
                            YA(-1, 0, -1) * (P(-1, 0, -1) - P(-1, -1, -1)));
        double zvel1_s =
            V3(zvel0, j, k, l) -
            stepbymass_s * (ZA(0, 0, 0) * (P(0, 0, 0) - P(0, 0, -1)) +
                            ZA(0, -1, 0) * (P(0, -1, 0) - P(0, -1, -1)) +
                            ZA(-1, 0, 0) * (P(-1, 0, 0) - P(-1, 0, -1)) +
                            ZA(-1, -1, 0) * (P(-1, -1, 0) - P(-1, -1, -1)));
        V3(xvel1, j, k, l) =
            xvel1_s - stepbymass_s * (XA(0, 0, 0) * (Q(0, 0, 0) - Q(-1, 0, 0)) +
                                      XA(0, -1, 0) * (Q(0, -1, 0) - Q(-1, -1, 0)) +
                                      XA(0, 0, -1) * (Q(0, 0, -1) - Q(-1, 0, -1)) +
                                      XA(0, -1, -1) * (Q(0, -1, -1) - Q(-1, -1, -1)));
        V3(yvel1, j, k, l) =
            yvel1_s - stepbymass_s * (YA(0, 0, 0) * (Q(0, 0, 0) - Q(0, -1, 0)) +
                                      YA(-1, 0, 0) * (Q(-1, 0, 0) - Q(-1, -1, 0)) +
                                      YA(0, 0, -1) * (Q(0, 0, -1) - Q(0, -1, -1)) +
                                      YA(-1, 0, -1) * (Q(-1, 0, -1) - Q(-1, -1, -1)));
        V3(zvel1, j, k, l) =
            zvel1_s - stepbymass_s * (ZA(0, 0, 0) * (Q(0, 0, 0) - Q(0, 0, -1)) +
                                      ZA(0, -1, 0) * (Q(0, -1, 0) - Q(0, -1, -1)) +
                                      ZA(-1, 0, 0) * (Q(-1, 0, 0) - Q(-1, 0, -1)) +
                                      ZA(-1, -1, 0) * (Q(-1, -1, 0) - Q(-1, -1, -1)));
#undef P
#undef Q
#undef XA
#undef YA
#undef ZA
      }
}

/* flux_calc_kernel.f90:58-91 */
void oracle_flux_calc_kernel(const int *x_min, const int *x_max, const int *y_min,
                             const int *y_max, const int *z_min, const int *z_max,
                             const double *dt, const double *xarea, const double *yarea,
                             const double *zarea, const double *xvel0, const double *yvel0,
                             const double *zvel0, const double *xvel1, const double *yvel1,
                             const double *zvel1, double *vol_flux_x, double *vol_flux_y,
                             double *vol_flux_z) {
  DECL_EXTENTS;
  const double dtv = *dt;
#pragma omp parallel for
  for (int l = *z_min; l <= *z_max; l++)
    for (int k = *y_min; k <= *y_max; k++)
      for (int j = *x_min; j <= *x_max + 1; j++)
        X3(vol_flux_x, j, k, l) =
            0.125 * dtv * X3(xarea, j, k, l) *
            (V3(xvel0, j, k, l) + V3(xvel0, j, k + 1, l) + V3(xvel0, j, k, l + 1) +
             V3(xvel0, j, k + 1, l + 1) + V3(xvel1, j, k, l) + V3(xvel1, j, k + 1, l) +
             V3(xvel1, j, k, l + 1) + V3(xvel1, j, k + 1, l + 1));
#pragma omp parallel for
  for (int l = *z_min; l <= *z_max; l++)
    for (int k = *y_min; k <= *y_max + 1; k++)
      for (int j = *x_min; j <= *x_max; j++)
        Y3(vol_flux_y, j, k, l) =
            0.125 * dtv * Y3(yarea, j, k, l) *
            (V3(yvel0, j, k, l) + V3(yvel0, j + 1, k, l) + V3(yvel0, j, k, l + 1) +
             V3(yvel0, j + 1, k, l + 1) + V3(yvel1, j, k, l) + V3(yvel1, j + 1, k, l) +
             V3(yvel1, j, k, l + 1) + V3(yvel1, j + 1, k, l + 1));
  /* the zvel0 sum repeats zvel0(j+1,k,l) and omits zvel0(j,k+1,l) (:86).
   * ORACLE_FLUX_Z_PDV (a test-only build, never the checker of a parity
   * test) takes the four nodes PdV_kernel.f90 sums instead, to show that the
   * FP64 run's mass drift comes from this sum alone. */
#ifdef ORACLE_FLUX_Z_PDV
#define FLUX_Z_NODE3 V3(zvel0, j, k + 1, l)
#else
#define FLUX_Z_NODE3 V3(zvel0, j + 1, k, l)
#endif
#pragma omp parallel for
  for (int l = *z_min; l <= *z_max + 1; l++)
    for (int k = *y_min; k <= *y_max; k++)
      for (int j = *x_min; j <= *x_max; j++)
        Z3(vol_flux_z, j, k, l) =
            0.125 * dtv * Z3(zarea, j, k, l) *
            (V3(zvel0, j, k, l) + V3(zvel0, j + 1, k, l) + FLUX_Z_NODE3 +
             V3(zvel0, j + 1, k + 1, l) + V3(zvel1, j, k, l) + V3(zvel1, j + 1, k, l) +
             V3(zvel1, j, k + 1, l) + V3(zvel1, j + 1, k + 1, l));
#undef FLUX_Z_NODE3
}

/* Van Leer limited face flux, shared by the three directions of
 * advec_cell_kernel.f90:129-169 (x), :224-264 (y), :319-359 (z). */
static inline double cell_limiter(double sig, double sigma3, double sigma4, double diffuw,
                                  double diffdw) {
  const double one_by_six = 1.0 / 6.0;
  if (diffuw * diffdw > 0.0) {
    return (1.0 - sig) * fsign(1.0, diffdw) *
           fmin2(fmin2(fabs(diffuw), fabs(diffdw)),
                 one_by_six * (sigma3 * fabs(diffuw) + sigma4 * fabs(diffdw)));
  }
  return 0.0;
}

/* advec_cell_kernel.f90:95-379 */
void oracle_advec_cell_kernel(const int *x_min, const int *x_max, const int *y_min,
                              const int *y_max, const int *z_min, const int *z_max,
                              const int *advect_x, const int *dir, const int *sweep_number,
                              const double *vertexdx, const double *vertexdy,
                              const double *vertexdz, const double *volume,
                              double *density1, double *energy1, double *mass_flux_x,
                              const double *vol_flux_x, double *mass_flux_y,
                              const double *vol_flux_y, double *mass_flux_z,
                              const double *vol_flux_z, double *pre_vol, double *post_vol,
                              double *pre_mass, double *post_mass, double *advec_vol,
                              double *post_ener, double *ener_flux) {
  DECL_EXTENTS;
  const int sweep = *sweep_number;
  const int ax = *advect_x != 0;

  if (*dir == 1) {
    if (sweep == 1) {
#pragma omp parallel for
      for (int l = *z_min - 2; l <= *z_max + 2; l++)
        for (int k = *y_min - 2; k <= *y_max + 2; k++)
          for (int j = *x_min - 2; j <= *x_max + 2; j++) {
            V3(pre_vol, j, k, l) =
                C3(volume, j, k, l) +
                (X3(vol_flux_x, j + 1, k, l) - X3(vol_flux_x, j, k, l) +
                 Y3(vol_flux_y, j, k + 1, l) - Y3(vol_flux_y, j, k, l) +
                 Z3(vol_flux_z, j, k, l + 1) - Z3(vol_flux_z, j, k, l));
            V3(post_vol, j, k, l) =
                V3(pre_vol, j, k, l) - (X3(vol_flux_x, j + 1, k, l) - X3(vol_flux_x, j, k, l));
          }
    } else if (sweep == 3) {
#pragma omp parallel for
      for (int l = *z_min - 2; l <= *z_max + 2; l++)
        for (int k = *y_min - 2; k <= *y_max + 2; k++)
          for (int j = *x_min - 2; j <= *x_max + 2; j++) {
            V3(pre_vol, j, k, l) =
                C3(volume, j, k, l) + X3(vol_flux_x, j + 1, k, l) - X3(vol_flux_x, j, k, l);
            V3(post_vol, j, k, l) = C3(volume, j, k, l);
          }
    }

#pragma omp parallel for
    for (int l = *z_min; l <= *z_max; l++)
      for (int k = *y_min; k <= *y_max; k++)
        for (int j = *x_min; j <= *x_max + 2; j++) {
          int upwind, donor, downwind, dif;
          if (X3(vol_flux_x, j, k, l) > 0.0) {
            upwind = j - 2; donor = j - 1; downwind = j; dif = donor;
          } else {
            upwind = (j + 1 < *x_max + 2) ? j + 1 : *x_max + 2;
            donor = j; downwind = j - 1; dif = upwind;
          }
          double sigmat = fabs(X3(vol_flux_x, j, k, l)) / V3(pre_vol, donor, k, l);
          double sigma3 = (1.0 + sigmat) * (DX(vertexdx, j) / DX(vertexdx, dif));
          double sigma4 = 2.0 - sigmat;
          double sigmav = sigmat;

          double diffuw = C3(density1, donor, k, l) - C3(density1, upwind, k, l);
          double diffdw = C3(density1, downwind, k, l) - C3(density1, donor, k, l);
          double limiter = cell_limiter(sigmav, sigma3, sigma4, diffuw, diffdw);
          X3(mass_flux_x, j, k, l) =
              X3(vol_flux_x, j, k, l) * (C3(density1, donor, k, l) + limiter);

          double sigmam = fabs(X3(mass_flux_x, j, k, l)) /
                          (C3(density1, donor, k, l) * V3(pre_vol, donor, k, l));
          diffuw = C3(energy1, donor, k, l) - C3(energy1, upwind, k, l);
          diffdw = C3(energy1, downwind, k, l) - C3(energy1, donor, k, l);
          limiter = cell_limiter(sigmam, sigma3, sigma4, diffuw, diffdw);
          V3(ener_flux, j, k, l) =
              X3(mass_flux_x, j, k, l) * (C3(energy1, donor, k, l) + limiter);
        }

#pragma omp parallel for
    for (int l = *z_min; l <= *z_max; l++)
      for (int k = *y_min; k <= *y_max; k++)
        for (int j = *x_min; j <= *x_max; j++) {
          V3(pre_mass, j, k, l) = C3(density1, j, k, l) * V3(pre_vol, j, k, l);
          V3(post_mass, j, k, l) = V3(pre_mass, j, k, l) + X3(mass_flux_x, j, k, l) -
                                   X3(mass_flux_x, j + 1, k, l);
          V3(post_ener, j, k, l) = (C3(energy1, j, k, l) * V3(pre_mass, j, k, l) +
                                    V3(ener_flux, j, k, l) - V3(ener_flux, j + 1, k, l)) /
                                   V3(post_mass, j, k, l);
          V3(advec_vol, j, k, l) = V3(pre_vol, j, k, l) + X3(vol_flux_x, j, k, l) -
                                   X3(vol_flux_x, j + 1, k, l);
          C3(density1, j, k, l) = V3(post_mass, j, k, l) / V3(advec_vol, j, k, l);
          C3(energy1, j, k, l) = V3(post_ener, j, k, l);
        }

  } else if (*dir == 2) {
    if (sweep == 2) {
      if (ax) {
#pragma omp parallel for
        for (int l = *z_min - 2; l <= *z_max + 2; l++)
          for (int k = *y_min - 2; k <= *y_max + 2; k++)
            for (int j = *x_min - 2; j <= *x_max + 2; j++) {
              V3(pre_vol, j, k, l) = C3(volume, j, k, l) + Y3(vol_flux_y, j, k + 1, l) -
                                     Y3(vol_flux_y, j, k, l) + Z3(vol_flux_z, j, k, l + 1) -
                                     Z3(vol_flux_z, j, k, l);
              V3(post_vol, j, k, l) = V3(pre_vol, j, k, l) -
                                      (Y3(vol_flux_y, j, k + 1, l) - Y3(vol_flux_y, j, k, l));
            }
      } else {
#pragma omp parallel for
        for (int l = *z_min - 2; l <= *z_max + 2; l++)
          for (int k = *y_min - 2; k <= *y_max + 2; k++)
            for (int j = *x_min - 2; j <= *x_max + 2; j++) {
              V3(pre_vol, j, k, l) = C3(volume, j, k, l) + Y3(vol_flux_y, j, k + 1, l) -
                                     Y3(vol_flux_y, j, k, l) + X3(vol_flux_x, j + 1, k, l) -
                                     X3(vol_flux_x, j, k, l);
              V3(post_vol, j, k, l) = V3(pre_vol, j, k, l) -
                                      (Y3(vol_flux_y, j, k + 1, l) - Y3(vol_flux_y, j, k, l));
            }
      }
    }

    /* the y flux pass runs l up to z_max+2 (:220); the test-only
     * ORACLE_SYMMETRIC_HALO build stops it at z_max, like the x and z passes
     * (the rotation tests use it to show that this range is what separates a
     * flow along y from the same flow along x) */
#ifdef ORACLE_SYMMETRIC_HALO
    const int y_flux_l_hi = *z_max;
#else
    const int y_flux_l_hi = *z_max + 2;
#endif
#pragma omp parallel for
    for (int l = *z_min; l <= y_flux_l_hi; l++)
      for (int k = *y_min; k <= *y_max + 2; k++)
        for (int j = *x_min; j <= *x_max; j++) {
          int upwind, donor, downwind, dif;
          if (Y3(vol_flux_y, j, k, l) > 0.0) {
            upwind = k - 2; donor = k - 1; downwind = k; dif = donor;
          } else {
            upwind = (k + 1 < *y_max + 2) ? k + 1 : *y_max + 2;
            donor = k; downwind = k - 1; dif = upwind;
          }
          double sigmat = fabs(Y3(vol_flux_y, j, k, l)) / V3(pre_vol, j, donor, l);
          double sigma3 = (1.0 + sigmat) * (DY(vertexdy, k) / DY(vertexdy, dif));
          double sigma4 = 2.0 - sigmat;
          double sigmav = sigmat;

          double diffuw = C3(density1, j, donor, l) - C3(density1, j, upwind, l);
          double diffdw = C3(density1, j, downwind, l) - C3(density1, j, donor, l);
          double limiter = cell_limiter(sigmav, sigma3, sigma4, diffuw, diffdw);
          Y3(mass_flux_y, j, k, l) =
              Y3(vol_flux_y, j, k, l) * (C3(density1, j, donor, l) + limiter);

          double sigmam = fabs(Y3(mass_flux_y, j, k, l)) /
                          (C3(density1, j, donor, l) * V3(pre_vol, j, donor, l));
          diffuw = C3(energy1, j, donor, l) - C3(energy1, j, upwind, l);
          diffdw = C3(energy1, j, downwind, l) - C3(energy1, j, donor, l);
          limiter = cell_limiter(sigmam, sigma3, sigma4, diffuw, diffdw);
          V3(ener_flux, j, k, l) =
              Y3(mass_flux_y, j, k, l) * (C3(energy1, j, donor, l) + limiter);
        }

#pragma omp parallel for
    for (int l = *z_min; l <= *z_max; l++)
      for (int k = *y_min; k <= *y_max; k++)
        for (int j = *x_min; j <= *x_max; j++) {
          V3(pre_mass, j, k, l) = C3(density1, j, k, l) * V3(pre_vol, j, k, l);
          V3(post_mass, j, k, l) = V3(pre_mass, j, k, l) + Y3(mass_flux_y, j, k, l) -
                                   Y3(mass_flux_y, j, k + 1, l);
          V3(post_ener, j, k, l) = (C3(energy1, j, k, l) * V3(pre_mass, j, k, l) +
                                    V3(ener_flux, j, k, l) - V3(ener_flux, j, k + 1, l)) /
                                   V3(post_mass, j, k, l);
          V3(advec_vol, j, k, l) = V3(pre_vol, j, k, l) + Y3(vol_flux_y, j, k, l) -
                                   Y3(vol_flux_y, j, k + 1, l);
          C3(density1, j, k, l) = V3(post_mass, j, k, l) / V3(advec_vol, j, k, l);
          C3(energy1, j, k, l) = V3(post_ener, j, k, l);
        }

  } else if (*dir == 3) {
    if (sweep == 1) {
#pragma omp parallel for
      for (int l = *z_min - 2; l <= *z_max + 2; l++)
        for (int k = *y_min - 2; k <= *y_max + 2; k++)
          for (int j = *x_min - 2; j <= *x_max + 2; j++) {
            V3(pre_vol, j, k, l) =
                C3(volume, j, k, l) +
                (X3(vol_flux_x, j + 1, k, l) - X3(vol_flux_x, j, k, l) +
                 Y3(vol_flux_y, j, k + 1, l) - Y3(vol_flux_y, j, k, l) +
                 Z3(vol_flux_z, j, k, l + 1) - Z3(vol_flux_z, j, k, l));
            V3(post_vol, j, k, l) =
                V3(pre_vol, j, k, l) - (Z3(vol_flux_z, j, k, l + 1) - Z3(vol_flux_z, j, k, l));
          }
    } else if (sweep == 3) {
#pragma omp parallel for
      for (int l = *z_min - 2; l <= *z_max + 2; l++)
        for (int k = *y_min - 2; k <= *y_max + 2; k++)
          for (int j = *x_min - 2; j <= *x_max + 2; j++) {
            V3(pre_vol, j, k, l) =
                C3(volume, j, k, l) + Z3(vol_flux_z, j, k, l + 1) - Z3(vol_flux_z, j, k, l);
            V3(post_vol, j, k, l) = C3(volume, j, k, l);
          }
    }

#pragma omp parallel for
    for (int l = *z_min; l <= *z_max + 2; l++)
      for (int k = *y_min; k <= *y_max; k++)
        for (int j = *x_min; j <= *x_max; j++) {
          int upwind, donor, downwind, dif;
          if (Z3(vol_flux_z, j, k, l) > 0.0) {
            upwind = l - 2; donor = l - 1; downwind = l; dif = donor;
          } else {
            upwind = (l + 1 < *z_max + 2) ? l + 1 : *z_max + 2;
            donor = l; downwind = l - 1; dif = upwind;
          }
          double sigmat = fabs(Z3(vol_flux_z, j, k, l)) / V3(pre_vol, j, k, donor);
          double sigma3 = (1.0 + sigmat) * (DZ(vertexdz, l) / DZ(vertexdz, dif));
          double sigma4 = 2.0 - sigmat;
          double sigmav = sigmat;

          double diffuw = C3(density1, j, k, donor) - C3(density1, j, k, upwind);
          double diffdw = C3(density1, j, k, downwind) - C3(density1, j, k, donor);
          double limiter = cell_limiter(sigmav, sigma3, sigma4, diffuw, diffdw);
          Z3(mass_flux_z, j, k, l) =
              Z3(vol_flux_z, j, k, l) * (C3(density1, j, k, donor) + limiter);

          double sigmam = fabs(Z3(mass_flux_z, j, k, l)) /
                          (C3(density1, j, k, donor) * V3(pre_vol, j, k, donor));
          diffuw = C3(energy1, j, k, donor) - C3(energy1, j, k, upwind);
          diffdw = C3(energy1, j, k, downwind) - C3(energy1, j, k, donor);
          limiter = cell_limiter(sigmam, sigma3, sigma4, diffuw, diffdw);
          V3(ener_flux, j, k, l) =
              Z3(mass_flux_z, j, k, l) * (C3(energy1, j, k, donor) + limiter);
        }

#pragma omp parallel for
    for (int l = *z_min; l <= *z_max; l++)
      for (int k = *y_min; k <= *y_max; k++)
        for (int j = *x_min; j <= *x_max; j++) {
          V3(pre_mass, j, k, l) = C3(density1, j, k, l) * V3(pre_vol, j, k, l);
          V3(post_mass, j, k, l) = V3(pre_mass, j, k, l) + Z3(mass_flux_z, j, k, l) -
                                   Z3(mass_flux_z, j, k, l + 1);
          V3(post_ener, j, k, l) = (C3(energy1, j, k, l) * V3(pre_mass, j, k, l) +
                                    V3(ener_flux, j, k, l) - V3(ener_flux, j, k, l + 1)) /
                                   V3(post_mass, j, k, l);
          V3(advec_vol, j, k, l) = V3(pre_vol, j, k, l) + Z3(vol_flux_z, j, k, l) -
                                   Z3(vol_flux_z, j, k, l + 1);
          C3(density1, j, k, l) = V3(post_mass, j, k, l) / V3(advec_vol, j, k, l);
          C3(energy1, j, k, l) = V3(post_ener, j, k, l);
        }
  }
}

/* Momentum limiter of advec_mom_kernel.f90:225-238 (x), :310-322 (y), :396-408 (z). */
static inline double mom_limiter(double sigma, double width, double celld_dif, double vdiffuw,
                                 double vdiffdw) {
  double limiter = 0.0;
  if (vdiffuw * vdiffdw > 0.0) {
    double auw = fabs(vdiffuw);
    double adw = fabs(vdiffdw);
    double wind = 1.0;
    if (vdiffdw <= 0.0) wind = -1.0;
    limiter = wind * fmin2(fmin2(width * ((2.0 - sigma) * adw / width +
                                          (1.0 + sigma) * auw / celld_dif) / 6.0,
                                 auw),
                           adw);
  }
  return limiter;
}

/* advec_mom_kernel.f90:95-423 */
void oracle_advec_mom_kernel(const int *x_min, const int *x_max, const int *y_min,
                             const int *y_max, const int *z_min, const int *z_max,
                             double *vel1, const double *mass_flux_x,
                             const double *vol_flux_x, const double *mass_flux_y,
                             const double *vol_flux_y, const double *mass_flux_z,
                             const double *vol_flux_z, const double *volume,
                             const double *density1, double *node_flux,
                             double *node_mass_post, double *node_mass_pre,
                             double *advec_vel, double *mom_flux, double *pre_vol,
                             double *post_vol, const double *celldx, const double *celldy,
                             const double *celldz, const int *advect_x,
                             const int *which_vel, const int *sweep_number,
                             const int *direction) {
  DECL_EXTENTS;
  (void)advec_vel;
  const int sweep = *sweep_number, dirn = *direction, ax = *advect_x != 0;

  /* :95-163 pre/post volume variants */
#pragma omp parallel for
  for (int l = *z_min - 2; l <= *z_max + 2; l++)
    for (int k = *y_min - 2; k <= *y_max + 2; k++)
      for (int j = *x_min - 2; j <= *x_max + 2; j++) {
        double vol = C3(volume, j, k, l);
        double fx1 = X3(vol_flux_x, j + 1, k, l), fx0 = X3(vol_flux_x, j, k, l);
        double fy1 = Y3(vol_flux_y, j, k + 1, l), fy0 = Y3(vol_flux_y, j, k, l);
        double fz1 = Z3(vol_flux_z, j, k, l + 1), fz0 = Z3(vol_flux_z, j, k, l);
        double post, pre;
        if (sweep == 1 && dirn == 1) {
          post = vol + fy1 - fy0 + fz1 - fz0;
          pre = post + fx1 - fx0;
        } else if (sweep == 1 && dirn == 3) {
          post = vol + fx1 - fx0 + fy1 - fy0;
          pre = post + fz1 - fz0;
        } else if (sweep == 2 && ax) {
          post = vol + fz1 - fz0;
          pre = post + fy1 - fy0;
        } else if (sweep == 2 && !ax) {
          post = vol + fx1 - fx0;
          pre = post + fy1 - fy0;
        } else if (sweep == 3 && dirn == 1) {
          post = vol;
          pre = post + fx1 - fx0;
        } else if (sweep == 3 && dirn == 3) {
          post = vol;
          pre = post + fz1 - fz0;
        } else {
          continue; /* no branch taken: the arrays keep their contents */
        }
        V3(post_vol, j, k, l) = post;
        V3(pre_vol, j, k, l) = pre;
      }

#define NMP(jj, kk, ll)                                                                     \
  (0.125 * (C3(density1, jj, kk - 1, ll) * V3(post_vol, jj, kk - 1, ll) +                   \
            C3(density1, jj, kk, ll) * V3(post_vol, jj, kk, ll) +                           \
            C3(density1, jj - 1, kk - 1, ll) * V3(post_vol, jj - 1, kk - 1, ll) +           \
            C3(density1, jj - 1, kk, ll) * V3(post_vol, jj - 1, kk, ll) +                   \
            C3(density1, jj, kk - 1, ll - 1) * V3(post_vol, jj, kk - 1, ll - 1) +           \
            C3(density1, jj, kk, ll - 1) * V3(post_vol, jj, kk, ll - 1) +                   \
            C3(density1, jj - 1, kk - 1, ll - 1) * V3(post_vol, jj - 1, kk - 1, ll - 1) +   \
            C3(density1, jj - 1, kk, ll - 1) * V3(post_vol, jj - 1, kk, ll - 1)))

  if (dirn == 1) {
    if (*which_vel == 1) {
#pragma omp parallel for
      for (int l = *z_min; l <= *z_max + 1; l++)
        for (int k = *y_min; k <= *y_max + 1; k++)
          for (int j = *x_min - 2; j <= *x_max + 2; j++)
            V3(node_flux, j, k, l) =
                0.125 * (X3(mass_flux_x, j, k - 1, l) + X3(mass_flux_x, j, k, l) +
                         X3(mass_flux_x, j + 1, k - 1, l) + X3(mass_flux_x, j + 1, k, l) +
                         X3(mass_flux_x, j, k - 1, l - 1) + X3(mass_flux_x, j, k, l - 1) +
                         X3(mass_flux_x, j + 1, k - 1, l - 1) + X3(mass_flux_x, j + 1, k, l - 1));
#pragma omp parallel for
      for (int l = *z_min; l <= *z_max + 1; l++)
        for (int k = *y_min; k <= *y_max + 1; k++)
          for (int j = *x_min - 1; j <= *x_max + 2; j++) V3(node_mass_post, j, k, l) = NMP(j, k, l);
#pragma omp parallel for
      for (int l = *z_min; l <= *z_max + 1; l++)
        for (int k = *y_min; k <= *y_max + 1; k++)
          for (int j = *x_min - 1; j <= *x_max + 2; j++)
            V3(node_mass_pre, j, k, l) = V3(node_mass_post, j, k, l) -
                                         V3(node_flux, j - 1, k, l) + V3(node_flux, j, k, l);
    }
#pragma omp parallel for
    for (int l = *z_min; l <= *z_max + 1; l++)
      for (int k = *y_min; k <= *y_max + 1; k++)
        for (int j = *x_min - 1; j <= *x_max + 1; j++) {
          int upwind, donor, downwind, dif;
          if (V3(node_flux, j, k, l) < 0.0) {
            upwind = j + 2; donor = j + 1; downwind = j; dif = donor;
          } else {
            upwind = j - 1; donor = j; downwind = j + 1; dif = upwind;
          }
          double sigma = fabs(V3(node_flux, j, k, l)) / V3(node_mass_pre, donor, k, l);
          double width = DX(celldx, j);
          double vdiffuw = V3(vel1, donor, k, l) - V3(vel1, upwind, k, l);
          double vdiffdw = V3(vel1, downwind, k, l) - V3(vel1, donor, k, l);
          double limiter = mom_limiter(sigma, width, DX(celldx, dif), vdiffuw, vdiffdw);
          double advec_vel_s = V3(vel1, donor, k, l) + (1.0 - sigma) * limiter;
          V3(mom_flux, j, k, l) = advec_vel_s * V3(node_flux, j, k, l);
        }
#pragma omp parallel for
    for (int l = *z_min; l <= *z_max + 1; l++)
      for (int k = *y_min; k <= *y_max + 1; k++)
        for (int j = *x_min; j <= *x_max + 1; j++)
          V3(vel1, j, k, l) = (V3(vel1, j, k, l) * V3(node_mass_pre, j, k, l) +
                               V3(mom_flux, j - 1, k, l) - V3(mom_flux, j, k, l)) /
                              V3(node_mass_post, j, k, l);
  } else if (dirn == 2) {
    if (*which_vel == 1) {
#pragma omp parallel for
      for (int l = *z_min; l <= *z_max + 1; l++)
        for (int k = *y_min - 2; k <= *y_max + 2; k++)
          for (int j = *x_min; j <= *x_max + 1; j++)
            V3(node_flux, j, k, l) =
                0.125 * (Y3(mass_flux_y, j - 1, k, l) + Y3(mass_flux_y, j, k, l) +
                         Y3(mass_flux_y, j - 1, k + 1, l) + Y3(mass_flux_y, j, k + 1, l) +
                         Y3(mass_flux_y, j - 1, k, l - 1) + Y3(mass_flux_y, j, k, l - 1) +
                         Y3(mass_flux_y, j - 1, k + 1, l - 1) + Y3(mass_flux_y, j, k + 1, l - 1));
#pragma omp parallel for
      for (int l = *z_min; l <= *z_max + 1; l++)
        for (int k = *y_min - 1; k <= *y_max + 2; k++)
          for (int j = *x_min; j <= *x_max + 1; j++) V3(node_mass_post, j, k, l) = NMP(j, k, l);
#pragma omp parallel for
      for (int l = *z_min; l <= *z_max + 1; l++)
        for (int k = *y_min - 1; k <= *y_max + 2; k++)
          for (int j = *x_min; j <= *x_max + 1; j++)
            V3(node_mass_pre, j, k, l) = V3(node_mass_post, j, k, l) -
                                         V3(node_flux, j, k - 1, l) + V3(node_flux, j, k, l);
    }
#pragma omp parallel for
    for (int l = *z_min; l <= *z_max + 1; l++)
      for (int k = *y_min - 1; k <= *y_max + 1; k++)
        for (int j = *x_min; j <= *x_max + 1; j++) {
          int upwind, donor, downwind, dif;
          if (V3(node_flux, j, k, l) < 0.0) {
            upwind = k + 2; donor = k + 1; downwind = k; dif = donor;
          } else {
            upwind = k - 1; donor = k; downwind = k + 1; dif = upwind;
          }
          double sigma = fabs(V3(node_flux, j, k, l)) / V3(node_mass_pre, j, donor, l);
          double width = DY(celldy, k);
          double vdiffuw = V3(vel1, j, donor, l) - V3(vel1, j, upwind, l);
          double vdiffdw = V3(vel1, j, downwind, l) - V3(vel1, j, donor, l);
          double limiter = mom_limiter(sigma, width, DY(celldy, dif), vdiffuw, vdiffdw);
          double advec_vel_s = V3(vel1, j, donor, l) + (1.0 - sigma) * limiter;
          V3(mom_flux, j, k, l) = advec_vel_s * V3(node_flux, j, k, l);
        }
#pragma omp parallel for
    for (int l = *z_min; l <= *z_max + 1; l++)
      for (int k = *y_min; k <= *y_max + 1; k++)
        for (int j = *x_min; j <= *x_max + 1; j++)
          V3(vel1, j, k, l) = (V3(vel1, j, k, l) * V3(node_mass_pre, j, k, l) +
                               V3(mom_flux, j, k - 1, l) - V3(mom_flux, j, k, l)) /
                              V3(node_mass_post, j, k, l);
  } else if (dirn == 3) {
    if (*which_vel == 1) {
#pragma omp parallel for
      for (int l = *z_min - 2; l <= *z_max + 2; l++)
        for (int k = *y_min; k <= *y_max + 1; k++)
          for (int j = *x_min; j <= *x_max + 1; j++)
            V3(node_flux, j, k, l) =
                0.125 * (Z3(mass_flux_z, j - 1, k, l) + Z3(mass_flux_z, j, k, l) +
                         Z3(mass_flux_z, j - 1, k, l + 1) + Z3(mass_flux_z, j, k, l + 1) +
                         Z3(mass_flux_z, j - 1, k - 1, l) + Z3(mass_flux_z, j, k - 1, l) +
                         Z3(mass_flux_z, j - 1, k - 1, l + 1) + Z3(mass_flux_z, j, k - 1, l + 1));
#pragma omp parallel for
      for (int l = *z_min - 1; l <= *z_max + 2; l++)
        for (int k = *y_min; k <= *y_max + 1; k++)
          for (int j = *x_min; j <= *x_max + 1; j++) V3(node_mass_post, j, k, l) = NMP(j, k, l);
#pragma omp parallel for
      for (int l = *z_min - 1; l <= *z_max + 2; l++)
        for (int k = *y_min; k <= *y_max + 1; k++)
          for (int j = *x_min; j <= *x_max + 1; j++)
            V3(node_mass_pre, j, k, l) = V3(node_mass_post, j, k, l) -
                                         V3(node_flux, j, k, l - 1) + V3(node_flux, j, k, l);
    }
#pragma omp parallel for
    for (int l = *z_min - 1; l <= *z_max + 1; l++)
      for (int k = *y_min; k <= *y_max + 1; k++)
        for (int j = *x_min; j <= *x_max + 1; j++) {
          int upwind, donor, downwind, dif;
          if (V3(node_flux, j, k, l) < 0.0) {
            upwind = l + 2; donor = l + 1; downwind = l; dif = donor;
          } else {
            upwind = l - 1; donor = l; downwind = l + 1; dif = upwind;
          }
          double sigma = fabs(V3(node_flux, j, k, l)) / V3(node_mass_pre, j, k, donor);
          double width = DZ(celldz, l);
          double vdiffuw = V3(vel1, j, k, donor) - V3(vel1, j, k, upwind);
          double vdiffdw = V3(vel1, j, k, downwind) - V3(vel1, j, k, donor);
          double limiter = mom_limiter(sigma, width, DZ(celldz, dif), vdiffuw, vdiffdw);
          double advec_vel_s = V3(vel1, j, k, donor) + (1.0 - sigma) * limiter;
          V3(mom_flux, j, k, l) = advec_vel_s * V3(node_flux, j, k, l);
        }
#pragma omp parallel for
    for (int l = *z_min; l <= *z_max + 1; l++)
      for (int k = *y_min; k <= *y_max + 1; k++)
        for (int j = *x_min; j <= *x_max + 1; j++)
          V3(vel1, j, k, l) = (V3(vel1, j, k, l) * V3(node_mass_pre, j, k, l) +
                               V3(mom_flux, j, k, l - 1) - V3(mom_flux, j, k, l)) /
                              V3(node_mass_post, j, k, l);
  }
#undef NMP
}

/* reset_field_kernel.f90:51-98 */
void oracle_reset_field_kernel(const int *x_min, const int *x_max, const int *y_min,
                               const int *y_max, const int *z_min, const int *z_max,
                               double *density0, const double *density1, double *energy0,
                               const double *energy1, double *xvel0, const double *xvel1,
                               double *yvel0, const double *yvel1, double *zvel0,
                               const double *zvel1) {
  DECL_EXTENTS;
#pragma omp parallel for
  for (int l = *z_min; l <= *z_max; l++)
    for (int k = *y_min; k <= *y_max; k++)
      for (int j = *x_min; j <= *x_max; j++) {
        C3(density0, j, k, l) = C3(density1, j, k, l);
        C3(energy0, j, k, l) = C3(energy1, j, k, l);
      }
#pragma omp parallel for
  for (int l = *z_min; l <= *z_max + 1; l++)
    for (int k = *y_min; k <= *y_max + 1; k++)
      for (int j = *x_min; j <= *x_max + 1; j++) {
        V3(xvel0, j, k, l) = V3(xvel1, j, k, l);
        V3(yvel0, j, k, l) = V3(yvel1, j, k, l);
        V3(zvel0, j, k, l) = V3(zvel1, j, k, l);
      }
}

/* field_summary_kernel.f90:52-77. The reference reduces with an OpenMP
 * REDUCTION(+) of unspecified order; this restatement sums each z-plane in
 * loop order and then adds the plane partials in z order, which is the serial
 * loop order when run on one thread and deterministic on any thread count. */
void oracle_field_summary_kernel(const int *x_min, const int *x_max, const int *y_min,
                                 const int *y_max, const int *z_min, const int *z_max,
                                 const double *volume, const double *density0,
                                 const double *energy0, const double *pressure,
                                 const double *xvel0, const double *yvel0,
                                 const double *zvel0, double *vol, double *mass, double *ie,
                                 double *ke, double *press) {
  DECL_EXTENTS;
  const int nz = *z_max - *z_min + 1;
  double *parts = (double *)malloc((size_t)(nz > 0 ? nz : 1) * 5 * sizeof(double));
#pragma omp parallel for
  for (int l = *z_min; l <= *z_max; l++) {
    double s_vol = 0.0, s_mass = 0.0, s_ie = 0.0, s_ke = 0.0, s_press = 0.0;
    for (int k = *y_min; k <= *y_max; k++)
      for (int j = *x_min; j <= *x_max; j++) {
        double vsqrd = 0.0;
        for (int lv = l; lv <= l + 1; lv++)
          for (int kv = k; kv <= k + 1; kv++)
            for (int jv = j; jv <= j + 1; jv++) {
              double u = V3(xvel0, jv, kv, lv), v = V3(yvel0, jv, kv, lv),
                     w = V3(zvel0, jv, kv, lv);
              vsqrd = vsqrd + 0.125 * (u * u + v * v + w * w);
            }
        double cell_vol = C3(volume, j, k, l);
        double cell_mass = cell_vol * C3(density0, j, k, l);
        s_vol = s_vol + cell_vol;
        s_mass = s_mass + cell_mass;
        s_ie = s_ie + cell_mass * C3(energy0, j, k, l);
        s_ke = s_ke + cell_mass * 0.5 * vsqrd;
        s_press = s_press + cell_vol * C3(pressure, j, k, l);
      }
    double *p = parts + 5 * (l - *z_min);
    p[0] = s_vol; p[1] = s_mass; p[2] = s_ie; p[3] = s_ke; p[4] = s_press;
  }
  double t[5] = {0.0, 0.0, 0.0, 0.0, 0.0};
  for (int i = 0; i < nz; i++)
    for (int q = 0; q < 5; q++) t[q] = t[q] + parts[5 * i + q];
  *vol = t[0]; *mass = t[1]; *ie = t[2]; *ke = t[3]; *press = t[4];
  free(parts);
}

/* initialise_chunk_kernel.f90:70-178 */
void oracle_initialise_chunk_kernel(const int *x_min, const int *x_max, const int *y_min,
                                    const int *y_max, const int *z_min, const int *z_max,
                                    const double *xmin, const double *ymin,
                                    const double *zmin, const double *dx, const double *dy,
                                    const double *dz, double *vertexx, double *vertexdx,
                                    double *vertexy, double *vertexdy, double *vertexz,
                                    double *vertexdz, double *cellx, double *celldx,
                                    double *celly, double *celldy, double *cellz,
                                    double *celldz, double *volume, double *xarea,
                                    double *yarea, double *zarea) {
  DECL_EXTENTS;
  /* float(j-x_min) is a default REAL; small integers convert exactly */
  for (int j = *x_min - 2; j <= *x_max + 3; j++) DX(vertexx, j) = *xmin + *dx * (double)(float)(j - *x_min);
  for (int j = *x_min - 2; j <= *x_max + 3; j++) DX(vertexdx, j) = *dx;
  for (int k = *y_min - 2; k <= *y_max + 3; k++) DY(vertexy, k) = *ymin + *dy * (double)(float)(k - *y_min);
  for (int k = *y_min - 2; k <= *y_max + 3; k++) DY(vertexdy, k) = *dy;
  for (int l = *z_min - 2; l <= *z_max + 3; l++) DZ(vertexz, l) = *zmin + *dz * (double)(float)(l - *z_min);
  for (int l = *z_min - 2; l <= *z_max + 3; l++) DZ(vertexdz, l) = *dz;
  for (int j = *x_min - 2; j <= *x_max + 2; j++) DX(cellx, j) = 0.5 * (DX(vertexx, j) + DX(vertexx, j + 1));
  for (int j = *x_min - 2; j <= *x_max + 2; j++) DX(celldx, j) = *dx;
  for (int k = *y_min - 2; k <= *y_max + 2; k++) DY(celly, k) = 0.5 * (DY(vertexy, k) + DY(vertexy, k + 1));
  for (int k = *y_min - 2; k <= *y_max + 2; k++) DY(celldy, k) = *dy;
  for (int l = *z_min - 2; l <= *z_max + 2; l++) DZ(cellz, l) = 0.5 * (DZ(vertexz, l) + DZ(vertexz, l + 1));
  for (int l = *z_min - 2; l <= *z_max + 2; l++) DZ(celldz, l) = *dz;
#pragma omp parallel for
  for (int l = *z_min - 2; l <= *z_max + 2; l++)
    for (int k = *y_min - 2; k <= *y_max + 2; k++)
      for (int j = *x_min - 2; j <= *x_max + 2; j++) {
        C3(volume, j, k, l) = *dx * *dy * *dz;
        X3(xarea, j, k, l) = DY(celldy, k) * DZ(celldz, l);
        Y3(yarea, j, k, l) = DX(celldx, j) * DZ(celldz, l);
        Z3(zarea, j, k, l) = DX(celldx, j) * DY(celldy, k);
      }
}

/* generate_chunk_kernel.f90:98-207 */
void oracle_generate_chunk_kernel(const int *x_min, const int *x_max, const int *y_min,
                                  const int *y_max, const int *z_min, const int *z_max,
                                  const double *vertexx, const double *vertexy,
                                  const double *vertexz, const double *cellx,
                                  const double *celly, const double *cellz,
                                  double *density0, double *energy0, double *xvel0,
                                  double *yvel0, double *zvel0, const int *number_of_states,
                                  const double *state_density, const double *state_energy,
                                  const double *state_xvel, const double *state_yvel,
                                  const double *state_zvel, const double *state_xmin,
                                  const double *state_xmax, const double *state_ymin,
                                  const double *state_ymax, const double *state_zmin,
                                  const double *state_zmax, const double *state_radius,
                                  const int *state_geometry, const int *g_rect,
                                  const int *g_circ, const int *g_point) {
  DECL_EXTENTS;
  for (int l = *z_min - 2; l <= *z_max + 2; l++)
    for (int k = *y_min - 2; k <= *y_max + 2; k++)
      for (int j = *x_min - 2; j <= *x_max + 2; j++) {
        C3(energy0, j, k, l) = state_energy[0];
        C3(density0, j, k, l) = state_density[0];
        V3(xvel0, j, k, l) = state_xvel[0];
        V3(yvel0, j, k, l) = state_yvel[0];
        V3(zvel0, j, k, l) = state_zvel[0];
      }
  for (int s = 1; s < *number_of_states; s++) {
    double x_cent = state_xmin[s], y_cent = state_ymin[s], z_cent = state_zmin[s];
    for (int l = *z_min - 2; l <= *z_max + 2; l++)
      for (int k = *y_min - 2; k <= *y_max + 2; k++)
        for (int j = *x_min - 2; j <= *x_max + 2; j++) {
          int hit = 0;
          if (state_geometry[s] == *g_rect) {
            hit = DX(vertexx, j + 1) >= state_xmin[s] && DX(vertexx, j) < state_xmax[s] &&
                  DY(vertexy, k + 1) >= state_ymin[s] && DY(vertexy, k) < state_ymax[s] &&
                  DZ(vertexz, l + 1) >= state_zmin[s] && DZ(vertexz, l) < state_zmax[s];
          } else if (state_geometry[s] == *g_circ) {
            double cx = DX(cellx, j) - x_cent, cy = DY(celly, k) - y_cent,
                   cz = DZ(cellz, l) - z_cent;
            double radius = sqrt(cx * cx + cy * cy + cz * cz);
            hit = radius <= state_radius[s];
          } else if (state_geometry[s] == *g_point) {
            hit = DX(vertexx, j) == x_cent && DY(vertexy, k) == y_cent &&
                  DZ(vertexz, l) == z_cent;
          }
          if (hit) {
            C3(energy0, j, k, l) = state_energy[s];
            C3(density0, j, k, l) = state_density[s];
            for (int lt = l; lt <= l + 1; lt++)
              for (int kt = k; kt <= k + 1; kt++)
                for (int jt = j; jt <= j + 1; jt++) {
                  V3(xvel0, jt, kt, lt) = state_xvel[s];
                  V3(yvel0, jt, kt, lt) = state_yvel[s];
                  V3(zvel0, jt, kt, lt) = state_zvel[s];
                }
          }
        }
  }
}
