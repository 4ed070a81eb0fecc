/*
 * CPU oracle: whole-run driver -- TEST INFRASTRUCTURE ONLY.
 *
 * One chunk, one tile, every face external. Restates start.f90:49-136 and
 * hydro.f90:46-192 with the phase drivers timestep.f90:56-126,
 * PdV.f90:50-107, advection.f90:43-179 and field_summary.f90:55-113.
 */
#define _POSIX_C_SOURCE 199309L
#include "clover_oracle.h"

#include <stdlib.h>
#include <string.h>
#include <time.h>

static double now_s(void) {
  struct timespec ts;
  clock_gettime(CLOCK_MONOTONIC, &ts);
  return (double)ts.tv_sec + 1e-9 * (double)ts.tv_nsec;
}

/* Wall time of the step loop after `timing_warmup` steps (CPU baseline). */
static int timing_warmup = -1;
static double timing_t0 = 0.0, timing_t1 = 0.0;

/* data.f90:30-31: both are default-REAL literals assigned to REAL(8). */
#define G_SMALL ((double)1.0e-16f)
#define G_BIG ((double)1.0e+21f)

enum {
  F_DENSITY0 = 1, F_DENSITY1, F_ENERGY0, F_ENERGY1, F_PRESSURE, F_VISCOSITY, F_SOUNDSPEED,
  F_XVEL0, F_XVEL1, F_YVEL0, F_YVEL1, F_ZVEL0, F_ZVEL1, F_VOL_FLUX_X, F_VOL_FLUX_Y,
  F_VOL_FLUX_Z, F_MASS_FLUX_X, F_MASS_FLUX_Y, F_MASS_FLUX_Z
};

typedef struct {
  int x_min, x_max, y_min, y_max, z_min, z_max;
  long ncell, nvert, nxf, nyf, nzf;
  double *density0, *density1, *energy0, *energy1, *pressure, *viscosity, *soundspeed;
  double *xvel0, *xvel1, *yvel0, *yvel1, *zvel0, *zvel1;
  double *vol_flux_x, *vol_flux_y, *vol_flux_z, *mass_flux_x, *mass_flux_y, *mass_flux_z;
  double *wa[7];
  double *cellx, *celly, *cellz, *vertexx, *vertexy, *vertexz;
  double *celldx, *celldy, *celldz, *vertexdx, *vertexdy, *vertexdz;
  double *volume, *xarea, *yarea, *zarea;
} tile_t;

static double *zalloc(long n) { return (double *)calloc((size_t)n, sizeof(double)); }

/* build_field.f90:41-229: every array allocated with the reference extents and zeroed */
static void build_field(tile_t *t, int nx, int ny, int nz) {
  t->x_min = 1; t->x_max = nx; t->y_min = 1; t->y_max = ny; t->z_min = 1; t->z_max = nz;
  long cx = nx + 4, cy = ny + 4, cz = nz + 4, vx = nx + 5, vy = ny + 5, vz = nz + 5;
  t->ncell = cx * cy * cz;
  t->nvert = vx * vy * vz;
  t->nxf = vx * cy * cz;
  t->nyf = cx * vy * cz;
  t->nzf = cx * cy * vz;
  t->density0 = zalloc(t->ncell); t->density1 = zalloc(t->ncell);
  t->energy0 = zalloc(t->ncell); t->energy1 = zalloc(t->ncell);
  t->pressure = zalloc(t->ncell); t->viscosity = zalloc(t->ncell);
  t->soundspeed = zalloc(t->ncell);
  t->xvel0 = zalloc(t->nvert); t->xvel1 = zalloc(t->nvert);
  t->yvel0 = zalloc(t->nvert); t->yvel1 = zalloc(t->nvert);
  t->zvel0 = zalloc(t->nvert); t->zvel1 = zalloc(t->nvert);
  t->vol_flux_x = zalloc(t->nxf); t->mass_flux_x = zalloc(t->nxf);
  t->vol_flux_y = zalloc(t->nyf); t->mass_flux_y = zalloc(t->nyf);
  t->vol_flux_z = zalloc(t->nzf); t->mass_flux_z = zalloc(t->nzf);
  for (int i = 0; i < 7; i++) t->wa[i] = zalloc(t->nvert);
  t->cellx = zalloc(cx); t->celly = zalloc(cy); t->cellz = zalloc(cz);
  t->vertexx = zalloc(vx); t->vertexy = zalloc(vy); t->vertexz = zalloc(vz);
  t->celldx = zalloc(cx); t->celldy = zalloc(cy); t->celldz = zalloc(cz);
  t->vertexdx = zalloc(vx); t->vertexdy = zalloc(vy); t->vertexdz = zalloc(vz);
  t->volume = zalloc(t->ncell);
  t->xarea = zalloc(t->nxf); t->yarea = zalloc(t->nyf); t->zarea = zalloc(t->nzf);
}

static void free_field(tile_t *t) {
  double *all[] = {t->density0, t->density1, t->energy0, t->energy1, t->pressure,
                   t->viscosity, t->soundspeed, t->xvel0, t->xvel1, t->yvel0, t->yvel1,
                   t->zvel0, t->zvel1, t->vol_flux_x, t->vol_flux_y, t->vol_flux_z,
                   t->mass_flux_x, t->mass_flux_y, t->mass_flux_z, t->cellx, t->celly,
                   t->cellz, t->vertexx, t->vertexy, t->vertexz, t->celldx, t->celldy,
                   t->celldz, t->vertexdx, t->vertexdy, t->vertexdz, t->volume, t->xarea,
                   t->yarea, t->zarea};
  for (size_t i = 0; i < sizeof(all) / sizeof(all[0]); i++) free(all[i]);
  for (int i = 0; i < 7; i++) free(t->wa[i]);
}

#define B(t) &(t)->x_min, &(t)->x_max, &(t)->y_min, &(t)->y_max, &(t)->z_min, &(t)->z_max

static void update_halo(tile_t *t, const int *fields, int depth) {
  static const int neighbours[6] = {-1, -1, -1, -1, -1, -1};
  oracle_update_halo_kernel(B(t), neighbours, neighbours, t->density0, t->energy0,
                            t->pressure, t->viscosity, t->soundspeed, t->density1,
                            t->energy1, t->xvel0, t->yvel0, t->zvel0, t->xvel1, t->yvel1,
                            t->zvel1, t->vol_flux_x, t->vol_flux_y, t->vol_flux_z,
                            t->mass_flux_x, t->mass_flux_y, t->mass_flux_z, fields, &depth);
}

static void set_fields(int *fields, const int *ids, int n) {
  memset(fields, 0, 19 * sizeof(int));
  for (int i = 0; i < n; i++) fields[ids[i] - 1] = 1;
}

/* ideal_gas.f90:38-66 */
static void ideal_gas(tile_t *t, int predict) {
  if (!predict)
    oracle_ideal_gas_kernel(B(t), t->density0, t->energy0, t->pressure, t->soundspeed);
  else
    oracle_ideal_gas_kernel(B(t), t->density1, t->energy1, t->pressure, t->soundspeed);
}

/* field_summary.f90:55-108 */
static void field_summary(tile_t *t, double out[5]) {
  ideal_gas(t, 0);
  oracle_field_summary_kernel(B(t), t->volume, t->density0, t->energy0, t->pressure,
                              t->xvel0, t->yvel0, t->zvel0, &out[0], &out[1], &out[2],
                              &out[3], &out[4]);
}

/* timestep.f90:56-126; returns 1 on the small-timestep error */
static int timestep(tile_t *t, const oracle_deck *dk, double *dt, double *dtold) {
  int fields[19];
  *dt = G_BIG;
  ideal_gas(t, 0);
  const int f1[] = {F_PRESSURE, F_ENERGY0, F_DENSITY0, F_XVEL0, F_YVEL0};
  set_fields(fields, f1, 5);
  update_halo(t, fields, 1);
  oracle_viscosity_kernel(B(t), t->xarea, t->yarea, t->zarea, t->celldx, t->celldy,
                          t->celldz, t->density0, t->pressure, t->viscosity, t->xvel0,
                          t->yvel0, t->zvel0);
  const int f2[] = {F_VISCOSITY};
  set_fields(fields, f2, 1);
  update_halo(t, fields, 1);

  const double g_small = G_SMALL, g_big = G_BIG, dtc_safe = 0.75, dtu_safe = 0.5,
               dtv_safe = 0.5, dtw_safe = 0.5, dtdiv_safe = 0.5;
  double dtlp, xl, yl, zl;
  int ctl, jl, kl, ll, small = 0;
  oracle_calc_dt_kernel(B(t), &g_small, &g_big, &dk->dtmin, &dtc_safe, &dtu_safe, &dtv_safe,
                        &dtw_safe, &dtdiv_safe, t->xarea, t->yarea, t->zarea, t->cellx,
                        t->celly, t->cellz, t->celldx, t->celldy, t->celldz, t->volume,
                        t->density0, t->energy0, t->pressure, t->viscosity, t->soundspeed,
                        t->xvel0, t->yvel0, t->zvel0, t->wa[0], &dtlp, &ctl, &xl, &yl, &zl,
                        &jl, &kl, &ll, &small);
  if (dtlp <= *dt) *dt = dtlp;
  double m = *dt;
  double r = *dtold * dk->dtrise;
  if (r < m) m = r;
  if (dk->dtmax < m) m = dk->dtmax;
  *dt = m;
  int err = *dt < dk->dtmin;
  *dtold = *dt;
  return err;
}

static void pdv(tile_t *t, int predict, double dt) {
  int fields[19];
  oracle_pdv_kernel(&predict, B(t), &dt, t->xarea, t->yarea, t->zarea, t->volume,
                    t->density0, t->density1, t->energy0, t->energy1, t->pressure,
                    t->viscosity, t->xvel0, t->xvel1, t->yvel0, t->yvel1, t->zvel0,
                    t->zvel1);
  if (predict) {
    ideal_gas(t, 1);
    const int f[] = {F_PRESSURE};
    set_fields(fields, f, 1);
    update_halo(t, fields, 1);
    oracle_revert_kernel(B(t), t->density0, t->density1, t->energy0, t->energy1);
  }
}

static void advec_cell(tile_t *t, int advect_x, int sweep, int dir) {
  oracle_advec_cell_kernel(B(t), &advect_x, &dir, &sweep, t->vertexdx, t->vertexdy,
                           t->vertexdz, t->volume, t->density1, t->energy1, t->mass_flux_x,
                           t->vol_flux_x, t->mass_flux_y, t->vol_flux_y, t->mass_flux_z,
                           t->vol_flux_z, t->wa[0], t->wa[1], t->wa[2], t->wa[3], t->wa[4],
                           t->wa[5], t->wa[6]);
}

static void advec_mom(tile_t *t, int advect_x, int which_vel, int dir, int sweep) {
  double *vel = which_vel == 1 ? t->xvel1 : which_vel == 2 ? t->yvel1 : t->zvel1;
  oracle_advec_mom_kernel(B(t), vel, t->mass_flux_x, t->vol_flux_x, t->mass_flux_y,
                          t->vol_flux_y, t->mass_flux_z, t->vol_flux_z, t->volume,
                          t->density1, t->wa[0], t->wa[1], t->wa[2], t->wa[3], t->wa[4],
                          t->wa[5], t->wa[6], t->celldx, t->celldy, t->celldz, &advect_x,
                          &which_vel, &sweep, &dir);
}

/* advection.f90:43-179 */
static void advection(tile_t *t, int advect_x) {
  int fields[19];
  const int fpre[] = {F_ENERGY1, F_DENSITY1, F_VOL_FLUX_X, F_VOL_FLUX_Y, F_VOL_FLUX_Z};
  const int fpost[] = {F_DENSITY1, F_ENERGY1, F_XVEL1, F_YVEL1, F_ZVEL1,
                       F_MASS_FLUX_X, F_MASS_FLUX_Y, F_MASS_FLUX_Z};
  int dir = advect_x ? 1 : 3;
  int sweep = 1;
  set_fields(fields, fpre, 5);
  update_halo(t, fields, 2);
  advec_cell(t, advect_x, sweep, dir);
  set_fields(fields, fpost, 8);
  update_halo(t, fields, 2);
  for (int v = 1; v <= 3; v++) advec_mom(t, advect_x, v, dir, sweep);

  sweep = 2;
  dir = 2;
  set_fields(fields, fpre, 5);
  update_halo(t, fields, 2);
  advec_cell(t, advect_x, sweep, dir);
  set_fields(fields, fpost, 8);
  update_halo(t, fields, 2);
  for (int v = 1; v <= 3; v++) advec_mom(t, advect_x, v, dir, sweep);

  sweep = 3;
  dir = advect_x ? 3 : 1;
  advec_cell(t, advect_x, sweep, dir); /* no halo refresh before this sweep */
  set_fields(fields, fpost, 8);
  update_halo(t, fields, 2);
  for (int v = 1; v <= 3; v++) advec_mom(t, advect_x, v, dir, sweep);
}

static void record(double *summary_out, int *summary_step_out, int *n, int cap, int step,
                   const double s[5]) {
  if (*n < cap) {
    if (summary_out) memcpy(summary_out + 5 * (*n), s, 5 * sizeof(double));
    if (summary_step_out) summary_step_out[*n] = step;
  }
  (*n)++;
}

/* The hydro loop on a built chunk t (the body of oracle_run). */
static int run_chunk(tile_t *t, const oracle_deck *dk, int max_steps, double *dt_out,
                     int max_summaries, double *summary_out, int *summary_step_out,
                     int *n_summaries) {
  int nsum = 0;

  /* initialise_chunk.f90:38-46 (float() of the cell count is a default REAL) */
  double dx = (dk->xmax - dk->xmin) / (double)(float)dk->x_cells;
  double dy = (dk->ymax - dk->ymin) / (double)(float)dk->y_cells;
  double dz = (dk->zmax - dk->zmin) / (double)(float)dk->z_cells;
  double xmin = dk->xmin + dx * (double)(float)0;
  double ymin = dk->ymin + dy * (double)(float)0;
  double zmin = dk->zmin + dz * (double)(float)0;
  oracle_initialise_chunk_kernel(B(t), &xmin, &ymin, &zmin, &dx, &dy, &dz, t->vertexx,
                                 t->vertexdx, t->vertexy, t->vertexdy, t->vertexz,
                                 t->vertexdz, t->cellx, t->celldx, t->celly, t->celldy,
                                 t->cellz, t->celldz, t->volume, t->xarea, t->yarea,
                                 t->zarea);

  /* read_input.f90:287-303: nudge the bounds of states 2.. by a hundredth of a cell */
  oracle_deck d = *dk;
  for (int n = 1; n < d.number_of_states; n++) {
    d.state_xmin[n] = d.state_xmin[n] + (dx / 100.0);
    d.state_ymin[n] = d.state_ymin[n] + (dy / 100.0);
    d.state_zmin[n] = d.state_zmin[n] + (dz / 100.0);
    d.state_xmax[n] = d.state_xmax[n] - (dx / 100.0);
    d.state_ymax[n] = d.state_ymax[n] - (dy / 100.0);
    d.state_zmax[n] = d.state_zmax[n] - (dz / 100.0);
  }
  const int g_rect = 1, g_circ = 2, g_point = 3;
  oracle_generate_chunk_kernel(B(t), t->vertexx, t->vertexy, t->vertexz, t->cellx, t->celly,
                               t->cellz, t->density0, t->energy0, t->xvel0, t->yvel0,
                               t->zvel0, &d.number_of_states, d.state_density,
                               d.state_energy, d.state_xvel, d.state_yvel, d.state_zvel,
                               d.state_xmin, d.state_xmax, d.state_ymin, d.state_ymax,
                               d.state_zmin, d.state_zmax, d.state_radius, d.state_geometry,
                               &g_rect, &g_circ, &g_point);

  /* start.f90:99-136 */
  int advect_x = 1;
  ideal_gas(t, 0);
  int fields[19];
  const int fstart[] = {F_DENSITY0, F_ENERGY0, F_PRESSURE, F_VISCOSITY, F_DENSITY1,
                        F_ENERGY1, F_XVEL0, F_YVEL0, F_ZVEL0, F_XVEL1, F_YVEL1, F_ZVEL1};
  set_fields(fields, fstart, 12);
  update_halo(t, fields, 2);
  double s[5];
  field_summary(t, s);
  record(summary_out, summary_step_out, &nsum, max_summaries, 0, s);

  /* hydro.f90:46-192 */
  double time = 0.0, dt = dk->dtinit, dtold = dk->dtinit;
  int step = 0;
  for (;;) {
    if (step == timing_warmup) timing_t0 = now_s();
    step = step + 1;
    if (timestep(t, dk, &dt, &dtold)) {
      step = -step; /* report_error('timestep','small timestep') */
      break;
    }
    if (step <= max_steps && dt_out) dt_out[step - 1] = dt;
    pdv(t, 1, dt);
    oracle_accelerate_kernel(B(t), &dt, t->xarea, t->yarea, t->zarea, t->volume,
                             t->density0, t->pressure, t->viscosity, t->xvel0, t->yvel0,
                             t->zvel0, t->xvel1, t->yvel1, t->zvel1);
    pdv(t, 0, dt);
    oracle_flux_calc_kernel(B(t), &dt, t->xarea, t->yarea, t->zarea, t->xvel0, t->yvel0,
                            t->zvel0, t->xvel1, t->yvel1, t->zvel1, t->vol_flux_x,
                            t->vol_flux_y, t->vol_flux_z);
    advection(t, advect_x);
    oracle_reset_field_kernel(B(t), t->density0, t->density1, t->energy0, t->energy1,
                              t->xvel0, t->xvel1, t->yvel0, t->yvel1, t->zvel0, t->zvel1);
    advect_x = !advect_x;
    time = time + dt;
    if (dk->summary_frequency != 0 && step % dk->summary_frequency == 0) {
      field_summary(t, s);
      record(summary_out, summary_step_out, &nsum, max_summaries, step, s);
    }
    if (time + G_SMALL > dk->end_time || step >= dk->end_step || step >= max_steps) {
      field_summary(t, s);
      record(summary_out, summary_step_out, &nsum, max_summaries, step, s);
      break;
    }
  }
  timing_t1 = now_s();
  if (n_summaries) *n_summaries = nsum;
  return step;
}

/* Field id (1..19, data.f90:55-74) of chunk t into out (its reference shape). */
static void copy_field(const tile_t *t, int id, double *out) {
  double *src[19] = {t->density0, t->density1, t->energy0, t->energy1, t->pressure,
                     t->viscosity, t->soundspeed, t->xvel0, t->xvel1, t->yvel0,
                     t->yvel1, t->zvel0, t->zvel1, t->vol_flux_x, t->vol_flux_y,
                     t->vol_flux_z, t->mass_flux_x, t->mass_flux_y, t->mass_flux_z};
  long n[19] = {t->ncell, t->ncell, t->ncell, t->ncell, t->ncell, t->ncell, t->ncell,
                t->nvert, t->nvert, t->nvert, t->nvert, t->nvert, t->nvert,
                t->nxf, t->nyf, t->nzf, t->nxf, t->nyf, t->nzf};
  memcpy(out, src[id - 1], (size_t)n[id - 1] * sizeof(double));
}

int oracle_run(const oracle_deck *dk, int max_steps, double *dt_out, int max_summaries,
               double *summary_out, int *summary_step_out, int *n_summaries,
               double **fields_out) {
  tile_t tt, *t = &tt;
  build_field(t, dk->x_cells, dk->y_cells, dk->z_cells);
  const int step = run_chunk(t, dk, max_steps, dt_out, max_summaries, summary_out,
                             summary_step_out, n_summaries);
  if (fields_out)
    for (int i = 0; i < 19; i++)
      if (fields_out[i]) copy_field(t, i + 1, fields_out[i]);
  free_field(t);
  return step;
}

/* oracle_run keeping the chunk: *steps receives its return value, and the
 * handle gives the fields one at a time (oracle_kept_field) until
 * oracle_kept_free, so that a large run is compared array by array. */
void *oracle_run_keep(const oracle_deck *dk, int max_steps, double *dt_out, int max_summaries,
                      double *summary_out, int *summary_step_out, int *n_summaries,
                      int *steps) {
  tile_t *t = (tile_t *)malloc(sizeof(tile_t));
  if (!t) return NULL;
  build_field(t, dk->x_cells, dk->y_cells, dk->z_cells);
  *steps = run_chunk(t, dk, max_steps, dt_out, max_summaries, summary_out, summary_step_out,
                     n_summaries);
  return t;
}

int oracle_kept_field(void *h, int id, double *out) {
  if (!h || id < 1 || id > 19) return -1;
  copy_field((const tile_t *)h, id, out);
  return 0;
}

void oracle_kept_free(void *h) {
  if (!h) return;
  free_field((tile_t *)h);
  free(h);
}

double oracle_run_timed(const oracle_deck *deck, int warmup, int steps) {
  timing_warmup = warmup;
  timing_t0 = timing_t1 = 0.0;
  oracle_run(deck, warmup + steps, NULL, 0, NULL, NULL, NULL, NULL);
  timing_warmup = -1;
  return timing_t1 - timing_t0;
}
