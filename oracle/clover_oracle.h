/*
 * CPU oracle for the CloverLeaf3D hydro cycle -- TEST INFRASTRUCTURE ONLY.
 *
 * A plain-C, loop-for-loop restatement of the reference's Fortran kernels
 * (UK-MAC/CloverLeaf3D_ref). Every routine keeps the reference argument list
 * (pointers only, Fortran pass-by-reference), the reference index ranges, the
 * reference operation order and the reference literals, so that with
 * -ffp-contract=off it reproduces the reference arithmetic bit for bit on one
 * thread. Arrays are column-major with lower bound (min-2) in every axis, laid
 * out with the extents the reference declares (cell: max-min+5, vertex/work:
 * max-min+6, x/y/z-face: vertex extent in the face-normal axis).
 *
 * Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg may
 * load this library, and only as the checker. The product path never calls it.
 *
 * Parity pin: the reference cannot be compiled in this environment (Fortran
 * with an MPI module, no Fortran compiler). The oracle is pinned against the
 * reference's own known-answer test, test_problem 1 (field_summary.f90:119-136:
 * final kinetic energy 3.64560737191257 within 0.001%), see tests/golden/.
 */
#ifndef CLOVER_ORACLE_H
#define CLOVER_ORACLE_H

#ifdef __cplusplus
extern "C" {
#endif

/* pack_kernel.f90:29-721, the twelve message routines as one (oracle_pack.c):
 * side 0..5 = left, right, bottom, top, back, front; field_type 1 cell,
 * 2 vertex, 3 x face, 4 y face, 5 z face. */
void oracle_pack_message(int side, int pack, const int *x_min, const int *x_max,
                         const int *y_min, const int *y_max, const int *z_min, const int *z_max,
                         double *field, double *buffer, const int *depth, const int *field_type,
                         const int *buffer_offset, const int *off_a, const int *off_b,
                         const int *g_x_max, const int *g_y_max, const int *g_z_max);

/* ideal_gas_kernel.f90:23-64 */
void oracle_ideal_gas_kernel(const int *x_min, const int *x_max, const int *y_min,
                             const int *y_max, const int *z_min, const int *z_max,
                             double *density, double *energy, double *pressure,
                             double *soundspeed);

/* viscosity_kernel.f90:28-141 */
void oracle_viscosity_kernel(const int *x_min, const int *x_max, const int *y_min,
                             const int *y_max, const int *z_min, const int *z_max,
                             const double *xarea, const double *yarea, const double *zarea,
                             const double *celldx, const double *celldy, const double *celldz,
                             const double *density0, const double *pressure,
                             double *viscosity, const double *xvel0, const double *yvel0,
                             const double *zvel0);

/* calc_dt_kernel.f90:28-183 */
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
                           int *small);

/* PdV_kernel.f90:28-175; predict is a Fortran LOGICAL (nonzero = .TRUE.) */
void oracle_pdv_kernel(const int *predict, const int *x_min, const int *x_max,
                       const int *y_min, const int *y_max, const int *z_min,
                       const int *z_max, const double *dt, const double *xarea,
                       const double *yarea, const double *zarea, const double *volume,
                       const double *density0, double *density1, const double *energy0,
                       double *energy1, const double *pressure, const double *viscosity,
                       const double *xvel0, const double *xvel1, const double *yvel0,
                       const double *yvel1, const double *zvel0, const double *zvel1);

/* revert_kernel.f90:23-67 */
void oracle_revert_kernel(const int *x_min, const int *x_max, const int *y_min,
                          const int *y_max, const int *z_min, const int *z_max,
                          const double *density0, double *density1,
                          const double *energy0, double *energy1);

/* accelerate_kernel.f90:27-115 */
void oracle_accelerate_kernel(const int *x_min, const int *x_max, const int *y_min,
                              const int *y_max, const int *z_min, const int *z_max,
                              const double *dt, const double *xarea, const double *yarea,
                              const double *zarea, const double *volume,
                              const double *density0, const double *pressure,
                              const double *viscosity, const double *xvel0,
                              const double *yvel0, const double *zvel0, double *xvel1,
                              double *yvel1, double *zvel1);

/* flux_calc_kernel.f90:26-95 */
void oracle_flux_calc_kernel(const int *x_min, const int *x_max, const int *y_min,
                             const int *y_max, const int *z_min, const int *z_max,
                             const double *dt, const double *xarea, const double *yarea,
                             const double *zarea, const double *xvel0, const double *yvel0,
                             const double *zvel0, const double *xvel1, const double *yvel1,
                             const double *zvel1, double *vol_flux_x, double *vol_flux_y,
                             double *vol_flux_z);

/* advec_cell_kernel.f90:30-383; advect_x is a Fortran LOGICAL */
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
                              double *post_ener, double *ener_flux);

/* advec_mom_kernel.f90:29-428 */
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
                             const int *direction);

/* reset_field_kernel.f90:27-101 */
void oracle_reset_field_kernel(const int *x_min, const int *x_max, const int *y_min,
                               const int *y_max, const int *z_min, const int *z_max,
                               double *density0, const double *density1, double *energy0,
                               const double *energy1, double *xvel0, const double *xvel1,
                               double *yvel0, const double *yvel1, double *zvel0,
                               const double *zvel1);

/* field_summary_kernel.f90:26-81 */
void oracle_field_summary_kernel(const int *x_min, const int *x_max, const int *y_min,
                                 const int *y_max, const int *z_min, const int *z_max,
                                 const double *volume, const double *density0,
                                 const double *energy0, const double *pressure,
                                 const double *xvel0, const double *yvel0,
                                 const double *zvel0, double *vol, double *mass, double *ie,
                                 double *ke, double *press);

/* update_halo_kernel.f90:32-1427 (external faces only; fields has 19 entries) */
void oracle_update_halo_kernel(const int *x_min, const int *x_max, const int *y_min,
                               const int *y_max, const int *z_min, const int *z_max,
                               const int *chunk_neighbours, const int *tile_neighbours,
                               double *density0, double *energy0, double *pressure,
                               double *viscosity, double *soundspeed, double *density1,
                               double *energy1, double *xvel0, double *yvel0, double *zvel0,
                               double *xvel1, double *yvel1, double *zvel1,
                               double *vol_flux_x, double *vol_flux_y, double *vol_flux_z,
                               double *mass_flux_x, double *mass_flux_y,
                               double *mass_flux_z, const int *fields, const int *depth);

/* initialise_chunk_kernel.f90:27-182 */
void oracle_initialise_chunk_kernel(const int *x_min, const int *x_max, const int *y_min,
                                    const int *y_max, const int *z_min, const int *z_max,
                                    const double *xmin, const double *ymin,
                                    const double *zmin, const double *dx, const double *dy,
                                    const double *dz, double *vertexx, double *vertexdx,
                                    double *vertexy, double *vertexdy, double *vertexz,
                                    double *vertexdz, double *cellx, double *celldx,
                                    double *celly, double *celldy, double *cellz,
                                    double *celldz, double *volume, double *xarea,
                                    double *yarea, double *zarea);

/* generate_chunk_kernel.f90:27-211 (geometry codes: 1 cuboid, 2 sphere, 3 point) */
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
                                  const int *g_circ, const int *g_point);

/*
 * Whole-run driver: start.f90 + hydro.f90 for one chunk with one tile.
 * The deck values are the parsed deck (read_input.f90 defaults applied by the
 * caller); the state-bound nudge of read_input.f90:287-303 is applied here.
 * Outputs: dt of every step (dt_out[step-1], capacity max_steps), the 5 summed
 * field_summary quantities (vol, mass, ie, ke, press) for every summary call
 * (summary_out[5*i], summary_step_out[i], capacity max_summaries).
 * The final state is written into fields_out (ORACLE_NUM_OUT arrays, each in
 * the reference layout) when non-NULL. Returns the number of steps taken.
 */
typedef struct {
  int x_cells, y_cells, z_cells;
  double xmin, ymin, zmin, xmax, ymax, zmax;
  double dtinit, dtmax, dtrise, dtmin;
  double end_time;
  int end_step;
  int summary_frequency;
  int number_of_states;
  double state_density[16], state_energy[16];
  double state_xvel[16], state_yvel[16], state_zvel[16];
  double state_xmin[16], state_xmax[16], state_ymin[16], state_ymax[16];
  double state_zmin[16], state_zmax[16], state_radius[16];
  int state_geometry[16];
} oracle_deck;

int oracle_run(const oracle_deck *deck, int max_steps, double *dt_out, int max_summaries,
               double *summary_out, int *summary_step_out, int *n_summaries,
               double **fields_out);

/* oracle_run keeping the chunk: *steps receives oracle_run's return value;
 * the handle gives field id 1..19 in its reference shape (oracle_kept_field)
 * until oracle_kept_free. For comparing a large run array by array. */
void *oracle_run_keep(const oracle_deck *deck, int max_steps, double *dt_out, int max_summaries,
                      double *summary_out, int *summary_step_out, int *n_summaries,
                      int *steps);
int oracle_kept_field(void *h, int id, double *out);
void oracle_kept_free(void *h);

/* CPU-baseline timing: run warmup + steps steps of the deck and return the
 * wall seconds of the last `steps` (the step loop including its field
 * summaries, without set-up). */
double oracle_run_timed(const oracle_deck *deck, int warmup, int steps);

#ifdef __cplusplus
}
#endif
#endif
