/*
 * Bounds check of the reference index ranges -- TEST INFRASTRUCTURE ONLY.
 * Built with -fsanitize=address,undefined (oracle/Makefile target `asan`) and
 * run on edge-case grids: one-cell-thick axes, two-cell axes, odd sizes,
 * every state geometry. The device kernels use the same index arithmetic on
 * a layout at least as large, so a clean run here means the device accesses
 * of these cases stay inside their arrays.
 */
#include <stdio.h>
#include <string.h>

#include "clover_oracle.h"

static void base(oracle_deck *d, int nx, int ny, int nz) {
  memset(d, 0, sizeof(*d));
  d->x_cells = nx; d->y_cells = ny; d->z_cells = nz;
  d->xmax = 10.0; d->ymax = 10.0; d->zmax = 10.0;
  d->dtinit = 0.04; d->dtmax = 0.04; d->dtrise = 1.5; d->dtmin = 1e-7;
  d->end_time = 1000.0; d->end_step = 6; d->summary_frequency = 2;
  d->number_of_states = 4;
  d->state_density[0] = 0.2; d->state_energy[0] = 1.0; d->state_xvel[0] = 0.1;
  d->state_density[1] = 1.0; d->state_energy[1] = 2.5; d->state_geometry[1] = 1;
  d->state_xmax[1] = 5.0; d->state_ymax[1] = 2.0; d->state_zmax[1] = 2.0;
  d->state_yvel[1] = -0.2;
  d->state_density[2] = 2.0; d->state_energy[2] = 0.5; d->state_geometry[2] = 2;
  d->state_xmin[2] = 7.0; d->state_ymin[2] = 3.0; d->state_zmin[2] = 6.0;
  d->state_radius[2] = 2.2; d->state_zvel[2] = 0.3;
  d->state_density[3] = 3.0; d->state_energy[3] = 4.0; d->state_geometry[3] = 3;
}

int main(void) {
  static const int sizes[][3] = {{1, 1, 1}, {1, 4, 3}, {5, 1, 2}, {2, 2, 1}, {3, 2, 2},
                                 {10, 2, 2}, {7, 5, 3}, {4, 9, 6}, {6, 6, 1}};
  double dt[64], sum[5 * 64];
  int steps[64], nsum = 0;
  for (size_t i = 0; i < sizeof(sizes) / sizeof(sizes[0]); i++) {
    oracle_deck d;
    base(&d, sizes[i][0], sizes[i][1], sizes[i][2]);
    int n = oracle_run(&d, 6, dt, 64, sum, steps, &nsum, NULL);
    printf("%dx%dx%d steps %d summaries %d\n", sizes[i][0], sizes[i][1], sizes[i][2], n, nsum);
  }
  return 0;
}
