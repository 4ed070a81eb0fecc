/*
 * CPU oracle: the halo messages of the reference's MPI exchange,
 * pack_kernel.f90 -- TEST INFRASTRUCTURE ONLY (the checker of the device
 * pack/unpack entry points and of the brick driver's exchange).
 *
 * One routine for the twelve pack_kernel.f90 subroutines: side 0..5 = left,
 * right, bottom, top, back, front; pack != 0 copies field -> buffer, else
 * buffer -> field. The loops, index expressions and source/target elements are
 * those of pack_kernel.f90 (:74-82 left, :190-198 right, :306-315 top,
 * :422-431 bottom, :538-547 back, :654-663 front and the matching unpack
 * loops). `field` has the reference's declared extents for its type (cell
 * nx+4, one more in each axis the type is node-centred in), lower bound -1 in
 * every axis; `buffer` is the reference's 1-based message buffer.
 */
#include "clover_oracle.h"

void oracle_pack_message(int side, int pack, const int *x_min, const int *x_max,
                         const int *y_min, const int *y_max, const int *z_min, const int *z_max,
                         double *field, double *buffer, const int *depth, const int *field_type,
                         const int *buffer_offset, const int *off_a, const int *off_b,
                         const int *g_x_max, const int *g_y_max, const int *g_z_max) {
  const int d = *depth, t = *field_type;
  /* x_inc, y_inc, z_inc: CELL, VERTEX, X_FACE, Y_FACE, Z_FACE (pack_kernel.f90:47-71) */
  const int xi = (t == 2 || t == 3), yi = (t == 2 || t == 4), zi = (t == 2 || t == 5);
  const long nx = *x_max - *x_min + 5 + xi, ny = *y_max - *y_min + 5 + yi;
  const int x0 = *x_min - 2, y0 = *y_min - 2, z0 = *z_min - 2;
#define F(j, k, l) field[((long)(j) - x0) + nx * (((long)(k) - y0) + ny * ((long)(l) - z0))]
  const long bo = *buffer_offset;
  if (side <= 1) {
    const long gy = *g_y_max + yi + 2 * d;
    for (int l = *z_min - d; l <= *z_max + zi + d; l++)
      for (int k = *y_min - d; k <= *y_max + yi + d; k++)
        for (int j = 1; j <= d; j++) {
          const long idx = bo + (j + (long)(k + *off_a + d - 1) * d) + ((long)(l + *off_b + d - 1) * gy * d);
          const int jj = side == 0 ? (pack ? *x_min + xi - 1 + j : *x_min - j)
                                   : (pack ? *x_max + 1 - j : *x_max + xi + j);
          if (pack) buffer[idx - 1] = F(jj, k, l);
          else F(jj, k, l) = buffer[idx - 1];
        }
  } else if (side <= 3) {
    const long gx = *g_x_max + xi + 2 * d, gz = *g_z_max + zi + 2 * d;
    for (int k = 1; k <= d; k++)
      for (int l = *z_min - d; l <= *z_max + zi + d; l++)
        for (int j = *x_min - d; j <= *x_max + xi + d; j++) {
          const long idx = bo + (j + *off_a + d) + (long)(l + *off_b - 1 + d) * gx + (long)(k - 1) * (gx * gz);
          const int kk = side == 2 ? (pack ? *y_min + yi - 1 + k : *y_min - k)
                                   : (pack ? *y_max + 1 - k : *y_max + yi + k);
          if (pack) buffer[idx - 1] = F(j, kk, l);
          else F(j, kk, l) = buffer[idx - 1];
        }
  } else {
    const long gx = *g_x_max + xi + 2 * d, gy = *g_y_max + yi + 2 * d;
    for (int l = 1; l <= d; l++)
      for (int k = *y_min - d; k <= *y_max + yi + d; k++)
        for (int j = *x_min - d; j <= *x_max + xi + d; j++) {
          const long idx = bo + (j + *off_a + d) + (long)(k + *off_b - 1 + d) * gx + (long)(l - 1) * (gx * gy);
          const int ll = side == 4 ? (pack ? *z_min + zi - 1 + l : *z_min - l)
                                   : (pack ? *z_max + 1 - l : *z_max + zi + l);
          if (pack) buffer[idx - 1] = F(j, k, ll);
          else F(j, k, ll) = buffer[idx - 1];
        }
  }
#undef F
}
