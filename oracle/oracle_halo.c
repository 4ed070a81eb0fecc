/*
 * CPU oracle: reflective external-face halo update -- TEST INFRASTRUCTURE ONLY.
 *
 * Restates update_halo_kernel.f90:32-1427. Every field/face block of the
 * reference is one call below, in the reference order (fields 1..19; faces
 * bottom, top, left, right, back, front), with the loop extents and the
 * source/destination index arithmetic written out exactly as in the
 * reference. Later faces read corner values that earlier faces wrote, and
 * some corner values keep whatever the array held before the call; both are
 * part of the reference behaviour and are reproduced here.
 */
#include "clover_oracle.h"

enum { AX_X = 0, AX_Y = 1, AX_Z = 2 };

/* ORACLE_SYMMETRIC_HALO (a test-only build, never the checker of a parity
 * test): the z-face loops of the x and y face fluxes run to max+1+d along
 * their own face axis, as those of the z face fluxes do along z, instead of
 * the reference's max+d, which leaves the corners at max+2+d stale. The
 * rotation tests use it to show that this asymmetry of update_halo_kernel.f90
 * (:1018-1142, :1156-1280 against :1294-1417) is what separates a flow along
 * x or y from the same flow along z. */
#ifdef ORACLE_SYMMETRIC_HALO
#define FACE_FLUX_Z_EXT 1
#else
#define FACE_FLUX_Z_EXT 0
#endif

/*
 * One face block. The face-normal axis is `ax`; the two other axes run over
 * [a0,a1] and [b0,b1] (a = the lower-numbered of the remaining axes j<k<l).
 * For m = 1..depth the element at normal index dst(m) receives
 * sign * element at normal index src(m):
 *   low face : dst = 1 - m,       src = src_base + m
 *   high face: dst = dst_base + m, src = src_base - m
 */
static void face(double *a, long nx, long ny, long xlo, long ylo, long zlo, int ax, int high,
                 int depth, int a0, int a1, int b0, int b1, int dst_base, int src_base,
                 double sign) {
  for (int b = b0; b <= b1; b++)
    for (int aa = a0; aa <= a1; aa++)
      for (int m = 1; m <= depth; m++) {
        int dst = high ? dst_base + m : 1 - m;
        int src = high ? src_base - m : src_base + m;
        long dj, dk, dl, sj, sk, sl;
        if (ax == AX_X) {
          dj = dst; sj = src; dk = sk = aa; dl = sl = b;
        } else if (ax == AX_Y) {
          dk = dst; sk = src; dj = sj = aa; dl = sl = b;
        } else {
          dl = dst; sl = src; dj = sj = aa; dk = sk = b;
        }
        double v = a[(sj - xlo) + (sk - ylo) * nx + (sl - zlo) * nx * ny];
        a[(dj - xlo) + (dk - ylo) * nx + (dl - zlo) * nx * ny] = sign * v;
      }
}

void oracle_update_halo_kernel(const int *x_min, const int *x_max, const int *y_min,
                               const int *y_max, const int *z_min, const int *z_max,
                               const int *chunk_neighbours, const int *tile_neighbours,
                               double *density0, double *energy0, double *pressure,
                               double *viscosity, double *soundspeed, double *density1,
                               double *energy1, double *xvel0, double *yvel0, double *zvel0,
                               double *xvel1, double *yvel1, double *zvel1,
                               double *vol_flux_x, double *vol_flux_y, double *vol_flux_z,
                               double *mass_flux_x, double *mass_flux_y,
                               double *mass_flux_z, const int *fields, const int *depth) {
  const int xmn = *x_min, xmx = *x_max, ymn = *y_min, ymx = *y_max, zmn = *z_min, zmx = *z_max;
  const int d = *depth;
  const long xlo = xmn - 2, ylo = ymn - 2, zlo = zmn - 2;
  const long nxc = xmx - xmn + 5, nyc = ymx - ymn + 5;
  const long nxv = xmx - xmn + 6, nyv = ymx - ymn + 6;
  /* face ids: 1 left, 2 right, 3 bottom, 4 top, 5 back, 6 front; -1 external */
  int ext[7];
  for (int f = 1; f <= 6; f++)
    ext[f] = chunk_neighbours[f - 1] == -1 && tile_neighbours[f - 1] == -1;
  const int LEFT = 1, RIGHT = 2, BOTTOM = 3, TOP = 4, BACK = 5, FRONT = 6;

  /* Cell-centred fields, update_halo_kernel.f90:121-590: mirror about the face
   * (1-m <- 0+m, max+m <- max+1-m); all loops run over [min-d, max+d]. */
  double *cells[7] = {density0, density1, energy0, energy1, pressure, viscosity, soundspeed};
  const int cell_ids[7] = {1, 2, 3, 4, 5, 6, 7};
  for (int c = 0; c < 7; c++) {
    if (fields[cell_ids[c] - 1] != 1) continue;
    double *a = cells[c];
    if (ext[BOTTOM]) face(a, nxc, nyc, xlo, ylo, zlo, AX_Y, 0, d, xmn - d, xmx + d, zmn - d, zmx + d, 0, 0, 1.0);
    if (ext[TOP]) face(a, nxc, nyc, xlo, ylo, zlo, AX_Y, 1, d, xmn - d, xmx + d, zmn - d, zmx + d, ymx, ymx + 1, 1.0);
    if (ext[LEFT]) face(a, nxc, nyc, xlo, ylo, zlo, AX_X, 0, d, ymn - d, ymx + d, zmn - d, zmx + d, 0, 0, 1.0);
    if (ext[RIGHT]) face(a, nxc, nyc, xlo, ylo, zlo, AX_X, 1, d, ymn - d, ymx + d, zmn - d, zmx + d, xmx, xmx + 1, 1.0);
    if (ext[BACK]) face(a, nxc, nyc, xlo, ylo, zlo, AX_Z, 0, d, xmn - d, xmx + d, ymn - d, ymx + d, 0, 0, 1.0);
    if (ext[FRONT]) face(a, nxc, nyc, xlo, ylo, zlo, AX_Z, 1, d, xmn - d, xmx + d, ymn - d, ymx + d, zmx, zmx + 1, 1.0);
  }

  /* Vertex velocities, update_halo_kernel.f90:597-1004: mirror about the
   * boundary node (1-m <- 1+m, max+1+m <- max+1-m), extents [min-d, max+1+d];
   * the component normal to the face is negated. */
  double *verts[6] = {xvel0, xvel1, yvel0, yvel1, zvel0, zvel1};
  const int vert_ids[6] = {8, 9, 10, 11, 12, 13};
  const int vert_comp[6] = {AX_X, AX_X, AX_Y, AX_Y, AX_Z, AX_Z};
  for (int c = 0; c < 6; c++) {
    if (fields[vert_ids[c] - 1] != 1) continue;
    double *a = verts[c];
    double sy = vert_comp[c] == AX_Y ? -1.0 : 1.0;
    double sx = vert_comp[c] == AX_X ? -1.0 : 1.0;
    double sz = vert_comp[c] == AX_Z ? -1.0 : 1.0;
    if (ext[BOTTOM]) face(a, nxv, nyv, xlo, ylo, zlo, AX_Y, 0, d, xmn - d, xmx + 1 + d, zmn - d, zmx + 1 + d, 0, 1, sy);
    if (ext[TOP]) face(a, nxv, nyv, xlo, ylo, zlo, AX_Y, 1, d, xmn - d, xmx + 1 + d, zmn - d, zmx + 1 + d, ymx + 1, ymx + 1, sy);
    if (ext[LEFT]) face(a, nxv, nyv, xlo, ylo, zlo, AX_X, 0, d, ymn - d, ymx + 1 + d, zmn - d, zmx + 1 + d, 0, 1, sx);
    if (ext[RIGHT]) face(a, nxv, nyv, xlo, ylo, zlo, AX_X, 1, d, ymn - d, ymx + 1 + d, zmn - d, zmx + 1 + d, xmx + 1, xmx + 1, sx);
    if (ext[BACK]) face(a, nxv, nyv, xlo, ylo, zlo, AX_Z, 0, d, xmn - d, xmx + 1 + d, ymn - d, ymx + 1 + d, 0, 1, sz);
    if (ext[FRONT]) face(a, nxv, nyv, xlo, ylo, zlo, AX_Z, 1, d, xmn - d, xmx + 1 + d, ymn - d, ymx + 1 + d, zmx + 1, zmx + 1, sz);
  }

  /* vol_flux_x / mass_flux_x, update_halo_kernel.f90:1018-1142 */
  double *fx[2] = {vol_flux_x, mass_flux_x};
  const int fx_ids[2] = {14, 17};
  for (int c = 0; c < 2; c++) {
    if (fields[fx_ids[c] - 1] != 1) continue;
    double *a = fx[c];
    /* bottom: a(j,1-m,l)=a(j,1+m,l), j in [min-d,max+1+d], l in [min-d,max+d] */
    if (ext[BOTTOM]) face(a, nxv, nyc, xlo, ylo, zlo, AX_Y, 0, d, xmn - d, xmx + 1 + d, zmn - d, zmx + d, 0, 1, 1.0);
    /* top: a(j,ymax+m,l)=a(j,ymax-m,l) */
    if (ext[TOP]) face(a, nxv, nyc, xlo, ylo, zlo, AX_Y, 1, d, xmn - d, xmx + 1 + d, zmn - d, zmx + d, ymx, ymx, 1.0);
    /* left: a(1-m,k,l)=-a(1+m,k,l), k in [min-d,max+d] */
    if (ext[LEFT]) face(a, nxv, nyc, xlo, ylo, zlo, AX_X, 0, d, ymn - d, ymx + d, zmn - d, zmx + d, 0, 1, -1.0);
    /* right: a(xmax+1+m,k,l)=-a(xmax+1-m,k,l) */
    if (ext[RIGHT]) face(a, nxv, nyc, xlo, ylo, zlo, AX_X, 1, d, ymn - d, ymx + d, zmn - d, zmx + d, xmx + 1, xmx + 1, -1.0);
    /* back: a(j,k,1-m)=a(j,k,1+m), j in [min-d,max+d] (not max+1+d) */
    if (ext[BACK]) face(a, nxv, nyc, xlo, ylo, zlo, AX_Z, 0, d, xmn - d, xmx + FACE_FLUX_Z_EXT + d, ymn - d, ymx + d, 0, 1, 1.0);
    /* front: a(j,k,zmax+m)=a(j,k,zmax-m) */
    if (ext[FRONT]) face(a, nxv, nyc, xlo, ylo, zlo, AX_Z, 1, d, xmn - d, xmx + FACE_FLUX_Z_EXT + d, ymn - d, ymx + d, zmx, zmx, 1.0);
  }

  /* vol_flux_y / mass_flux_y, update_halo_kernel.f90:1156-1280 */
  double *fy[2] = {vol_flux_y, mass_flux_y};
  const int fy_ids[2] = {15, 18};
  for (int c = 0; c < 2; c++) {
    if (fields[fy_ids[c] - 1] != 1) continue;
    double *a = fy[c];
    /* bottom: a(j,1-m,l)=-a(j,1+m,l), j,l in [min-d,max+d] */
    if (ext[BOTTOM]) face(a, nxc, nyv, xlo, ylo, zlo, AX_Y, 0, d, xmn - d, xmx + d, zmn - d, zmx + d, 0, 1, -1.0);
    /* top: a(j,ymax+1+m,l)=-a(j,ymax+1-m,l) */
    if (ext[TOP]) face(a, nxc, nyv, xlo, ylo, zlo, AX_Y, 1, d, xmn - d, xmx + d, zmn - d, zmx + d, ymx + 1, ymx + 1, -1.0);
    /* left: a(1-m,k,l)=a(1+m,k,l), k in [min-d,max+1+d] */
    if (ext[LEFT]) face(a, nxc, nyv, xlo, ylo, zlo, AX_X, 0, d, ymn - d, ymx + 1 + d, zmn - d, zmx + d, 0, 1, 1.0);
    /* right: a(xmax+m,k,l)=a(xmax-m,k,l) */
    if (ext[RIGHT]) face(a, nxc, nyv, xlo, ylo, zlo, AX_X, 1, d, ymn - d, ymx + 1 + d, zmn - d, zmx + d, xmx, xmx, 1.0);
    /* back: a(j,k,1-m)=a(j,k,1+m), k in [min-d,max+d] */
    if (ext[BACK]) face(a, nxc, nyv, xlo, ylo, zlo, AX_Z, 0, d, xmn - d, xmx + d, ymn - d, ymx + FACE_FLUX_Z_EXT + d, 0, 1, 1.0);
    /* front: a(j,k,zmax+m)=a(j,k,zmax-m) */
    if (ext[FRONT]) face(a, nxc, nyv, xlo, ylo, zlo, AX_Z, 1, d, xmn - d, xmx + d, ymn - d, ymx + FACE_FLUX_Z_EXT + d, zmx, zmx, 1.0);
  }

  /* vol_flux_z, update_halo_kernel.f90:1294-1349 */
  if (fields[16 - 1] == 1) {
    double *a = vol_flux_z;
    /* bottom: l in [min-d,max+d] */
    if (ext[BOTTOM]) face(a, nxc, nyc, xlo, ylo, zlo, AX_Y, 0, d, xmn - d, xmx + d, zmn - d, zmx + d, 0, 1, 1.0);
    /* top: l in [min-d,max+1+d]; a(j,ymax+m,l)=a(j,ymax-m,l) */
    if (ext[TOP]) face(a, nxc, nyc, xlo, ylo, zlo, AX_Y, 1, d, xmn - d, xmx + d, zmn - d, zmx + 1 + d, ymx, ymx, 1.0);
    /* left: a(1-m,k,l)=a(1+m,k,l), l in [min-d,max+1+d] */
    if (ext[LEFT]) face(a, nxc, nyc, xlo, ylo, zlo, AX_X, 0, d, ymn - d, ymx + d, zmn - d, zmx + 1 + d, 0, 1, 1.0);
    /* right: a(xmax+m,k,l)=a(xmax-m,k,l) */
    if (ext[RIGHT]) face(a, nxc, nyc, xlo, ylo, zlo, AX_X, 1, d, ymn - d, ymx + d, zmn - d, zmx + 1 + d, xmx, xmx, 1.0);
    /* back: a(j,k,1-m)=-a(j,k,1+m) */
    if (ext[BACK]) face(a, nxc, nyc, xlo, ylo, zlo, AX_Z, 0, d, xmn - d, xmx + d, ymn - d, ymx + d, 0, 1, -1.0);
    /* front: a(j,k,zmax+1+m)=-a(j,k,zmax+1-m) */
    if (ext[FRONT]) face(a, nxc, nyc, xlo, ylo, zlo, AX_Z, 1, d, xmn - d, xmx + d, ymn - d, ymx + d, zmx + 1, zmx + 1, -1.0);
  }

  /* mass_flux_z, update_halo_kernel.f90:1362-1417 (bottom also runs to max+1+d) */
  if (fields[19 - 1] == 1) {
    double *a = mass_flux_z;
    if (ext[BOTTOM]) face(a, nxc, nyc, xlo, ylo, zlo, AX_Y, 0, d, xmn - d, xmx + d, zmn - d, zmx + 1 + d, 0, 1, 1.0);
    if (ext[TOP]) face(a, nxc, nyc, xlo, ylo, zlo, AX_Y, 1, d, xmn - d, xmx + d, zmn - d, zmx + 1 + d, ymx, ymx, 1.0);
    if (ext[LEFT]) face(a, nxc, nyc, xlo, ylo, zlo, AX_X, 0, d, ymn - d, ymx + d, zmn - d, zmx + 1 + d, 0, 1, 1.0);
    if (ext[RIGHT]) face(a, nxc, nyc, xlo, ylo, zlo, AX_X, 1, d, ymn - d, ymx + d, zmn - d, zmx + 1 + d, xmx, xmx, 1.0);
    if (ext[BACK]) face(a, nxc, nyc, xlo, ylo, zlo, AX_Z, 0, d, xmn - d, xmx + d, ymn - d, ymx + d, 0, 1, -1.0);
    if (ext[FRONT]) face(a, nxc, nyc, xlo, ylo, zlo, AX_Z, 1, d, xmn - d, xmx + d, ymn - d, ymx + d, zmx + 1, zmx + 1, -1.0);
  }
}
