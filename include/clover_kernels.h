/*
 * Drop-in C ABI of the CloverLeaf3D hydro-cycle kernels, B200 (sm_100a).
 *
 * Each entry point replaces one Fortran module procedure of the reference
 * (UK-MAC/CloverLeaf3D_ref) and keeps its argument list and argument order.
 * Every argument is a pointer, as Fortran passes them by reference; LOGICAL
 * arguments arrive as int32 (nonzero = .TRUE.). Array arguments point at
 * element (x_min-2, y_min-2, z_min-2) of a column-major array with the shape
 * the reference declares for that argument.
 *
 * Host arrays are mirrored on the GPU: the first call that sees a host
 * pointer allocates a device buffer in the chunk layout and copies the array
 * up; every later call works on the resident copy and the host copy goes
 * stale. Scalar outputs (calc_dt, field_summary) come back on return.
 * clover_gpu_sync_to_host() copies every mirrored array back;
 * clover_gpu_invalidate() marks one host array as changed on the host.
 * A pointer to device memory is used in place and must already follow the
 * chunk layout that clover_gpu_layout() describes.
 *
 * One chunk with one tile per process: every call must pass the same
 * x_min..z_max. Calls are asynchronous on one library stream, except those
 * that return scalars. Not re-entrant. Errors never cross the ABI: they set
 * bits of clover_gpu_status().
 */
#ifndef CLOVER_KERNELS_H
#define CLOVER_KERNELS_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ideal_gas_kernel_module::ideal_gas_kernel, ideal_gas_kernel.f90:23-64 */
void clover_ideal_gas_kernel(const int *x_min, const int *x_max, const int *y_min,
                             const int *y_max, const int *z_min, const int *z_max,
                             double *density, double *energy, double *pressure,
                             double *soundspeed);

/* viscosity_kernel_module::viscosity_kernel, viscosity_kernel.f90:28-141 */
void clover_viscosity_kernel(const int *x_min, const int *x_max, const int *y_min,
                             const int *y_max, const int *z_min, const int *z_max,
                             double *xarea, double *yarea, double *zarea, double *celldx,
                             double *celldy, double *celldz, double *density0,
                             double *pressure, double *viscosity, double *xvel0,
                             double *yvel0, double *zvel0);

/* calc_dt_kernel_module::calc_dt_kernel, calc_dt_kernel.f90:28-183.
 * Synchronises: dt_min_val and the location outputs are host scalars. */
void clover_calc_dt_kernel(const int *x_min, const int *x_max, const int *y_min,
                           const int *y_max, const int *z_min, const int *z_max,
                           const double *g_small, const double *g_big, const double *dtmin,
                           const double *dtc_safe, const double *dtu_safe,
                           const double *dtv_safe, const double *dtw_safe,
                           const double *dtdiv_safe, double *xarea, double *yarea,
                           double *zarea, double *cellx, double *celly, double *cellz,
                           double *celldx, double *celldy, double *celldz, double *volume,
                           double *density0, double *energy0, double *pressure,
                           double *viscosity_a, double *soundspeed, double *xvel0,
                           double *yvel0, double *zvel0, double *dt_min, double *dt_min_val,
                           int *dtl_control, double *xl_pos, double *yl_pos, double *zl_pos,
                           int *jldt, int *kldt, int *lldt, int *small);

/* PdV_kernel_module::PdV_kernel, PdV_kernel.f90:28-175 */
void clover_pdv_kernel(const int32_t *predict, const int *x_min, const int *x_max,
                       const int *y_min, const int *y_max, const int *z_min, const int *z_max,
                       const double *dt, double *xarea, double *yarea, double *zarea,
                       double *volume, double *density0, double *density1, double *energy0,
                       double *energy1, double *pressure, double *viscosity, double *xvel0,
                       double *xvel1, double *yvel0, double *yvel1, double *zvel0,
                       double *zvel1);

/* revert_kernel_module::revert_kernel, revert_kernel.f90:23-67 */
void clover_revert_kernel(const int *x_min, const int *x_max, const int *y_min,
                          const int *y_max, const int *z_min, const int *z_max,
                          double *density0, double *density1, double *energy0,
                          double *energy1);

/* accelerate_kernel_module::accelerate_kernel, accelerate_kernel.f90:27-115 */
void clover_accelerate_kernel(const int *x_min, const int *x_max, const int *y_min,
                              const int *y_max, const int *z_min, const int *z_max,
                              const double *dt, double *xarea, double *yarea, double *zarea,
                              double *volume, double *density0, double *pressure,
                              double *viscosity, double *xvel0, double *yvel0, double *zvel0,
                              double *xvel1, double *yvel1, double *zvel1);

/* flux_calc_kernel_module::flux_calc_kernel, flux_calc_kernel.f90:26-95 */
void clover_flux_calc_kernel(const int *x_min, const int *x_max, const int *y_min,
                             const int *y_max, const int *z_min, const int *z_max,
                             const double *dt, double *xarea, double *yarea, double *zarea,
                             double *xvel0, double *yvel0, double *zvel0, double *xvel1,
                             double *yvel1, double *zvel1, double *vol_flux_x,
                             double *vol_flux_y, double *vol_flux_z);

/* advec_cell_kernel_module::advec_cell_kernel, advec_cell_kernel.f90:30-383 */
void clover_advec_cell_kernel(const int *x_min, const int *x_max, const int *y_min,
                              const int *y_max, const int *z_min, const int *z_max,
                              const int32_t *advect_x, const int *dir, const int *sweep_number,
                              double *vertexdx, double *vertexdy, double *vertexdz,
                              double *volume, double *density1, double *energy1,
                              double *mass_flux_x, double *vol_flux_x, double *mass_flux_y,
                              double *vol_flux_y, double *mass_flux_z, double *vol_flux_z,
                              double *pre_vol, double *post_vol, double *pre_mass,
                              double *post_mass, double *advec_vol, double *post_ener,
                              double *ener_flux);

/* advec_mom_kernel_mod::advec_mom_kernel, advec_mom_kernel.f90:29-428 */
void clover_advec_mom_kernel(const int *x_min, const int *x_max, const int *y_min,
                             const int *y_max, const int *z_min, const int *z_max,
                             double *vel1, double *mass_flux_x, double *vol_flux_x,
                             double *mass_flux_y, double *vol_flux_y, double *mass_flux_z,
                             double *vol_flux_z, double *volume, double *density1,
                             double *node_flux, double *node_mass_post, double *node_mass_pre,
                             double *advec_vel, double *mom_flux, double *pre_vol,
                             double *post_vol, double *celldx, double *celldy, double *celldz,
                             const int32_t *advect_x, const int *which_vel,
                             const int *sweep_number, const int *direction);

/* reset_field_kernel_module::reset_field_kernel, reset_field_kernel.f90:27-101 */
void clover_reset_field_kernel(const int *x_min, const int *x_max, const int *y_min,
                               const int *y_max, const int *z_min, const int *z_max,
                               double *density0, double *density1, double *energy0,
                               double *energy1, double *xvel0, double *xvel1, double *yvel0,
                               double *yvel1, double *zvel0, double *zvel1);

/* field_summary_kernel_module::field_summary_kernel, field_summary_kernel.f90:26-81.
 * Synchronises: the five sums are host scalars. */
void clover_field_summary_kernel(const int *x_min, const int *x_max, const int *y_min,
                                 const int *y_max, const int *z_min, const int *z_max,
                                 double *volume, double *density0, double *energy0,
                                 double *pressure, double *xvel0, double *yvel0, double *zvel0,
                                 double *vol, double *mass, double *ie, double *ke,
                                 double *press);

/* field_summary for callers that cannot let the library allocate device
 * memory. No counterpart in the reference. Meant for a host code whose GPU
 * memory is all owned by its own pool allocator or held under a fixed budget,
 * where a cudaMalloc made inside the library could fail or fragment that
 * pool. It allocates nothing: the arrays are the caller's DEVICE arrays in
 * the chunk layout of clover_gpu_layout(), on the current device (host
 * arrays and another GPU's arrays are rejected), the five sums come back in
 * host scalars, and the reduction scratch is a fixed 320 KiB file-scope
 * device array that every GPU loading the library holds until the process
 * exits. At most CLOVER_NOALLOC_MAX_Z_CELLS cells along z (larger grids
 * return CLOVER_STATUS_BAD_ARG with a message on stderr).
 * It runs on the library's stream when the drop-in context exists on the
 * current device, so it reads the arrays after every clover_*_kernel call
 * queued before it (those return without waiting); otherwise on the legacy
 * default stream. Work the caller queued on its own streams must be finished
 * first. Returns when the sums are on the host; 0 on success, else a
 * CLOVER_STATUS_* bit. The first call on a device looks up the scratch
 * address (once per device; a cudaDeviceReset after it is not supported);
 * make that first call before any stream capture. All calls share the one
 * scratch array: calls that overlap on the GPU race. Sums agree with
 * clover_field_summary_kernel to rounding (both compensated, in different
 * fixed orders). */
#define CLOVER_NOALLOC_MAX_Z_CELLS 4096
int clover_field_summary_kernel_noalloc(const int *x_min, const int *x_max, const int *y_min,
                                        const int *y_max, const int *z_min, const int *z_max,
                                        const double *volume, const double *density0,
                                        const double *energy0, const double *pressure,
                                        const double *xvel0, const double *yvel0,
                                        const double *zvel0, double *vol, double *mass,
                                        double *ie, double *ke, double *press);

/* update_halo_kernel_module::update_halo_kernel, update_halo_kernel.f90:32-1427.
 * Reflective copies on the faces where both neighbour entries are -1. */
void clover_update_halo_kernel(const int *x_min, const int *x_max, const int *y_min,
                               const int *y_max, const int *z_min, const int *z_max,
                               const int *chunk_neighbours, const int *tile_neighbours,
                               double *density0, double *energy0, double *pressure,
                               double *viscosity, double *soundspeed, double *density1,
                               double *energy1, double *xvel0, double *yvel0, double *zvel0,
                               double *xvel1, double *yvel1, double *zvel1,
                               double *vol_flux_x, double *vol_flux_y, double *vol_flux_z,
                               double *mass_flux_x, double *mass_flux_y, double *mass_flux_z,
                               const int *fields, const int *depth);

/* initialise_chunk_kernel_module::initialise_chunk_kernel,
 * initialise_chunk_kernel.f90:27-182 */
void clover_initialise_chunk_kernel(const int *x_min, const int *x_max, const int *y_min,
                                    const int *y_max, const int *z_min, const int *z_max,
                                    const double *xmin, const double *ymin, const double *zmin,
                                    const double *dx, const double *dy, const double *dz,
                                    double *vertexx, double *vertexdx, double *vertexy,
                                    double *vertexdy, double *vertexz, double *vertexdz,
                                    double *cellx, double *celldx, double *celly,
                                    double *celldy, double *cellz, double *celldz,
                                    double *volume, double *xarea, double *yarea,
                                    double *zarea);

/* generate_chunk_kernel_module::generate_chunk_kernel, generate_chunk_kernel.f90:27-211
 * (at most 16 states) */
void clover_generate_chunk_kernel(const int *x_min, const int *x_max, const int *y_min,
                                  const int *y_max, const int *z_min, const int *z_max,
                                  double *vertexx, double *vertexy, double *vertexz,
                                  double *cellx, double *celly, double *cellz,
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

/* pack_kernel_module (pack_kernel.f90): the halo messages of the reference's
 * MPI exchange, called per field by clover.f90:715-4457 (clover_pack_left and
 * the like). pack copies `depth` layers of `field` next to the side into the
 * caller's buffer at the 1-based indices pack_kernel.f90 forms from
 * buffer_offset, the two tile offsets and g_x/y/z_max; unpack copies them into
 * the halo on that side. The field is the device mirror of the host array; the
 * message is formed on the device and copied to or from `buffer` (host memory)
 * before the call returns. field_type is compared with the five *_DATA
 * arguments (data.f90 CELL_DATA..Z_FACE_DATA) as the reference does. */
/* pack_kernel_module::clover_pack_message_left, pack_kernel.f90:29-85 */
void clover_pack_message_left(const int *x_min, const int *x_max, const int *y_min, const int *y_max,
                          const int *z_min, const int *z_max, double *field, double *buffer,
                          const int *cell_data, const int *vertex_data, const int *x_face_data,
                          const int *y_face_data, const int *z_face_data, const int *depth,
                          const int *field_type, const int *buffer_offset, const int *y_offset,
                          const int *z_offset, const int *g_x_max, const int *g_y_max,
                          const int *g_z_max);
/* pack_kernel_module::clover_unpack_message_left, pack_kernel.f90:87-143 */
void clover_unpack_message_left(const int *x_min, const int *x_max, const int *y_min, const int *y_max,
                          const int *z_min, const int *z_max, double *field, double *buffer,
                          const int *cell_data, const int *vertex_data, const int *x_face_data,
                          const int *y_face_data, const int *z_face_data, const int *depth,
                          const int *field_type, const int *buffer_offset, const int *y_offset,
                          const int *z_offset, const int *g_x_max, const int *g_y_max,
                          const int *g_z_max);
/* pack_kernel_module::clover_pack_message_right, pack_kernel.f90:145-201 */
void clover_pack_message_right(const int *x_min, const int *x_max, const int *y_min, const int *y_max,
                          const int *z_min, const int *z_max, double *field, double *buffer,
                          const int *cell_data, const int *vertex_data, const int *x_face_data,
                          const int *y_face_data, const int *z_face_data, const int *depth,
                          const int *field_type, const int *buffer_offset, const int *y_offset,
                          const int *z_offset, const int *g_x_max, const int *g_y_max,
                          const int *g_z_max);
/* pack_kernel_module::clover_unpack_message_right, pack_kernel.f90:203-259 */
void clover_unpack_message_right(const int *x_min, const int *x_max, const int *y_min, const int *y_max,
                          const int *z_min, const int *z_max, double *field, double *buffer,
                          const int *cell_data, const int *vertex_data, const int *x_face_data,
                          const int *y_face_data, const int *z_face_data, const int *depth,
                          const int *field_type, const int *buffer_offset, const int *y_offset,
                          const int *z_offset, const int *g_x_max, const int *g_y_max,
                          const int *g_z_max);
/* pack_kernel_module::clover_pack_message_bottom, pack_kernel.f90:377-433 */
void clover_pack_message_bottom(const int *x_min, const int *x_max, const int *y_min, const int *y_max,
                          const int *z_min, const int *z_max, double *field, double *buffer,
                          const int *cell_data, const int *vertex_data, const int *x_face_data,
                          const int *y_face_data, const int *z_face_data, const int *depth,
                          const int *field_type, const int *buffer_offset, const int *x_offset,
                          const int *z_offset, const int *g_x_max, const int *g_y_max,
                          const int *g_z_max);
/* pack_kernel_module::clover_unpack_message_bottom, pack_kernel.f90:435-491 */
void clover_unpack_message_bottom(const int *x_min, const int *x_max, const int *y_min, const int *y_max,
                          const int *z_min, const int *z_max, double *field, double *buffer,
                          const int *cell_data, const int *vertex_data, const int *x_face_data,
                          const int *y_face_data, const int *z_face_data, const int *depth,
                          const int *field_type, const int *buffer_offset, const int *x_offset,
                          const int *z_offset, const int *g_x_max, const int *g_y_max,
                          const int *g_z_max);
/* pack_kernel_module::clover_pack_message_top, pack_kernel.f90:261-317 */
void clover_pack_message_top(const int *x_min, const int *x_max, const int *y_min, const int *y_max,
                          const int *z_min, const int *z_max, double *field, double *buffer,
                          const int *cell_data, const int *vertex_data, const int *x_face_data,
                          const int *y_face_data, const int *z_face_data, const int *depth,
                          const int *field_type, const int *buffer_offset, const int *x_offset,
                          const int *z_offset, const int *g_x_max, const int *g_y_max,
                          const int *g_z_max);
/* pack_kernel_module::clover_unpack_message_top, pack_kernel.f90:319-375 */
void clover_unpack_message_top(const int *x_min, const int *x_max, const int *y_min, const int *y_max,
                          const int *z_min, const int *z_max, double *field, double *buffer,
                          const int *cell_data, const int *vertex_data, const int *x_face_data,
                          const int *y_face_data, const int *z_face_data, const int *depth,
                          const int *field_type, const int *buffer_offset, const int *x_offset,
                          const int *z_offset, const int *g_x_max, const int *g_y_max,
                          const int *g_z_max);
/* pack_kernel_module::clover_pack_message_back, pack_kernel.f90:493-549 */
void clover_pack_message_back(const int *x_min, const int *x_max, const int *y_min, const int *y_max,
                          const int *z_min, const int *z_max, double *field, double *buffer,
                          const int *cell_data, const int *vertex_data, const int *x_face_data,
                          const int *y_face_data, const int *z_face_data, const int *depth,
                          const int *field_type, const int *buffer_offset, const int *x_offset,
                          const int *y_offset, const int *g_x_max, const int *g_y_max,
                          const int *g_z_max);
/* pack_kernel_module::clover_unpack_message_back, pack_kernel.f90:551-607 */
void clover_unpack_message_back(const int *x_min, const int *x_max, const int *y_min, const int *y_max,
                          const int *z_min, const int *z_max, double *field, double *buffer,
                          const int *cell_data, const int *vertex_data, const int *x_face_data,
                          const int *y_face_data, const int *z_face_data, const int *depth,
                          const int *field_type, const int *buffer_offset, const int *x_offset,
                          const int *y_offset, const int *g_x_max, const int *g_y_max,
                          const int *g_z_max);
/* pack_kernel_module::clover_pack_message_front, pack_kernel.f90:609-664 */
void clover_pack_message_front(const int *x_min, const int *x_max, const int *y_min, const int *y_max,
                          const int *z_min, const int *z_max, double *field, double *buffer,
                          const int *cell_data, const int *vertex_data, const int *x_face_data,
                          const int *y_face_data, const int *z_face_data, const int *depth,
                          const int *field_type, const int *buffer_offset, const int *x_offset,
                          const int *y_offset, const int *g_x_max, const int *g_y_max,
                          const int *g_z_max);
/* pack_kernel_module::clover_unpack_message_front, pack_kernel.f90:666-721 */
void clover_unpack_message_front(const int *x_min, const int *x_max, const int *y_min, const int *y_max,
                          const int *z_min, const int *z_max, double *field, double *buffer,
                          const int *cell_data, const int *vertex_data, const int *x_face_data,
                          const int *y_face_data, const int *z_face_data, const int *depth,
                          const int *field_type, const int *buffer_offset, const int *x_offset,
                          const int *y_offset, const int *g_x_max, const int *g_y_max,
                          const int *g_z_max);

/* ---- mirror management (no counterpart in the reference: the reference
 * arrays live in host memory only) ---- */

/* Status bits. */
#define CLOVER_STATUS_CUDA_ERROR 0x1   /* a CUDA call or launch failed */
#define CLOVER_STATUS_BOUNDS 0x2       /* an array passed with another chunk's bounds */
#define CLOVER_STATUS_SMALL_DT 0x4     /* calc_dt returned small=1 */
#define CLOVER_STATUS_NO_DEVICE 0x8    /* no CUDA device */
#define CLOVER_STATUS_BAD_ARG 0x10     /* unsupported argument (e.g. >16 states) */
#define CLOVER_STATUS_TIMEOUT 0x20     /* a bounded device wait gave up */

int clover_gpu_status(void);
const char *clover_gpu_error_string(void);
void clover_gpu_clear_status(void);
/* Copy every mirrored array back into its host array (waits for the GPU). */
void clover_gpu_sync_to_host(void);
/* The host copy of this array changed: upload it again at its next use. */
void clover_gpu_invalidate(const void *host_array);
/* Every mirrored host array changed (e.g. the caller restored its state on
 * the host): each is uploaded again at its next use. */
void clover_gpu_invalidate_all(void);
/* Wait for all queued work. */
void clover_gpu_synchronize(void);
/* Allow (1, the default) or forbid (0) the staged forms of the kernels that
 * have one (planes copied into shared memory by bulk-tensor copies): both
 * forms give the same bits. A staged kernel whose bounded wait for its copies
 * gives up sets CLOVER_STATUS_TIMEOUT, seen at the next synchronisation. */
void clover_gpu_use_staging(int on);
/* Failure-path check of the above: queue on the library stream a bounded wait
 * that runs out (cycles SM clocks at most) and reports through the library's
 * device status word, as a staged kernel whose copies do not arrive would; the
 * next synchronisation sets CLOVER_STATUS_TIMEOUT. 0, or a status bit if no
 * library context exists yet or the launch failed. */
int clover_gpu_wait_selftest_queued(long long cycles);
/* Free every mirror and the library stream. */
void clover_gpu_release(void);
/* Chunk layout for device pointers passed in place: element (j,k,l) is at
 * (j-x_min+2) + (k-y_min+2)*px + (l-z_min+2)*pxy from the pointer. */
void clover_gpu_layout(const int *x_min, const int *x_max, const int *y_min, const int *y_max,
                       const int *z_min, const int *z_max, int *px, long long *pxy,
                       long long *elems);
/* Number of host arrays currently mirrored, and their total device bytes. */
void clover_gpu_mirror_stats(int *arrays, long long *bytes);
/* One halo message between two chunks mirrored in this process, on the
 * device: side's message of `src` (a host array of the chunk with bounds
 * src_bounds = x_min,x_max,y_min,y_max,z_min,z_max) packed as pack_kernel.f90
 * packs it and unpacked into the opposite side of `dst` (chunk dst_bounds).
 * side 0..5 = left, right, bottom, top, back, front; field_type 1 cell,
 * 2 vertex, 3 x face, 4 y face, 5 z face; depth 1 or 2. The transport of the
 * brick driver when its bricks share a device. */
void clover_gpu_face_copy(const int *src_bounds, double *src, const int *dst_bounds, double *dst,
                          int side, int field_type, int depth);
/* n halo messages between chunks of this process in one launch, message m
 * as clover_gpu_face_copy(src_bounds + 6m, src[m], dst_bounds + 6m, dst[m],
 * sides[m], field_types[m], depth) would move it; the messages must not write
 * what another of them reads (one axis phase of an exchange). 0, or -1 with
 * the status set. */
int clover_gpu_face_copy_many(int n, const int *src_bounds, double *const *src,
                              const int *dst_bounds, double *const *dst, const int *sides,
                              const int *field_types, int depth);
/* Length in doubles of one halo message (pack_kernel.f90 layout, no tile
 * offsets) of a chunk with bounds x_min..z_max; -1 for a bad argument. */
long long clover_gpu_message_len(const int *bounds, int side, int field_type, int depth);
/* Pack (unpack = 0) side's message of `field` (host array of the chunk with
 * `bounds`, mirrored) into the device buffer dev_msg, or unpack (unpack = 1)
 * it from there into the halo on that side; queued on the library stream.
 * Returns 0, or -1 with the status set. */
int clover_gpu_pack_device(const int *bounds, double *field, int side, int field_type, int depth,
                           double *dev_msg, int unpack);

#ifdef __cplusplus
}
#endif
#endif
