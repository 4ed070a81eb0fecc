// Bulk-tensor (TMA) staging of chunk-layout planes into shared memory.
//
// A z-marching stencil block (32 x 8 columns) needs, per plane of the march,
// a box of each input array: its 32 columns plus halo columns on both sides,
// and its 8 rows plus halo rows. One thread issues the box copies of a whole
// plane (cp.async.bulk.tensor.3d, completion counted in bytes on an
// mbarrier) a few planes ahead of the plane the block computes, so the loads
// stay in flight without registers, and the block reads every stencil
// neighbour from shared memory.
//
// Tensor maps describe one array of one chunk in the chunk layout
// (clover_layout.cuh): dimensions (px, rows, planes), row and plane strides
// in bytes. A copy must start on a 16-byte boundary along x, so the map's
// base is the element H = 16 / sizeof(T) columns before x_min (element
// x_min is 128-byte aligned in every array) and a tile whose first column is
// x_min + 32 t starts its box at x coordinate 32 t, H columns before it; the
// box is 32 + 2 H columns wide. Rows and planes have no alignment rule, and a
// box that runs past the array's end reads zeros there.
//
// Only loads (no multicast): each block reads this GPU's own arrays.
#pragma once

#include <cuda.h>
#include <cuda_runtime.h>

#include "clover_launch.h"

namespace clover {

// Columns a box carries on each side of its 32 for element type T.
template <class T>
constexpr int kTmaHalo = 16 / (int)sizeof(T);
template <class T>
constexpr int kTmaWidth = 32 + 2 * kTmaHalo<T>;

// Encode the map of one chunk-layout array (base: its element
// (x_min-2, y_min-2, z_min-2), the pointer every kernel indexes with off3)
// with boxes of kTmaWidth<T> x box_rows x 1 (x-y planes), or kTmaWidth<T> x 1
// x box_rows (x-z slices) with rows_along_z. False if the driver refuses it.
bool encode_plane_map(CUtensorMap* map, const void* base, int elem_bytes, const Geom& g,
                      int box_rows, bool rows_along_z = false);

// The tensor maps of the arrays the viscosity/calc_dt stencil reads.
struct ViscMaps {
  CUtensorMap u, v, w, d, e;
};

// The maps of the arrays the x momentum sweep reads: mass_flux_x, density1,
// vol_flux_y and vol_flux_z (rows k0-1.., 9 and 10 rows), and the three
// time-level-1 velocities it advects (rows k0.., 8 rows).
struct MomXMaps {
  CUtensorMap mf, d, vfy, vfz, u, v, w;
};
template <class S>
bool mom_x_tma_prepare();
// The x momentum sweep of one chunk (sweep 1 or 3 of the step), its planes
// staged by bulk-tensor copies; seg planes per block along z.
template <class S>
void launch_mom_x_tma(const Geom& g, cudaStream_t s, int sweep, int seg, const MomXMaps& maps,
                      const GeomArrays& ga, typename S::vel_t* const* vel_out,
                      const Level0<S>& level0, int* status);

// The maps of the one-cell-per-thread stencils: the PdV predictor + EOS
// (node velocities 9 rows, density0, energy0, pressure, viscosity 8 rows),
// accelerate (density0, pressure, viscosity 9 rows from k0-1, node
// velocities 8 rows) and the PdV corrector + flux_calc (time level 0 and 1
// velocities, 9 rows).
struct PdvMaps {
  CUtensorMap u, v, w, d, e, p, q;
};
struct AccMaps {
  CUtensorMap d, p, q, u, v, w;
};
struct FluxMaps {
  CUtensorMap u0, v0, w0, u1, v1, w1;
};
template <class S>
bool stencils_tma_prepare();
template <class S>
void launch_pdv_predict_eos_tma(const Geom& g, cudaStream_t s, const double* dt_ptr,
                                const PdvMaps& maps, typename S::cs_t* pressure, int* status);
template <class S>
void launch_accelerate_tma(const Geom& g, cudaStream_t s, const double* dt_ptr, const AccMaps& maps,
                           typename S::vel_t* xvel1, typename S::vel_t* yvel1,
                           typename S::vel_t* zvel1, int* status);
template <class S>
void launch_pdv_flux_tma(const Geom& g, cudaStream_t s, const double* dt_ptr, const FluxMaps& maps,
                         const typename S::rho_t* density0, typename S::rho_t* density1,
                         const typename S::ene_t* energy0, typename S::ene_t* energy1,
                         const typename S::cs_t* pressure, const typename S::cs_t* viscosity,
                         typename S::vf_t* vol_flux_x, typename S::vf_t* vol_flux_y,
                         typename S::vf_t* vol_flux_z, int* status);

// The maps of the drop-in PdV (clover_pdv_kernel over the caller's arrays):
// time level 0 and (corrector) time level 1 node velocities and yarea, 9
// rows; xarea and zarea, 8 rows.
struct PdvDropMaps {
  CUtensorMap u0, v0, w0, u1, v1, w1, xa, ya, za;
};
bool pdv_dropin_tma_prepare();
// PdV_kernel.f90:72-166 (predict or correct) over the caller's arrays, planes
// staged by bulk-tensor copies; FP64, one chunk.
void launch_pdv_dropin_tma(const Geom& g, cudaStream_t s, bool predict, double dt,
                           const PdvDropMaps& maps, const double* volume, const double* density0,
                           double* density1, const double* energy0, double* energy1,
                           const double* pressure, const double* viscosity, int* status);

// The maps of the drop-in calc_dt (node velocities 9 rows; sound speed,
// viscosity, density0, volume and the face areas 8 rows), viscosity (node
// velocities 9 rows, pressure 10 rows from k0-1, face areas and density0 8
// rows) and accelerate (density0, volume, pressure, viscosity, xarea and
// zarea 9 rows from k0-1, yarea and the node velocities 8 rows).
struct DtDropMaps {
  CUtensorMap u, v, w, ss, q, d, vol, xa, ya, za;
};
struct ViscDropMaps {
  CUtensorMap u, v, w, p, xa, ya, za, d;
};
struct AccDropMaps {
  CUtensorMap d, vol, p, q, xa, za, ya, u, v, w;
};
bool stencils_dropin_tma_prepare();
void launch_calc_dt_dropin_tma(const Geom& g, cudaStream_t s, const GeomArrays& ga, double g_small,
                               double dtc_safe, double dtu_safe, double dtv_safe, double dtw_safe,
                               double dtdiv_safe, const DtDropMaps& maps, double* dt_min,
                               unsigned long long* min_key, int* status);
void launch_viscosity_dropin_tma(const Geom& g, cudaStream_t s, const GeomArrays& ga,
                                 const ViscDropMaps& maps, double* viscosity, int* status);
void launch_accelerate_dropin_tma(const Geom& g, cudaStream_t s, double dt,
                                  const AccDropMaps& maps, double* xvel1, double* yvel1,
                                  double* zvel1, int* status);

// The maps of the drop-in momentum node pass: the sweep's mass flux,
// density1 and post_vol, 9 rows (x-z slices for the y sweep).
struct NodeDropMaps {
  CUtensorMap mf, d, pv;
};
bool mom_node_dropin_tma_prepare();
void launch_mom_node_dropin_tma(const Geom& g, cudaStream_t s, int dir, const NodeDropMaps& maps,
                                double* node_flux, double* node_mass_post, double* node_mass_pre,
                                int* status);

// The maps of the x cell sweep reading one buffer of the density1/energy1
// pair: density1, energy1, vol_flux_x and vol_flux_z (8 rows), vol_flux_y
// (9 rows).
struct CellXMaps {
  CUtensorMap d, e, vfx, vfy, vfz;
};
template <class S>
bool cell_sweep_x_tma_prepare();
// The x cell sweep of the step's sweep 1 or 3, out of place into (d_out,
// e_out), planes staged by bulk-tensor copies (interior cells only).
template <class S>
void launch_cell_sweep_x_tma(const Geom& g, cudaStream_t s, int sweep, const CellXMaps& maps,
                             const GeomArrays& ga, typename S::rho_t* d_out,
                             typename S::ene_t* e_out, typename S::mf_t* mass_flux_x,
                             const Level0<S>& level0, int* status);

// The bounded wait of the staged kernels made to run out (a barrier phase
// nothing completes, cycles SM clocks at most), CLOVER_STATUS_TIMEOUT or'd
// into *status on the device, queued on stream s.
void launch_wait_selftest(cudaStream_t s, long long cycles, int* status);

// The maps of the y/z momentum node pass: mass flux of the sweep direction
// and density1 (9 rows from c0-1), and the volume fluxes its post volumes
// take (vol_flux_x 9 rows, the row-direction flux 10 rows: vol_flux_y for
// the z sweep's variant 1, vol_flux_z for the y sweep's variant 2). Rows run
// along y for the z sweep and along z for the y sweep.
struct NodeMaps {
  CUtensorMap mf, d, vfx, vfr;
};
template <class S>
bool mom_node_tma_prepare();
// The node pass of the y (dir 2) or z (dir 3) momentum sweep with post-volume
// variant var, planes staged by bulk-tensor copies.
template <class S>
void launch_mom_node_tma(const Geom& g, cudaStream_t s, int dir, int var, const NodeMaps& maps,
                         typename S::nd_t* node_flux, typename S::nd_t* node_mass_post,
                         typename S::nd_t* node_mass_pre, int* status);

// The maps of the y/z momentum velocity pass: node flux, node mass pre and
// post (the work arrays as the node pass stores them) and the three
// velocities it advects, 8 rows from c0 (along y for the z sweep, along z for
// the y sweep).
struct VelMaps {
  CUtensorMap nf, pre, post, u, v, w;
};
template <class S>
bool mom_vel_tma_prepare();
template <class S>
void launch_mom_vel_tma(const Geom& g, cudaStream_t s, int dir, const VelMaps& maps,
                        const GeomArrays& ga, const typename S::nd_t* node_flux,
                        const typename S::nd_t* node_mass_pre, typename S::vel_t* const* vel_in,
                        typename S::vel_t* const* vel_out, const Level0<S>& level0, int* status);

// The maps of the staged y/z cell sweep: density1 and energy1 of the input
// buffer, the sweep direction's volume flux (8 rows from c0), vol_flux_x (8
// rows) and the volume flux along the rows (9 rows: vol_flux_z for the y
// sweep's variant 2, vol_flux_y for the z sweep's variant 4).
struct CellMaps {
  CUtensorMap d, e, vfd, vfx, vfr;
};
template <class S>
bool cell_sweep_tma_prepare();
// The y (dir 2) or z (dir 3) cell sweep with pre-volume variant var, out of
// place from (d_in, e_in) into (d_out, e_out), planes staged by bulk-tensor
// copies. Needs a depth-2 halo update of density1/energy1 after it.
template <class S>
void launch_cell_sweep_tma(const Geom& g, cudaStream_t s, int dir, int var, const CellMaps& maps,
                           const GeomArrays& ga, const typename S::rho_t* d_in,
                           const typename S::ene_t* e_in, typename S::rho_t* d_out,
                           typename S::ene_t* e_out, const typename S::vf_t* vfx,
                           const typename S::vf_t* vfy, const typename S::vf_t* vfz,
                           typename S::mf_t* mass_flux, const Level0<S>& level0, int* status);

// The maps of a chunk's velocities (time level 0), density0 and energy0.
template <class S>
bool visc_dt_tma_maps(const Geom& g, const typename S::vel_t* xvel0, const typename S::vel_t* yvel0,
                      const typename S::vel_t* zvel0, const typename S::rho_t* density0,
                      const typename S::ene_t* energy0, ViscMaps* maps);
// Once per process before the first launch (outside any stream capture):
// the kernel's shared-memory size.
template <class S>
bool visc_dt_tma_prepare();
// viscosity + calc_dt (+ ideal_gas) of every interior cell of one chunk, the
// planes staged by bulk-tensor copies; the cell minimum folds into *min_key,
// and a block whose copies do not arrive sets CLOVER_STATUS_TIMEOUT in
// *status.
template <class S>
void launch_visc_dt_tma(const Geom& g, cudaStream_t s, const ViscMaps& maps, const GeomArrays& ga,
                        double g_small, double dtc_safe, double dtu_safe, double dtv_safe,
                        double dtw_safe, double dtdiv_safe, typename S::cs_t* pressure,
                        typename S::cs_t* viscosity, typename S::cs_t* soundspeed,
                        unsigned long long* min_key, int* status);

// Bytes of one box.
template <class T>
constexpr unsigned box_bytes(int rows) {
  return (unsigned)(rows * kTmaWidth<T> * (int)sizeof(T));
}

#ifdef __CUDACC__
__device__ __forceinline__ unsigned smem_u32(const void* p) {
  return (unsigned)__cvta_generic_to_shared(p);
}

__device__ __forceinline__ void mbar_init(unsigned long long* bar, unsigned count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count)
               : "memory");
}

// make the initialised barriers visible to the copy engine
__device__ __forceinline__ void mbar_init_fence() {
  asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}

// one arrival that also expects `bytes` of copies to complete this phase
__device__ __forceinline__ void mbar_arrive_expect_tx(unsigned long long* bar, unsigned bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)),
               "r"(bytes)
               : "memory");
}

__device__ __forceinline__ bool mbar_try_wait(unsigned long long* bar, unsigned parity) {
  unsigned done;
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
      "selp.u32 %0, 1, 0, p;\n\t}"
      : "=r"(done)
      : "r"(smem_u32(bar)), "r"(parity)
      : "memory");
  return done != 0;
}

// Cycles a block waits for a plane's copies before it gives up (about one
// second at the B200's clocks): the wait then reports failure instead of
// spinning on.
constexpr long long kTmaWaitCycles = 2000000000ll;

// Wait for the phase of the given parity; false if it did not complete
// within `limit` cycles.
__device__ __forceinline__ bool mbar_wait_bounded(unsigned long long* bar, unsigned parity,
                                                  long long limit = kTmaWaitCycles) {
  if (mbar_try_wait(bar, parity)) return true;
  const long long t0 = clock64();
  while (!mbar_try_wait(bar, parity))
    if (clock64() - t0 > limit) return false;
  return true;
}

// Box (x, y, z) of the map into shared memory (16-byte aligned), completion
// counted on bar.
__device__ __forceinline__ void tma_load_box(void* dst, const CUtensorMap* map,
                                             unsigned long long* bar, int x, int y, int z) {
  asm volatile(
      "cp.async.bulk.tensor.3d.shared::cluster.global.tile.mbarrier::complete_tx::bytes"
      " [%0], [%1, {%3, %4, %5}], [%2];" ::"r"(smem_u32(dst)),
      "l"((unsigned long long)map), "r"(smem_u32(bar)), "r"(x), "r"(y), "r"(z)
      : "memory");
}

__device__ __forceinline__ void tma_prefetch_map(const CUtensorMap* map) {
  asm volatile("prefetch.tensormap [%0];" ::"l"((unsigned long long)map) : "memory");
}
#endif

}  // namespace clover
