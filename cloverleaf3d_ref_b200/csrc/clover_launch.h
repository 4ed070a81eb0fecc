// Host-side launchers of the hydro-cycle kernels (C++, internal to the
// library). Every launcher takes device pointers in the chunk layout of
// clover_layout.cuh, a stream, and the scalar arguments of the reference
// kernel it replaces. dt is passed either by value (dt_ptr == nullptr) or as a
// device pointer, so the same kernels serve the drop-in ABI (dt from the
// caller) and the graph-captured native step (dt computed on the device).
//
// The launchers of the native step take a Target: one chunk (a Geom, which
// may carry offsets into shared allocations) or every deck of an ensemble's
// BatchPlan, in which case the same kernels run over all decks in one
// persistent launch (clover_sched.cuh, clover_batch.cu).
#pragma once

#include <cuda_runtime.h>

#include <cstring>
#include <utility>

#include "clover_layout.cuh"
#include "clover_sched.cuh"

namespace clover {

// Device-resident state of one deck of a native run (timestep.f90 and
// hydro.f90 scalars, the calc_dt reduction key, the status word and the
// deck's timestep controls). Kernels find deck d's copy kScalarStride
// doubles after deck 0's.
struct DevScalars {
  double dt, dtold, time;
  unsigned long long key;
  int step;
  int status;
  int dt_cap;
  int pad;
  double dtrise, dtmax, dtmin, pad2;
};
constexpr int kScalarStride = (int)(sizeof(DevScalars) / sizeof(double));
static_assert(sizeof(DevScalars) % sizeof(double) == 0, "deck scalars stride");

// ---- batched launches over the decks of an ensemble ----
struct BatchPlan;  // clover_batch.cu

// One deck's tile grid for a launch; aux is the segment length of a marching
// kernel or the depth of a halo update.
using GridFn = dim3 (*)(const Geom& g, int aux);

struct BatchLaunch {
  const int4* items;  // (deck, tile x, y, z), in schedule order
  const Geom* decks;
  int n;              // items
  int grid;           // blocks to launch (0: nothing to launch)
  int aux;            // segment length / depth the schedule was built for
};

// The schedule of one batched launch. key names the launch (kernel and the
// variant that fixes its grid); seg_tunable says whether aux is a segment
// length the plan may choose. Builds the schedule on first use (not while a
// stream is being captured): its upload is ordered on s and waited for.
BatchLaunch batch_launch(BatchPlan* plan, cudaStream_t s, unsigned key, GridFn grid_fn, int aux,
                         bool seg_tunable, const void* kernel, int threads);
void batch_mark(BatchPlan* plan, unsigned key, cudaStream_t s, bool begin);

struct Target {
  Geom g;
  BatchPlan* plan;
  Target(const Geom& g_) : g(g_), plan(nullptr) {}
  explicit Target(BatchPlan* p) : g(), plan(p) {}
};

// Launch kernel ks over one chunk (grid from grid_fn) or kb over the plan's
// schedule; both get the map first and then args.
template <class MB, class... P, class... A>
inline void launch_mapped(const Target& tg, cudaStream_t s, unsigned key, GridFn grid_fn, int aux,
                          bool seg_tunable, dim3 blk, void (*ks)(MapSingle, P...),
                          void (*kb)(MB, P...), A&&... args) {
  if (!tg.plan) {
    const dim3 gr = grid_fn(tg.g, aux);
    if (gr.x && gr.y && gr.z) ks<<<gr, blk, 0, s>>>(MapSingle{tg.g, aux}, std::forward<A>(args)...);
    return;
  }
  const BatchLaunch bl = batch_launch(tg.plan, s, key, grid_fn, aux, seg_tunable, (const void*)kb,
                                      (int)(blk.x * blk.y * blk.z));
  if (bl.grid <= 0) return;
  batch_mark(tg.plan, key, s, true);
  kb<<<bl.grid, blk, 0, s>>>(MB{bl.items, bl.decks, bl.n, bl.aux}, std::forward<A>(args)...);
  batch_mark(tg.plan, key, s, false);
}

// The same with another grid function for the batched launch (kernels whose
// tiles a batch lays out differently, e.g. flattened (j, k) planes).
template <class MB, class... P, class... A>
inline void launch_mapped2(const Target& tg, cudaStream_t s, unsigned key, GridFn grid_single,
                           GridFn grid_batch, int aux, bool seg_tunable, dim3 blk,
                           void (*ks)(MapSingle, P...), void (*kb)(MB, P...),
                           A&&... args) {
  if (!tg.plan) {
    launch_mapped(tg, s, key, grid_single, aux, seg_tunable, blk, ks, kb, std::forward<A>(args)...);
    return;
  }
  launch_mapped(tg, s, key, grid_batch, aux, seg_tunable, blk, ks, kb, std::forward<A>(args)...);
}

// Launch keys: kernel id in the high bits, the variant fixing the grid low.
enum : unsigned {
  kKeyIdealGas = 1u << 8, kKeyCalcDt = 2u << 8, kKeyReset = 3u << 8, kKeyHalo = 4u << 8,
  kKeyTimestepVisc = 5u << 8, kKeyPdvPredict = 6u << 8, kKeyPdvFlux = 7u << 8,
  kKeyCellSweepX = 8u << 8, kKeyCellShell = 9u << 8, kKeyCellSweep = 10u << 8,
  kKeyMomSweepX = 11u << 8, kKeyMomNode = 12u << 8, kKeyMomVel3 = 13u << 8,
  kKeyShellCopy = 14u << 8, kKeySummary = 15u << 8, kKeyAccelerate = 16u << 8,
  kKeyHaloX = 17u << 8
};

// Storage policy: FP64 everywhere (the drop-in / parity path).
struct F64 {
  using rho_t = double;  // density0, density1
  using ene_t = double;  // energy0, energy1
  using cs_t = double;   // pressure, viscosity, soundspeed
  using vel_t = double;  // xvel0..zvel1
  using vf_t = double;   // vol_flux_x/y/z
  using mf_t = double;   // mass_flux_x/y/z
  using wk_t = double;   // work arrays
  using nd_t = double;   // node flux and node masses of the y/z momentum sweeps
  using arith_t = double;  // arithmetic of the stencils the mixed path runs in FP32
};

// Storage policy of the mixed-precision native path: FP32 storage for the
// stencilled fields (energy, pressure, viscosity, sound speed, velocities)
// and the volume fluxes, FP64 kept where conservation needs it: density, the
// work arrays and all the arithmetic on volumes. The volume fluxes' differences
// form the advection's pre/post volumes and must cancel against the PdV volume
// change for mass to be conserved: the PdV corrector takes its face fluxes as
// they are stored (flux_calc's expression, rounded to FP32), so the two see
// the same values and the volumes are formed from them in FP64.
// The cell sweeps update mass and energy from their FP64 face fluxes; the
// mass flux is stored in FP32 (mf_t) for the momentum sweep, which forms its
// node fluxes and node masses from it in FP64. The y/z momentum sweeps hand
// those node values to the velocity pass, which reads them in the FP32
// arithmetic: they are stored as FP32 (nd_t), the rounding the velocity pass
// would apply. The momentum advection's flux limiter and velocity update,
// accelerate's gradients and the EOS/viscosity/dt stencils run in FP32
// (arith_t), with FP32 division and square root to within 2 ulp and FP32
// subnormals flushed (the library's single-precision build flags); all other
// arithmetic is FP64.
struct F32Mixed {
  using rho_t = double;
  using ene_t = float;
  using cs_t = float;
  using vel_t = float;
  using vf_t = float;
  using mf_t = float;
  using wk_t = double;
  using nd_t = float;
  using arith_t = float;  // momentum flux and update, accelerate (node and cell masses stay FP64)
};

// The node arrays of the y/z momentum sweeps (node flux, node masses) as nd_t
// views of work arrays of wk_t: an FP32 view of an FP64 work array starts two
// elements in, so that its column x_min sits on a 128-byte boundary like every
// other array's (the work array's x_min is 16 bytes after its base).
template <class S>
typename S::nd_t* nd_array(typename S::wk_t* w) {
  using ND = typename S::nd_t;
  return reinterpret_cast<ND*>(w) + (sizeof(ND) == 4 && sizeof(typename S::wk_t) == 8 ? 2 : 0);
}

// The time level 0 arrays, which the step's last sweep also writes: the final
// density1/energy1 of every interior cell and vel1 of every node in
// [min, max+1]^3, i.e. reset_field_kernel.f90:51-98 folded into the kernels
// that produce those values. All null in the other sweeps.
template <class S>
struct Level0 {
  typename S::rho_t* density0;
  typename S::ene_t* energy0;
  typename S::vel_t* xvel0;
  typename S::vel_t* yvel0;
  typename S::vel_t* zvel0;
};

// Geometry arrays (always FP64).
struct GeomArrays {
  const double *volume, *xarea, *yarea, *zarea;
  const double *cellx, *celly, *cellz;
  const double *celldx, *celldy, *celldz;
  const double *vertexx, *vertexy, *vertexz;
  const double *vertexdx, *vertexdy, *vertexdz;
};

// The 19 halo-exchangeable fields in reference id order (data.f90:55-74).
struct HaloFields {
  void* f[19];
};

template <class S>
void launch_ideal_gas(const Target& tg, cudaStream_t s, const typename S::rho_t* density,
                      const typename S::ene_t* energy, typename S::cs_t* pressure,
                      typename S::cs_t* soundspeed);

template <class S>
void launch_viscosity(const Geom& g, cudaStream_t s, const GeomArrays& ga,
                      const typename S::rho_t* density0, const typename S::cs_t* pressure,
                      typename S::cs_t* viscosity, const typename S::vel_t* xvel0,
                      const typename S::vel_t* yvel0, const typename S::vel_t* zvel0);

// Writes dt_min per interior cell (when dt_min_arr != nullptr) and folds the
// minimum into *min_key (an order-preserving 64-bit key of a double, see
// clover_kernels.cu); the caller initialises *min_key. Over a plan, deck d
// folds into min_key[d * kScalarStride]; dt_ptr arguments are read the same
// way (deck d's dt at dt_ptr[d * kScalarStride]).
template <class S>
void launch_calc_dt(const Target& tg, cudaStream_t s, const GeomArrays& ga, double g_small,
                    double dtc_safe, double dtu_safe, double dtv_safe, double dtw_safe,
                    double dtdiv_safe, const typename S::rho_t* density0,
                    const typename S::cs_t* viscosity, const typename S::cs_t* soundspeed,
                    const typename S::vel_t* xvel0, const typename S::vel_t* yvel0,
                    const typename S::vel_t* zvel0, typename S::wk_t* dt_min_arr,
                    unsigned long long* min_key);

// Doubles mapped to an order-preserving 64-bit key: an atomic minimum over
// keys gives exactly the serial minimum of the values (NaNs are skipped by
// the callers, as the reference's .LT. skips them).
__host__ __device__ __forceinline__ unsigned long long key_of(double v) {
#ifdef __CUDA_ARCH__
  unsigned long long b = (unsigned long long)__double_as_longlong(v);
#else
  unsigned long long b;
  memcpy(&b, &v, sizeof(b));
#endif
  return (b >> 63) ? ~b : (b | 0x8000000000000000ull);
}
unsigned long long min_key_of(double v);
double min_key_value(unsigned long long key);

template <class S>
void launch_pdv(const Geom& g, cudaStream_t s, int predict, double dt_val, const double* dt_ptr,
                const GeomArrays& ga, const typename S::rho_t* density0,
                typename S::rho_t* density1, const typename S::ene_t* energy0,
                typename S::ene_t* energy1, const typename S::cs_t* pressure,
                const typename S::cs_t* viscosity, const typename S::vel_t* xvel0,
                const typename S::vel_t* xvel1, const typename S::vel_t* yvel0,
                const typename S::vel_t* yvel1, const typename S::vel_t* zvel0,
                const typename S::vel_t* zvel1);

template <class S>
void launch_revert(const Geom& g, cudaStream_t s, const typename S::rho_t* density0,
                   typename S::rho_t* density1, const typename S::ene_t* energy0,
                   typename S::ene_t* energy1);

template <class S>
void launch_accelerate(const Target& tg, cudaStream_t s, double dt_val, const double* dt_ptr,
                       const GeomArrays& ga, const typename S::rho_t* density0,
                       const typename S::cs_t* pressure, const typename S::cs_t* viscosity,
                       const typename S::vel_t* xvel0, const typename S::vel_t* yvel0,
                       const typename S::vel_t* zvel0, typename S::vel_t* xvel1,
                       typename S::vel_t* yvel1, typename S::vel_t* zvel1,
                       bool uniform_mesh = false);  // volume and areas from Geom::vol, xa, ya, za

template <class S>
void launch_flux_calc(const Geom& g, cudaStream_t s, double dt_val, const double* dt_ptr,
                      const GeomArrays& ga, const typename S::vel_t* xvel0,
                      const typename S::vel_t* yvel0, const typename S::vel_t* zvel0,
                      const typename S::vel_t* xvel1, const typename S::vel_t* yvel1,
                      const typename S::vel_t* zvel1, typename S::vf_t* vol_flux_x,
                      typename S::vf_t* vol_flux_y, typename S::vf_t* vol_flux_z);

// work: the 7 work arrays (advec_cell_driver.f90:56-62 order).
template <class S>
void launch_advec_cell(const Geom& g, cudaStream_t s, int advect_x, int dir, int sweep,
                       const GeomArrays& ga, typename S::rho_t* density1,
                       typename S::ene_t* energy1, typename S::mf_t* mass_flux_x,
                       const typename S::vf_t* vol_flux_x, typename S::mf_t* mass_flux_y,
                       const typename S::vf_t* vol_flux_y, typename S::mf_t* mass_flux_z,
                       const typename S::vf_t* vol_flux_z, typename S::wk_t* const* work);

// advec_mom's pre/post volume form for a sweep (-1: none).
int mom_vol_variant(int advect_x, int sweep, int direction);

// work: the 7 work arrays (advec_mom_driver.f90:51-57 order). skip_volumes:
// pre_vol/post_vol already hold this sweep's values (the caller knows that
// nothing changed them or their inputs since they were formed).
// The parts of one advec_mom call: the pre/post volumes, the node pass
// (which_vel 1) and the momentum flux + velocity update; a caller that runs
// the node pass itself launches the first and the last part around it.
constexpr int kMomVolumes = 1, kMomNodePass = 2, kMomFluxUpdate = 4;
constexpr int kMomAllParts = kMomVolumes | kMomNodePass | kMomFluxUpdate;

template <class S>
void launch_advec_mom(const Geom& g, cudaStream_t s, typename S::vel_t* vel1,
                      const typename S::mf_t* mass_flux_x, const typename S::vf_t* vol_flux_x,
                      const typename S::mf_t* mass_flux_y, const typename S::vf_t* vol_flux_y,
                      const typename S::mf_t* mass_flux_z, const typename S::vf_t* vol_flux_z,
                      const GeomArrays& ga, const typename S::rho_t* density1,
                      typename S::wk_t* const* work, int advect_x, int which_vel, int sweep,
                      int direction, bool skip_volumes = false, int parts = kMomAllParts);

template <class S>
void launch_reset_field(const Target& tg, cudaStream_t s, typename S::rho_t* density0,
                        const typename S::rho_t* density1, typename S::ene_t* energy0,
                        const typename S::ene_t* energy1, typename S::vel_t* xvel0,
                        const typename S::vel_t* xvel1, typename S::vel_t* yvel0,
                        const typename S::vel_t* yvel1, typename S::vel_t* zvel0,
                        const typename S::vel_t* zvel1);

// Per-deck sums of a plan's decks: out holds 5 doubles per deck. Each deck
// sums its z planes (one block each, a fixed tree order) into
// partials[(plane_base[d] + plane) * 10 ...] (five compensated sums, then
// their five compensation terms), then one block per deck merges its planes in
// a fixed tree. plane_base: device array of the decks' first plane index.
template <class S>
void launch_field_summary_batch(BatchPlan* plan, int n_decks, cudaStream_t s,
                                const int* plane_base, const double* volume,
                                const typename S::rho_t* density0, const typename S::ene_t* energy0,
                                const typename S::cs_t* pressure, const typename S::vel_t* xvel0,
                                const typename S::vel_t* yvel0, const typename S::vel_t* zvel0,
                                double* partials, double* out);

// Sums (vol, mass, ie, ke, press) into out5 (device), deterministic order,
// each with a Neumaier compensation term through every stage (clover_sum.cuh).
// partials: device scratch of summary_partials_len() doubles.
int summary_partials_len();
template <class S>
void launch_field_summary(const Geom& g, cudaStream_t s, const double* volume,
                          const typename S::rho_t* density0, const typename S::ene_t* energy0,
                          const typename S::cs_t* pressure, const typename S::vel_t* xvel0,
                          const typename S::vel_t* yvel0, const typename S::vel_t* zvel0,
                          double* partials, double* out5);

// update_halo_kernel: fields[i] != 0 selects field id i+1; all faces external.
// Element size of every selected field comes from the policy S.
template <class S>
void launch_update_halo(const Target& tg, cudaStream_t s, const HaloFields& f, const int* fields,
                        int depth, const int* external_faces /*6: left..front*/);

// initialise_chunk_kernel + generate_chunk_kernel on the device.
struct StateTable {
  int n;
  double density[16], energy[16], xvel[16], yvel[16], zvel[16];
  double xmin[16], xmax[16], ymin[16], ymax[16], zmin[16], zmax[16], radius[16];
  int geometry[16];
};
void launch_initialise_chunk(const Geom& g, cudaStream_t s, double xmin, double ymin,
                             double zmin, double dx, double dy, double dz, double* vertexx,
                             double* vertexdx, double* vertexy, double* vertexdy,
                             double* vertexz, double* vertexdz, double* cellx, double* celldx,
                             double* celly, double* celldy, double* cellz, double* celldz,
                             double* volume, double* xarea, double* yarea, double* zarea);
template <class S>
void launch_generate_chunk(const Geom& g, cudaStream_t s, const GeomArrays& ga,
                           typename S::rho_t* density0, typename S::ene_t* energy0,
                           typename S::vel_t* xvel0, typename S::vel_t* yvel0,
                           typename S::vel_t* zvel0, const StateTable& st);

// ---- fused kernels of the native step (clover_fused.cu) ----
// viscosity and calc_dt of every interior cell in one pass; the cell minimum
// folds into min_key (per deck over a plan).
template <class S>
void launch_visc_dt(const Target& tg, cudaStream_t s, const GeomArrays& ga, double g_small,
                    double dtc_safe, double dtu_safe, double dtv_safe, double dtw_safe,
                    double dtdiv_safe, const typename S::rho_t* density0,
                    const typename S::ene_t* energy0, typename S::cs_t* pressure,
                    typename S::cs_t* viscosity, typename S::cs_t* soundspeed,
                    const typename S::vel_t* xvel0, const typename S::vel_t* yvel0,
                    const typename S::vel_t* zvel0, unsigned long long* min_key);
template <class S>
void launch_pdv_predict_eos(const Target& tg, cudaStream_t s, const double* dt_ptr,
                            const GeomArrays& ga, const typename S::rho_t* density0,
                            const typename S::ene_t* energy0, typename S::cs_t* pressure,
                            const typename S::cs_t* viscosity, const typename S::vel_t* xvel0,
                            const typename S::vel_t* yvel0, const typename S::vel_t* zvel0);
template <class S>
void launch_pdv_flux(const Target& tg, cudaStream_t s, const double* dt_ptr, const GeomArrays& ga,
                     const typename S::rho_t* density0, typename S::rho_t* density1,
                     const typename S::ene_t* energy0, typename S::ene_t* energy1,
                     const typename S::cs_t* pressure, const typename S::cs_t* viscosity,
                     const typename S::vel_t* xvel0, const typename S::vel_t* xvel1,
                     const typename S::vel_t* yvel0, const typename S::vel_t* yvel1,
                     const typename S::vel_t* zvel0, const typename S::vel_t* zvel1,
                     typename S::vf_t* vol_flux_x, typename S::vf_t* vol_flux_y,
                     typename S::vf_t* vol_flux_z);
template <class S>
void launch_advec_cell_fused(const Target& tg, cudaStream_t s, int advect_x, int dir, int sweep,
                             const GeomArrays& ga, typename S::rho_t* density1,
                             typename S::ene_t* energy1, typename S::mf_t* mass_flux_x,
                             const typename S::vf_t* vol_flux_x, typename S::mf_t* mass_flux_y,
                             const typename S::vf_t* vol_flux_y, typename S::mf_t* mass_flux_z,
                             const typename S::vf_t* vol_flux_z, typename S::wk_t* ener_flux,
                             const Level0<S>& level0);
// The x cell sweep out of place: density1/energy1 in one buffer pair, the
// updated values in the other, and with copy_shell a copy of every cell
// outside the interior (left out where a depth-2 halo update of density1 and
// energy1 follows, which rewrites all of them from the interior).
struct CellXMaps;  // clover_tma.cuh
template <class S>
void launch_advec_cell_x(const Target& tg, cudaStream_t s, int sweep, const GeomArrays& ga,
                         const typename S::rho_t* density1_in, const typename S::ene_t* energy1_in,
                         typename S::rho_t* density1_out, typename S::ene_t* energy1_out,
                         const typename S::vf_t* vol_flux_x, const typename S::vf_t* vol_flux_y,
                         const typename S::vf_t* vol_flux_z, typename S::mf_t* mass_flux_x,
                         bool copy_shell, const Level0<S>& level0,
                         const CellXMaps* maps = nullptr, int* status = nullptr);
// All three velocities of one sweep; vel_in/vel_out are the two buffers of
// each velocity pair, and with copy_shell the shell outside [min,max+1]^3 is
// copied across (left out where a depth-2 halo update of the velocities
// comes before the next read of the shell).
// vol: the uniform cell volume of the chunk (dx*dy*dz).
// x_maps (one chunk, x sweep): the tensor maps of the sweep's inputs, to run
// its shared-memory staged form (clover_tma.cu), which reports a copy that
// did not arrive in *status; null: the register-marching form.
// node_maps, vel_maps (one chunk, y/z sweep): the maps of the node pass's and
// the velocity pass's inputs, to run their staged forms.
struct MomXMaps;
struct NodeMaps;
struct VelMaps;
template <class S>
void launch_advec_mom_fused(const Target& tg, cudaStream_t s, int advect_x, int sweep, int dir,
                            double vol, const GeomArrays& ga, const typename S::rho_t* density1,
                            const typename S::mf_t* mass_flux_x, const typename S::mf_t* mass_flux_y,
                            const typename S::mf_t* mass_flux_z, const typename S::vf_t* vol_flux_x,
                            const typename S::vf_t* vol_flux_y, const typename S::vf_t* vol_flux_z,
                            typename S::wk_t* node_flux, typename S::wk_t* node_mass_post,
                            typename S::wk_t* node_mass_pre, typename S::vel_t* const* vel_in,
                            typename S::vel_t* const* vel_out, bool copy_shell,
                            const Level0<S>& level0, const MomXMaps* x_maps = nullptr,
                            int* status = nullptr, const NodeMaps* node_maps = nullptr,
                            const VelMaps* vel_maps = nullptr);

// Fill every element of an array (size elems after the pad) with a value.
template <class T>
void launch_fill(cudaStream_t s, T* base_after_pad, long long elems, T value);

}  // namespace clover
