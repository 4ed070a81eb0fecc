// Fused kernels of the native step (clover_native.cu).
//
// Every value these kernels produce is computed with the operation order of
// the reference expression it stands for, so the native step stays bit for
// bit equal to the drop-in kernels and to the oracle. What changes is the
// traffic: intermediate arrays that the reference writes and reads back
// (pre/post volumes, node fluxes and masses, momentum fluxes, the predictor
// density/energy) live in registers, dead writes are dropped, and passes that
// read the same inputs are merged.
//
//  k_visc_dt         viscosity with the compression test first (where the
//                    divergence is non-negative the viscosity is zero whatever
//                    the limiter, so its thirteen divisions are skipped), then
//                    calc_dt on the same cell and the per-deck minimum.
//  k_pdv_predict_eos PdV predictor + ideal_gas on the predicted state; only
//                    the pressure is stored (revert then restores time level
//                    0, and the corrector overwrites density1/energy1).
//  k_pdv_flux        PdV corrector + flux_calc (shared velocity loads).
//  k_cell_sweep_x    the whole x cell sweep in one pass (neighbouring cells by
//                    warp shuffles), out of place into the other buffer of the
//                    density1/energy1 pair.
//  k_cell_sweep_march  the whole y or z cell sweep in one pass, each thread
//                    marching a segment of a column with the stencil in
//                    registers (the segments of a column share a block).
//  k_mom_sweep_x     the whole x momentum sweep (three velocities) in one pass:
//                    neighbouring nodes along x through warp shuffles, the
//                    previous z plane in registers.
//  k_mom_node_march / k_mom_vel3_march  y and z momentum sweeps: node pass and
//                    velocity pass, each marching along the sweep axis with the
//                    previous node's values in registers.
//  Updated velocities go to the other buffer of each velocity pair.
#include <cfloat>
#include <type_traits>

#include "clover_launch.h"
#include "clover_stencil.cuh"
#include "clover_tma.cuh"

namespace clover {
namespace {

constexpr int BX = 32, BY = 8;
constexpr int kViscCellsZ = 2;  // cells along z per thread of k_visc_dt

struct Box {
  int j0, j1, k0, k1, l0, l1;
};

inline dim3 grid_of(const Box& b, int march = 1) {
  int nj = b.j1 - b.j0 + 1, nk = b.k1 - b.k0 + 1, nl = b.l1 - b.l0 + 1;
  if (nj <= 0 || nk <= 0 || nl <= 0) return dim3(0, 0, 0);
  return dim3((nj + BX - 1) / BX, (nk + BY - 1) / BY, (nl + march - 1) / march);
}

// The thread's (j, k) in tile t of box b: 32 x 8 tiles for one chunk; for a
// batch, tile t.x holds the 256 consecutive cells t.x*256.. of the box's
// (j, k) plane in row order (MapBatch::kFlat). False outside the box.
template <class M>
__device__ __forceinline__ bool tile_jk(const Box& b, const Tile& t, int& j, int& k) {
  if (M::kFlat) {
    const int nj = b.j1 - b.j0 + 1, nk = b.k1 - b.k0 + 1;
    const int i = t.x * (BX * BY) + (int)threadIdx.y * BX + (int)threadIdx.x;
    j = b.j0 + i % nj;
    k = b.k0 + i / nj;
    return i < nj * nk;
  }
  j = b.j0 + t.x * BX + (int)threadIdx.x;
  k = b.k0 + t.y * BY + (int)threadIdx.y;
  return j <= b.j1 && k <= b.k1;
}
inline dim3 grid_flat(const Box& b, int zdiv = 1) {
  const long long nj = b.j1 - b.j0 + 1, nk = b.k1 - b.k0 + 1, nl = b.l1 - b.l0 + 1;
  if (nj <= 0 || nk <= 0 || nl <= 0) return dim3(0, 0, 0);
  return dim3((unsigned)((nj * nk + BX * BY - 1) / (BX * BY)), 1, (unsigned)((nl + zdiv - 1) / zdiv));
}

// Index ranges of the kernels, from a chunk's geometry (device: per tile of
// a mapped kernel; host: the tile grid of a launch).
__host__ __device__ inline Box interior(const Geom& g) {
  return Box{g.x_min, g.x_max, g.y_min, g.y_max, g.z_min, g.z_max};
}
__host__ __device__ inline Box nodes(const Geom& g) {
  return Box{g.x_min, g.x_max + 1, g.y_min, g.y_max + 1, g.z_min, g.z_max + 1};
}

#define E(a, jj, kk, ll) (a)[off3(g, (jj), (kk), (ll))]
#define GX(a, jj) (a)[g.o1 + (jj) - g.x_min + 2]
#define GY(a, kk) (a)[g.o1 + (kk) - g.y_min + 2]
#define GZ(a, ll) (a)[g.o1 + (ll) - g.z_min + 2]

__device__ __forceinline__ double ld(const double* p) { return __ldg(p); }
__device__ __forceinline__ double ld(const float* p) { return (double)__ldg(p); }
#define L(a, jj, kk, ll) ld(&E(a, jj, kk, ll))
// the same with the three indices given by one macro (expanded first)
#define EI(a, idx) EI_(a, idx)
#define EI_(a, jj, kk, ll) (a)[off3(g, (jj), (kk), (ll))]
#define LI(a, idx) ld(&EI_(a, idx))

// ---------------------------------------------------------------------------
// viscosity_kernel.f90:71-134 followed by calc_dt_kernel.f90:102-149 on the
// same cell: both read the cell's 24 corner velocities, its face areas and
// density, and calc_dt reads the viscosity of its own cell only, so it needs
// no halo of the viscosity just computed. The viscosity's
// IF((limiter.GT.0.0).OR.(div.GE.0.0)) is taken as "div >= 0 -> 0, else
// limiter > 0 -> 0, else ..." (the same outcome). The cell minimum folds into
// deck d's key at min_key[d * kScalarStride] (warp, block, one atomic).
template <class S, class M>
__global__ void __launch_bounds__(BX * BY, sizeof(typename S::arith_t) == 4 || M::kFlat ? 4 : 3) k_visc_dt(M m, GeomArrays ga, double g_small,
    double dtc_safe, double dtu_safe, double dtv_safe, double dtw_safe, double dtdiv_safe,
    const typename S::rho_t* __restrict__ density0, const typename S::ene_t* __restrict__ energy0,
    typename S::cs_t* __restrict__ pressure, typename S::cs_t* __restrict__ viscosity,
    typename S::cs_t* __restrict__ soundspeed,
    const typename S::vel_t* __restrict__ xvel0, const typename S::vel_t* __restrict__ yvel0,
    const typename S::vel_t* __restrict__ zvel0, unsigned long long* __restrict__ min_key) {
  __shared__ unsigned long long wmin[BX * BY / 32];
  m.run([&](const Geom& g, const Tile& t) {
  // viscosity and dt criteria in the policy's arithmetic (FP64, or FP32 in
  // the mixed path); the minimum folds as a double key
  using A = typename S::arith_t;
#define LA(a, jj, kk, ll) lda<A>(&E(a, jj, kk, ll))
#define EGA(a, jj, kk, ll) ((A)E(a, jj, kk, ll))
#define AG(G, a, i) ((A)G(a, i))
  const A a_gs = (A)g_small, a_dtc = (A)dtc_safe, a_dtu = (A)dtu_safe, a_dtv = (A)dtv_safe;
  const A a_dtw = (A)dtw_safe, a_dtdiv = (A)dtdiv_safe;
  const Box b = interior(g);
  int j, k;
  const bool in_jk = tile_jk<M>(b, t, j, k);
  unsigned long long key = ~0ull;
  // kViscCellsZ cells along z per thread, one after another (not unrolled,
  // which keeps the FP64 form's spills small); the node values of a cell's
  // upper plane are the next cell's lower plane
  A cp[12];
  bool carried = false;
#pragma unroll 1
  for (int iz = 0; iz < kViscCellsZ; iz++) {
  const int l = b.l0 + t.z * kViscCellsZ + iz;
  if (in_jk && l <= b.l1) {
  A u000, u100, u010, u110, v000, v100, v010, v110, w000, w100, w010, w110;
  if (carried) {
    u000 = cp[0]; u100 = cp[1]; u010 = cp[2]; u110 = cp[3];
    v000 = cp[4]; v100 = cp[5]; v010 = cp[6]; v110 = cp[7];
    w000 = cp[8]; w100 = cp[9]; w010 = cp[10]; w110 = cp[11];
  } else {
    u000 = LA(xvel0, j, k, l); u100 = LA(xvel0, j + 1, k, l);
    u010 = LA(xvel0, j, k + 1, l); u110 = LA(xvel0, j + 1, k + 1, l);
    v000 = LA(yvel0, j, k, l); v100 = LA(yvel0, j + 1, k, l);
    v010 = LA(yvel0, j, k + 1, l); v110 = LA(yvel0, j + 1, k + 1, l);
    w000 = LA(zvel0, j, k, l); w100 = LA(zvel0, j + 1, k, l);
    w010 = LA(zvel0, j, k + 1, l); w110 = LA(zvel0, j + 1, k + 1, l);
  }
  const A u001 = LA(xvel0, j, k, l + 1), u101 = LA(xvel0, j + 1, k, l + 1);
  const A u011 = LA(xvel0, j, k + 1, l + 1), u111 = LA(xvel0, j + 1, k + 1, l + 1);
  const A v001 = LA(yvel0, j, k, l + 1), v101 = LA(yvel0, j + 1, k, l + 1);
  const A v011 = LA(yvel0, j, k + 1, l + 1), v111 = LA(yvel0, j + 1, k + 1, l + 1);
  const A w001 = LA(zvel0, j, k, l + 1), w101 = LA(zvel0, j + 1, k, l + 1);
  const A w011 = LA(zvel0, j, k + 1, l + 1), w111 = LA(zvel0, j + 1, k + 1, l + 1);
  cp[0] = u001; cp[1] = u101; cp[2] = u011; cp[3] = u111;
  cp[4] = v001; cp[5] = v101; cp[6] = v011; cp[7] = v111;
  cp[8] = w001; cp[9] = w101; cp[10] = w011; cp[11] = w111;
  carried = true;

  const A ugradx1 = u000 + u010 + u001 + u011;
  const A ugradx2 = u100 + u110 + u101 + u111;
  const A vgrady1 = v000 + v100 + v001 + v101;
  const A vgrady2 = v010 + v110 + v011 + v111;
  const A wgradz1 = w000 + w100 + w010 + w110;
  const A wgradz2 = w001 + w101 + w011 + w111;
  const A xa = (A)g.xa, ya = (A)g.ya, za = (A)g.za;
  const A div = (xa * (ugradx2 - ugradx1) + ya * (vgrady2 - vgrady1)) +
                     za * (wgradz2 - wgradz1);
  A q = A(A(0.0));
  if (!(div >= A(0.0))) {
    const A ugrady1 = u000 + u100 + u001 + u101;
    const A ugrady2 = u010 + u110 + u011 + u111;
    const A ugradz1 = u000 + u100 + u010 + u110;
    const A ugradz2 = u001 + u101 + u011 + u111;
    const A vgradx1 = v000 + v010 + v001 + v011;
    const A vgradx2 = v100 + v110 + v101 + v111;
    const A vgradz1 = v000 + v100 + v010 + v110;
    const A vgradz2 = v001 + v101 + v011 + v111;
    const A wgradx1 = w000 + w010 + w001 + w011;
    const A wgradx2 = w100 + w110 + w101 + w111;
    const A wgrady1 = w000 + w100 + w001 + w101;
    const A wgrady2 = w010 + w110 + w011 + w111;
    const A cdx = AG(GX, ga.celldx, j), cdy = AG(GY, ga.celldy, k), cdz = AG(GZ, ga.celldz, l);
    const A xx = A(0.25) * (ugradx2 - ugradx1) / cdx;
    const A yy = A(0.25) * (vgrady2 - vgrady1) / cdy;
    const A zz = A(0.25) * (wgradz2 - wgradz1) / cdz;
    const A xy = A(0.25) * (ugrady2 - ugrady1) / cdy + A(0.25) * (vgradx2 - vgradx1) / cdx;
    const A xz = A(0.25) * (ugradz2 - ugradz1) / cdz + A(0.25) * (wgradx2 - wgradx1) / cdx;
    const A yz = A(0.25) * (vgradz2 - vgradz1) / cdz + A(0.25) * (wgrady2 - wgrady1) / cdy;
    // the neighbours' pressures as ideal_gas stores them (density0 and
    // energy0 carry the halo the pressure's would mirror)
    using C = typename S::cs_t;
#define PN(jj, kk, ll) \
  ((A)st<C>(((A(1.4) - A(1.0)) * LA(density0, jj, kk, ll) * LA(energy0, jj, kk, ll))))
    A pgradx = (PN(j + 1, k, l) - PN(j - 1, k, l)) / (cdx + AG(GX, ga.celldx, j + 1));
    A pgrady = (PN(j, k + 1, l) - PN(j, k - 1, l)) / (cdy + AG(GY, ga.celldy, k + 1));
    A pgradz = (PN(j, k, l + 1) - PN(j, k, l - 1)) / (cdz + AG(GZ, ga.celldz, l + 1));
#undef PN
    const A pgradx2 = pgradx * pgradx;
    const A pgrady2 = pgrady * pgrady;
    const A pgradz2 = pgradz * pgradz;
    const A limiter = (xx * pgradx2 + yy * pgrady2 + zz * pgradz2 + xy * pgradx * pgrady +
                            xz * pgradx * pgradz + yz * pgrady * pgradz) /
                           fmax2(pgradx2 + pgrady2 + pgradz2, A(1.0e-16));
    if (!(limiter > A(0.0))) {
      pgradx = copysign(fmax2(A(1.0e-16), fabs(pgradx)), pgradx);
      pgrady = copysign(fmax2(A(1.0e-16), fabs(pgrady)), pgrady);
      pgradz = copysign(fmax2(A(1.0e-16), fabs(pgradz)), pgradz);
      const A pgrad = sqrt(pgradx * pgradx + pgrady * pgrady + pgradz * pgradz);
      const A xgrad = fabs(cdx * pgrad / pgradx);
      const A ygrad = fabs(cdy * pgrad / pgrady);
      const A zgrad = fabs(cdz * pgrad / pgradz);
      const A grad = fmin2(fmin2(xgrad, ygrad), zgrad);
      const A grad2 = grad * grad;
      q = A(2.0) * LA(density0, j, k, l) * grad2 * limiter * limiter;
    }
  }
  using C = typename S::cs_t;
  E(viscosity, j, k, l) = st<C>(q);
  // calc_dt_kernel.f90:102-149 (the viscosity as stored)
  const A visc = (A)st<C>(q);
  const A d0 = LA(density0, j, k, l);
  // 1/min(celldx, celldy, celldz)^2 of the chunk's uniform mesh
  const A ds = geo_ds<A>(g);
  // ideal_gas_kernel.f90:47-58 on this cell, stored as ideal_gas stores it
  A ss;
  {
    const A v_eos = A(1.0) / d0;
    const A p_eos = (A(1.4) - A(1.0)) * d0 * LA(energy0, j, k, l);
    const A pbe = (A(1.4) - A(1.0)) * d0;
    const A pbv = -d0 * p_eos;
    const A ss2 = v_eos * v_eos * (p_eos * pbe - pbv);
    E(pressure, j, k, l) = st<C>(p_eos);
    const C ss_st = st<C>(sqrt(ss2));
    E(soundspeed, j, k, l) = ss_st;
    ss = (A)ss_st;
  }
  A cc = ss * ss;
  cc = cc + A(2.0) * visc / d0;
  A dtct = ds * cc;
  dtct = a_dtc * A(1.0) / fmax2(sqrt(dtct), a_gs);
  const A vol = (A)g.vol;
  const A du1 = ugradx1 * xa, du2 = ugradx2 * xa;
  const A dtut = a_dtu * A(4.0) * vol / fmax2(fmax2(fabs(du1), fabs(du2)), A(1.0e-5) * vol);
  const A dv1 = vgrady1 * ya, dv2 = vgrady2 * ya;
  const A dtvt = a_dtv * A(4.0) * vol / fmax2(fmax2(fabs(dv1), fabs(dv2)), A(1.0e-5) * vol);
  // both z faces use zarea(j,k,l); its sums add (j,k+1) before (j+1,k)
  const A dw1 = (w000 + w010 + w100 + w110) * za;
  const A dw2 = (w001 + w011 + w101 + w111) * za;
  const A dtwt = a_dtw * A(4.0) * vol / fmax2(fmax2(fabs(dw1), fabs(dw2)), A(1.0e-5) * vol);
  const A dvg = du2 - du1 + dv2 - dv1 + dw2 - dw1;
  const A dtdivt = a_dtdiv * A(4.0) * vol / fmax2(vol * A(1.0e-05), fabs(dvg));
  const A mn = fmin2(fmin2(fmin2(fmin2(dtct, dtut), dtvt), dtwt), dtdivt);
  if (!(mn != mn)) {
    const unsigned long long kc = key_of(mn);
    key = kc < key ? kc : key;
  }
  }
  }
  // warp then block minimum, one atomic per block
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    unsigned long long other = __shfl_xor_sync(0xffffffffu, key, o);
    key = other < key ? other : key;
  }
  const int lane = threadIdx.x, warp = threadIdx.y;
  if (lane == 0) wmin[warp] = key;
  __syncthreads();
  if (warp == 0) {
    key = lane < BX * BY / 32 ? wmin[lane] : ~0ull;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
      unsigned long long other = __shfl_xor_sync(0xffffffffu, key, o);
      key = other < key ? other : key;
    }
    if (lane == 0 && key != ~0ull) atomicMin(min_key + (long long)t.d * kScalarStride, key);
  }
#undef AG
#undef EGA
#undef LA
  });
}

// ---------------------------------------------------------------------------
// PdV_kernel.f90:72-118 (predict) followed by ideal_gas_kernel.f90:47-58 on
// the predicted density1/energy1; the pressure is stored in place (each
// thread reads and writes only its own cell).
template <class S, class M>
__global__ void __launch_bounds__(BX * BY, M::kFlat ? 6 : 8) k_pdv_predict_eos(M m, const double* dt_ptr,
    GeomArrays ga, const typename S::rho_t* __restrict__ density0,
    const typename S::ene_t* __restrict__ energy0, typename S::cs_t* __restrict__ pressure,
    const typename S::cs_t* __restrict__ viscosity, const typename S::vel_t* __restrict__ xvel0,
    const typename S::vel_t* __restrict__ yvel0, const typename S::vel_t* __restrict__ zvel0) {
  m.run([&](const Geom& g, const Tile& t) {
  const Box b = interior(g);
  int j, k;
  if (!tile_jk<M>(b, t, j, k)) return;
  const int l = b.l0 + t.z;
  // predictor and EOS in the policy's arithmetic (FP64, or FP32 in the mixed
  // path: only the pressure, stored in FP32 there, comes out of it)
  using A = typename S::arith_t;
#define LA(a, jj, kk, ll) lda<A>(&E(a, jj, kk, ll))
#define EGA(a, jj, kk, ll) ((A)E(a, jj, kk, ll))
  const A dt = (A)dt_ptr[(long long)t.d * kScalarStride];
#define XS(jj) (LA(xvel0, jj, k, l) + LA(xvel0, jj, k + 1, l) + LA(xvel0, jj, k, l + 1) + LA(xvel0, jj, k + 1, l + 1))
#define YS(kk) (LA(yvel0, j, kk, l) + LA(yvel0, j + 1, kk, l) + LA(yvel0, j, kk, l + 1) + LA(yvel0, j + 1, kk, l + 1))
#define ZS(ll) (LA(zvel0, j, k, ll) + LA(zvel0, j + 1, k, ll) + LA(zvel0, j, k + 1, ll) + LA(zvel0, j + 1, k + 1, ll))
  // the predictor sums the same four node values twice (vel0 + vel0)
  A s;
  s = XS(j);
  const A left_flux = ((A)g.xa * (s + LA(xvel0, j, k, l) + LA(xvel0, j, k + 1, l) +
                            LA(xvel0, j, k, l + 1) + LA(xvel0, j, k + 1, l + 1))) * A(0.125) * dt * A(0.5);
  s = XS(j + 1);
  const A right_flux = ((A)g.xa * (s + LA(xvel0, j + 1, k, l) + LA(xvel0, j + 1, k + 1, l) +
                             LA(xvel0, j + 1, k, l + 1) + LA(xvel0, j + 1, k + 1, l + 1))) * A(0.125) * dt * A(0.5);
  s = YS(k);
  const A bottom_flux = ((A)g.ya * (s + LA(yvel0, j, k, l) + LA(yvel0, j + 1, k, l) +
                              LA(yvel0, j, k, l + 1) + LA(yvel0, j + 1, k, l + 1))) * A(0.125) * dt * A(0.5);
  s = YS(k + 1);
  const A top_flux = ((A)g.ya * (s + LA(yvel0, j, k + 1, l) + LA(yvel0, j + 1, k + 1, l) +
                           LA(yvel0, j, k + 1, l + 1) + LA(yvel0, j + 1, k + 1, l + 1))) * A(0.125) * dt * A(0.5);
  s = ZS(l);
  const A back_flux = ((A)g.za * (s + LA(zvel0, j, k, l) + LA(zvel0, j + 1, k, l) +
                            LA(zvel0, j, k + 1, l) + LA(zvel0, j + 1, k + 1, l))) * A(0.125) * dt * A(0.5);
  s = ZS(l + 1);
  const A front_flux = ((A)g.za * (s + LA(zvel0, j, k, l + 1) + LA(zvel0, j + 1, k, l + 1) +
                             LA(zvel0, j, k + 1, l + 1) + LA(zvel0, j + 1, k + 1, l + 1))) * A(0.125) * dt * A(0.5);
#undef XS
#undef YS
#undef ZS
  const A total_flux = right_flux - left_flux + top_flux - bottom_flux + front_flux - back_flux;
  const A vol = (A)g.vol;
  const A vol_change_s = div_rn(vol, vol + total_flux);
  const A recip_volume = geo_rvol<A>(g);  // 1/volume
  const A d0 = LA(density0, j, k, l);
  const A energy_change =
      quot_pair_sum(LA(pressure, j, k, l), LA(viscosity, j, k, l), d0) * total_flux * recip_volume;
  using R = typename S::rho_t;
  using En = typename S::ene_t;
  // the predicted state goes through the storage types, as it would in memory
  const A e1 = (A)st<En>((LA(energy0, j, k, l) - energy_change));
  const A d1 = (A)st<R>((d0 * vol_change_s));
  E(pressure, j, k, l) = st<typename S::cs_t>(((A(1.4) - A(1.0)) * d1 * e1));
#undef EGA
#undef LA
  });
}

// ---------------------------------------------------------------------------
// PdV_kernel.f90:120-166 (corrector) + flux_calc_kernel.f90:58-91 over the
// node box [min, max+1]^3: cells in the interior run the corrector, faces in
// the flux ranges get their volume flux.
template <class S, class M>
__global__ void __launch_bounds__(BX * BY, M::kFlat ? 5 : 8) k_pdv_flux(M m, const double* dt_ptr,
    GeomArrays ga, const typename S::rho_t* __restrict__ density0,
    typename S::rho_t* __restrict__ density1, const typename S::ene_t* __restrict__ energy0,
    typename S::ene_t* __restrict__ energy1, const typename S::cs_t* __restrict__ pressure,
    const typename S::cs_t* __restrict__ viscosity, const typename S::vel_t* __restrict__ xvel0,
    const typename S::vel_t* __restrict__ xvel1, const typename S::vel_t* __restrict__ yvel0,
    const typename S::vel_t* __restrict__ yvel1, const typename S::vel_t* __restrict__ zvel0,
    const typename S::vel_t* __restrict__ zvel1, typename S::vf_t* __restrict__ vol_flux_x,
    typename S::vf_t* __restrict__ vol_flux_y, typename S::vf_t* __restrict__ vol_flux_z) {
  m.run([&](const Geom& g, const Tile& t) {
  const Box b = nodes(g);
  int j, k;
  if (!tile_jk<M>(b, t, j, k)) return;
  const int l = b.l0 + t.z;
  const double dt = dt_ptr[(long long)t.d * kScalarStride];
  const bool jin = j <= g.x_max, kin = k <= g.y_max, lin = l <= g.z_max;
  using F = typename S::vf_t;
  // face sums of the node velocities, reference order (vel0 x4 then vel1 x4),
  // in the policy's arithmetic: FP64, or in the mixed path the FP32 sum of
  // the FP32 velocities, widened once per face (the fluxes, the corrector and
  // its volume change stay FP64, and the corrector and the volume fluxes see
  // the same face sums, as in FP64)
  using A = typename S::arith_t;
#define LA(a, jj, kk, ll) lda<A>(&E(a, jj, kk, ll))
  auto xsum = [&](int jj) {
    return (double)(LA(xvel0, jj, k, l) + LA(xvel0, jj, k + 1, l) + LA(xvel0, jj, k, l + 1) +
                    LA(xvel0, jj, k + 1, l + 1) + LA(xvel1, jj, k, l) + LA(xvel1, jj, k + 1, l) +
                    LA(xvel1, jj, k, l + 1) + LA(xvel1, jj, k + 1, l + 1));
  };
  auto ysum = [&](int kk) {
    return (double)(LA(yvel0, j, kk, l) + LA(yvel0, j + 1, kk, l) + LA(yvel0, j, kk, l + 1) +
                    LA(yvel0, j + 1, kk, l + 1) + LA(yvel1, j, kk, l) + LA(yvel1, j + 1, kk, l) +
                    LA(yvel1, j, kk, l + 1) + LA(yvel1, j + 1, kk, l + 1));
  };
  auto zsum = [&](int ll) {
    return (double)(LA(zvel0, j, k, ll) + LA(zvel0, j + 1, k, ll) + LA(zvel0, j, k + 1, ll) +
                    LA(zvel0, j + 1, k + 1, ll) + LA(zvel1, j, k, ll) + LA(zvel1, j + 1, k, ll) +
                    LA(zvel1, j, k + 1, ll) + LA(zvel1, j + 1, k + 1, ll));
  };
  double sx = 0, sy = 0, sz = 0;
  F vfx0 = F(0), vfy0 = F(0);
  if (kin && lin) {
    sx = xsum(j);
    vfx0 = st<F>(0.125 * dt * g.xa * sx);
    E(vol_flux_x, j, k, l) = vfx0;
  }
  if (jin && lin) {
    sy = ysum(k);
    vfy0 = st<F>(0.125 * dt * g.ya * sy);
    E(vol_flux_y, j, k, l) = vfy0;
  }
  if (jin && kin) {
    // flux_calc_kernel.f90:86 repeats zvel0(j+1,k,l) and omits zvel0(j,k+1,l)
    const double bz = (double)(LA(zvel0, j, k, l) + LA(zvel0, j + 1, k, l) +
                               LA(zvel0, j + 1, k, l) + LA(zvel0, j + 1, k + 1, l) +
                               LA(zvel1, j, k, l) + LA(zvel1, j + 1, k, l) +
                               LA(zvel1, j, k + 1, l) + LA(zvel1, j + 1, k + 1, l));
    E(vol_flux_z, j, k, l) = st<F>(0.125 * dt * g.za * bz);
    sz = zsum(l);
  }
  if (!(jin && kin && lin)) return;
  double left_flux, right_flux, bottom_flux, top_flux, back_flux, front_flux;
  if (sizeof(F) == 8) {  // PdV_kernel.f90:120-131 order
    left_flux = (g.xa * sx) * 0.125 * dt;
    right_flux = (g.xa * xsum(j + 1)) * 0.125 * dt;
    bottom_flux = (g.ya * sy) * 0.125 * dt;
    top_flux = (g.ya * ysum(k + 1)) * 0.125 * dt;
    back_flux = (g.za * sz) * 0.125 * dt;
    front_flux = (g.za * zsum(l + 1)) * 0.125 * dt;
  } else {
    // FP32 volume fluxes: the corrector's face fluxes as the volume fluxes are
    // stored (the same expression and rounding; the z faces from the
    // corrector's own node sums), so that the advection's pre/post volumes
    // cancel against this volume change
    auto stored = [&](double area, double s) { return (double)st<F>(0.125 * dt * area * s); };
    left_flux = (double)vfx0;
    right_flux = stored(g.xa, xsum(j + 1));
    bottom_flux = (double)vfy0;
    top_flux = stored(g.ya, ysum(k + 1));
    back_flux = stored(g.za, sz);
    front_flux = stored(g.za, zsum(l + 1));
  }
  const double total_flux = right_flux - left_flux + top_flux - bottom_flux + front_flux - back_flux;
  const double vol = g.vol;
  const double vol_change_s = vol / (vol + total_flux);
  const double d0 = L(density0, j, k, l);
  // the energy change in the policy's arithmetic (an FP32 stencil in the
  // mixed path); the density, which carries the mass, stays FP64
  const A ad0 = (A)d0;
  const A energy_change = (LA(pressure, j, k, l) / ad0 + LA(viscosity, j, k, l) / ad0) *
                          (A)total_flux * geo_rvol<A>(g);
  E(energy1, j, k, l) = st<typename S::ene_t>((LA(energy0, j, k, l) - energy_change));
  E(density1, j, k, l) = st<typename S::rho_t>(d0 * vol_change_s);
#undef LA
  });
}

// ---------------------------------------------------------------------------
// advec_cell pre_vol (advec_cell_kernel.f90:97-121, :190-216, :287-311),
// the variants of launch_advec_cell in clover_kernels.cu.
template <class S>
__device__ __forceinline__ double cell_pre_vol(const Geom& g, int variant, const GeomArrays& ga,
    const typename S::vf_t* vfx, const typename S::vf_t* vfy, const typename S::vf_t* vfz,
    int j, int k, int l) {
  const double vol = g.vol;
  switch (variant) {
    case 0:
    case 4: {
      const double fx1 = L(vfx, j + 1, k, l), fx0 = L(vfx, j, k, l);
      const double fy1 = L(vfy, j, k + 1, l), fy0 = L(vfy, j, k, l);
      const double fz1 = L(vfz, j, k, l + 1), fz0 = L(vfz, j, k, l);
      return vol + (fx1 - fx0 + fy1 - fy0 + fz1 - fz0);
    }
    case 1:
      return vol + L(vfx, j + 1, k, l) - L(vfx, j, k, l);
    case 2:
      return vol + L(vfy, j, k + 1, l) - L(vfy, j, k, l) + L(vfz, j, k, l + 1) - L(vfz, j, k, l);
    case 3:
      return vol + L(vfy, j, k + 1, l) - L(vfy, j, k, l) + L(vfx, j + 1, k, l) - L(vfx, j, k, l);
    default:
      return vol + L(vfz, j, k, l + 1) - L(vfz, j, k, l);
  }
}

// advec_cell x sweep as ONE pass (advec_cell_kernel.f90:125-185), out of
// place. Lane L of a warp holds cell c = x_min-2+28t+L of a row: its old
// density, energy, pre-volume, volume flux and vertexdx are loaded once, the
// neighbours c-2..c+1 come from the lanes around it, lanes 2..30 form the
// face c fluxes and lanes 2..29 own cell c (28 per warp): they store the
// fluxes of face c and update cell c from faces c and c+1 into the output
// arrays, so no thread reads a value another one writes.
template <class S, int VAR, class M>
__global__ void __launch_bounds__(BX * BY, M::kFlat ? 4 : (sizeof(typename S::arith_t) == 4 ? 6 : 5)) k_cell_sweep_x(M m, GeomArrays ga,
    const typename S::rho_t* __restrict__ d_in, const typename S::ene_t* __restrict__ e_in,
    typename S::rho_t* __restrict__ d_out, typename S::ene_t* __restrict__ e_out,
    const typename S::vf_t* __restrict__ vfx, const typename S::vf_t* __restrict__ vfy,
    const typename S::vf_t* __restrict__ vfz, typename S::mf_t* __restrict__ mass_flux,
    Level0<S> lz) {
  m.run([&](const Geom& g, const Tile& t) {
  const int lane = threadIdx.x;
  const int c = g.x_min - 2 + t.x * 28 + lane;
  const int k = g.y_min + t.y * BY + threadIdx.y;
  const int l = g.z_min + t.z;
  const bool row = k <= g.y_max;  // every lane of a row stays for the shuffles
  const bool lds = row && c <= g.x_max + 2;
  const int top = g.x_max + 2;
  const unsigned full = 0xffffffffu;
  double d = 0.0, e = 0.0, pv = 0.0, vf = 0.0, vd = 1.0;
  if (lds) {
    d = L(d_in, c, k, l);
    e = L(e_in, c, k, l);
    pv = cell_pre_vol<S>(g, VAR, ga, vfx, vfy, vfz, c, k, l);
    vf = L(vfx, c, k, l);
    vd = GX(ga.vertexdx, c);
  }
  const double d_m2 = __shfl_up_sync(full, d, 2), d_m1 = __shfl_up_sync(full, d, 1);
  const double d_p1 = __shfl_down_sync(full, d, 1);
  const double e_m2 = __shfl_up_sync(full, e, 2), e_m1 = __shfl_up_sync(full, e, 1);
  const double e_p1 = __shfl_down_sync(full, e, 1);
  const double pv_m1 = __shfl_up_sync(full, pv, 1);
  const double vd_m1 = __shfl_up_sync(full, vd, 1), vd_p1 = __shfl_down_sync(full, vd, 1);
  const bool face = lds && lane >= 2 && lane <= 30 && c >= g.x_min;
  using MF = typename S::mf_t;
  double mf_st = 0.0, ef = 0.0;
  if (face) {
    // advec_cell_kernel.f90:131-169 at face c; the upwind index clamps to x_max+2
    double d_up, d_don, d_dn, e_up, e_don, e_dn, pv_don, vd_dif;
    if (vf > 0.0) {  // upwind c-2, donor c-1, downwind c
      d_up = d_m2; d_don = d_m1; d_dn = d; e_up = e_m2; e_don = e_m1; e_dn = e;
      pv_don = pv_m1; vd_dif = vd_m1;
    } else {  // upwind min(c+1, x_max+2), donor c, downwind c-1
      const bool clamp = c + 1 > top;
      d_up = clamp ? d : d_p1; d_don = d; d_dn = d_m1;
      e_up = clamp ? e : e_p1; e_don = e; e_dn = e_m1;
      pv_don = pv; vd_dif = clamp ? vd : vd_p1;
    }
    using AL = typename S::arith_t;  // the limiters' arithmetic
    const AL sigmat = div_rn((AL)fabs(vf), (AL)pv_don);
    const AL sigma3 = (AL(1.0) + sigmat) * (AL)width_ratio(vd, vd_dif);
    const AL sigma4 = AL(2.0) - sigmat;
    AL diffuw = (AL)(d_don - d_up);
    AL diffdw = (AL)(d_dn - d_don);
    AL limiter = cell_limiter<AL>(sigmat, sigma3, sigma4, diffuw, diffdw);
    const double mflux = vf * (d_don + (double)limiter);
    // the cell update takes the FP64 face fluxes; the stored mass flux
    // (mf_t) feeds only the momentum sweep
    mf_st = mflux;
    if (lane <= 29) E(mass_flux, c, k, l) = st<MF>(mflux);
    const AL sigmam = div_rn((AL)fabs(mflux), (AL)d_don * (AL)pv_don);
    diffuw = (AL)(e_don - e_up);
    diffdw = (AL)(e_dn - e_don);
    limiter = cell_limiter<AL>(sigmam, sigma3, sigma4, diffuw, diffdw);
    ef = mflux * (e_don + (double)limiter);
  }
  // advec_cell_kernel.f90:173-185 for cell c from faces c and c+1
  const double mf_p = __shfl_down_sync(full, mf_st, 1);
  const double ef_p = __shfl_down_sync(full, ef, 1);
  const double vf_p = __shfl_down_sync(full, vf, 1);
  if (face && lane <= 29 && c <= g.x_max) {
    const double pm = d * pv;
    const double pom = pm + mf_st - mf_p;
    const double poe = (e * pm + ef - ef_p) / pom;
    const double av = pv + vf - vf_p;
    const typename S::rho_t dn = st<typename S::rho_t>(pom / av);
    const typename S::ene_t en = st<typename S::ene_t>(poe);
    E(d_out, c, k, l) = dn;
    E(e_out, c, k, l) = en;
    if (lz.density0) {  // last sweep of the step: reset_field
      E(lz.density0, c, k, l) = dn;
      E(lz.energy0, c, k, l) = en;
    }
  }
  });
}

// Copy the cells of two cell arrays outside the interior (the halo shell
// [min-2, max+2]^3 minus [min, max]^3) from one buffer to the other.
template <class R, class En, class M>
__global__ void k_cell_shell_copy(M m, const R* __restrict__ a_in, const En* __restrict__ b_in,
                                  R* __restrict__ a_out, En* __restrict__ b_out) {
  m.run([&](const Geom& g, const Tile& t) {
  int j, k;
  if (!tile_jk<M>(Box{g.x_min - 2, g.x_max + 2, g.y_min - 2, g.y_max + 2, 0, 0}, t, j, k)) return;
  const int l = g.z_min - 2 + t.z;
  const bool inside = j >= g.x_min && j <= g.x_max && k >= g.y_min && k <= g.y_max &&
                      l >= g.z_min && l <= g.z_max;
  if (inside) return;
  const long long o = off3(g, j, k, l);
  a_out[o] = a_in[o];
  b_out[o] = b_in[o];
  });
}

// ---------------------------------------------------------------------------
// advec_mom post_vol (advec_mom_kernel.f90:95-163); pre_vol is not needed by
// the node masses, only post_vol.
template <class S>
__device__ __forceinline__ double mom_post_vol(const Geom& g, int variant, const GeomArrays& ga,
    const typename S::vf_t* vfx, const typename S::vf_t* vfy, const typename S::vf_t* vfz,
    int j, int k, int l) {
  const double vol = g.vol;
  switch (variant) {
    case 0:
      return vol + L(vfy, j, k + 1, l) - L(vfy, j, k, l) + L(vfz, j, k, l + 1) - L(vfz, j, k, l);
    case 1:
      return vol + L(vfx, j + 1, k, l) - L(vfx, j, k, l) + L(vfy, j, k + 1, l) - L(vfy, j, k, l);
    case 2:
      return vol + L(vfz, j, k, l + 1) - L(vfz, j, k, l);
    case 3:
      return vol + L(vfx, j + 1, k, l) - L(vfx, j, k, l);
    default:
      return vol;
  }
}

// The reference's node-flux sum for direction DIR at node (j,k,l).
template <class S, int DIR>
__device__ __forceinline__ double node_flux_at(const Geom& g, const typename S::mf_t* mf, int j,
                                               int k, int l) {
  if (DIR == 1)
    return 0.125 * (L(mf, j, k - 1, l) + L(mf, j, k, l) + L(mf, j + 1, k - 1, l) + L(mf, j + 1, k, l) +
                    L(mf, j, k - 1, l - 1) + L(mf, j, k, l - 1) + L(mf, j + 1, k - 1, l - 1) +
                    L(mf, j + 1, k, l - 1));
  if (DIR == 2)
    return 0.125 * (L(mf, j - 1, k, l) + L(mf, j, k, l) + L(mf, j - 1, k + 1, l) + L(mf, j, k + 1, l) +
                    L(mf, j - 1, k, l - 1) + L(mf, j, k, l - 1) + L(mf, j - 1, k + 1, l - 1) +
                    L(mf, j, k + 1, l - 1));
  return 0.125 * (L(mf, j - 1, k, l) + L(mf, j, k, l) + L(mf, j - 1, k, l + 1) + L(mf, j, k, l + 1) +
                  L(mf, j - 1, k - 1, l) + L(mf, j, k - 1, l) + L(mf, j - 1, k - 1, l + 1) +
                  L(mf, j, k - 1, l + 1));
}

template <class S>
__device__ __forceinline__ double cell_product(const Geom& g, int variant, const GeomArrays& ga,
    const typename S::rho_t* density1, const typename S::vf_t* vfx, const typename S::vf_t* vfy,
    const typename S::vf_t* vfz, int j, int k, int l) {
  return L(density1, j, k, l) * mom_post_vol<S>(g, variant, ga, vfx, vfy, vfz, j, k, l);
}

// Node pass for direction y or z, marching along the sweep axis p: thread
// (j, c) walks a segment of p carrying the mass fluxes of plane p and the cell
// products of the plane below. Lane L of a warp holds column j = jlo-1+31t+L:
// the values at column j-1 (mass fluxes and cell products) come from lane
// L-1, so lane 0 only serves lane 1 and lanes 1..31 store nodes.
// DIR 2: p = k, c = l; DIR 3: p = l, c = k. Sums keep the reference order
// (advec_mom_kernel.f90:166-190 and the y/z forms).
template <class S, int DIR, int VAR, class M>
__global__ void __launch_bounds__(BX * BY, M::kFlat || sizeof(typename S::arith_t) == 4 ? 5 : 6) k_mom_node_march(M m, GeomArrays ga,
    const typename S::mf_t* __restrict__ mf, const typename S::rho_t* __restrict__ density1,
    const typename S::vf_t* __restrict__ vfx, const typename S::vf_t* __restrict__ vfy,
    const typename S::vf_t* __restrict__ vfz, typename S::nd_t* __restrict__ node_flux,
    typename S::nd_t* __restrict__ node_mass_post, typename S::nd_t* __restrict__ node_mass_pre) {
  m.run([&](const Geom& g, const Tile& t) {
  const MarchRange r = mom_node_range<DIR>(g);
  const int plo = r.plo, phi = r.phi;
  const int seg = m.seg;
  const int lane = threadIdx.x;
  const int j = r.jlo - 1 + t.x * 31 + lane;
  const int c = r.clo + t.y * BY + threadIdx.y;
  if (c > r.chi) return;  // the whole warp: c depends on the row only
  const bool lds = j <= r.jhi;            // lanes that load (lane 0 holds column j-1 of lane 1)
  const bool own = lds && lane >= 1;      // lanes that store
  const int p0 = plo + t.z * seg;
  int p1 = p0 + seg - 1;
  if (p1 > phi) p1 = phi;
  const unsigned full = 0xffffffffu;
  using W = typename S::nd_t;
  // (j,k,l) of the node at march index p, and the same with c-1
#define IDX(p) j, (DIR == 2 ? (p) : c), (DIR == 2 ? c : (p))
#define IDXM(p) j, (DIR == 2 ? (p) : c - 1), (DIR == 2 ? c - 1 : (p))
  auto P = [&](int jj, int kk, int ll) {
    return cell_product<S>(g, VAR, ga, density1, vfx, vfy, vfz, jj, kk, ll);
  };
  auto up = [&](double v) { return __shfl_up_sync(full, v, 1); };
  // mass fluxes of plane p at (j, c) and (j, c-1); the node flux of node p
  // adds, in the reference order, (j-1,c,p) (j,c,p) (j-1,c,p+1) (j,c,p+1)
  // (j-1,c-1,p) (j,c-1,p) (j-1,c-1,p+1) (j,c-1,p+1)
  double a0 = 0.0, b0 = 0.0;
  if (lds) { a0 = LI(mf, IDX(p0)); b0 = LI(mf, IDXM(p0)); }
  double a0m = up(a0), b0m = up(b0);
  // node flux of the node before the segment and the plane of products below
  // the first node (cells at march index p0-1); the first segment starts at
  // the first node-flux index, whose node mass is not computed
  double nf_prev = 0.0;
  double q_a = 0.0, q_b = 0.0, q_c = 0.0, q_d = 0.0;  // lower-plane products
  if (p0 - 1 >= plo) {
    double am = 0.0, bm = 0.0;
    if (lds) { am = LI(mf, IDX(p0 - 1)); bm = LI(mf, IDXM(p0 - 1)); }
    const double amm = up(am), bmm = up(bm);
    nf_prev = 0.125 * (amm + am + a0m + a0 + bmm + bm + b0m + b0);
    const int p = p0;
    double x0 = 0.0, x1 = 0.0;
    if (DIR == 3) {  // lower plane l-1: P(j,k-1,l-1), P(j,k,l-1), P(j-1,k-1,l-1), P(j-1,k,l-1)
      if (lds) { x0 = P(j, c - 1, p - 1); x1 = P(j, c, p - 1); }
      q_a = x0; q_b = x1; q_c = up(x0); q_d = up(x1);
    } else {  // lower plane k-1: P(j,k-1,l), P(j-1,k-1,l), P(j,k-1,l-1), P(j-1,k-1,l-1)
      if (lds) { x0 = P(j, p - 1, c); x1 = P(j, p - 1, c - 1); }
      q_a = x0; q_b = up(x0); q_c = x1; q_d = up(x1);
    }
  }
  for (int p = p0; p <= p1; p++) {
    double a1 = 0.0, b1 = 0.0;
    if (lds) { a1 = LI(mf, IDX(p + 1)); b1 = LI(mf, IDXM(p + 1)); }
    const double a1m = up(a1), b1m = up(b1);
    const double nf = 0.125 * (a0m + a0 + a1m + a1 + b0m + b0 + b1m + b1);
    if (own) EI(node_flux, IDX(p)) = st<W>(nf);
    double u_a, u_b, u_c, u_d;  // upper-plane products
    double nmp;
    double x0 = 0.0, x1 = 0.0;
    if (DIR == 3) {  // upper plane l: P(j,k-1,l), P(j,k,l), P(j-1,k-1,l), P(j-1,k,l)
      if (lds) { x0 = P(j, c - 1, p); x1 = P(j, c, p); }
      u_a = x0; u_b = x1; u_c = up(x0); u_d = up(x1);
      nmp = node_mass_sum(u_a, u_b, u_c, u_d, q_a, q_b, q_c, q_d);
    } else {  // upper plane k: P(j,k,l), P(j-1,k,l), P(j,k,l-1), P(j-1,k,l-1)
      if (lds) { x0 = P(j, p, c); x1 = P(j, p, c - 1); }
      u_a = x0; u_b = up(x0); u_c = x1; u_d = up(x1);
      // order: P(j,k-1,l) P(j,k,l) P(j-1,k-1,l) P(j-1,k,l) P(j,k-1,l-1) P(j,k,l-1) P(j-1,k-1,l-1) P(j-1,k,l-1)
      nmp = node_mass_sum(q_a, u_a, q_b, u_b, q_c, u_c, q_d, u_d);
    }
    if (own && p >= plo + 1) {  // node masses run from one node after the flux range start
      EI(node_mass_post, IDX(p)) = st<W>(nmp);
      EI(node_mass_pre, IDX(p)) = st<W>(nmp - nf_prev + nf);
    }
    nf_prev = nf;
    q_a = u_a; q_b = u_b; q_c = u_c; q_d = u_d;
    a0 = a1; b0 = b1; a0m = a1m; b0m = b1m;
  }
#undef IDXM
#undef IDX
  });
}

// Velocity pass for direction y or z, marching along the sweep axis with the
// previous momentum fluxes and the velocity window in registers.
template <class S, int DIR, class M>
__global__ void __launch_bounds__(BX * BY, sizeof(typename S::arith_t) == 4 && !M::kFlat ? 5 : 3) k_mom_vel3_march(M m, GeomArrays ga,
    const typename S::nd_t* __restrict__ node_flux, const typename S::nd_t* __restrict__ node_mass_post,
    const typename S::nd_t* __restrict__ node_mass_pre, const typename S::vel_t* __restrict__ u_in,
    const typename S::vel_t* __restrict__ v_in, const typename S::vel_t* __restrict__ w_in,
    typename S::vel_t* __restrict__ u_out, typename S::vel_t* __restrict__ v_out,
    typename S::vel_t* __restrict__ w_out, Level0<S> lz) {
  m.run([&](const Geom& g, const Tile& t) {
  const MarchRange r = mom_vel_range<DIR>(g);
  const int jlo = r.jlo, jhi = r.jhi, clo = r.clo, chi = r.chi, plo = r.plo, phi = r.phi;
  const int seg = m.seg;
  int j, c;
  if (!tile_jk<M>(Box{jlo, jhi, clo, chi, 0, 0}, t, j, c)) return;
  const int p0 = plo + t.z * seg;
  int p1 = p0 + seg - 1;
  if (p1 > phi) p1 = phi;
#define IDX(p) j, (DIR == 2 ? (p) : c), (DIR == 2 ? c : (p))
  const double* cd = DIR == 2 ? ga.celldy : ga.celldz;
  const int cdlo = DIR == 2 ? g.y_min : g.z_min;
#define CD(p) cd[g.o1 + (p) - cdlo + 2]
  using V = typename S::vel_t;
  using A = typename S::arith_t;  // arithmetic of the flux and update
#define LA(a, idx) lda<A>(&EI_(a, idx))
  const typename S::vel_t* in[3] = {u_in, v_in, w_in};
  typename S::vel_t* out[3] = {u_out, v_out, w_out};
  typename S::vel_t* lev0[3] = {lz.xvel0, lz.yvel0, lz.zvel0};
  // window at node p: v(p-2), v(p-1), v(p), v(p+1) ; loaded v(p+2) each step
  A vw[3][4];
  A mf_prev[3];
  A nf_m = LA(node_flux, IDX(p0 - 1));
  A pre_m = LA(node_mass_pre, IDX(p0 - 1));
  A pre_0 = LA(node_mass_pre, IDX(p0));
  {
    // mom_flux(p0-1)
    const MomNodeTerms<A> nt =
        mom_node_terms<A>(nf_m, pre_m, pre_0, (A)CD(p0 - 1), (A)CD(p0 - 2), (A)CD(p0));
#pragma unroll
    for (int q = 0; q < 3; q++) {
      vw[q][0] = LA(in[q], IDX(p0 - 2));
      vw[q][1] = LA(in[q], IDX(p0 - 1));
      vw[q][2] = LA(in[q], IDX(p0));
      vw[q][3] = LA(in[q], IDX(p0 + 1));
      mf_prev[q] = mom_flux_v<A>(nt, vw[q][0], vw[q][1], vw[q][2], vw[q][3]);
    }
  }
  for (int p = p0; p <= p1; p++) {
    const A nf_0 = LA(node_flux, IDX(p));
    const A pre_p = LA(node_mass_pre, IDX(p + 1));
    const A post_0 = LA(node_mass_post, IDX(p));
    A vn[3];
#pragma unroll
    for (int q = 0; q < 3; q++) vn[q] = LA(in[q], IDX(p + 2));
    const MomNodeTerms<A> nt =
        mom_node_terms<A>(nf_0, pre_0, pre_p, (A)CD(p), (A)CD(p - 1), (A)CD(p + 1));
#pragma unroll
    for (int q = 0; q < 3; q++) {
      const A vp2 = vn[q];
      const A mf_0 = mom_flux_v<A>(nt, vw[q][1], vw[q][2], vw[q][3], vp2);
      vn[q] = vw[q][2] * pre_0 + mf_prev[q] - mf_0;
      mf_prev[q] = mf_0;
      vw[q][0] = vw[q][1];
      vw[q][1] = vw[q][2];
      vw[q][2] = vw[q][3];
      vw[q][3] = vp2;
    }
    div3_rn(vn, post_0);  // the three updates share node_mass_post
#pragma unroll
    for (int q = 0; q < 3; q++) {
      const V vn1 = st<V>(vn[q]);
      EI(out[q], IDX(p)) = vn1;
      if (lz.xvel0) EI(lev0[q], IDX(p)) = vn1;  // last sweep of the step: reset_field
    }
    pre_0 = pre_p;
  }
#undef LA
#undef CD
#undef IDX
  });
}

// ---------------------------------------------------------------------------
// advec_cell sweep along y or z as ONE pass. A block holds 32 columns j of
// one cross-axis index c and splits the sweep axis p (k for DIR 2, l for
// DIR 3) into BY segments, one per threadIdx.y. Each thread walks its segment
// [c0, c1] face by face, holding the old density/energy of cells p-2..p+1
// and the pre-volumes of cells p-1, p in registers, so the donor/upwind
// selection needs no dependent loads, and updates cell p-1 in place as soon
// as face p is known. The faces at a segment's ends read two old cells of
// each neighbouring segment, which those segments overwrite: every thread
// reads them (c0-2, c0-1, c1+1, c1+2) before the block's barrier, and only
// then does any thread write. Faces p in [pmin, pmax+2] (c up to chi), cells p
// in [pmin, pmax] (c <= cmax); face c1+1 is computed by both neighbours and
// stored by the segment that starts there.
template <class S, int DIR, int VAR, class M>
__global__ void __launch_bounds__(BX * BY, sizeof(typename S::arith_t) == 4 && M::kFlat ? 4 : 3) k_cell_sweep_march(M m, GeomArrays ga,
    typename S::rho_t* __restrict__ density1, typename S::ene_t* __restrict__ energy1,
    const typename S::vf_t* __restrict__ vfx, const typename S::vf_t* __restrict__ vfy,
    const typename S::vf_t* __restrict__ vfz, typename S::mf_t* __restrict__ mass_flux,
    Level0<S> lz) {
  // old density/energy of cells c1+1, c1+2 of each thread's segment
  __shared__ double s_end[4][BY][BX];
  m.run([&](const Geom& g, const Tile& t) {
  const MarchRange r = cell_sweep_range<DIR>(g);
  // one chunk: 32 columns j of one cross index c per block; a batch: 32
  // consecutive columns of the deck's (j, c) plane in row order
  int j, c;
  bool col;
  if (M::kFlat) {
    const int nj = r.jhi - r.jlo + 1, nc = r.chi - r.clo + 1;
    const int i = t.x * BX + (int)threadIdx.x;
    j = r.jlo + i % nj;
    c = r.clo + i / nj;
    col = i < nj * nc;
  } else {
    j = r.jlo + t.x * BX + (int)threadIdx.x;
    c = r.clo + t.y;
    col = j <= r.jhi && c <= r.chi;
  }
  const int pmin = DIR == 2 ? g.y_min : g.z_min;
  const int pmax = DIR == 2 ? g.y_max : g.z_max;
  const int len = (pmax - pmin + 1 + BY - 1) / BY;  // cells per segment
  const int c0 = pmin + (int)threadIdx.y * len;
  const int c1 = c0 + len - 1 < pmax ? c0 + len - 1 : pmax;
  const bool active = col && c0 <= pmax;
  const bool last = c1 == pmax;  // this segment also walks the faces pmax+1, pmax+2
#define IDX(p) j, (DIR == 2 ? (p) : c), (DIR == 2 ? c : (p))
  const int top = pmax + 2;
  // old values at the segment's ends (cells of the neighbouring segments)
  double d0 = 0.0, d1 = 0.0, e0 = 0.0, e1 = 0.0;
  const int ty = threadIdx.y, tx = threadIdx.x;
  if (active) {
    d0 = LI(density1, IDX(c0 - 2)); d1 = LI(density1, IDX(c0 - 1));
    e0 = LI(energy1, IDX(c0 - 2)); e1 = LI(energy1, IDX(c0 - 1));
    const int q1 = c1 + 1 < top ? c1 + 1 : top, q2 = c1 + 2 < top ? c1 + 2 : top;
    s_end[0][ty][tx] = LI(density1, IDX(q1));
    s_end[1][ty][tx] = LI(density1, IDX(q2));
    s_end[2][ty][tx] = LI(energy1, IDX(q1));
    s_end[3][ty][tx] = LI(energy1, IDX(q2));
  }
  __syncthreads();
  if (!active) return;
  const typename S::vf_t* vf_d = DIR == 2 ? vfy : vfz;
  const double* vd = DIR == 2 ? ga.vertexdy : ga.vertexdz;
#define VD(p) vd[g.o1 + (p) - pmin + 2]
  const bool update = c <= r.cmax;
  using R = typename S::rho_t;
  using En = typename S::ene_t;
  using MF = typename S::mf_t;
  auto prevol = [&](int p) {
    return cell_pre_vol<S>(g, VAR, ga, vfx, vfy, vfz, IDX(p));
  };
  // window: d0..d3 = density1(p-2..p+1), e0..e3 = energy1(p-2..p+1), old values
  double d2 = LI(density1, IDX(c0)), d3;
  double e2 = LI(energy1, IDX(c0)), e3;
  double pv_m = prevol(c0 - 1), pv_0;  // pre_vol(p-1), pre_vol(p)
  double vf_prev = 0.0, mf_prev = 0.0, ef_prev = 0.0;
  const int pend = last ? top : c1 + 1;
  for (int p = c0; p <= pend; p++) {
    // cell p+1 is read by face p (the upwind index clamps to pmax+2 at the top);
    // beyond c1 it comes from the values read before the barrier
    const int pn = p + 1 <= top ? p + 1 : top;
    if (pn <= c1) {
      d3 = LI(density1, IDX(pn));
      e3 = LI(energy1, IDX(pn));
    } else {
      const int w = pn == c1 + 1 ? 0 : 1;
      d3 = s_end[w][ty][tx];
      e3 = s_end[2 + w][ty][tx];
    }
    pv_0 = prevol(p);
    const double vf = LI(vf_d, IDX(p));
    // advec_cell_kernel.f90:226-264 (y) / :321-359 (z) at face p
    double d_up, d_don, d_dn, e_up, e_don, e_dn, pv_don;
    int dif;
    if (vf > 0.0) {  // upwind p-2, donor p-1, downwind p
      d_up = d0; d_don = d1; d_dn = d2; e_up = e0; e_don = e1; e_dn = e2; pv_don = pv_m;
      dif = p - 1;
    } else {  // upwind min(p+1, pmax+2), donor p, downwind p-1
      d_up = d3; d_don = d2; d_dn = d1; e_up = e3; e_don = e2; e_dn = e1; pv_don = pv_0;
      dif = p + 1 < top ? p + 1 : top;
    }
    using AL = typename S::arith_t;  // the limiters' arithmetic
    const AL sigmat = div_rn((AL)fabs(vf), (AL)pv_don);
    const AL sigma3 = (AL(1.0) + sigmat) * (AL)width_ratio(VD(p), VD(dif));
    const AL sigma4 = AL(2.0) - sigmat;
    AL diffuw = (AL)(d_don - d_up);
    AL diffdw = (AL)(d_dn - d_don);
    AL limiter = cell_limiter<AL>(sigmat, sigma3, sigma4, diffuw, diffdw);
    const double mflux = vf * (d_don + (double)limiter);
    if (p <= c1 || last) EI(mass_flux, IDX(p)) = st<MF>(mflux);
    const double mf_stored = mflux;  // FP64 in the cell update; mf_t storage feeds the momentum sweep
    const AL sigmam = div_rn((AL)fabs(mflux), (AL)d_don * (AL)pv_don);
    diffuw = (AL)(e_don - e_up);
    diffdw = (AL)(e_dn - e_don);
    limiter = cell_limiter<AL>(sigmam, sigma3, sigma4, diffuw, diffdw);
    const double eflux = mflux * (e_don + (double)limiter);
    // advec_cell_kernel.f90:270-281 (y) / :365-376 (z) for cell p-1
    if (update && p - 1 >= c0 && p - 1 <= c1) {
      const double pm = d1 * pv_m;
      const double pom = pm + mf_prev - mf_stored;
      const double poe = (e1 * pm + ef_prev - eflux) / pom;
      const double av = pv_m + vf_prev - vf;
      const R dn = st<R>(pom / av);
      const En en = st<En>(poe);
      EI(density1, IDX(p - 1)) = dn;
      EI(energy1, IDX(p - 1)) = en;
      if (lz.density0) {  // last sweep of the step: reset_field
        EI(lz.density0, IDX(p - 1)) = dn;
        EI(lz.energy0, IDX(p - 1)) = en;
      }
    }
    vf_prev = vf;
    mf_prev = mf_stored;
    ef_prev = eflux;
    d0 = d1; d1 = d2; d2 = d3;
    e0 = e1; e1 = e2; e2 = e3;
    pv_m = pv_0;
  }
#undef VD
#undef IDX
  });
}

// ---------------------------------------------------------------------------
// advec_mom x sweep as ONE pass for the three velocities. Lane L of a warp
// holds node j = j0 - 2 + L of row k and walks l over a segment; node_flux(j)
// and the cell masses density1*post_vol of column j come from loads, the
// values of column j-1 / node j+1 from the neighbouring lanes (shuffles), and
// the plane l-1 terms from the previous step. Lanes 1..31 form node masses,
// lanes 1..30 momentum fluxes, lanes 2..30 update (29 nodes per warp). Sums
// and the momentum limiter keep the reference order
// (advec_mom_kernel.f90:166-252).
template <class S, int VAR, class M>
__global__ void __launch_bounds__(BX * BY, M::kFlat || sizeof(typename S::arith_t) == 8 ? 4 : 6) k_mom_sweep_x(M m,
    GeomArrays ga, const typename S::mf_t* __restrict__ mfx,
    const typename S::rho_t* __restrict__ density1, const typename S::vf_t* __restrict__ vfx,
    const typename S::vf_t* __restrict__ vfy, const typename S::vf_t* __restrict__ vfz,
    const typename S::vel_t* __restrict__ u_in, const typename S::vel_t* __restrict__ v_in,
    const typename S::vel_t* __restrict__ w_in, typename S::vel_t* __restrict__ u_out,
    typename S::vel_t* __restrict__ v_out, typename S::vel_t* __restrict__ w_out,
    Level0<S> lz) {
  m.run([&](const Geom& g, const Tile& t) {
  const int seg = m.seg;
  const int lane = threadIdx.x;
  const int j = g.x_min - 2 + t.x * 29 + lane;  // node of this lane
  const int k = g.y_min + t.y * BY + threadIdx.y;
  const int l0 = g.z_min + t.z * seg;
  int l1 = l0 + seg - 1;
  if (l1 > g.z_max + 1) l1 = g.z_max + 1;
  const bool row = k <= g.y_max + 1;                // every lane of a row stays for the shuffles
  const bool has_nf = row && j <= g.x_max + 2;     // node_flux range j in [x_min-2, x_max+2]
  const bool has_mf = row && lane >= 1 && lane <= 30 && j >= g.x_min - 1 && j <= g.x_max + 1;
  const bool has_up = row && lane >= 2 && lane <= 30 && j >= g.x_min && j <= g.x_max + 1;
  auto P = [&](int kk, int ll) {
    return cell_product<S>(g, VAR, ga, density1, vfx, vfy, vfz, j, kk, ll);
  };
  using V = typename S::vel_t;
  const typename S::vel_t* in[3] = {u_in, v_in, w_in};
  typename S::vel_t* out[3] = {u_out, v_out, w_out};
  typename S::vel_t* lev0[3] = {lz.xvel0, lz.yvel0, lz.zvel0};
  const double cd_0 = has_nf ? GX(ga.celldx, j) : 1.0;
  const double cd_m1 = has_mf ? GX(ga.celldx, j - 1) : 1.0;
  const double cd_p1 = has_mf ? GX(ga.celldx, j + 1) : 1.0;
  // plane l-1 terms: mass fluxes at (j, k-1), (j, k), (j+1, k-1), (j+1, k); cell
  // masses at (j, k-1), (j, k)
  double fm_a = 0.0, fm_b = 0.0, fm_c = 0.0, fm_d = 0.0, pm_a = 0.0, pm_b = 0.0;
  if (has_nf) {
    fm_a = L(mfx, j, k - 1, l0 - 1); fm_b = L(mfx, j, k, l0 - 1);
    fm_c = L(mfx, j + 1, k - 1, l0 - 1); fm_d = L(mfx, j + 1, k, l0 - 1);
    pm_a = P(k - 1, l0 - 1); pm_b = P(k, l0 - 1);
  }
  for (int l = l0; l <= l1; l++) {
    double f_a = 0.0, f_b = 0.0, f_c = 0.0, f_d = 0.0, p_a = 0.0, p_b = 0.0;
    if (has_nf) {
      f_a = L(mfx, j, k - 1, l); f_b = L(mfx, j, k, l);
      f_c = L(mfx, j + 1, k - 1, l); f_d = L(mfx, j + 1, k, l);
      p_a = P(k - 1, l); p_b = P(k, l);
    }
    const double nf = 0.125 * (f_a + f_b + f_c + f_d + fm_a + fm_b + fm_c + fm_d);
    const double q_a = __shfl_up_sync(0xffffffffu, p_a, 1);
    const double q_b = __shfl_up_sync(0xffffffffu, p_b, 1);
    const double qm_a = __shfl_up_sync(0xffffffffu, pm_a, 1);
    const double qm_b = __shfl_up_sync(0xffffffffu, pm_b, 1);
    const double nmp = node_mass_sum(p_a, p_b, q_a, q_b, pm_a, pm_b, qm_a, qm_b);
    const double nf_m = __shfl_up_sync(0xffffffffu, nf, 1);
    const double nmpre = nmp - nf_m + nf;
    const double nmpre_p = __shfl_down_sync(0xffffffffu, nmpre, 1);
    // flux and update in the momentum arithmetic A (node masses are FP64)
    using A = typename S::arith_t;
    const MomNodeTerms<A> nt =
        mom_node_terms<A>((A)nf, (A)nmpre, (A)nmpre_p, (A)cd_0, (A)cd_m1, (A)cd_p1);
    A vn[3];
#pragma unroll
    for (int q = 0; q < 3; q++) {
      A mf = A(0.0), v0 = A(0.0);
      if (has_mf) {
        const A vm1 = lda<A>(&E(in[q], j - 1, k, l));
        v0 = lda<A>(&E(in[q], j, k, l));
        const A vp1 = lda<A>(&E(in[q], j + 1, k, l)), vp2 = lda<A>(&E(in[q], j + 2, k, l));
        mf = mom_flux_v<A>(nt, vm1, v0, vp1, vp2);
      }
      const A mf_m = __shfl_up_sync(0xffffffffu, mf, 1);
      vn[q] = v0 * (A)nmpre + mf_m - mf;
    }
    if (has_up) {
      div3_rn(vn, (A)nmp);  // the three updates share node_mass_post
#pragma unroll
      for (int q = 0; q < 3; q++) {
        const V vn1 = st<V>(vn[q]);
        E(out[q], j, k, l) = vn1;
        if (lz.xvel0) E(lev0[q], j, k, l) = vn1;  // last sweep of the step: reset_field
      }
    }
    fm_a = f_a; fm_b = f_b; fm_c = f_c; fm_d = f_d;
    pm_a = p_a; pm_b = p_b;
  }
  });
}

// Copy the halo shell of three vertex arrays (every node of [min-2, max+3]^3
// outside [min, max+1]^3) from one buffer of a pair to the other, touching
// the shell only: k_vert_shell_planes takes the four halo planes l whole
// (tile z 0..3: z_min-2, z_min-1, z_max+2, z_max+3), k_vert_shell_ring the
// ring of each interior plane (the four shell rows k whole, then the four
// shell columns j of each interior row).
template <class T>
__device__ __forceinline__ void copy3_at(long long o, const T* __restrict__ a_in,
                                         const T* __restrict__ b_in, const T* __restrict__ c_in,
                                         T* __restrict__ a_out, T* __restrict__ b_out,
                                         T* __restrict__ c_out) {
  a_out[o] = a_in[o];
  b_out[o] = b_in[o];
  c_out[o] = c_in[o];
}

template <class T, class M>
__global__ void k_vert_shell_planes(M m, const T* __restrict__ a_in, const T* __restrict__ b_in,
                                    const T* __restrict__ c_in, T* __restrict__ a_out,
                                    T* __restrict__ b_out, T* __restrict__ c_out) {
  m.run([&](const Geom& g, const Tile& t) {
  int j, k;
  if (!tile_jk<M>(Box{g.x_min - 2, g.x_max + 3, g.y_min - 2, g.y_max + 3, 0, 0}, t, j, k)) return;
  const int l = t.z < 2 ? g.z_min - 2 + t.z : g.z_max + t.z;
  copy3_at(off3(g, j, k, l), a_in, b_in, c_in, a_out, b_out, c_out);
  });
}

template <class T, class M>
__global__ void k_vert_shell_ring(M m, const T* __restrict__ a_in, const T* __restrict__ b_in,
                                  const T* __restrict__ c_in, T* __restrict__ a_out,
                                  T* __restrict__ b_out, T* __restrict__ c_out) {
  m.run([&](const Geom& g, const Tile& t) {
  const int w = g.x_max - g.x_min + 6;        // nodes of a shell row
  const int rows = g.y_max - g.y_min + 2;     // interior rows k in [y_min, y_max+1]
  const int e = t.x * (BX * BY) + (int)threadIdx.y * BX + (int)threadIdx.x;
  const int l = g.z_min + t.z;                // interior planes [z_min, z_max+1]
  int j, k;
  if (e < 4 * w) {
    const int r = e / w;
    j = g.x_min - 2 + e % w;
    k = r < 2 ? g.y_min - 2 + r : g.y_max + r;
  } else {
    const int f = e - 4 * w;
    if (f >= 4 * rows) return;
    const int c = f % 4;
    k = g.y_min + f / 4;
    j = c < 2 ? g.x_min - 2 + c : g.x_max + c;
  }
  copy3_at(off3(g, j, k, l), a_in, b_in, c_in, a_out, b_out, c_out);
  });
}

// ===========================================================================
// Tile grids of the launches (aux: segment length of a marching kernel)
constexpr int kMarchSeg = 32;

dim3 grid_interior(const Geom& g, int) { return grid_of(interior(g)); }
dim3 grid_nodes(const Geom& g, int) { return grid_of(nodes(g)); }
dim3 grid_visc(const Geom& g, int) { return grid_of(interior(g), kViscCellsZ); }
// the same laid out for a batch (tile_jk)
dim3 grid_interior_flat(const Geom& g, int) { return grid_flat(interior(g)); }
dim3 grid_nodes_flat(const Geom& g, int) { return grid_flat(nodes(g)); }
dim3 grid_visc_flat(const Geom& g, int) { return grid_flat(interior(g), kViscCellsZ); }
// 28 cells per warp along x (faces x_min..x_max+2), rows of 8, one plane
dim3 grid_cell_sweep_x(const Geom& g, int) {
  return dim3((g.x_max + 2 - g.x_min + 1 + 27) / 28, (g.y_max - g.y_min + 1 + BY - 1) / BY,
              g.z_max - g.z_min + 1);
}
dim3 grid_cell_shell(const Geom& g, int) {
  return dim3((g.x_max - g.x_min + 5 + BX - 1) / BX, (g.y_max - g.y_min + 5 + BY - 1) / BY,
              g.z_max - g.z_min + 5);
}
dim3 grid_cell_shell_flat(const Geom& g, int) {
  return grid_flat(Box{g.x_min - 2, g.x_max + 2, g.y_min - 2, g.y_max + 2, g.z_min - 2, g.z_max + 2});
}
// the vertex shell: four whole halo planes, and the ring of each interior plane
dim3 grid_shell_planes_flat(const Geom& g, int) {
  dim3 d = grid_flat(Box{g.x_min - 2, g.x_max + 3, g.y_min - 2, g.y_max + 3, 0, 0});
  d.z = 4;
  return d;
}
dim3 grid_shell_planes(const Geom& g, int) {
  dim3 d = grid_of(Box{g.x_min - 2, g.x_max + 3, g.y_min - 2, g.y_max + 3, 0, 0});
  d.z = 4;
  return d;
}
dim3 grid_shell_ring(const Geom& g, int) {
  const int ring = 4 * (g.x_max - g.x_min + 6) + 4 * (g.y_max - g.y_min + 2);
  return dim3((ring + BX * BY - 1) / (BX * BY), 1, g.z_max - g.z_min + 2);
}
// 32 columns j of one cross-axis index per block, BY segments along the sweep
template <int DIR>
dim3 grid_cell_sweep(const Geom& g, int) {
  const MarchRange r = cell_sweep_range<DIR>(g);
  return dim3((r.jhi - r.jlo + 1 + BX - 1) / BX, r.chi - r.clo + 1, 1);
}
// 31 nodes per warp along x (lane 0 holds the column below), rows of 8, segments
template <int DIR>
dim3 grid_mom_node(const Geom& g, int seg) {
  const MarchRange r = mom_node_range<DIR>(g);
  return dim3((r.jhi - r.jlo + 1 + 30) / 31, (r.chi - r.clo + 1 + BY - 1) / BY,
              (r.phi - r.plo + 1 + seg - 1) / seg);
}
template <int DIR>
dim3 grid_cell_sweep_flat(const Geom& g, int) {
  const MarchRange r = cell_sweep_range<DIR>(g);
  const long long n = (long long)(r.jhi - r.jlo + 1) * (r.chi - r.clo + 1);
  return dim3((unsigned)((n + BX - 1) / BX), 1, 1);
}
template <int DIR>
dim3 grid_mom_vel_flat(const Geom& g, int seg) {
  const MarchRange r = mom_vel_range<DIR>(g);
  const long long n = (long long)(r.jhi - r.jlo + 1) * (r.chi - r.clo + 1);
  return dim3((unsigned)((n + BX * BY - 1) / (BX * BY)), 1, (r.phi - r.plo + 1 + seg - 1) / seg);
}
template <int DIR>
dim3 grid_mom_vel(const Geom& g, int seg) {
  const MarchRange r = mom_vel_range<DIR>(g);
  return dim3((r.jhi - r.jlo + 1 + BX - 1) / BX, (r.chi - r.clo + 1 + BY - 1) / BY,
              (r.phi - r.plo + 1 + seg - 1) / seg);
}
// 29 nodes per warp along x, rows of 8 along y, segments of seg planes along z
dim3 grid_mom_sweep_x(const Geom& g, int seg) {
  return dim3((g.x_max + 1 - g.x_min + 1 + 28) / 29, (g.y_max + 1 - g.y_min + 1 + BY - 1) / BY,
              (g.z_max + 1 - g.z_min + 1 + seg - 1) / seg);
}

}  // namespace

const dim3 kBlk(BX, BY);

template <class S>
void launch_visc_dt(const Target& tg, cudaStream_t s, const GeomArrays& ga, double g_small,
                    double dtc_safe, double dtu_safe, double dtv_safe, double dtw_safe,
                    double dtdiv_safe, const typename S::rho_t* density0,
                    const typename S::ene_t* energy0, typename S::cs_t* pressure,
                    typename S::cs_t* viscosity, typename S::cs_t* soundspeed,
                    const typename S::vel_t* xvel0, const typename S::vel_t* yvel0,
                    const typename S::vel_t* zvel0, unsigned long long* min_key) {
  launch_mapped2(tg, s, kKeyTimestepVisc, grid_visc, grid_visc_flat, 0, false, kBlk, k_visc_dt<S, MapSingle>,
                k_visc_dt<S, MapBatch>, ga, g_small, dtc_safe, dtu_safe, dtv_safe, dtw_safe,
                dtdiv_safe, density0, energy0, pressure, viscosity, soundspeed, xvel0, yvel0,
                zvel0, min_key);
}

template <class S>
void launch_pdv_predict_eos(const Target& tg, cudaStream_t s, const double* dt_ptr,
                            const GeomArrays& ga, const typename S::rho_t* density0,
                            const typename S::ene_t* energy0, typename S::cs_t* pressure,
                            const typename S::cs_t* viscosity, const typename S::vel_t* xvel0,
                            const typename S::vel_t* yvel0, const typename S::vel_t* zvel0) {
  launch_mapped2(tg, s, kKeyPdvPredict, grid_interior, grid_interior_flat, 0, false, kBlk,
                k_pdv_predict_eos<S, MapSingle>, k_pdv_predict_eos<S, MapBatchFree>, dt_ptr, ga,
                density0, energy0, pressure, viscosity, xvel0, yvel0, zvel0);
}

template <class S>
void launch_pdv_flux(const Target& tg, cudaStream_t s, const double* dt_ptr, const GeomArrays& ga,
                     const typename S::rho_t* density0, typename S::rho_t* density1,
                     const typename S::ene_t* energy0, typename S::ene_t* energy1,
                     const typename S::cs_t* pressure, const typename S::cs_t* viscosity,
                     const typename S::vel_t* xvel0, const typename S::vel_t* xvel1,
                     const typename S::vel_t* yvel0, const typename S::vel_t* yvel1,
                     const typename S::vel_t* zvel0, const typename S::vel_t* zvel1,
                     typename S::vf_t* vol_flux_x, typename S::vf_t* vol_flux_y,
                     typename S::vf_t* vol_flux_z) {
  launch_mapped2(tg, s, kKeyPdvFlux, grid_nodes, grid_nodes_flat, 0, false, kBlk, k_pdv_flux<S, MapSingle>,
                k_pdv_flux<S, MapBatchFree>, dt_ptr, ga, density0, density1, energy0, energy1,
                pressure, viscosity, xvel0, xvel1, yvel0, yvel1, zvel0, zvel1, vol_flux_x,
                vol_flux_y, vol_flux_z);
}

template <class S>
void launch_advec_cell_fused(const Target& tg, cudaStream_t s, int advect_x, int dir, int sweep,
                             const GeomArrays& ga, typename S::rho_t* density1,
                             typename S::ene_t* energy1, typename S::mf_t* mass_flux_x,
                             const typename S::vf_t* vol_flux_x, typename S::mf_t* mass_flux_y,
                             const typename S::vf_t* vol_flux_y, typename S::mf_t* mass_flux_z,
                             const typename S::vf_t* vol_flux_z, typename S::wk_t* ener_flux,
                             const Level0<S>& level0) {
  (void)ener_flux;
  // pre_vol variant (the sweep's volume-flux terms) as a kernel template
  // argument: y is sweep 2 (2: after x, 3: after z); z is sweep 1 (4) or 3 (5)
  if (dir == 1) return;  // the x sweep is out of place: launch_advec_cell_x
  auto sweep_y = [&](auto var) {
    constexpr int V = decltype(var)::value;
    launch_mapped2(tg, s, kKeyCellSweep | 2u | (V << 4), grid_cell_sweep<2>,
                   grid_cell_sweep_flat<2>, 0, false, kBlk,
                   k_cell_sweep_march<S, 2, V, MapSingle>, k_cell_sweep_march<S, 2, V, MapBatch>,
                   ga, density1, energy1, vol_flux_x, vol_flux_y, vol_flux_z, mass_flux_y, level0);
  };
  auto sweep_z = [&](auto var) {
    constexpr int V = decltype(var)::value;
    launch_mapped2(tg, s, kKeyCellSweep | 3u | (V << 4), grid_cell_sweep<3>,
                   grid_cell_sweep_flat<3>, 0, false, kBlk,
                   k_cell_sweep_march<S, 3, V, MapSingle>, k_cell_sweep_march<S, 3, V, MapBatch>,
                   ga, density1, energy1, vol_flux_x, vol_flux_y, vol_flux_z, mass_flux_z, level0);
  };
  // one marching pass, in place
  if (dir == 2) {
    if (advect_x) sweep_y(std::integral_constant<int, 2>{});
    else sweep_y(std::integral_constant<int, 3>{});
  } else {
    if (sweep == 1) sweep_z(std::integral_constant<int, 4>{});
    else sweep_z(std::integral_constant<int, 5>{});
  }
}

template <class S>
void launch_advec_cell_x(const Target& tg, cudaStream_t s, int sweep, const GeomArrays& ga,
                         const typename S::rho_t* density1_in, const typename S::ene_t* energy1_in,
                         typename S::rho_t* density1_out, typename S::ene_t* energy1_out,
                         const typename S::vf_t* vol_flux_x, const typename S::vf_t* vol_flux_y,
                         const typename S::vf_t* vol_flux_z, typename S::mf_t* mass_flux_x,
                         bool copy_shell, const Level0<S>& level0, const CellXMaps* maps,
                         int* status) {
  // pre_vol variant: 0 on sweep 1 (all three flux differences), 1 on sweep 3
  if (maps && !tg.plan)  // one chunk: planes staged by bulk-tensor copies
    launch_cell_sweep_x_tma<S>(tg.g, s, sweep, *maps, ga, density1_out, energy1_out, mass_flux_x,
                               level0, status);
  else if (sweep == 1)
    launch_mapped(tg, s, kKeyCellSweepX, grid_cell_sweep_x, 0, false, kBlk,
                  k_cell_sweep_x<S, 0, MapSingle>, k_cell_sweep_x<S, 0, MapBatchFree>, ga,
                  density1_in, energy1_in, density1_out, energy1_out, vol_flux_x, vol_flux_y,
                  vol_flux_z, mass_flux_x, level0);
  else
    launch_mapped(tg, s, kKeyCellSweepX | (1u << 4), grid_cell_sweep_x, 0, false, kBlk,
                  k_cell_sweep_x<S, 1, MapSingle>, k_cell_sweep_x<S, 1, MapBatchFree>, ga,
                  density1_in, energy1_in, density1_out, energy1_out, vol_flux_x, vol_flux_y,
                  vol_flux_z, mass_flux_x, level0);
  // the cells the sweep does not update keep their values in the output pair
  if (copy_shell) {
    using R = typename S::rho_t;
    using En = typename S::ene_t;
    launch_mapped2(tg, s, kKeyCellShell, grid_cell_shell, grid_cell_shell_flat, 0, false, kBlk,
                   k_cell_shell_copy<R, En, MapSingle>, k_cell_shell_copy<R, En, MapBatchFree>,
                   density1_in, energy1_in, density1_out, energy1_out);
  }
}

template <class S>
void launch_advec_mom_fused(const Target& tg, cudaStream_t s, int advect_x, int sweep, int dir,
                            double vol, const GeomArrays& ga, const typename S::rho_t* density1,
                            const typename S::mf_t* mass_flux_x, const typename S::mf_t* mass_flux_y,
                            const typename S::mf_t* mass_flux_z, const typename S::vf_t* vol_flux_x,
                            const typename S::vf_t* vol_flux_y, const typename S::vf_t* vol_flux_z,
                            typename S::wk_t* node_flux, typename S::wk_t* node_mass_post,
                            typename S::wk_t* node_mass_pre, typename S::vel_t* const* vel_in,
                            typename S::vel_t* const* vel_out, bool copy_shell,
                            const Level0<S>& level0, const MomXMaps* x_maps, int* status,
                            const NodeMaps* node_maps, const VelMaps* vel_maps) {
  // the node arrays of the y/z sweeps live in three work arrays, as nd_t
  using ND = typename S::nd_t;
  static_assert(sizeof(ND) <= sizeof(typename S::wk_t), "node arrays fit the work arrays");
  ND* nd_flux = nd_array<S>(node_flux);
  ND* nd_post = nd_array<S>(node_mass_post);
  ND* nd_pre = nd_array<S>(node_mass_pre);
  (void)vol;
  // post_vol variant (mom_post_vol) as a kernel template argument: x is sweep
  // 1 (0) or 3 (4); y is sweep 2 (2: after x, 3: after z); z is sweep 1 (1) or 3 (4)
  auto node_vel = [&](auto dir_c, auto var) {
    constexpr int D = decltype(dir_c)::value, V = decltype(var)::value;
    // node pass then velocity pass, each marching along the sweep axis in segments
    if (node_maps && !tg.plan)
      launch_mom_node_tma<S>(tg.g, s, D, V, *node_maps, nd_flux, nd_post, nd_pre, status);
    else
      launch_mapped(tg, s, kKeyMomNode | D | (V << 4), grid_mom_node<D>, kMarchSeg, true, kBlk,
                    k_mom_node_march<S, D, V, MapSingle>, k_mom_node_march<S, D, V, MapBatchFree>,
                    ga, D == 2 ? mass_flux_y : mass_flux_z, density1, vol_flux_x, vol_flux_y,
                    vol_flux_z, nd_flux, nd_post, nd_pre);
    if (vel_maps && !tg.plan)
      launch_mom_vel_tma<S>(tg.g, s, D, *vel_maps, ga, nd_flux, nd_pre, vel_in, vel_out, level0,
                            status);
    else
      launch_mapped2(tg, s, kKeyMomVel3 | D, grid_mom_vel<D>, grid_mom_vel_flat<D>, kMarchSeg,
                     true, kBlk, k_mom_vel3_march<S, D, MapSingle>,
                     k_mom_vel3_march<S, D, MapBatchFree>, ga, nd_flux, nd_post, nd_pre,
                     vel_in[0], vel_in[1], vel_in[2], vel_out[0], vel_out[1], vel_out[2], level0);
  };
  using I2 = std::integral_constant<int, 2>;
  using I3 = std::integral_constant<int, 3>;
  if (dir == 1 && x_maps && !tg.plan) {
    // one pass, its planes staged in shared memory
    launch_mom_x_tma<S>(tg.g, s, sweep, kMarchSeg, *x_maps, ga, vel_out, level0, status);
  } else if (dir == 1) {
    // one pass for the three velocities
    auto sweep_x = [&](auto var) {
      constexpr int V = decltype(var)::value;
      launch_mapped(tg, s, kKeyMomSweepX | (V << 4), grid_mom_sweep_x, kMarchSeg, true, kBlk,
                    k_mom_sweep_x<S, V, MapSingle>, k_mom_sweep_x<S, V, MapBatchFree>, ga,
                    mass_flux_x, density1, vol_flux_x, vol_flux_y, vol_flux_z, vel_in[0],
                    vel_in[1], vel_in[2], vel_out[0], vel_out[1], vel_out[2], level0);
    };
    if (sweep == 1) sweep_x(std::integral_constant<int, 0>{});
    else sweep_x(std::integral_constant<int, 4>{});
  } else if (dir == 2) {
    if (advect_x) node_vel(I2{}, std::integral_constant<int, 2>{});
    else node_vel(I2{}, std::integral_constant<int, 3>{});
  } else {
    if (sweep == 1) node_vel(I3{}, std::integral_constant<int, 1>{});
    else node_vel(I3{}, std::integral_constant<int, 4>{});
  }
  // the updated buffers take the halo shell of the inputs
  if (copy_shell) {
    using V = typename S::vel_t;
    launch_mapped2(tg, s, kKeyShellCopy, grid_shell_planes, grid_shell_planes_flat, 0, false,
                   kBlk, k_vert_shell_planes<V, MapSingle>, k_vert_shell_planes<V, MapBatchFree>,
                   vel_in[0], vel_in[1], vel_in[2], vel_out[0], vel_out[1], vel_out[2]);
    launch_mapped(tg, s, kKeyShellCopy | 1u, grid_shell_ring, 0, false, kBlk,
                  k_vert_shell_ring<V, MapSingle>, k_vert_shell_ring<V, MapBatchFree>, vel_in[0],
                  vel_in[1], vel_in[2], vel_out[0], vel_out[1], vel_out[2]);
  }
}

#define INSTF(S)                                                                               \
  template void launch_visc_dt<S>(const Target&, cudaStream_t, const GeomArrays&, double, double,  \
                                  double, double, double, double, const S::rho_t*,             \
                                  const S::ene_t*, S::cs_t*, S::cs_t*, S::cs_t*,               \
                                  const S::vel_t*, const S::vel_t*, const S::vel_t*,           \
                                  unsigned long long*);                                        \
  template void launch_pdv_predict_eos<S>(const Target&, cudaStream_t, const double*,            \
                                          const GeomArrays&, const S::rho_t*, const S::ene_t*, \
                                          S::cs_t*, const S::cs_t*, const S::vel_t*,           \
                                          const S::vel_t*, const S::vel_t*);                   \
  template void launch_pdv_flux<S>(const Target&, cudaStream_t, const double*, const GeomArrays&, \
                                   const S::rho_t*, S::rho_t*, const S::ene_t*, S::ene_t*,     \
                                   const S::cs_t*, const S::cs_t*, const S::vel_t*,            \
                                   const S::vel_t*, const S::vel_t*, const S::vel_t*,          \
                                   const S::vel_t*, const S::vel_t*, S::vf_t*, S::vf_t*,       \
                                   S::vf_t*);                                                  \
  template void launch_advec_cell_fused<S>(const Target&, cudaStream_t, int, int, int,           \
                                           const GeomArrays&, S::rho_t*, S::ene_t*, S::mf_t*,  \
                                           const S::vf_t*, S::mf_t*, const S::vf_t*, S::mf_t*, \
                                           const S::vf_t*, S::wk_t*, const Level0<S>&);        \
  template void launch_advec_cell_x<S>(const Target&, cudaStream_t, int, const GeomArrays&,      \
                                       const S::rho_t*, const S::ene_t*, S::rho_t*, S::ene_t*,  \
                                       const S::vf_t*, const S::vf_t*, const S::vf_t*,          \
                                       S::mf_t*, bool, const Level0<S>&, const CellXMaps*, int*); \
  template void launch_advec_mom_fused<S>(const Target&, cudaStream_t, int, int, int, double,    \
                                          const GeomArrays&, const S::rho_t*, const S::mf_t*,  \
                                          const S::mf_t*, const S::mf_t*, const S::vf_t*,      \
                                          const S::vf_t*, const S::vf_t*, S::wk_t*, S::wk_t*,  \
                                          S::wk_t*, S::vel_t* const*, S::vel_t* const*, bool,  \
                                          const Level0<S>&, const MomXMaps*, int*,            \
                                          const NodeMaps*, const VelMaps*);

INSTF(F64)
INSTF(F32Mixed)

}  // namespace clover
