// Hydro-cycle kernels for sm_100a, one family per reference *_kernel.
//
// Each kernel computes exactly the elements the reference loop nest computes,
// over the same index ranges, with the same operation order. The library is
// built with -fmad=false, so FP64 results are bit-identical to a serial
// IEEE evaluation of the reference expressions (the reductions excepted,
// whose order differs). All arithmetic is FP64 whatever the storage type.
//
// Threads map one-to-one onto elements: x (the contiguous axis) across the
// 32 lanes of a warp, y across warps, z across the grid, so every warp load
// is a coalesced 256-byte row segment of the pitched layout.
#include <cfloat>
#include <cstdio>

#include "../../include/clover_b200.h"
#include "../../include/clover_kernels.h"
#include "clover_div.cuh"
#include "clover_launch.h"
#include "clover_sum.cuh"

namespace clover {

namespace {

constexpr int BX = 32, BY = 8;

struct Box {
  int j0, j1, k0, k1, l0, l1;
};

inline dim3 grid_of(const Box& b) {
  int nj = b.j1 - b.j0 + 1, nk = b.k1 - b.k0 + 1, nl = b.l1 - b.l0 + 1;
  if (nj <= 0 || nk <= 0 || nl <= 0) return dim3(0, 0, 0);
  return dim3((nj + BX - 1) / BX, (nk + BY - 1) / BY, nl);
}

inline bool launchable(const dim3& gr) { return gr.x > 0 && gr.y > 0 && gr.z > 0; }

__host__ __device__ inline Box interior(const Geom& g) {
  return Box{g.x_min, g.x_max, g.y_min, g.y_max, g.z_min, g.z_max};
}
__host__ __device__ inline Box nodes(const Geom& g) {
  return Box{g.x_min, g.x_max + 1, g.y_min, g.y_max + 1, g.z_min, g.z_max + 1};
}
__host__ __device__ inline Box halo2(const Geom& g) {
  return Box{g.x_min - 2, g.x_max + 2, g.y_min - 2, g.y_max + 2, g.z_min - 2, g.z_max + 2};
}
inline dim3 grid_interior(const Geom& g, int) { return grid_of(interior(g)); }
inline dim3 grid_nodes(const Geom& g, int) { return grid_of(nodes(g)); }

#define BOX_THREAD(b)                                    \
  const int j = (b).j0 + blockIdx.x * BX + threadIdx.x;  \
  const int k = (b).k0 + blockIdx.y * BY + threadIdx.y;  \
  const int l = (b).l0 + blockIdx.z;                     \
  if (j > (b).j1 || k > (b).k1) return

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
// flattened tile grid of a box for a batch: 256 cells of the (j, k) plane per
// tile, planes along z
inline dim3 grid_flat(const Box& b, int zdiv = 1) {
  const long long nj = b.j1 - b.j0 + 1, nk = b.k1 - b.k0 + 1, nl = b.l1 - b.l0 + 1;
  if (nj <= 0 || nk <= 0 || nl <= 0) return dim3(0, 0, 0);
  return dim3((unsigned)((nj * nk + BX * BY - 1) / (BX * BY)), 1, (unsigned)((nl + zdiv - 1) / zdiv));
}

inline dim3 grid_interior_flat(const Geom& g, int) { return grid_flat(interior(g)); }
inline dim3 grid_nodes_flat(const Geom& g, int) { return grid_flat(nodes(g)); }

// the same for tile t of a mapped kernel (clover_sched.cuh)
#define TILE_THREAD(box, t)                            \
  const Box b = (box);                                 \
  int j, k;                                            \
  if (!tile_jk<M>(b, (t), j, k)) return;               \
  const int l = b.l0 + (t).z

// 3D element, 1D coordinate arrays
#define E(a, jj, kk, ll) (a)[off3(g, (jj), (kk), (ll))]
#define GX(a, jj) (a)[g.o1 + (jj) - g.x_min + 2]
#define GY(a, kk) (a)[g.o1 + (kk) - g.y_min + 2]
#define GZ(a, ll) (a)[g.o1 + (ll) - g.z_min + 2]

__device__ __forceinline__ double ld(const double* p) { return __ldg(p); }
__device__ __forceinline__ double ld(const float* p) { return (double)__ldg(p); }
#define L(a, jj, kk, ll) ld(&E(a, jj, kk, ll))

// a value in storage type T, converted once from the arithmetic it was
// formed in (no detour through double for an FP32 value stored as FP32)
template <class T, class U>
__device__ __forceinline__ T st(U v) { return (T)v; }

__device__ __forceinline__ double fmin2(double a, double b) { return b < a ? b : a; }
__device__ __forceinline__ double fmax2(double a, double b) { return b > a ? b : a; }

__device__ __forceinline__ double dt_of(double v, const double* p) { return p ? *p : v; }

// ---------------------------------------------------------------------------
// ideal_gas_kernel.f90:47-58
template <class S, class M>
__global__ void __launch_bounds__(BX * BY) k_ideal_gas(M m,
    const typename S::rho_t* __restrict__ density, const typename S::ene_t* __restrict__ energy,
    typename S::cs_t* __restrict__ pressure, typename S::cs_t* __restrict__ soundspeed) {
  m.run([&](const Geom& g, const Tile& t) {
  TILE_THREAD(interior(g), t);
  // in the policy's arithmetic (FP64, or FP32 where pressure and sound speed
  // are stored in FP32)
  using A = typename S::arith_t;
  const A d = (A)L(density, j, k, l);
  const A v = div_rn(A(1.0), d);
  const A p = (A(1.4) - A(1.0)) * d * (A)L(energy, j, k, l);
  const A pressurebyenergy = (A(1.4) - A(1.0)) * d;
  const A pressurebyvolume = -d * p;
  const A ss2 = v * v * (p * pressurebyenergy - pressurebyvolume);
  using C = typename S::cs_t;
  E(pressure, j, k, l) = st<C>(p);
  E(soundspeed, j, k, l) = st<C>(sqrt(ss2));
  });
}

// ---------------------------------------------------------------------------
// viscosity_kernel.f90:71-134
template <class S>
__global__ void __launch_bounds__(BX * BY, 4) k_viscosity(Geom g, Box b, GeomArrays ga,
    const typename S::rho_t* __restrict__ density0, const typename S::cs_t* __restrict__ pressure,
    typename S::cs_t* __restrict__ viscosity, const typename S::vel_t* __restrict__ xvel0,
    const typename S::vel_t* __restrict__ yvel0, const typename S::vel_t* __restrict__ zvel0) {
  BOX_THREAD(b);
  const double u000 = L(xvel0, j, k, l), u100 = L(xvel0, j + 1, k, l);
  const double u010 = L(xvel0, j, k + 1, l), u110 = L(xvel0, j + 1, k + 1, l);
  const double u001 = L(xvel0, j, k, l + 1), u101 = L(xvel0, j + 1, k, l + 1);
  const double u011 = L(xvel0, j, k + 1, l + 1), u111 = L(xvel0, j + 1, k + 1, l + 1);
  const double v000 = L(yvel0, j, k, l), v100 = L(yvel0, j + 1, k, l);
  const double v010 = L(yvel0, j, k + 1, l), v110 = L(yvel0, j + 1, k + 1, l);
  const double v001 = L(yvel0, j, k, l + 1), v101 = L(yvel0, j + 1, k, l + 1);
  const double v011 = L(yvel0, j, k + 1, l + 1), v111 = L(yvel0, j + 1, k + 1, l + 1);
  const double w000 = L(zvel0, j, k, l), w100 = L(zvel0, j + 1, k, l);
  const double w010 = L(zvel0, j, k + 1, l), w110 = L(zvel0, j + 1, k + 1, l);
  const double w001 = L(zvel0, j, k, l + 1), w101 = L(zvel0, j + 1, k, l + 1);
  const double w011 = L(zvel0, j, k + 1, l + 1), w111 = L(zvel0, j + 1, k + 1, l + 1);

  const double ugradx1 = u000 + u010 + u001 + u011;
  const double ugradx2 = u100 + u110 + u101 + u111;
  const double vgrady1 = v000 + v100 + v001 + v101;
  const double vgrady2 = v010 + v110 + v011 + v111;
  const double wgradz1 = w000 + w100 + w010 + w110;
  const double wgradz2 = w001 + w101 + w011 + w111;
  const double div = (E(ga.xarea, j, k, l) * (ugradx2 - ugradx1) +
                      E(ga.yarea, j, k, l) * (vgrady2 - vgrady1)) +
                     E(ga.zarea, j, k, l) * (wgradz2 - wgradz1);
  // IF((limiter.GT.0.0).OR.(div.GE.0.0)) q=0: with div >= 0 the limiter
  // cannot change q, so the strain terms, pressure gradients and limiter are
  // formed only for compressing cells (a NaN div takes that path too)
  double q = 0.0;
  if (!(div >= 0.0)) {
    const double ugrady1 = u000 + u100 + u001 + u101;
    const double ugrady2 = u010 + u110 + u011 + u111;
    const double ugradz1 = u000 + u100 + u010 + u110;
    const double ugradz2 = u001 + u101 + u011 + u111;
    const double vgradx1 = v000 + v010 + v001 + v011;
    const double vgradx2 = v100 + v110 + v101 + v111;
    const double vgradz1 = v000 + v100 + v010 + v110;
    const double vgradz2 = v001 + v101 + v011 + v111;
    const double wgradx1 = w000 + w010 + w001 + w011;
    const double wgradx2 = w100 + w110 + w101 + w111;
    const double wgrady1 = w000 + w100 + w001 + w101;
    const double wgrady2 = w010 + w110 + w011 + w111;

    const double cdx = GX(ga.celldx, j), cdy = GY(ga.celldy, k), cdz = GZ(ga.celldz, l);
    const double xx = 0.25 * (ugradx2 - ugradx1) / cdx;
    const double yy = 0.25 * (vgrady2 - vgrady1) / cdy;
    const double zz = 0.25 * (wgradz2 - wgradz1) / cdz;
    const double xy = 0.25 * (ugrady2 - ugrady1) / cdy + 0.25 * (vgradx2 - vgradx1) / cdx;
    const double xz = 0.25 * (ugradz2 - ugradz1) / cdz + 0.25 * (wgradx2 - wgradx1) / cdx;
    const double yz = 0.25 * (vgradz2 - vgradz1) / cdz + 0.25 * (wgrady2 - wgrady1) / cdy;

    double pgradx = (L(pressure, j + 1, k, l) - L(pressure, j - 1, k, l)) / (cdx + GX(ga.celldx, j + 1));
    double pgrady = (L(pressure, j, k + 1, l) - L(pressure, j, k - 1, l)) / (cdy + GY(ga.celldy, k + 1));
    double pgradz = (L(pressure, j, k, l + 1) - L(pressure, j, k, l - 1)) / (cdz + GZ(ga.celldz, l + 1));

    const double pgradx2 = pgradx * pgradx;
    const double pgrady2 = pgrady * pgrady;
    const double pgradz2 = pgradz * pgradz;

    const double limiter = (xx * pgradx2 + yy * pgrady2 + zz * pgradz2 + xy * pgradx * pgrady +
                            xz * pgradx * pgradz + yz * pgrady * pgradz) /
                           fmax2(pgradx2 + pgrady2 + pgradz2, 1.0e-16);
    if (!(limiter > 0.0)) {
      pgradx = copysign(fmax2(1.0e-16, fabs(pgradx)), pgradx);
      pgrady = copysign(fmax2(1.0e-16, fabs(pgrady)), pgrady);
      pgradz = copysign(fmax2(1.0e-16, fabs(pgradz)), pgradz);
      const double pgrad = sqrt(pgradx * pgradx + pgrady * pgrady + pgradz * pgradz);
      const double xgrad = fabs(cdx * pgrad / pgradx);
      const double ygrad = fabs(cdy * pgrad / pgrady);
      const double zgrad = fabs(cdz * pgrad / pgradz);
      const double grad = fmin2(fmin2(xgrad, ygrad), zgrad);
      const double grad2 = grad * grad;
      q = 2.0 * L(density0, j, k, l) * grad2 * limiter * limiter;
    }
  }
  E(viscosity, j, k, l) = st<typename S::cs_t>(q);
}

// ---------------------------------------------------------------------------
// calc_dt_kernel.f90:102-149 with the minimum of :141-147 folded into an
// atomic minimum. Doubles are mapped to an order-preserving 64-bit key, so the
// atomic gives exactly the serial minimum; NaNs never win, as with .LT..

template <class S, class M>
__global__ void __launch_bounds__(BX * BY, 6) k_calc_dt(M m, GeomArrays ga,
    double g_small, double dtc_safe, double dtu_safe, double dtv_safe, double dtw_safe,
    double dtdiv_safe, const typename S::rho_t* __restrict__ density0,
    const typename S::cs_t* __restrict__ viscosity_a, const typename S::cs_t* __restrict__ soundspeed,
    const typename S::vel_t* __restrict__ xvel0, const typename S::vel_t* __restrict__ yvel0,
    const typename S::vel_t* __restrict__ zvel0, typename S::wk_t* __restrict__ dt_min,
    unsigned long long* __restrict__ min_key) {
  __shared__ unsigned long long wmin[BX * BY / 32];
  m.run([&](const Geom& g, const Tile& t) {
  const Box b = interior(g);
  const int j = b.j0 + t.x * BX + threadIdx.x;
  const int k = b.k0 + t.y * BY + threadIdx.y;
  const int l = b.l0 + t.z;
  unsigned long long key = ~0ull;
  if (j <= b.j1 && k <= b.k1) {
    const double m = fmin2(fmin2(GX(ga.celldx, j), GY(ga.celldy, k)), GZ(ga.celldz, l));
    const double ds = 1.0 / (m * m);
    const double ss = L(soundspeed, j, k, l);
    double cc = ss * ss;
    cc = cc + 2.0 * L(viscosity_a, j, k, l) / L(density0, j, k, l);
    double dtct = ds * cc;
    dtct = dtc_safe * 1.0 / fmax2(sqrt(dtct), g_small);

    const double vol = E(ga.volume, j, k, l);
    const double xa = E(ga.xarea, j, k, l);
    const double du1 = (L(xvel0, j, k, l) + L(xvel0, j, k + 1, l) + L(xvel0, j, k, l + 1) +
                        L(xvel0, j, k + 1, l + 1)) * xa;
    const double du2 = (L(xvel0, j + 1, k, l) + L(xvel0, j + 1, k + 1, l) +
                        L(xvel0, j + 1, k, l + 1) + L(xvel0, j + 1, k + 1, l + 1)) * xa;
    const double dtut = dtu_safe * 4.0 * vol / fmax2(fmax2(fabs(du1), fabs(du2)), 1.0e-5 * vol);

    const double ya = E(ga.yarea, j, k, l);
    const double dv1 = (L(yvel0, j, k, l) + L(yvel0, j + 1, k, l) + L(yvel0, j, k, l + 1) +
                        L(yvel0, j + 1, k, l + 1)) * ya;
    const double dv2 = (L(yvel0, j, k + 1, l) + L(yvel0, j + 1, k + 1, l) +
                        L(yvel0, j, k + 1, l + 1) + L(yvel0, j + 1, k + 1, l + 1)) * ya;
    const double dtvt = dtv_safe * 4.0 * vol / fmax2(fmax2(fabs(dv1), fabs(dv2)), 1.0e-5 * vol);

    const double za = E(ga.zarea, j, k, l);  // both z faces use zarea(j,k,l)
    const double dw1 = (L(zvel0, j, k, l) + L(zvel0, j, k + 1, l) + L(zvel0, j + 1, k, l) +
                        L(zvel0, j + 1, k + 1, l)) * za;
    const double dw2 = (L(zvel0, j, k, l + 1) + L(zvel0, j, k + 1, l + 1) +
                        L(zvel0, j + 1, k, l + 1) + L(zvel0, j + 1, k + 1, l + 1)) * za;
    const double dtwt = dtw_safe * 4.0 * vol / fmax2(fmax2(fabs(dw1), fabs(dw2)), 1.0e-5 * vol);

    const double div = du2 - du1 + dv2 - dv1 + dw2 - dw1;
    const double dtdivt = dtdiv_safe * 4.0 * vol / fmax2(vol * 1.0e-05, fabs(div));

    const double mn = fmin2(fmin2(fmin2(fmin2(dtct, dtut), dtvt), dtwt), dtdivt);
    if (dt_min) E(dt_min, j, k, l) = st<typename S::wk_t>(mn);
    if (!(mn != mn)) key = key_of(mn);
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
  });
}

// ---------------------------------------------------------------------------
// PdV_kernel.f90:72-166
template <class S>
__global__ void __launch_bounds__(BX * BY, 8) k_pdv(Geom g, Box b, int predict, double dt_val,
    const double* dt_ptr, GeomArrays ga, const typename S::rho_t* __restrict__ density0,
    typename S::rho_t* __restrict__ density1, const typename S::ene_t* __restrict__ energy0,
    typename S::ene_t* __restrict__ energy1, const typename S::cs_t* __restrict__ pressure,
    const typename S::cs_t* __restrict__ viscosity, const typename S::vel_t* __restrict__ xvel0,
    const typename S::vel_t* __restrict__ xvel1, const typename S::vel_t* __restrict__ yvel0,
    const typename S::vel_t* __restrict__ yvel1, const typename S::vel_t* __restrict__ zvel0,
    const typename S::vel_t* __restrict__ zvel1) {
  BOX_THREAD(b);
  const double dt = dt_of(dt_val, dt_ptr);
  // predictor: the second velocity set is vel0 again and the flux carries *0.5
  const typename S::vel_t* xb = predict ? xvel0 : xvel1;
  const typename S::vel_t* yb = predict ? yvel0 : yvel1;
  const typename S::vel_t* zb = predict ? zvel0 : zvel1;
#define XF(jj)                                                                            \
  (E(ga.xarea, jj, k, l) * (L(xvel0, jj, k, l) + L(xvel0, jj, k + 1, l) + L(xvel0, jj, k, l + 1) + \
                            L(xvel0, jj, k + 1, l + 1) + L(xb, jj, k, l) + L(xb, jj, k + 1, l) +   \
                            L(xb, jj, k, l + 1) + L(xb, jj, k + 1, l + 1)))
#define YF(kk)                                                                            \
  (E(ga.yarea, j, kk, l) * (L(yvel0, j, kk, l) + L(yvel0, j + 1, kk, l) + L(yvel0, j, kk, l + 1) + \
                            L(yvel0, j + 1, kk, l + 1) + L(yb, j, kk, l) + L(yb, j + 1, kk, l) +   \
                            L(yb, j, kk, l + 1) + L(yb, j + 1, kk, l + 1)))
#define ZF(ll)                                                                            \
  (E(ga.zarea, j, k, ll) * (L(zvel0, j, k, ll) + L(zvel0, j + 1, k, ll) + L(zvel0, j, k + 1, ll) + \
                            L(zvel0, j + 1, k + 1, ll) + L(zb, j, k, ll) + L(zb, j + 1, k, ll) +   \
                            L(zb, j, k + 1, ll) + L(zb, j + 1, k + 1, ll)))
  double left_flux, right_flux, bottom_flux, top_flux, back_flux, front_flux;
  if (predict) {
    left_flux = XF(j) * 0.125 * dt * 0.5;
    right_flux = XF(j + 1) * 0.125 * dt * 0.5;
    bottom_flux = YF(k) * 0.125 * dt * 0.5;
    top_flux = YF(k + 1) * 0.125 * dt * 0.5;
    back_flux = ZF(l) * 0.125 * dt * 0.5;
    front_flux = ZF(l + 1) * 0.125 * dt * 0.5;
  } else if (sizeof(typename S::vf_t) == 8) {
    left_flux = XF(j) * 0.125 * dt;
    right_flux = XF(j + 1) * 0.125 * dt;
    bottom_flux = YF(k) * 0.125 * dt;
    top_flux = YF(k + 1) * 0.125 * dt;
    back_flux = ZF(l) * 0.125 * dt;
    front_flux = ZF(l + 1) * 0.125 * dt;
  } else {
    // FP32 volume fluxes (mixed storage): the corrector's face fluxes as
    // k_flux_calc stores them (its expression and rounding; the z faces from
    // the corrector's own node sums), so that the advection's pre/post
    // volumes cancel against this volume change
    using F = typename S::vf_t;
#define XS(jj) (0.125 * dt * E(ga.xarea, jj, k, l) *                                              \
    (L(xvel0, jj, k, l) + L(xvel0, jj, k + 1, l) + L(xvel0, jj, k, l + 1) + L(xvel0, jj, k + 1, l + 1) + \
     L(xb, jj, k, l) + L(xb, jj, k + 1, l) + L(xb, jj, k, l + 1) + L(xb, jj, k + 1, l + 1)))
#define YS(kk) (0.125 * dt * E(ga.yarea, j, kk, l) *                                              \
    (L(yvel0, j, kk, l) + L(yvel0, j + 1, kk, l) + L(yvel0, j, kk, l + 1) + L(yvel0, j + 1, kk, l + 1) + \
     L(yb, j, kk, l) + L(yb, j + 1, kk, l) + L(yb, j, kk, l + 1) + L(yb, j + 1, kk, l + 1)))
#define ZS(ll) (0.125 * dt * E(ga.zarea, j, k, ll) *                                              \
    (L(zvel0, j, k, ll) + L(zvel0, j + 1, k, ll) + L(zvel0, j, k + 1, ll) + L(zvel0, j + 1, k + 1, ll) + \
     L(zb, j, k, ll) + L(zb, j + 1, k, ll) + L(zb, j, k + 1, ll) + L(zb, j + 1, k + 1, ll)))
    left_flux = (double)st<F>(XS(j));
    right_flux = (double)st<F>(XS(j + 1));
    bottom_flux = (double)st<F>(YS(k));
    top_flux = (double)st<F>(YS(k + 1));
    back_flux = (double)st<F>(ZS(l));
    front_flux = (double)st<F>(ZS(l + 1));
#undef XS
#undef YS
#undef ZS
  }
#undef XF
#undef YF
#undef ZF
  const double total_flux = right_flux - left_flux + top_flux - bottom_flux + front_flux - back_flux;
  const double vol = E(ga.volume, j, k, l);
  const double vol_change_s = div_rn(vol, vol + total_flux);
  const double recip_volume = div_rn(1.0, vol);
  const double d0 = L(density0, j, k, l);
  const double energy_change =
      quot_pair_sum(L(pressure, j, k, l), L(viscosity, j, k, l), d0) * total_flux * recip_volume;
  E(energy1, j, k, l) = st<typename S::ene_t>(L(energy0, j, k, l) - energy_change);
  E(density1, j, k, l) = st<typename S::rho_t>(d0 * vol_change_s);
}

// ---------------------------------------------------------------------------
// revert_kernel.f90:41-61
template <class S>
__global__ void __launch_bounds__(BX * BY) k_revert(Geom g, Box b,
    const typename S::rho_t* __restrict__ density0, typename S::rho_t* __restrict__ density1,
    const typename S::ene_t* __restrict__ energy0, typename S::ene_t* __restrict__ energy1) {
  BOX_THREAD(b);
  E(density1, j, k, l) = E(density0, j, k, l);
  E(energy1, j, k, l) = E(energy0, j, k, l);
}

// ---------------------------------------------------------------------------
// accelerate_kernel.f90:61-109. UM: the cell volume and face areas come from
// the chunk's uniform-mesh constants (Geom::vol, xa, ya, za) instead of the
// arrays.
template <class S, class M, bool UM>
__global__ void __launch_bounds__(BX * BY, UM ? 5 : 4) k_accelerate(M m, double dt_val,
    const double* dt_ptr, GeomArrays ga, const typename S::rho_t* __restrict__ density0,
    const typename S::cs_t* __restrict__ pressure, const typename S::cs_t* __restrict__ viscosity,
    const typename S::vel_t* __restrict__ xvel0, const typename S::vel_t* __restrict__ yvel0,
    const typename S::vel_t* __restrict__ zvel0, typename S::vel_t* __restrict__ xvel1,
    typename S::vel_t* __restrict__ yvel1, typename S::vel_t* __restrict__ zvel1) {
  m.run([&](const Geom& g, const Tile& t) {
  TILE_THREAD(nodes(g), t);
  const double dt = dt_ptr ? dt_ptr[(long long)t.d * kScalarStride] : dt_val;
#define DV(a, bb, c) (L(density0, j + (a), k + (bb), l + (c)) * (UM ? g.vol : E(ga.volume, j + (a), k + (bb), l + (c))))
  const double nodal_mass = (DV(-1, -1, 0) + DV(0, -1, 0) + DV(0, 0, 0) + DV(-1, 0, 0) +
                             DV(-1, -1, -1) + DV(0, -1, -1) + DV(0, 0, -1) + DV(-1, 0, -1)) * 0.125;
#undef DV
  const double stepbymass_d = 0.25 * dt / nodal_mass;
  // the pressure and viscosity gradients and the update in the policy's
  // arithmetic (FP64, or FP32 in the mixed path; the nodal mass stays FP64)
  using A = typename S::arith_t;
  const A stepbymass_s = (A)stepbymass_d;
  auto la = [](const auto* p) { return (A)__ldg(p); };
#define LA(a, jj, kk, ll) la(&E(a, jj, kk, ll))
  const A p000 = LA(pressure, j, k, l), p100 = LA(pressure, j - 1, k, l);
  const A p010 = LA(pressure, j, k - 1, l), p110 = LA(pressure, j - 1, k - 1, l);
  const A p001 = LA(pressure, j, k, l - 1), p101 = LA(pressure, j - 1, k, l - 1);
  const A p011 = LA(pressure, j, k - 1, l - 1), p111 = LA(pressure, j - 1, k - 1, l - 1);
  const A q000 = LA(viscosity, j, k, l), q100 = LA(viscosity, j - 1, k, l);
  const A q010 = LA(viscosity, j, k - 1, l), q110 = LA(viscosity, j - 1, k - 1, l);
  const A q001 = LA(viscosity, j, k, l - 1), q101 = LA(viscosity, j - 1, k, l - 1);
  const A q011 = LA(viscosity, j, k - 1, l - 1), q111 = LA(viscosity, j - 1, k - 1, l - 1);
#define AR(a, c, jj, kk, ll) (UM ? (A)g.c : LA(ga.a, jj, kk, ll))
  const A xa0 = AR(xarea, xa, j, k, l), xa1 = AR(xarea, xa, j, k - 1, l);
  const A xa2 = AR(xarea, xa, j, k, l - 1), xa3 = AR(xarea, xa, j, k - 1, l - 1);
  const A ya0 = AR(yarea, ya, j, k, l), ya1 = AR(yarea, ya, j - 1, k, l);
  const A ya2 = AR(yarea, ya, j, k, l - 1), ya3 = AR(yarea, ya, j - 1, k, l - 1);
  const A za0 = AR(zarea, za, j, k, l), za1 = AR(zarea, za, j, k - 1, l);
  const A za2 = AR(zarea, za, j - 1, k, l), za3 = AR(zarea, za, j - 1, k - 1, l);
#undef AR

  const A xvel1_s = LA(xvel0, j, k, l) -
      stepbymass_s * (xa0 * (p000 - p100) + xa1 * (p010 - p110) + xa2 * (p001 - p101) +
                      xa3 * (p011 - p111));
  const A yvel1_s = LA(yvel0, j, k, l) -
      stepbymass_s * (ya0 * (p000 - p010) + ya1 * (p100 - p110) + ya2 * (p001 - p011) +
                      ya3 * (p101 - p111));
  const A zvel1_s = LA(zvel0, j, k, l) -
      stepbymass_s * (za0 * (p000 - p001) + za1 * (p010 - p011) + za2 * (p100 - p101) +
                      za3 * (p110 - p111));
#undef LA
  using V = typename S::vel_t;
  E(xvel1, j, k, l) = st<V>(xvel1_s -
      stepbymass_s * (xa0 * (q000 - q100) + xa1 * (q010 - q110) + xa2 * (q001 - q101) +
                      xa3 * (q011 - q111)));
  E(yvel1, j, k, l) = st<V>(yvel1_s -
      stepbymass_s * (ya0 * (q000 - q010) + ya1 * (q100 - q110) + ya2 * (q001 - q011) +
                      ya3 * (q101 - q111)));
  E(zvel1, j, k, l) = st<V>(zvel1_s -
      stepbymass_s * (za0 * (q000 - q001) + za1 * (q010 - q011) + za2 * (q100 - q101) +
                      za3 * (q110 - q111)));
  });
}

// ---------------------------------------------------------------------------
// flux_calc_kernel.f90:58-91: one launch over the union of the three face
// ranges. The z sum repeats zvel0(j+1,k,l) and omits zvel0(j,k+1,l) (:86).
template <class S>
__global__ void __launch_bounds__(BX * BY) k_flux_calc(Geom g, Box b, double dt_val,
    const double* dt_ptr, GeomArrays ga, const typename S::vel_t* __restrict__ xvel0,
    const typename S::vel_t* __restrict__ yvel0, const typename S::vel_t* __restrict__ zvel0,
    const typename S::vel_t* __restrict__ xvel1, const typename S::vel_t* __restrict__ yvel1,
    const typename S::vel_t* __restrict__ zvel1, typename S::vf_t* __restrict__ vol_flux_x,
    typename S::vf_t* __restrict__ vol_flux_y, typename S::vf_t* __restrict__ vol_flux_z) {
  BOX_THREAD(b);
  const double dt = dt_of(dt_val, dt_ptr);
  using F = typename S::vf_t;
  const bool jin = j <= g.x_max, kin = k <= g.y_max, lin = l <= g.z_max;
  if (kin && lin)
    E(vol_flux_x, j, k, l) = st<F>(0.125 * dt * E(ga.xarea, j, k, l) *
        (L(xvel0, j, k, l) + L(xvel0, j, k + 1, l) + L(xvel0, j, k, l + 1) + L(xvel0, j, k + 1, l + 1) +
         L(xvel1, j, k, l) + L(xvel1, j, k + 1, l) + L(xvel1, j, k, l + 1) + L(xvel1, j, k + 1, l + 1)));
  if (jin && lin)
    E(vol_flux_y, j, k, l) = st<F>(0.125 * dt * E(ga.yarea, j, k, l) *
        (L(yvel0, j, k, l) + L(yvel0, j + 1, k, l) + L(yvel0, j, k, l + 1) + L(yvel0, j + 1, k, l + 1) +
         L(yvel1, j, k, l) + L(yvel1, j + 1, k, l) + L(yvel1, j, k, l + 1) + L(yvel1, j + 1, k, l + 1)));
  if (jin && kin)
    E(vol_flux_z, j, k, l) = st<F>(0.125 * dt * E(ga.zarea, j, k, l) *
        (L(zvel0, j, k, l) + L(zvel0, j + 1, k, l) + L(zvel0, j + 1, k, l) + L(zvel0, j + 1, k + 1, l) +
         L(zvel1, j, k, l) + L(zvel1, j + 1, k, l) + L(zvel1, j, k + 1, l) + L(zvel1, j + 1, k + 1, l)));
}

// ---------------------------------------------------------------------------
// advec_cell_kernel.f90: pre/post volume pass (:97-121, :190-216, :287-311)
template <class S>
__global__ void __launch_bounds__(BX * BY) k_cell_vol(Geom g, Box b, int variant, GeomArrays ga,
    const typename S::vf_t* __restrict__ vfx, const typename S::vf_t* __restrict__ vfy,
    const typename S::vf_t* __restrict__ vfz, typename S::wk_t* __restrict__ pre_vol,
    typename S::wk_t* __restrict__ post_vol) {
  BOX_THREAD(b);
  const double vol = E(ga.volume, j, k, l);
  const double fx1 = L(vfx, j + 1, k, l), fx0 = L(vfx, j, k, l);
  const double fy1 = L(vfy, j, k + 1, l), fy0 = L(vfy, j, k, l);
  const double fz1 = L(vfz, j, k, l + 1), fz0 = L(vfz, j, k, l);
  double pre, post;
  switch (variant) {
    case 0:  // x, sweep 1
      pre = vol + (fx1 - fx0 + fy1 - fy0 + fz1 - fz0);
      post = pre - (fx1 - fx0);
      break;
    case 1:  // x, sweep 3
      pre = vol + fx1 - fx0;
      post = vol;
      break;
    case 2:  // y, sweep 2, advect_x
      pre = vol + fy1 - fy0 + fz1 - fz0;
      post = pre - (fy1 - fy0);
      break;
    case 3:  // y, sweep 2, not advect_x
      pre = vol + fy1 - fy0 + fx1 - fx0;
      post = pre - (fy1 - fy0);
      break;
    case 4:  // z, sweep 1
      pre = vol + (fx1 - fx0 + fy1 - fy0 + fz1 - fz0);
      post = pre - (fz1 - fz0);
      break;
    default:  // z, sweep 3
      pre = vol + fz1 - fz0;
      post = vol;
      break;
  }
  using W = typename S::wk_t;
  E(pre_vol, j, k, l) = st<W>(pre);
  E(post_vol, j, k, l) = st<W>(post);
}

__device__ __forceinline__ double cell_limiter(double sig, double sigma3, double sigma4,
                                               double diffuw, double diffdw) {
  const double one_by_six = 1.0 / 6.0;
  if (diffuw * diffdw > 0.0)
    return (1.0 - sig) * copysign(1.0, diffdw) *
           fmin2(fmin2(fabs(diffuw), fabs(diffdw)),
                 one_by_six * (sigma3 * fabs(diffuw) + sigma4 * fabs(diffdw)));
  return 0.0;
}

// Warp-row helpers of the x sweeps: lane m holds element b+m of a row chunk
// (cur), b+32+m (nxt) and b-32+m (prv).
constexpr unsigned kFull = 0xffffffffu;

// element b+m+s of the row (s = 1, 2): lanes past 31 read the next chunk
__device__ __forceinline__ double row_dn(double cur, double nxt, int s) {
  const int m = threadIdx.x & 31;
  return __shfl_sync(kFull, m >= s ? cur : nxt, (m + s) & 31);
}
// element b+m-1: lane 0 reads the previous chunk's last
__device__ __forceinline__ double row_up(double cur, double prv) {
  const int m = threadIdx.x & 31;
  return __shfl_sync(kFull, m == 31 ? prv : cur, (m + 31) & 31);
}

// A loaded element of an array the kernel also writes (a plain load: the
// read-only path is for arrays nobody writes during the launch).
template <class T>
__device__ __forceinline__ double ldw(const T* p) { return (double)*p; }

// Per-thread prefetch rings of the line marches: each thread copies the
// elements it will need kLineRing - 1 steps ahead into its own shared-memory
// slots with cp.async (one commit group per step) and reads back only its own
// slots after its own cp.async.wait_group, so no barrier orders them. A copy
// whose element is not wanted zero-fills its slot without reading memory.
constexpr int kLineRing = 4;
constexpr int kLineStreams = 4;
constexpr int kLineSlots = kLineRing * kLineStreams * BX * BY;  // doubles per block

template <class T>
__device__ __forceinline__ void cp_elem(double* slot, const T* src, bool want) {
  const unsigned d = (unsigned)__cvta_generic_to_shared(slot);
  asm volatile("cp.async.ca.shared.global [%0], [%1], %2, %3;\n" ::"r"(d), "l"(src),
               "n"((int)sizeof(T)), "r"(want ? (int)sizeof(T) : 0)
               : "memory");
}
__device__ __forceinline__ void cp_commit() { asm volatile("cp.async.commit_group;\n" ::: "memory"); }
__device__ __forceinline__ void cp_wait_step() {
  asm volatile("cp.async.wait_group %0;\n" ::"n"(kLineRing - 1) : "memory");
}
__device__ __forceinline__ void cp_wait_all() { asm volatile("cp.async.wait_group 0;\n" ::: "memory"); }
template <class T>
__device__ __forceinline__ double slot_val(const double* slot) {
  return (double)*(const volatile T*)slot;
}
// this thread's slot of stream q for step t
__device__ __forceinline__ double* line_slot(double* ring, int t, int q) {
  return ring + ((t & (kLineRing - 1)) * kLineStreams + q) * (BX * BY) + threadIdx.y * BX + threadIdx.x;
}

// The fluxes at one face of a cell sweep (advec_cell_kernel.f90:125-171 x,
// :220-266 y, :315-361 z), from the cells' old values: du/dd/dw (density) and
// eu/ed/ew (energy) at the upwind, donor and downwind cells, pvd the donor's
// pre_vol, rw = vertexd(i) / vertexd(dif). mf and ef are the mass and energy
// fluxes as formed (the energy flux takes the mass flux before storage).
__device__ __forceinline__ void cell_face_flux(double vf, double pvd, double rw, double du,
                                               double dd, double dw, double eu, double ed,
                                               double ew, double& mf, double& ef) {
  const double sigmat = div_rn(fabs(vf), pvd);
  const double sigma3 = (1.0 + sigmat) * rw;
  const double sigma4 = 2.0 - sigmat;
  double limiter = cell_limiter(sigmat, sigma3, sigma4, dd - du, dw - dd);
  mf = vf * (dd + limiter);
  const double sigmam = div_rn(fabs(mf), dd * pvd);
  limiter = cell_limiter(sigmam, sigma3, sigma4, ed - eu, ew - ed);
  ef = mf * (ed + limiter);
}

// The cell update (advec_cell_kernel.f90:175-186 x, :270-281 y, :365-376 z) of
// a cell with old density d, energy e, pre_vol pv, from the stored fluxes at
// its low (ml, el, vl) and high (mh, eh, vh) faces.
template <class S>
__device__ __forceinline__ void cell_update(long long at, double d, double e, double pv,
                                            double ml, double mh, double el, double eh,
                                            double vl, double vh,
                                            typename S::rho_t* __restrict__ density1,
                                            typename S::ene_t* __restrict__ energy1,
                                            typename S::wk_t* __restrict__ pre_mass,
                                            typename S::wk_t* __restrict__ post_mass,
                                            typename S::wk_t* __restrict__ advec_vol,
                                            typename S::wk_t* __restrict__ post_ener) {
  const double pm = d * pv;
  const double pom = pm + ml - mh;
  const double poe = (e * pm + el - eh) / pom;
  const double av = pv + vl - vh;
  using W = typename S::wk_t;
  if (pre_mass) {
    pre_mass[at] = st<W>(pm);
    post_mass[at] = st<W>(pom);
    post_ener[at] = st<W>(poe);
    advec_vol[at] = st<W>(av);
  }
  density1[at] = st<typename S::rho_t>(pom / av);
  energy1[at] = st<typename S::ene_t>(poe);
}

// The x cell sweep, flux pass and update in one: a warp per (k, l) row of the
// interior marches along x in chunks of 32 cells. Lane m of the chunk at b
// holds the old values of cell b+m, forms the fluxes at face b+m+1 (faces
// x_min..x_max+2) and updates cell b+m from them and the fluxes lane m-1
// formed at face b+m (lane 0: lane 31 of the previous chunk). A face reads
// cells b+m-1 .. b+m+2, all held in registers (this chunk, the next, and the
// previous chunk's last), and the next chunks are loaded before this one is
// written: density1 and energy1 are updated in place and no element is read
// after it has been written.
template <class S>
__global__ void __launch_bounds__(BX * BY, 3) k_cell_line_x(Geom g, GeomArrays ga,
    typename S::rho_t* __restrict__ density1, typename S::ene_t* __restrict__ energy1,
    const typename S::vf_t* __restrict__ vol_flux, typename S::mf_t* __restrict__ mass_flux,
    const typename S::wk_t* __restrict__ pre_vol, typename S::wk_t* __restrict__ pre_mass,
    typename S::wk_t* __restrict__ post_mass, typename S::wk_t* __restrict__ advec_vol,
    typename S::wk_t* __restrict__ post_ener, typename S::wk_t* __restrict__ ener_flux) {
  __shared__ double ring[kLineSlots];
  const int k = g.y_min + blockIdx.x * BY + threadIdx.y;
  const int l = g.z_min + blockIdx.y;
  if (k > g.y_max) return;  // the warp's row: every lane leaves together
  const int m = threadIdx.x;
  const int x0 = g.x_min, x1 = g.x_max;
  const long long row = off3(g, 0, k, l);  // element j of the row at row + j
  const double* vd = ga.vertexdx + g.o1 + 2 - x0;
  auto in_row = [&](int j) { return j >= x0 - 2 && j <= x1 + 2; };
  auto lw = [&](const auto* a, int j) { return in_row(j) ? ldw(a + row + j) : 0.0; };
  auto lr = [&](const auto* a, int j) { return in_row(j) ? ld(a + row + j) : 0.0; };
  // step t marches the chunk at b = x0-32+32t; its ring entry is the chunk
  // two ahead (b+64), copied kLineRing-1 steps before it is shifted in
  const int steps = (x1 + 1 - (x0 - 32)) / 32 + 1;
  auto issue = [&](int t) {
    const int j = x0 + 32 + 32 * t + m;
    const bool want = t < steps && in_row(j);
    const long long at = row + (want ? j : x0);
    cp_elem(line_slot(ring, t, 0), density1 + at, want);
    cp_elem(line_slot(ring, t, 1), energy1 + at, want);
    cp_elem(line_slot(ring, t, 2), pre_vol + at, want);
    cp_elem(line_slot(ring, t, 3), vol_flux + at, want);
    cp_commit();
  };
  for (int t = 0; t < kLineRing - 1; t++) issue(t);
  int b = x0 - 32;
  double dp = 0.0, dc = lw(density1, b + m), dn = lw(density1, b + 32 + m);
  double ep = 0.0, ec = lw(energy1, b + m), en = lw(energy1, b + 32 + m);
  double pc = lr(pre_vol, b + m), pn = lr(pre_vol, b + 32 + m);
  double fc = lr(vol_flux, b + m), fn = lr(vol_flux, b + 32 + m);
  double m_last = 0.0, e_last = 0.0;  // this lane's stored fluxes of the previous chunk
  for (int t = 0; t < steps; t++, b += 32) {
    issue(t + kLineRing - 1);
    cp_wait_step();
    const double dnn = slot_val<typename S::rho_t>(line_slot(ring, t, 0));
    const double enn = slot_val<typename S::ene_t>(line_slot(ring, t, 1));
    const double pnn = slot_val<typename S::wk_t>(line_slot(ring, t, 2));
    const double fnn = slot_val<typename S::vf_t>(line_slot(ring, t, 3));
    const int c = b + m, i = c + 1;  // this lane's cell and face
    const double da = row_up(dc, dp), d1 = row_dn(dc, dn, 1), d2 = row_dn(dc, dn, 2);
    const double ea = row_up(ec, ep), e1 = row_dn(ec, en, 1), e2 = row_dn(ec, en, 2);
    const double vf = row_dn(fc, fn, 1), pv1 = row_dn(pc, pn, 1);
    double mflux = 0.0, eflux = 0.0;
    if (i >= x0 && i <= x1 + 2) {
      // vf > 0: upwind i-2, donor i-1, downwind i; else upwind MIN(i+1, x_max+2),
      // donor i, downwind i-1 (the donor's vertexdx over the upwind's)
      const bool pos = vf > 0.0, clamp = i + 1 > x1 + 2;
      const int dif = pos ? i - 1 : (clamp ? x1 + 2 : i + 1);
      double mf, ef;
      cell_face_flux(vf, pos ? pc : pv1, vd[i] / vd[dif], pos ? da : (clamp ? d1 : d2),
                     pos ? dc : d1, pos ? d1 : dc, pos ? ea : (clamp ? e1 : e2), pos ? ec : e1,
                     pos ? e1 : ec, mf, ef);
      const typename S::mf_t ms = st<typename S::mf_t>(mf);
      const typename S::wk_t es = st<typename S::wk_t>(ef);
      mass_flux[row + i] = ms;
      ener_flux[row + i] = es;
      mflux = (double)ms;
      eflux = (double)es;
    }
    const double ml = row_up(mflux, m_last), el = row_up(eflux, e_last);
    if (c >= x0 && c <= x1)
      cell_update<S>(row + c, dc, ec, pc, ml, mflux, el, eflux, fc, vf, density1, energy1,
                     pre_mass, post_mass, advec_vol, post_ener);
    m_last = mflux;
    e_last = eflux;
    dp = dc; dc = dn; dn = dnn;
    ep = ec; ec = en; en = enn;
    pc = pn; pn = pnn;
    fc = fn; fn = fnn;
  }
  cp_wait_all();
}

// The y or z cell sweep (DIR 2 or 3), flux pass and update in one. A block
// holds 32 columns along the sweep axis (consecutive in x, then in the other
// index: l for y, over z_min..z_max+2 as the reference's y flux range, k for
// z) and splits the faces min..max+2 into one segment per warp.
// A warp marches its segment face by face with the old cells i-2..i+1 in
// registers, stores the fluxes at face i and updates cell i-1. Before the
// block's barrier each warp reads the old cells it needs that the
// neighbouring segments will overwrite: the first window (cells f0-3..f0,
// starting with the face f0-1 below its segment, formed again and not stored)
// and cells f1 and f1+1 above its last face f1. After the barrier a warp
// writes only its own cells and reads from memory only its own cells not yet
// written, so the update is in place.
template <class S, int DIR>
__global__ void __launch_bounds__(BX * BY, 3) k_cell_line_yz(Geom g, GeomArrays ga,
    typename S::rho_t* __restrict__ density1, typename S::ene_t* __restrict__ energy1,
    const typename S::vf_t* __restrict__ vol_flux, typename S::mf_t* __restrict__ mass_flux,
    const typename S::wk_t* __restrict__ pre_vol, typename S::wk_t* __restrict__ pre_mass,
    typename S::wk_t* __restrict__ post_mass, typename S::wk_t* __restrict__ advec_vol,
    typename S::wk_t* __restrict__ post_ener, typename S::wk_t* __restrict__ ener_flux) {
  __shared__ double ring[kLineSlots];
  // columns (j, o) numbered j fastest: lane x of block b holds column 32b+x
  const int nj = g.x_max - g.x_min + 1;
  const int no = DIR == 2 ? g.z_max + 3 - g.z_min : g.y_max + 1 - g.y_min;
  const int col = blockIdx.x * BX + threadIdx.x;
  const int j = g.x_min + col % nj;
  const int o = (DIR == 2 ? g.z_min : g.y_min) + col / nj;
  const int imin = DIR == 2 ? g.y_min : g.z_min, imax = DIR == 2 ? g.y_max : g.z_max;
  const int top = imax + 2;  // last face, and last cell a face reads
  // faces imin..top in BY segments
  const int per = (top - imin + BY) / BY;
  const int f0 = imin + (int)threadIdx.y * per;
  const int f1 = f0 + per - 1 < top ? f0 + per - 1 : top;
  const bool act = col < nj * no && f0 <= f1;
  const bool upd = DIR == 3 || o <= g.z_max;  // the y sweep's planes z_max+1, z_max+2: fluxes only
  const long long step = DIR == 2 ? g.px : g.pxy;
  const long long base = DIR == 2 ? off3(g, j, 0, o) : off3(g, j, o, 0);  // + i * step
  const double* vd = (DIR == 2 ? ga.vertexdy : ga.vertexdz) + g.o1 + 2 - imin;
  const int i0 = f0 > imin ? f0 - 1 : f0;  // first face formed
  const int steps = f1 - i0 + 1;
  // cells f1 and MIN(f1+1, top) above the segment (the next segment's), read
  // before the barrier and kept in shared memory until the segment's end
  __shared__ double edge[4][BX * BY];
  const int me = threadIdx.y * BX + threadIdx.x;
  // step t (face i = i0+t) shifts in cell MIN(i+2, top) (below f1; the cells
  // at and above f1 come from the pre-read pair), pre_vol and vol_flux at
  // i+1; ia is the element offset of face i0+ti, the next step to issue
  int ti = 0;
  long long ia = base + i0 * step;
  auto issue = [&]() {
    const int i = i0 + ti;
    const bool wc = ti < steps && i + 2 < f1, wf = ti < steps && i < f1;
    const long long ac = wc ? ia + 2 * step : base, af = wf ? ia + step : base;
    double* sl = line_slot(ring, ti, 0);
    cp_elem(sl, density1 + ac, wc);
    cp_elem(sl + BX * BY, energy1 + ac, wc);
    cp_elem(sl + 2 * BX * BY, pre_vol + af, wf);
    cp_elem(sl + 3 * BX * BY, vol_flux + af, wf);
    cp_commit();
    ia += step;
    ti++;
  };
  double d0 = 0, d1 = 0, d2 = 0, d3 = 0, e0 = 0, e1 = 0, e2 = 0, e3 = 0;  // cells i-2..i+1
  if (act) {
    for (int t = 0; t < kLineRing - 1; t++) issue();
    const int c3 = i0 + 1 < top ? i0 + 1 : top;
    d0 = ldw(density1 + base + (i0 - 2) * step); e0 = ldw(energy1 + base + (i0 - 2) * step);
    d1 = ldw(density1 + base + (i0 - 1) * step); e1 = ldw(energy1 + base + (i0 - 1) * step);
    d2 = ldw(density1 + base + i0 * step);       e2 = ldw(energy1 + base + i0 * step);
    d3 = ldw(density1 + base + c3 * step);       e3 = ldw(energy1 + base + c3 * step);
    const int r1 = f1 + 1 < top ? f1 + 1 : top;
    edge[0][me] = ldw(density1 + base + f1 * step);
    edge[1][me] = ldw(density1 + base + r1 * step);
    edge[2][me] = ldw(energy1 + base + f1 * step);
    edge[3][me] = ldw(energy1 + base + r1 * step);
  }
  __syncthreads();
  if (!act) return;
  double p0 = ld(pre_vol + base + (i0 - 1) * step), p1 = ld(pre_vol + base + i0 * step);
  double v0 = ld(vol_flux + base + (i0 - 1) * step), v1 = ld(vol_flux + base + i0 * step);
  // vertex widths at i-1, i and MIN(i+1, top)
  double xm = vd[i0 - 1], xc = vd[i0], xp = vd[i0 + 1 < top ? i0 + 1 : top];
  long long at = base + i0 * step;  // face i
  double m_last = 0.0, e_last = 0.0;  // stored fluxes at face i-1
  for (int t = 0; t < steps; t++) {
    issue();
    const int i = i0 + t, cn = i + 2 < top ? i + 2 : top;
    const double xn = vd[cn];
    cp_wait_step();
    const double* sl = line_slot(ring, t, 0);
    // (at the segment's last face cn may be f1+2: that shift-in is never used)
    const int eg = cn > f1 ? 1 : 0;
    const double dn = cn < f1 ? slot_val<typename S::rho_t>(sl) : edge[eg][me];
    const double en = cn < f1 ? slot_val<typename S::ene_t>(sl + BX * BY) : edge[2 + eg][me];
    const double pn = slot_val<typename S::wk_t>(sl + 2 * BX * BY);
    const double vn = slot_val<typename S::vf_t>(sl + 3 * BX * BY);
    // face i: cells d0 (i-2), d1 (i-1), d2 (i), d3 (MIN(i+1, top)); the
    // donor's width over the upwind's: i-1 for v > 0, else MIN(i+1, top)
    const bool pos = v1 > 0.0;
    double mf, ef;
    cell_face_flux(v1, pos ? p0 : p1, xc / (pos ? xm : xp), pos ? d0 : d3, pos ? d1 : d2,
                   pos ? d2 : d1, pos ? e0 : e3, pos ? e1 : e2, pos ? e2 : e1, mf, ef);
    const typename S::mf_t ms = st<typename S::mf_t>(mf);
    const typename S::wk_t es = st<typename S::wk_t>(ef);
    if (i >= f0) {
      mass_flux[at] = ms;
      ener_flux[at] = es;
    }
    const int c = i - 1;
    if (upd && i > i0 && c >= imin && c <= imax)
      cell_update<S>(at - step, d1, e1, p0, m_last, (double)ms, e_last, (double)es, v0, v1,
                     density1, energy1, pre_mass, post_mass, advec_vol, post_ener);
    m_last = (double)ms;
    e_last = (double)es;
    d0 = d1; d1 = d2; d2 = d3; d3 = dn;
    e0 = e1; e1 = e2; e2 = e3; e3 = en;
    p0 = p1; p1 = pn;
    v0 = v1; v1 = vn;
    xm = xc; xc = xp; xp = xn;
    at += step;
  }
  cp_wait_all();
}

// ---------------------------------------------------------------------------
// advec_mom_kernel.f90 pre/post volume variants (:95-163)
template <class S>
__global__ void __launch_bounds__(BX * BY) k_mom_vol(Geom g, Box b, int variant, GeomArrays ga,
    const typename S::vf_t* __restrict__ vfx, const typename S::vf_t* __restrict__ vfy,
    const typename S::vf_t* __restrict__ vfz, typename S::wk_t* __restrict__ pre_vol,
    typename S::wk_t* __restrict__ post_vol) {
  BOX_THREAD(b);
  const double vol = E(ga.volume, j, k, l);
  const double fx1 = L(vfx, j + 1, k, l), fx0 = L(vfx, j, k, l);
  const double fy1 = L(vfy, j, k + 1, l), fy0 = L(vfy, j, k, l);
  const double fz1 = L(vfz, j, k, l + 1), fz0 = L(vfz, j, k, l);
  double post, pre;
  switch (variant) {
    case 0:  // sweep 1, direction x
      post = vol + fy1 - fy0 + fz1 - fz0;
      pre = post + fx1 - fx0;
      break;
    case 1:  // sweep 1, direction z
      post = vol + fx1 - fx0 + fy1 - fy0;
      pre = post + fz1 - fz0;
      break;
    case 2:  // sweep 2, advect_x
      post = vol + fz1 - fz0;
      pre = post + fy1 - fy0;
      break;
    case 3:  // sweep 2, not advect_x
      post = vol + fx1 - fx0;
      pre = post + fy1 - fy0;
      break;
    case 4:  // sweep 3, direction x
      post = vol;
      pre = post + fx1 - fx0;
      break;
    default:  // sweep 3, direction z
      post = vol;
      pre = post + fz1 - fz0;
      break;
  }
  using W = typename S::wk_t;
  E(post_vol, j, k, l) = st<W>(post);
  E(pre_vol, j, k, l) = st<W>(pre);
}

// node_flux (:166-176 x, :254-263 y, :339-349 z), node_mass_post
// (:177-193, :264-279, :350-365) and node_mass_pre (:194-202, :280-288,
// :366-374) over the union of their ranges, one pass: a node of the mass
// range forms the node flux of its lower neighbour along the sweep again (the
// same sum, so the same bits) for its node_mass_pre.
template <class S, int DIR>
__device__ __forceinline__ double node_flux_at(const Geom& g, const typename S::mf_t* __restrict__ mf,
                                               int j, int k, int l) {
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

template <class S, int DIR>
__global__ void __launch_bounds__(BX * BY) k_mom_node(Geom g, Box b, Box bflux, Box bmass,
    const typename S::mf_t* __restrict__ mf, const typename S::rho_t* __restrict__ density1,
    const typename S::wk_t* __restrict__ post_vol, typename S::wk_t* __restrict__ node_flux,
    typename S::wk_t* __restrict__ node_mass_post, typename S::wk_t* __restrict__ node_mass_pre) {
  BOX_THREAD(b);
  using W = typename S::wk_t;
  const bool in_flux = j >= bflux.j0 && j <= bflux.j1 && k >= bflux.k0 && k <= bflux.k1 &&
                       l >= bflux.l0 && l <= bflux.l1;
  const bool in_mass = j >= bmass.j0 && j <= bmass.j1 && k >= bmass.k0 && k <= bmass.k1 &&
                       l >= bmass.l0 && l <= bmass.l1;
  double nf = 0.0;
  if (in_flux || in_mass) {
    nf = (double)st<W>(node_flux_at<S, DIR>(g, mf, j, k, l));
    if (in_flux) E(node_flux, j, k, l) = st<W>(nf);
  }
  if (in_mass) {
#define DP(a, bb, c) (L(density1, j + (a), k + (bb), l + (c)) * L(post_vol, j + (a), k + (bb), l + (c)))
    const double nm = (double)st<W>(0.125 * (DP(0, -1, 0) + DP(0, 0, 0) + DP(-1, -1, 0) + DP(-1, 0, 0) +
                                             DP(0, -1, -1) + DP(0, 0, -1) + DP(-1, -1, -1) + DP(-1, 0, -1)));
#undef DP
    E(node_mass_post, j, k, l) = st<W>(nm);
    // the lower neighbour's node flux (inside the flux range for every mass node)
    const double prev = (double)st<W>(DIR == 1 ? node_flux_at<S, DIR>(g, mf, j - 1, k, l)
                                      : DIR == 2 ? node_flux_at<S, DIR>(g, mf, j, k - 1, l)
                                                 : node_flux_at<S, DIR>(g, mf, j, k, l - 1));
    E(node_mass_pre, j, k, l) = st<W>(nm - prev + nf);
  }
}

__device__ __forceinline__ double mom_limiter(double sigma, double width, double celld_dif,
                                              double vdiffuw, double vdiffdw) {
  double limiter = 0.0;
  if (vdiffuw * vdiffdw > 0.0) {
    const double auw = fabs(vdiffuw);
    const double adw = fabs(vdiffdw);
    double wind = 1.0;
    if (vdiffdw <= 0.0) wind = -1.0;
    // ... / 6.0_8 correctly rounded by div6 (clover_div.cuh)
    limiter = wind * fmin2(fmin2(div6(width * ((2.0 - sigma) * adw / width +
                                               (1.0 + sigma) * auw / celld_dif)),
                                 auw),
                           adw);
  }
  return limiter;
}

// The momentum flux at node i (advec_mom_kernel.f90:211-242 x, :295-327 y,
// :381-413 z) from the old velocities vm1, v0, vp1, vp2 at i-1..i+2, the node
// flux nf, node_mass_pre at i and i+1, and the cell widths cd at i-1, i, i+1.
__device__ __forceinline__ double mom_node_flux(double nf, double vm1, double v0, double vp1,
                                                double vp2, double nmp0, double nmp1, double cdm,
                                                double cd0, double cdp) {
  // nf < 0: upwind i+2, donor i+1, downwind i (width of the donor);
  // else upwind i-1, donor i, downwind i+1 (width of the upwind)
  const bool neg = nf < 0.0;
  const double v_donor = neg ? vp1 : v0;
  const double sigma = div_rn(fabs(nf), neg ? nmp1 : nmp0);
  const double vdiffuw = v_donor - (neg ? vp2 : vm1);
  const double vdiffdw = (neg ? v0 : vp1) - v_donor;
  const double limiter = mom_limiter(sigma, cd0, neg ? cdp : cdm, vdiffuw, vdiffdw);
  const double advec_vel_s = v_donor + (1.0 - sigma) * limiter;
  return advec_vel_s * nf;
}

// The x momentum flux and velocity update of one velocity in one pass: a warp
// per (k, l) node row (nodes y_min..y_max+1, z_min..z_max+1) marches along x
// in chunks of 32 nodes. Lane m of the chunk at b forms the flux at node b+m
// (nodes x_min-1..x_max+1) from the old velocities b+m-1..b+m+2 held in
// registers (this chunk, the next and the previous chunk's last) and updates
// node b+m (x_min..x_max+1) with the flux lane m-1 formed (lane 0: lane 31 of
// the previous chunk); the velocity is updated in place.
template <class S>
__global__ void __launch_bounds__(BX * BY, 4) k_mom_line_x(Geom g, GeomArrays ga,
    typename S::vel_t* __restrict__ vel1, const typename S::wk_t* __restrict__ node_flux,
    const typename S::wk_t* __restrict__ node_mass_pre,
    const typename S::wk_t* __restrict__ node_mass_post, typename S::wk_t* __restrict__ mom_flux) {
  __shared__ double ring[kLineSlots];
  const int k = g.y_min + blockIdx.x * BY + threadIdx.y;
  const int l = g.z_min + blockIdx.y;
  if (k > g.y_max + 1) return;  // the warp's row: every lane leaves together
  const int m = threadIdx.x;
  const int x0 = g.x_min, x1 = g.x_max;
  const long long row = off3(g, 0, k, l);
  const double* cd = ga.celldx + g.o1 + 2 - x0;
  auto in_row = [&](int j) { return j >= x0 - 2 && j <= x1 + 3; };
  auto lw = [&](const auto* a, int j) { return in_row(j) ? ldw(a + row + j) : 0.0; };
  auto lr = [&](const auto* a, int j) { return in_row(j) ? ld(a + row + j) : 0.0; };
  // step t marches the chunk at b = x0-32+32t: its ring entries are the
  // velocity and node_mass_pre two chunks ahead (b+64) and the node flux and
  // node_mass_post of the chunk itself
  const int steps = (x1 + 1 - (x0 - 32)) / 32 + 1;
  auto issue = [&](int t) {
    const int ja = x0 + 32 + 32 * t + m, jc = x0 - 32 + 32 * t + m;
    const bool wa = t < steps && in_row(ja), wc = t < steps && in_row(jc);
    const long long aa = row + (wa ? ja : x0), ac = row + (wc ? jc : x0);
    cp_elem(line_slot(ring, t, 0), vel1 + aa, wa);
    cp_elem(line_slot(ring, t, 1), node_mass_pre + aa, wa);
    cp_elem(line_slot(ring, t, 2), node_flux + ac, wc);
    cp_elem(line_slot(ring, t, 3), node_mass_post + ac, wc);
    cp_commit();
  };
  for (int t = 0; t < kLineRing - 1; t++) issue(t);
  int b = x0 - 32;
  double vp = 0.0, vc = lw(vel1, b + m), vn = lw(vel1, b + 32 + m);
  double qc = lr(node_mass_pre, b + m), qn = lr(node_mass_pre, b + 32 + m);
  double f_last = 0.0;  // this lane's stored flux of the previous chunk
  for (int t = 0; t < steps; t++, b += 32) {
    issue(t + kLineRing - 1);
    cp_wait_step();
    const double vnn = slot_val<typename S::vel_t>(line_slot(ring, t, 0));
    const double qnn = slot_val<typename S::wk_t>(line_slot(ring, t, 1));
    const double nf = slot_val<typename S::wk_t>(line_slot(ring, t, 2));
    const double post = slot_val<typename S::wk_t>(line_slot(ring, t, 3));
    const int i = b + m;
    const double vm1 = row_up(vc, vp), vp1 = row_dn(vc, vn, 1), vp2 = row_dn(vc, vn, 2);
    const double q1 = row_dn(qc, qn, 1);
    double flux = 0.0;
    if (i >= x0 - 1 && i <= x1 + 1) {
      const typename S::wk_t fs = st<typename S::wk_t>(
          mom_node_flux(nf, vm1, vc, vp1, vp2, qc, q1, cd[i - 1], cd[i], cd[i + 1]));
      mom_flux[row + i] = fs;
      flux = (double)fs;
    }
    const double fl = row_up(flux, f_last);
    if (i >= x0 && i <= x1 + 1)
      vel1[row + i] = st<typename S::vel_t>(div_rn(vc * qc + fl - flux, post));
    f_last = flux;
    vp = vc; vc = vn; vn = vnn;
    qc = qn; qn = qnn;
  }
  cp_wait_all();
}

// The y or z momentum flux and velocity update of one velocity in one pass
// (DIR 2 or 3). A block holds 32 node columns along the sweep axis
// (consecutive in x, then in the other index) and splits the nodes min..max+1
// into one segment per warp. A warp marches its segment node by node with the
// old velocities i-1..i+2 in registers, starting at the node below its
// segment (whose flux only the first segment stores), stores the flux at node
// i and updates node i. Before the block's barrier each warp reads the old
// velocities the neighbouring segments will overwrite: n0-2, n0-1 below its
// first node n0 and n1+1, n1+2 above its last n1; so the update is in place.
template <class S, int DIR>
__global__ void __launch_bounds__(BX * BY, 4) k_mom_line_yz(Geom g, GeomArrays ga,
    typename S::vel_t* __restrict__ vel1, const typename S::wk_t* __restrict__ node_flux,
    const typename S::wk_t* __restrict__ node_mass_pre,
    const typename S::wk_t* __restrict__ node_mass_post, typename S::wk_t* __restrict__ mom_flux) {
  __shared__ double ring[kLineSlots];
  // node columns (j, o) numbered j fastest: lane x of block b holds column 32b+x
  const int nj = g.x_max + 2 - g.x_min;
  const int no = DIR == 2 ? g.z_max + 2 - g.z_min : g.y_max + 2 - g.y_min;
  const int col = blockIdx.x * BX + threadIdx.x;
  const int j = g.x_min + col % nj;
  const int o = (DIR == 2 ? g.z_min : g.y_min) + col / nj;
  const int imin = DIR == 2 ? g.y_min : g.z_min;
  const int top = (DIR == 2 ? g.y_max : g.z_max) + 1;  // last node
  const int per = (top - imin + BY) / BY;
  const int n0 = imin + (int)threadIdx.y * per;
  const int n1 = n0 + per - 1 < top ? n0 + per - 1 : top;
  const bool act = col < nj * no && n0 <= n1;
  const long long step = DIR == 2 ? g.px : g.pxy;
  const long long base = DIR == 2 ? off3(g, j, 0, o) : off3(g, j, o, 0);
  const double* cd = (DIR == 2 ? ga.celldy : ga.celldz) + g.o1 + 2 - imin;
  const int i0 = n0 - 1;  // first node whose flux is formed
  const int steps = n1 - i0 + 1;
  // the velocities n1+1, n1+2 above the segment (the next segment's), read
  // before the barrier and kept in shared memory until the segment's end
  __shared__ double edge[2][BX * BY];
  const int me = threadIdx.y * BX + threadIdx.x;
  // step t (node i = i0+t): the velocity at i+2 (up to n1; above it the
  // pre-read pair), node_mass_pre at i+1, the node flux and node_mass_post
  // at i; ia is the element offset of node i0+ti, the next step to issue
  int ti = 0;
  long long ia = base + i0 * step;
  auto issue = [&]() {
    const bool wn = ti < steps, wv = wn && i0 + ti + 2 <= n1;
    const long long a = wn ? ia : base;
    double* sl = line_slot(ring, ti, 0);
    cp_elem(sl, vel1 + (wv ? ia + 2 * step : base), wv);
    cp_elem(sl + BX * BY, node_mass_pre + a + (wn ? step : 0), wn);
    cp_elem(sl + 2 * BX * BY, node_flux + a, wn);
    cp_elem(sl + 3 * BX * BY, node_mass_post + a, wn);
    cp_commit();
    ia += step;
    ti++;
  };
  double w0 = 0, w1 = 0, w2 = 0;  // old velocities i-1..i+1
  if (act) {
    for (int t = 0; t < kLineRing - 1; t++) issue();
    w0 = ldw(vel1 + base + (i0 - 1) * step);
    w1 = ldw(vel1 + base + i0 * step);
    w2 = ldw(vel1 + base + (i0 + 1) * step);
    edge[0][me] = ldw(vel1 + base + (n1 + 1) * step);
    edge[1][me] = ldw(vel1 + base + (n1 + 2) * step);
  }
  __syncthreads();
  if (!act) return;
  double q0 = ld(node_mass_pre + base + i0 * step);
  long long at = base + i0 * step;  // node i
  double f_last = 0.0;  // stored flux at node i-1
  for (int t = 0; t < steps; t++) {
    issue();
    const int i = i0 + t;
    cp_wait_step();
    const double* sl = line_slot(ring, t, 0);
    // (i + 2 is n1 + 1 or n1 + 2 here)
    const double w3 = i + 2 <= n1 ? slot_val<typename S::vel_t>(sl) : edge[i + 1 - n1][me];
    const double q1 = slot_val<typename S::wk_t>(sl + BX * BY);
    const double nf = slot_val<typename S::wk_t>(sl + 2 * BX * BY);
    const double post = slot_val<typename S::wk_t>(sl + 3 * BX * BY);
    const typename S::wk_t fs =
        st<typename S::wk_t>(mom_node_flux(nf, w0, w1, w2, w3, q0, q1, cd[i - 1], cd[i], cd[i + 1]));
    if (i >= n0 || n0 == imin) mom_flux[at] = fs;
    if (i >= n0) vel1[at] = st<typename S::vel_t>(div_rn(w1 * q0 + f_last - (double)fs, post));
    f_last = (double)fs;
    w0 = w1; w1 = w2; w2 = w3;
    q0 = q1;
    at += step;
  }
  cp_wait_all();
}

// ---------------------------------------------------------------------------
// reset_field_kernel.f90:51-98 (cell part over the interior, vertex part over
// the interior nodes; one launch over the node box)
template <class S, class M>
__global__ void __launch_bounds__(BX * BY) k_reset(M m,
    typename S::rho_t* __restrict__ density0, const typename S::rho_t* __restrict__ density1,
    typename S::ene_t* __restrict__ energy0, const typename S::ene_t* __restrict__ energy1,
    typename S::vel_t* __restrict__ xvel0, const typename S::vel_t* __restrict__ xvel1,
    typename S::vel_t* __restrict__ yvel0, const typename S::vel_t* __restrict__ yvel1,
    typename S::vel_t* __restrict__ zvel0, const typename S::vel_t* __restrict__ zvel1) {
  m.run([&](const Geom& g, const Tile& t) {
  TILE_THREAD(nodes(g), t);
  if (j <= g.x_max && k <= g.y_max && l <= g.z_max) {
    E(density0, j, k, l) = E(density1, j, k, l);
    E(energy0, j, k, l) = E(energy1, j, k, l);
  }
  E(xvel0, j, k, l) = E(xvel1, j, k, l);
  E(yvel0, j, k, l) = E(yvel1, j, k, l);
  E(zvel0, j, k, l) = E(zvel1, j, k, l);
  });
}

// ---------------------------------------------------------------------------
// field_summary_kernel.f90:57-77: a fixed grid of SUM_BLOCKS blocks strides
// over the interior cells in a fixed assignment; each block tree-reduces its
// five partials; a one-block pass adds the partials in block order. Every sum
// carries a Neumaier compensation term through the thread's loop, the block
// tree and the second stage (clover_sum.cuh). The result is the same on every
// run.
constexpr int SUM_THREADS = 256;
constexpr int SUM_BLOCKS = 148 * 4;

// field_summary_kernel.f90:60-75 for cell (j,k,l), added to the compensated
// sums (s, c)
template <class S>
__device__ __forceinline__ void summary_cell(const Geom& g, int j, int k, int l,
    const double* __restrict__ volume, const typename S::rho_t* __restrict__ density0,
    const typename S::ene_t* __restrict__ energy0, const typename S::cs_t* __restrict__ pressure,
    const typename S::vel_t* __restrict__ xvel0, const typename S::vel_t* __restrict__ yvel0,
    const typename S::vel_t* __restrict__ zvel0, double s[kSumQ], double c[kSumQ]) {
  double vsqrd = 0.0;
  for (int lv = l; lv <= l + 1; lv++)
    for (int kv = k; kv <= k + 1; kv++)
      for (int jv = j; jv <= j + 1; jv++) {
        const double u = L(xvel0, jv, kv, lv), v = L(yvel0, jv, kv, lv), w = L(zvel0, jv, kv, lv);
        vsqrd = vsqrd + 0.125 * (u * u + v * v + w * w);
      }
  const double cell_vol = E(volume, j, k, l);
  const double cell_mass = cell_vol * L(density0, j, k, l);
  csum_add(s[0], c[0], cell_vol);
  csum_add(s[1], c[1], cell_mass);
  csum_add(s[2], c[2], cell_mass * L(energy0, j, k, l));
  csum_add(s[3], c[3], cell_mass * 0.5 * vsqrd);
  csum_add(s[4], c[4], cell_vol * L(pressure, j, k, l));
}

// partials: per block (or plane) the five sums s then their five compensations c
__device__ __forceinline__ void store_csum(double* o, const double s[kSumQ], const double c[kSumQ]) {
  for (int q = 0; q < kSumQ; q++) {
    o[q] = s[q];
    o[kSumQ + q] = c[q];
  }
}

template <class S>
__global__ void __launch_bounds__(SUM_THREADS) k_summary(Geom g, const double* __restrict__ volume,
    const typename S::rho_t* __restrict__ density0, const typename S::ene_t* __restrict__ energy0,
    const typename S::cs_t* __restrict__ pressure, const typename S::vel_t* __restrict__ xvel0,
    const typename S::vel_t* __restrict__ yvel0, const typename S::vel_t* __restrict__ zvel0,
    double* __restrict__ partials) {
  __shared__ double sh[2 * kSumQ * SUM_THREADS];
  const int nx = g.x_max - g.x_min + 1, ny = g.y_max - g.y_min + 1, nz = g.z_max - g.z_min + 1;
  const long long n = (long long)nx * ny * nz;
  double s[kSumQ] = {0.0, 0.0, 0.0, 0.0, 0.0}, c[kSumQ] = {0.0, 0.0, 0.0, 0.0, 0.0};
  for (long long i = (long long)blockIdx.x * SUM_THREADS + threadIdx.x; i < n;
       i += (long long)SUM_BLOCKS * SUM_THREADS) {
    const int j = g.x_min + (int)(i % nx);
    const long long r = i / nx;
    const int k = g.y_min + (int)(r % ny);
    const int l = g.z_min + (int)(r / ny);
    summary_cell<S>(g, j, k, l, volume, density0, energy0, pressure, xvel0, yvel0, zvel0, s, c);
  }
  block_csum<SUM_THREADS>(s, c, sh);
  if (threadIdx.x == 0) store_csum(partials + blockIdx.x * 2 * kSumQ, s, c);
}

// The block partials merged in a fixed tree; out5 = s + c per quantity.
__global__ void __launch_bounds__(SUM_THREADS) k_summary_final(const double* __restrict__ partials,
                                                               double* __restrict__ out5) {
  __shared__ double sh[2 * kSumQ * SUM_THREADS];
  double s[kSumQ] = {0.0, 0.0, 0.0, 0.0, 0.0}, c[kSumQ] = {0.0, 0.0, 0.0, 0.0, 0.0};
  for (int i = threadIdx.x; i < SUM_BLOCKS; i += SUM_THREADS)
    for (int q = 0; q < kSumQ; q++)
      csum_merge(s[q], c[q], partials[i * 2 * kSumQ + q], partials[i * 2 * kSumQ + kSumQ + q]);
  block_csum<SUM_THREADS>(s, c, sh);
  if (threadIdx.x == 0)
    for (int q = 0; q < kSumQ; q++) out5[q] = s[q] + c[q];
}

// Per-deck summaries of an ensemble: tile z = one z plane of one deck, its
// cells strided over the block in a fixed order and tree-reduced.
template <class S, class M>
__global__ void __launch_bounds__(SUM_THREADS) k_summary_plane(M m,
    const int* __restrict__ plane_base, const double* __restrict__ volume,
    const typename S::rho_t* __restrict__ density0, const typename S::ene_t* __restrict__ energy0,
    const typename S::cs_t* __restrict__ pressure, const typename S::vel_t* __restrict__ xvel0,
    const typename S::vel_t* __restrict__ yvel0, const typename S::vel_t* __restrict__ zvel0,
    double* __restrict__ partials) {
  __shared__ double sh[2 * kSumQ * SUM_THREADS];
  m.run([&](const Geom& g, const Tile& t) {
    const int nx = g.x_max - g.x_min + 1, ny = g.y_max - g.y_min + 1;
    const int l = g.z_min + t.z;
    double s[kSumQ] = {0.0, 0.0, 0.0, 0.0, 0.0}, c[kSumQ] = {0.0, 0.0, 0.0, 0.0, 0.0};
    for (int i = threadIdx.x; i < nx * ny; i += SUM_THREADS)
      summary_cell<S>(g, g.x_min + i % nx, g.y_min + i / nx, l, volume, density0, energy0,
                      pressure, xvel0, yvel0, zvel0, s, c);
    block_csum<SUM_THREADS>(s, c, sh);
    if (threadIdx.x == 0) store_csum(partials + 2 * kSumQ * ((long long)plane_base[t.d] + t.z), s, c);
  });
}

// One block per deck: its plane partials merged in a fixed tree.
__global__ void __launch_bounds__(SUM_THREADS) k_summary_decks(const int* __restrict__ plane_base,
    const double* __restrict__ partials, double* __restrict__ out) {
  __shared__ double sh[2 * kSumQ * SUM_THREADS];
  const int d = blockIdx.x;
  const int p0 = plane_base[d], p1 = plane_base[d + 1];
  double s[kSumQ] = {0.0, 0.0, 0.0, 0.0, 0.0}, c[kSumQ] = {0.0, 0.0, 0.0, 0.0, 0.0};
  for (int i = p0 + (int)threadIdx.x; i < p1; i += SUM_THREADS)
    for (int q = 0; q < kSumQ; q++)
      csum_merge(s[q], c[q], partials[i * 2 * kSumQ + q], partials[i * 2 * kSumQ + kSumQ + q]);
  block_csum<SUM_THREADS>(s, c, sh);
  if (threadIdx.x == 0)
    for (int q = 0; q < kSumQ; q++) out[d * kSumQ + q] = s[q] + c[q];
}

// ---------------------------------------------------------------------------
// update_halo_kernel.f90:115-1423, table driven. For a face of normal axis A
// and m = 1..depth:
//   low face : dst = 1 - m,        src = low_src + m
//   high face: dst = max + hi_dst + m, src = max + hi_src - m
// with sign -1 where the reference negates. The two tangential loops run over
// [min-depth, max+depth+ext] with ext (0 or 1) per field, face and axis.
struct HaloRule {
  signed char sign, low_src, hi_dst, hi_src;
  signed char ext_lo[3], ext_hi[3];  // per axis x,y,z: extent of the low / high face loops
};

// kind: 0 cell, 1 vertex (comp = velocity component), 2 face (comp = normal)
inline HaloRule make_rule(int kind, int comp, int face_axis, int field_id) {
  HaloRule r;
  for (int a = 0; a < 3; a++) { r.ext_lo[a] = 0; r.ext_hi[a] = 0; }
  if (kind == 0) {  // :121-590
    r.sign = 1; r.low_src = 0; r.hi_dst = 0; r.hi_src = 1;
  } else if (kind == 1) {  // :604-1004
    r.sign = comp == face_axis ? -1 : 1;
    r.low_src = 1; r.hi_dst = 1; r.hi_src = 1;
    for (int a = 0; a < 3; a++) { r.ext_lo[a] = 1; r.ext_hi[a] = 1; }
  } else {  // :1018-1417
    if (comp == face_axis) {
      r.sign = -1; r.low_src = 1; r.hi_dst = 1; r.hi_src = 1;
    } else {
      r.sign = 1; r.low_src = 1; r.hi_dst = 0; r.hi_src = 0;
    }
    // Tangential extents: the face-normal axis of the field runs one further,
    // except on the z faces (back/front), which never extend.
    if (face_axis != 2 && comp != face_axis) { r.ext_lo[comp] = 1; r.ext_hi[comp] = 1; }
    // vol_flux_z (id 16) on the bottom face stops at z_max+depth (:1297-1303)
    if (field_id == 16 && face_axis == 1) r.ext_lo[2] = 0;
  }
  return r;
}

struct HaloLaunch {
  void* f[19];
  int elem_bytes[19];
  HaloRule rule[19];
  int nfields;
  int ids[19];
};

template <int AX, class M>
__global__ void k_halo(M m, HaloLaunch h, int depth, int do_low, int do_high) {
  m.run([&](const Geom& g, const Tile& t) {
  // tangential axes: y faces (j,l), x faces (k,l), z faces (j,k)
  const int ta = AX == 0 ? 1 : 0;  // first tangential axis
  const int tb = AX == 2 ? 1 : 2;  // second tangential axis
  const int mins[3] = {g.x_min, g.y_min, g.z_min};
  const int maxs[3] = {g.x_max, g.y_max, g.z_max};
  int a, bb;
  if (!tile_jk<M>(Box{mins[ta] - depth, maxs[ta] + 1 + depth, mins[tb] - depth,
                      maxs[tb] + 1 + depth, 0, 0}, t, a, bb))
    return;
  const int n = maxs[AX];
  for (int fi = 0; fi < h.nfields; fi++) {
    const HaloRule r = h.rule[fi];
    const int id = h.ids[fi];
    for (int side = 0; side < 2; side++) {
      if (side == 0 ? !do_low : !do_high) continue;
      const signed char* ext = side == 0 ? r.ext_lo : r.ext_hi;
      if (a > maxs[ta] + depth + ext[ta] || bb > maxs[tb] + depth + ext[tb]) continue;
      for (int m = 1; m <= depth; m++) {
        const int dst = side == 0 ? 1 - m : n + r.hi_dst + m;
        const int src = side == 0 ? r.low_src + m : n + r.hi_src - m;
        int dj, dk, dl, sj, sk, sl;
        if (AX == 0) { dj = dst; sj = src; dk = sk = a; dl = sl = bb; }
        else if (AX == 1) { dk = dst; sk = src; dj = sj = a; dl = sl = bb; }
        else { dl = dst; sl = src; dj = sj = a; dk = sk = bb; }
        const long long od = off3(g, dj, dk, dl), os = off3(g, sj, sk, sl);
        if (h.elem_bytes[fi] == 8) {
          double* p = (double*)h.f[fi];
          p[od] = r.sign < 0 ? -p[os] : p[os];
        } else {
          float* p = (float*)h.f[fi];
          p[od] = r.sign < 0 ? -p[os] : p[os];
        }
      }
    }
    (void)id;
  }
  });
}

// The x faces, one copy per thread: task = ((row * nfields + field) * 2 +
// side) * depth + m - 1 over the rows (k, l) of the face, so that the copies
// are all in flight at once (a row's halo cells lie in different sectors;
// the y and z faces are coalesced along x instead). On an axis shorter than
// three cells the high side reads cells the low side writes: there one thread
// per row does the row's copies in the reference order.
template <class M>
__global__ void k_halo_x(M m, HaloLaunch h, int depth, int do_low, int do_high) {
  m.run([&](const Geom& g, const Tile& t) {
  const int na = g.y_max - g.y_min + 2 + 2 * depth;  // k in [y_min-depth, y_max+1+depth]
  const int nb = g.z_max - g.z_min + 2 + 2 * depth;  // l likewise
  const int per_row = h.nfields * 2 * depth;
  const long long task = (long long)t.x * (BX * BY) + threadIdx.y * BX + threadIdx.x;
  if (task >= (long long)na * nb * per_row) return;
  const long long row = task / per_row;
  int rem = (int)(task % per_row);
  const int a = g.y_min - depth + (int)(row % na);
  const int bb = g.z_min - depth + (int)(row / na);
  const int n = g.x_max - g.x_min + 1;
  auto copy = [&](int fi, int side, int mm) {
    if (side == 0 ? !do_low : !do_high) return;
    const HaloRule r = h.rule[fi];
    const signed char* ext = side == 0 ? r.ext_lo : r.ext_hi;
    if (a > g.y_max + depth + ext[1] || bb > g.z_max + depth + ext[2]) return;
    const int dst = side == 0 ? 1 - mm : n + r.hi_dst + mm;
    const int src = side == 0 ? r.low_src + mm : n + r.hi_src - mm;
    const long long od = off3(g, dst, a, bb), os = off3(g, src, a, bb);
    if (h.elem_bytes[fi] == 8) {
      double* p = (double*)h.f[fi];
      p[od] = r.sign < 0 ? -p[os] : p[os];
    } else {
      float* p = (float*)h.f[fi];
      p[od] = r.sign < 0 ? -p[os] : p[os];
    }
  };
  if (n < 3) {
    if (rem != 0) return;
    for (int fi = 0; fi < h.nfields; fi++)
      for (int side = 0; side < 2; side++)
        for (int mm = 1; mm <= depth; mm++) copy(fi, side, mm);
    return;
  }
  const int mm = rem % depth + 1;
  rem /= depth;
  copy(rem / 2, rem % 2, mm);
  });
}

// tasks of k_halo_x in blocks of BX * BY; aux = tasks per row (fields * 2 * depth)
dim3 grid_halo_x_tasks(const Geom& g, int per_row, int depth) {
  const long long na = g.y_max - g.y_min + 2 + 2 * depth, nb = g.z_max - g.z_min + 2 + 2 * depth;
  return dim3((unsigned)((na * nb * per_row + BX * BY - 1) / (BX * BY)), 1, 1);
}
template <int D>
dim3 grid_halo_x(const Geom& g, int per_row) { return grid_halo_x_tasks(g, per_row, D); }

// tile grid of the halo update of the faces normal to AX (32 x 8 tiles over
// the two tangential axes, each extended by depth)
template <int AX>
dim3 grid_halo_flat(const Geom& g, int depth) {
  const int mins[3] = {g.x_min, g.y_min, g.z_min}, maxs[3] = {g.x_max, g.y_max, g.z_max};
  const int ta = AX == 0 ? 1 : 0, tb = AX == 2 ? 1 : 2;
  return grid_flat(Box{mins[ta] - depth, maxs[ta] + 1 + depth, mins[tb] - depth,
                       maxs[tb] + 1 + depth, 0, 0});
}
template <int AX>
dim3 grid_halo(const Geom& g, int depth) {
  const int mins[3] = {g.x_min, g.y_min, g.z_min}, maxs[3] = {g.x_max, g.y_max, g.z_max};
  const int ta = AX == 0 ? 1 : 0, tb = AX == 2 ? 1 : 2;
  const int na = maxs[ta] - mins[ta] + 2 + 2 * depth, nb = maxs[tb] - mins[tb] + 2 + 2 * depth;
  return dim3((na + 31) / 32, (nb + 7) / 8, 1);
}

// ---------------------------------------------------------------------------
// initialise_chunk_kernel.f90:70-178 and generate_chunk_kernel.f90:98-207
__global__ void k_init_1d(Geom g, double xmin, double ymin, double zmin, double dx, double dy,
                          double dz, double* vertexx, double* vertexdx, double* vertexy,
                          double* vertexdy, double* vertexz, double* vertexdz, double* cellx,
                          double* celldx, double* celly, double* celldy, double* cellz,
                          double* celldz) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  const int jx = g.x_min - 2 + t, ky = g.y_min - 2 + t, lz = g.z_min - 2 + t;
  // float(j-x_min) is a default REAL; small integers convert exactly
  auto vx = [&](int j) { return xmin + dx * (double)(float)(j - g.x_min); };
  auto vy = [&](int k) { return ymin + dy * (double)(float)(k - g.y_min); };
  auto vz = [&](int l) { return zmin + dz * (double)(float)(l - g.z_min); };
  if (jx <= g.x_max + 3) { GX(vertexx, jx) = vx(jx); GX(vertexdx, jx) = dx; }
  if (ky <= g.y_max + 3) { GY(vertexy, ky) = vy(ky); GY(vertexdy, ky) = dy; }
  if (lz <= g.z_max + 3) { GZ(vertexz, lz) = vz(lz); GZ(vertexdz, lz) = dz; }
  if (jx <= g.x_max + 2) { GX(cellx, jx) = 0.5 * (vx(jx) + vx(jx + 1)); GX(celldx, jx) = dx; }
  if (ky <= g.y_max + 2) { GY(celly, ky) = 0.5 * (vy(ky) + vy(ky + 1)); GY(celldy, ky) = dy; }
  if (lz <= g.z_max + 2) { GZ(cellz, lz) = 0.5 * (vz(lz) + vz(lz + 1)); GZ(celldz, lz) = dz; }
}

__global__ void __launch_bounds__(BX * BY) k_init_3d(Geom g, Box b, double dx, double dy, double dz,
    const double* celldx, const double* celldy, const double* celldz, double* volume,
    double* xarea, double* yarea, double* zarea) {
  BOX_THREAD(b);
  E(volume, j, k, l) = dx * dy * dz;
  E(xarea, j, k, l) = GY(celldy, k) * GZ(celldz, l);
  E(yarea, j, k, l) = GX(celldx, j) * GZ(celldz, l);
  E(zarea, j, k, l) = GX(celldx, j) * GY(celldy, k);
}

template <class S>
__global__ void __launch_bounds__(BX * BY) k_generate_bg(Geom g, Box b, StateTable st,
    typename S::rho_t* density0, typename S::ene_t* energy0, typename S::vel_t* xvel0,
    typename S::vel_t* yvel0, typename S::vel_t* zvel0) {
  BOX_THREAD(b);
  E(energy0, j, k, l) = st.energy[0];
  E(density0, j, k, l) = st.density[0];
  E(xvel0, j, k, l) = st.xvel[0];
  E(yvel0, j, k, l) = st.yvel[0];
  E(zvel0, j, k, l) = st.zvel[0];
}

template <class S>
__global__ void __launch_bounds__(BX * BY) k_generate_state(Geom g, Box b, GeomArrays ga, int s,
    StateTable st, typename S::rho_t* density0, typename S::ene_t* energy0,
    typename S::vel_t* xvel0, typename S::vel_t* yvel0, typename S::vel_t* zvel0) {
  BOX_THREAD(b);
  bool hit = false;
  if (st.geometry[s] == 1) {
    hit = GX(ga.vertexx, j + 1) >= st.xmin[s] && GX(ga.vertexx, j) < st.xmax[s] &&
          GY(ga.vertexy, k + 1) >= st.ymin[s] && GY(ga.vertexy, k) < st.ymax[s] &&
          GZ(ga.vertexz, l + 1) >= st.zmin[s] && GZ(ga.vertexz, l) < st.zmax[s];
  } else if (st.geometry[s] == 2) {
    const double cx = GX(ga.cellx, j) - st.xmin[s], cy = GY(ga.celly, k) - st.ymin[s],
                 cz = GZ(ga.cellz, l) - st.zmin[s];
    hit = sqrt(cx * cx + cy * cy + cz * cz) <= st.radius[s];
  } else if (st.geometry[s] == 3) {
    hit = GX(ga.vertexx, j) == st.xmin[s] && GY(ga.vertexy, k) == st.ymin[s] &&
          GZ(ga.vertexz, l) == st.zmin[s];
  }
  if (!hit) return;
  E(energy0, j, k, l) = st.energy[s];
  E(density0, j, k, l) = st.density[s];
  // every writer of a node writes the same state's value
  for (int lt = l; lt <= l + 1; lt++)
    for (int kt = k; kt <= k + 1; kt++)
      for (int jt = j; jt <= j + 1; jt++) {
        E(xvel0, jt, kt, lt) = st.xvel[s];
        E(yvel0, jt, kt, lt) = st.yvel[s];
        E(zvel0, jt, kt, lt) = st.zvel[s];
      }
}

template <class T>
__global__ void k_fill(T* p, long long n, T v) {
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n;
       i += (long long)gridDim.x * blockDim.x)
    p[i] = v;
}

}  // namespace

// ===========================================================================
// Launchers
#define LAUNCH(kern, box, ...)                                          \
  do {                                                                  \
    const Box _b = (box);                                               \
    const dim3 _gr = grid_of(_b);                                       \
    if (launchable(_gr)) kern<<<_gr, dim3(BX, BY), 0, s>>>(g, _b, __VA_ARGS__); \
  } while (0)


unsigned long long min_key_of(double v) { return key_of(v); }
double min_key_value(unsigned long long key) {
  unsigned long long b = (key >> 63) ? (key & 0x7fffffffffffffffull) : ~key;
  double v;
  memcpy(&v, &b, sizeof(v));
  return v;
}

template <class S>
void launch_ideal_gas(const Target& tg, cudaStream_t s, const typename S::rho_t* density,
                      const typename S::ene_t* energy, typename S::cs_t* pressure,
                      typename S::cs_t* soundspeed) {
  launch_mapped2(tg, s, kKeyIdealGas, grid_interior, grid_interior_flat, 0, false, dim3(BX, BY),
                k_ideal_gas<S, MapSingle>, k_ideal_gas<S, MapBatchFree>, density, energy, pressure,
                soundspeed);
}

template <class S>
void launch_viscosity(const Geom& g, cudaStream_t s, const GeomArrays& ga,
                      const typename S::rho_t* density0, const typename S::cs_t* pressure,
                      typename S::cs_t* viscosity, const typename S::vel_t* xvel0,
                      const typename S::vel_t* yvel0, const typename S::vel_t* zvel0) {
  LAUNCH(k_viscosity<S>, interior(g), ga, density0, pressure, viscosity, xvel0, yvel0, zvel0);
}

template <class S>
void launch_calc_dt(const Target& tg, cudaStream_t s, const GeomArrays& ga, double g_small,
                    double dtc_safe, double dtu_safe, double dtv_safe, double dtw_safe,
                    double dtdiv_safe, const typename S::rho_t* density0,
                    const typename S::cs_t* viscosity, const typename S::cs_t* soundspeed,
                    const typename S::vel_t* xvel0, const typename S::vel_t* yvel0,
                    const typename S::vel_t* zvel0, typename S::wk_t* dt_min_arr,
                    unsigned long long* min_key) {
  launch_mapped(tg, s, kKeyCalcDt, grid_interior, 0, false, dim3(BX, BY), k_calc_dt<S, MapSingle>,
                k_calc_dt<S, MapBatch>, ga, g_small, dtc_safe, dtu_safe, dtv_safe, dtw_safe,
                dtdiv_safe, density0, viscosity, soundspeed, xvel0, yvel0, zvel0, dt_min_arr,
                min_key);
}

template <class S>
void launch_pdv(const Geom& g, cudaStream_t s, int predict, double dt_val, const double* dt_ptr,
                const GeomArrays& ga, const typename S::rho_t* density0,
                typename S::rho_t* density1, const typename S::ene_t* energy0,
                typename S::ene_t* energy1, const typename S::cs_t* pressure,
                const typename S::cs_t* viscosity, const typename S::vel_t* xvel0,
                const typename S::vel_t* xvel1, const typename S::vel_t* yvel0,
                const typename S::vel_t* yvel1, const typename S::vel_t* zvel0,
                const typename S::vel_t* zvel1) {
  LAUNCH(k_pdv<S>, interior(g), predict, dt_val, dt_ptr, ga, density0, density1, energy0,
         energy1, pressure, viscosity, xvel0, xvel1, yvel0, yvel1, zvel0, zvel1);
}

template <class S>
void launch_revert(const Geom& g, cudaStream_t s, const typename S::rho_t* density0,
                   typename S::rho_t* density1, const typename S::ene_t* energy0,
                   typename S::ene_t* energy1) {
  LAUNCH(k_revert<S>, interior(g), density0, density1, energy0, energy1);
}

template <class S>
void launch_accelerate(const Target& tg, cudaStream_t s, double dt_val, const double* dt_ptr,
                       const GeomArrays& ga, const typename S::rho_t* density0,
                       const typename S::cs_t* pressure, const typename S::cs_t* viscosity,
                       const typename S::vel_t* xvel0, const typename S::vel_t* yvel0,
                       const typename S::vel_t* zvel0, typename S::vel_t* xvel1,
                       typename S::vel_t* yvel1, typename S::vel_t* zvel1, bool uniform_mesh) {
  if (uniform_mesh)
    launch_mapped2(tg, s, kKeyAccelerate, grid_nodes, grid_nodes_flat, 0, false, dim3(BX, BY),
                   k_accelerate<S, MapSingle, true>, k_accelerate<S, MapBatchFree, true>, dt_val,
                   dt_ptr, ga, density0, pressure, viscosity, xvel0, yvel0, zvel0, xvel1, yvel1,
                   zvel1);
  else
    launch_mapped2(tg, s, kKeyAccelerate, grid_nodes, grid_nodes_flat, 0, false, dim3(BX, BY),
                   k_accelerate<S, MapSingle, false>, k_accelerate<S, MapBatchFree, false>, dt_val,
                   dt_ptr, ga, density0, pressure, viscosity, xvel0, yvel0, zvel0, xvel1, yvel1,
                   zvel1);
}

template <class S>
void launch_flux_calc(const Geom& g, cudaStream_t s, double dt_val, const double* dt_ptr,
                      const GeomArrays& ga, const typename S::vel_t* xvel0,
                      const typename S::vel_t* yvel0, const typename S::vel_t* zvel0,
                      const typename S::vel_t* xvel1, const typename S::vel_t* yvel1,
                      const typename S::vel_t* zvel1, typename S::vf_t* vol_flux_x,
                      typename S::vf_t* vol_flux_y, typename S::vf_t* vol_flux_z) {
  LAUNCH(k_flux_calc<S>, nodes(g), dt_val, dt_ptr, ga, xvel0, yvel0, zvel0, xvel1, yvel1,
         zvel1, vol_flux_x, vol_flux_y, vol_flux_z);
}

template <class S>
void launch_advec_cell(const Geom& g, cudaStream_t s, int advect_x, int dir, int sweep,
                       const GeomArrays& ga, typename S::rho_t* density1,
                       typename S::ene_t* energy1, typename S::mf_t* mass_flux_x,
                       const typename S::vf_t* vol_flux_x, typename S::mf_t* mass_flux_y,
                       const typename S::vf_t* vol_flux_y, typename S::mf_t* mass_flux_z,
                       const typename S::vf_t* vol_flux_z, typename S::wk_t* const* work) {
  typename S::wk_t *pre_vol = work[0], *post_vol = work[1], *pre_mass = work[2],
                   *post_mass = work[3], *advec_vol = work[4], *post_ener = work[5],
                   *ener_flux = work[6];
  int variant = -1;
  if (dir == 1) variant = sweep == 1 ? 0 : sweep == 3 ? 1 : -1;
  else if (dir == 2) variant = sweep == 2 ? (advect_x ? 2 : 3) : -1;
  else if (dir == 3) variant = sweep == 1 ? 4 : sweep == 3 ? 5 : -1;
  if (variant >= 0)
    LAUNCH(k_cell_vol<S>, halo2(g), variant, ga, vol_flux_x, vol_flux_y, vol_flux_z, pre_vol, post_vol);
  const int nx = g.x_max - g.x_min + 1, ny = g.y_max - g.y_min + 1, nz = g.z_max - g.z_min + 1;
  const dim3 blk(BX, BY);
  if (dir == 1)
    k_cell_line_x<S><<<dim3((ny + BY - 1) / BY, nz), blk, 0, s>>>(g, ga, density1, energy1,
        vol_flux_x, mass_flux_x, pre_vol, pre_mass, post_mass, advec_vol, post_ener, ener_flux);
  else if (dir == 2)  // columns on the planes z_min..z_max+2 (the reference's y flux range)
    k_cell_line_yz<S, 2><<<dim3((nx * (nz + 2) + BX - 1) / BX), blk, 0, s>>>(g, ga, density1,
        energy1, vol_flux_y, mass_flux_y, pre_vol, pre_mass, post_mass, advec_vol, post_ener,
        ener_flux);
  else if (dir == 3)
    k_cell_line_yz<S, 3><<<dim3((nx * ny + BX - 1) / BX), blk, 0, s>>>(g, ga, density1, energy1,
        vol_flux_z, mass_flux_z, pre_vol, pre_mass, post_mass, advec_vol, post_ener, ener_flux);
}

static inline Box box_union(const Box& a, const Box& b) {
  return Box{a.j0 < b.j0 ? a.j0 : b.j0, a.j1 > b.j1 ? a.j1 : b.j1,
             a.k0 < b.k0 ? a.k0 : b.k0, a.k1 > b.k1 ? a.k1 : b.k1,
             a.l0 < b.l0 ? a.l0 : b.l0, a.l1 > b.l1 ? a.l1 : b.l1};
}

// advec_mom_kernel.f90:106-162: which pre/post volume form a sweep takes
// (-1: none)
int mom_vol_variant(int advect_x, int sweep, int direction) {
  if (sweep == 1 && direction == 1) return 0;
  if (sweep == 1 && direction == 3) return 1;
  if (sweep == 2) return advect_x ? 2 : 3;
  if (sweep == 3 && direction == 1) return 4;
  if (sweep == 3 && direction == 3) return 5;
  return -1;
}

template <class S>
void launch_advec_mom(const Geom& g, cudaStream_t s, typename S::vel_t* vel1,
                      const typename S::mf_t* mass_flux_x, const typename S::vf_t* vol_flux_x,
                      const typename S::mf_t* mass_flux_y, const typename S::vf_t* vol_flux_y,
                      const typename S::mf_t* mass_flux_z, const typename S::vf_t* vol_flux_z,
                      const GeomArrays& ga, const typename S::rho_t* density1,
                      typename S::wk_t* const* work, int advect_x, int which_vel, int sweep,
                      int direction, bool skip_volumes, int parts) {
  typename S::wk_t *node_flux = work[0], *node_mass_post = work[1], *node_mass_pre = work[2],
                   *mom_flux = work[4], *pre_vol = work[5], *post_vol = work[6];
  const int variant = mom_vol_variant(advect_x, sweep, direction);
  if (variant >= 0 && !skip_volumes && (parts & kMomVolumes))
    LAUNCH(k_mom_vol<S>, halo2(g), variant, ga, vol_flux_x, vol_flux_y, vol_flux_z, pre_vol, post_vol);
  const int x0 = g.x_min, x1 = g.x_max, y0 = g.y_min, y1 = g.y_max, z0 = g.z_min, z1 = g.z_max;
  if (!(parts & kMomNodePass)) {
  } else if (direction == 1) {
    if (which_vel == 1) {
      const Box bf{x0 - 2, x1 + 2, y0, y1 + 1, z0, z1 + 1}, bm{x0 - 1, x1 + 2, y0, y1 + 1, z0, z1 + 1};
      LAUNCH((k_mom_node<S, 1>), box_union(bf, bm), bf, bm, mass_flux_x, density1, post_vol,
             node_flux, node_mass_post, node_mass_pre);
    }
  } else if (direction == 2) {
    if (which_vel == 1) {
      const Box bf{x0, x1 + 1, y0 - 2, y1 + 2, z0, z1 + 1}, bm{x0, x1 + 1, y0 - 1, y1 + 2, z0, z1 + 1};
      LAUNCH((k_mom_node<S, 2>), box_union(bf, bm), bf, bm, mass_flux_y, density1, post_vol,
             node_flux, node_mass_post, node_mass_pre);
    }
  } else if (direction == 3) {
    if (which_vel == 1) {
      const Box bf{x0, x1 + 1, y0, y1 + 1, z0 - 2, z1 + 2}, bm{x0, x1 + 1, y0, y1 + 1, z0 - 1, z1 + 2};
      LAUNCH((k_mom_node<S, 3>), box_union(bf, bm), bf, bm, mass_flux_z, density1, post_vol,
             node_flux, node_mass_post, node_mass_pre);
    }
  }
  if (!(parts & kMomFluxUpdate)) return;
  // the flux at nodes min-1..max+1 and the update of nodes min..max+1 along
  // the sweep, in one pass per velocity
  const int nx = x1 - x0 + 1, ny = y1 - y0 + 1, nz = z1 - z0 + 1;
  const dim3 blk(BX, BY);
  if (direction == 1)
    k_mom_line_x<S><<<dim3((ny + 1 + BY - 1) / BY, nz + 1), blk, 0, s>>>(g, ga, vel1, node_flux,
        node_mass_pre, node_mass_post, mom_flux);
  else if (direction == 2)
    k_mom_line_yz<S, 2><<<dim3(((nx + 1) * (nz + 1) + BX - 1) / BX), blk, 0, s>>>(g, ga, vel1,
        node_flux, node_mass_pre, node_mass_post, mom_flux);
  else if (direction == 3)
    k_mom_line_yz<S, 3><<<dim3(((nx + 1) * (ny + 1) + BX - 1) / BX), blk, 0, s>>>(g, ga, vel1,
        node_flux, node_mass_pre, node_mass_post, mom_flux);
}

template <class S>
void launch_reset_field(const Target& tg, cudaStream_t s, typename S::rho_t* density0,
                        const typename S::rho_t* density1, typename S::ene_t* energy0,
                        const typename S::ene_t* energy1, typename S::vel_t* xvel0,
                        const typename S::vel_t* xvel1, typename S::vel_t* yvel0,
                        const typename S::vel_t* yvel1, typename S::vel_t* zvel0,
                        const typename S::vel_t* zvel1) {
  launch_mapped2(tg, s, kKeyReset, grid_nodes, grid_nodes_flat, 0, false, dim3(BX, BY), k_reset<S, MapSingle>,
                k_reset<S, MapBatchFree>, density0, density1, energy0, energy1, xvel0, xvel1, yvel0,
                yvel1, zvel0, zvel1);
}

int summary_partials_len() { return SUM_BLOCKS * 2 * kSumQ; }

template <class S>
void launch_field_summary(const Geom& g, cudaStream_t s, const double* volume,
                          const typename S::rho_t* density0, const typename S::ene_t* energy0,
                          const typename S::cs_t* pressure, const typename S::vel_t* xvel0,
                          const typename S::vel_t* yvel0, const typename S::vel_t* zvel0,
                          double* partials, double* out5) {
  k_summary<S><<<SUM_BLOCKS, SUM_THREADS, 0, s>>>(g, volume, density0, energy0, pressure, xvel0,
                                                  yvel0, zvel0, partials);
  k_summary_final<<<1, SUM_THREADS, 0, s>>>(partials, out5);
}

inline dim3 grid_planes(const Geom& g, int) { return dim3(1, 1, g.z_max - g.z_min + 1); }

template <class S>
void launch_field_summary_batch(BatchPlan* plan, int n_decks, cudaStream_t s,
                                const int* plane_base, const double* volume,
                                const typename S::rho_t* density0, const typename S::ene_t* energy0,
                                const typename S::cs_t* pressure, const typename S::vel_t* xvel0,
                                const typename S::vel_t* yvel0, const typename S::vel_t* zvel0,
                                double* partials, double* out) {
  launch_mapped(Target(plan), s, kKeySummary, grid_planes, 0, false, dim3(SUM_THREADS),
                k_summary_plane<S, MapSingle>, k_summary_plane<S, MapBatch>, plane_base, volume,
                density0, energy0, pressure, xvel0, yvel0, zvel0, partials);
  if (n_decks > 0)
    k_summary_decks<<<n_decks, SUM_THREADS, 0, s>>>(plane_base, partials, out);
}

template <class S>
static int elem_bytes_of(int id) {
  if (id == 1 || id == 2) return sizeof(typename S::rho_t);
  if (id == 3 || id == 4) return sizeof(typename S::ene_t);
  if (id >= 5 && id <= 7) return sizeof(typename S::cs_t);
  if (id >= 8 && id <= 13) return sizeof(typename S::vel_t);
  if (id >= 14 && id <= 16) return sizeof(typename S::vf_t);
  return sizeof(typename S::mf_t);
}

template <class S>
void launch_update_halo(const Target& tg, cudaStream_t s, const HaloFields& f, const int* fields,
                        int depth, const int* external_faces) {
  // field id -> (kind, component)
  static const int kind[19] = {0, 0, 0, 0, 0, 0, 0, 1, 1, 1, 1, 1, 1, 2, 2, 2, 2, 2, 2};
  static const int comp[19] = {0, 0, 0, 0, 0, 0, 0, 0, 0, 1, 1, 2, 2, 0, 1, 2, 0, 1, 2};
  // faces: 0 left, 1 right, 2 bottom, 3 top, 4 back, 5 front; axis order y, x, z
  const int axes[3] = {1, 0, 2};
  for (int ai = 0; ai < 3; ai++) {
    const int ax = axes[ai];
    const int lo_face = ax == 0 ? 0 : ax == 1 ? 2 : 4;
    const int do_low = external_faces[lo_face] ? 1 : 0, do_high = external_faces[lo_face + 1] ? 1 : 0;
    if (!do_low && !do_high) continue;
    HaloLaunch h;
    h.nfields = 0;
    for (int id = 1; id <= 19; id++) {
      if (fields[id - 1] != 1) continue;
      const int i = h.nfields++;
      h.f[i] = f.f[id - 1];
      h.ids[i] = id;
      h.elem_bytes[i] = elem_bytes_of<S>(id);
      h.rule[i] = make_rule(kind[id - 1], comp[id - 1], ax, id);
    }
    if (h.nfields == 0) return;
    const dim3 blk(32, 8);
    const unsigned key = kKeyHalo | (unsigned)(ax << 4) | (unsigned)depth;
    if (ax == 0) {
      const int per_row = h.nfields * 2 * depth;
      // the schedule depends on the depth as well as the tasks per row (a
      // depth-1 and a depth-2 update can have the same number per row)
      const unsigned kx = kKeyHaloX | (unsigned)((depth - 1) << 7) | (unsigned)per_row;
      if (depth == 1)
        launch_mapped(tg, s, kx, grid_halo_x<1>, per_row, false, blk, k_halo_x<MapSingle>,
                      k_halo_x<MapBatchFree>, h, depth, do_low, do_high);
      else
        launch_mapped(tg, s, kx, grid_halo_x<2>, per_row, false, blk, k_halo_x<MapSingle>,
                      k_halo_x<MapBatchFree>, h, depth, do_low, do_high);
    }
    else if (ax == 1)
      launch_mapped2(tg, s, key, grid_halo<1>, grid_halo_flat<1>, depth, false, blk,
                     k_halo<1, MapSingle>, k_halo<1, MapBatchFree>, h, depth, do_low, do_high);
    else
      launch_mapped2(tg, s, key, grid_halo<2>, grid_halo_flat<2>, depth, false, blk,
                     k_halo<2, MapSingle>, k_halo<2, MapBatchFree>, h, depth, do_low, do_high);
  }
}

void launch_initialise_chunk(const Geom& g, cudaStream_t s, double xmin, double ymin,
                             double zmin, double dx, double dy, double dz, double* vertexx,
                             double* vertexdx, double* vertexy, double* vertexdy,
                             double* vertexz, double* vertexdz, double* cellx, double* celldx,
                             double* celly, double* celldy, double* cellz, double* celldz,
                             double* volume, double* xarea, double* yarea, double* zarea) {
  int n = g.x_max - g.x_min;
  if (g.y_max - g.y_min > n) n = g.y_max - g.y_min;
  if (g.z_max - g.z_min > n) n = g.z_max - g.z_min;
  n += 6;
  k_init_1d<<<(n + 127) / 128, 128, 0, s>>>(g, xmin, ymin, zmin, dx, dy, dz, vertexx, vertexdx,
                                            vertexy, vertexdy, vertexz, vertexdz, cellx, celldx,
                                            celly, celldy, cellz, celldz);
  LAUNCH(k_init_3d, halo2(g), dx, dy, dz, celldx, celldy, celldz, volume, xarea, yarea, zarea);
}

template <class S>
void launch_generate_chunk(const Geom& g, cudaStream_t s, const GeomArrays& ga,
                           typename S::rho_t* density0, typename S::ene_t* energy0,
                           typename S::vel_t* xvel0, typename S::vel_t* yvel0,
                           typename S::vel_t* zvel0, const StateTable& st) {
  LAUNCH(k_generate_bg<S>, halo2(g), st, density0, energy0, xvel0, yvel0, zvel0);
  for (int state = 1; state < st.n; state++)
    LAUNCH(k_generate_state<S>, halo2(g), ga, state, st, density0, energy0, xvel0, yvel0, zvel0);
}

template <class T>
void launch_fill(cudaStream_t s, T* p, long long elems, T value) {
  k_fill<T><<<148 * 8, 256, 0, s>>>(p, elems, value);
}

#define INST(S)                                                                               \
  template void launch_ideal_gas<S>(const Target&, cudaStream_t, const S::rho_t*, const S::ene_t*, \
                                    S::cs_t*, S::cs_t*);                                      \
  template void launch_viscosity<S>(const Geom&, cudaStream_t, const GeomArrays&, const S::rho_t*, \
                                    const S::cs_t*, S::cs_t*, const S::vel_t*, const S::vel_t*, \
                                    const S::vel_t*);                                         \
  template void launch_calc_dt<S>(const Target&, cudaStream_t, const GeomArrays&, double, double, \
                                  double, double, double, double, const S::rho_t*,             \
                                  const S::cs_t*, const S::cs_t*, const S::vel_t*,              \
                                  const S::vel_t*, const S::vel_t*, S::wk_t*,                  \
                                  unsigned long long*);                                        \
  template void launch_pdv<S>(const Geom&, cudaStream_t, int, double, const double*,             \
                              const GeomArrays&, const S::rho_t*, S::rho_t*, const S::ene_t*,  \
                              S::ene_t*, const S::cs_t*, const S::cs_t*, const S::vel_t*,       \
                              const S::vel_t*, const S::vel_t*, const S::vel_t*,               \
                              const S::vel_t*, const S::vel_t*);                               \
  template void launch_revert<S>(const Geom&, cudaStream_t, const S::rho_t*, S::rho_t*,          \
                                 const S::ene_t*, S::ene_t*);                                  \
  template void launch_accelerate<S>(const Target&, cudaStream_t, double, const double*,           \
                                     const GeomArrays&, const S::rho_t*, const S::cs_t*,       \
                                     const S::cs_t*, const S::vel_t*, const S::vel_t*,          \
                                     const S::vel_t*, S::vel_t*, S::vel_t*, S::vel_t*, bool);  \
  template void launch_flux_calc<S>(const Geom&, cudaStream_t, double, const double*,            \
                                    const GeomArrays&, const S::vel_t*, const S::vel_t*,       \
                                    const S::vel_t*, const S::vel_t*, const S::vel_t*,          \
                                    const S::vel_t*, S::vf_t*, S::vf_t*, S::vf_t*);            \
  template void launch_advec_cell<S>(const Geom&, cudaStream_t, int, int, int, const GeomArrays&, \
                                     S::rho_t*, S::ene_t*, S::mf_t*, const S::vf_t*, S::mf_t*, \
                                     const S::vf_t*, S::mf_t*, const S::vf_t*, S::wk_t* const*); \
  template void launch_advec_mom<S>(const Geom&, cudaStream_t, S::vel_t*, const S::mf_t*,        \
                                    const S::vf_t*, const S::mf_t*, const S::vf_t*,            \
                                    const S::mf_t*, const S::vf_t*, const GeomArrays&,         \
                                    const S::rho_t*, S::wk_t* const*, int, int, int, int,      \
                                    bool, int);                                                \
  template void launch_reset_field<S>(const Target&, cudaStream_t, S::rho_t*, const S::rho_t*,     \
                                      S::ene_t*, const S::ene_t*, S::vel_t*, const S::vel_t*,  \
                                      S::vel_t*, const S::vel_t*, S::vel_t*, const S::vel_t*); \
  template void launch_field_summary<S>(const Geom&, cudaStream_t, const double*,               \
                                        const S::rho_t*, const S::ene_t*, const S::cs_t*,      \
                                        const S::vel_t*, const S::vel_t*, const S::vel_t*,     \
                                        double*, double*);                                     \
  template void launch_field_summary_batch<S>(BatchPlan*, int, cudaStream_t, const int*,        \
                                              const double*, const S::rho_t*, const S::ene_t*, \
                                              const S::cs_t*, const S::vel_t*, const S::vel_t*, \
                                              const S::vel_t*, double*, double*);              \
  template void launch_update_halo<S>(const Target&, cudaStream_t, const HaloFields&, const int*,  \
                                      int, const int*);                                        \
  template void launch_generate_chunk<S>(const Geom&, cudaStream_t, const GeomArrays&,          \
                                         S::rho_t*, S::ene_t*, S::vel_t*, S::vel_t*,           \
                                         S::vel_t*, const StateTable&);

INST(F64)
INST(F32Mixed)

template void launch_fill<double>(cudaStream_t, double*, long long, double);
template void launch_fill<float>(cudaStream_t, float*, long long, float);

}  // namespace clover

// ---------------------------------------------------------------------------
// Self-test of the shared-reciprocal quotient (clover_div.cuh): q[i] = x[i] /
// b[i] through recip_for + quot_rn where both lie in its range (fast[i] = 1),
// else by IEEE division (fast[i] = 0).
namespace clover {
namespace {
__global__ void k_quotient_selftest(const double* __restrict__ x, const double* __restrict__ b,
                                    double* __restrict__ q, int* __restrict__ fast, long long n) {
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n;
       i += (long long)gridDim.x * blockDim.x) {
    const Recip r = recip_for(b[i]);
    const bool ok = r.ok && quot_in_range(x[i]);
    q[i] = ok ? quot_rn(x[i], r) : x[i] / b[i];
    fast[i] = ok ? 1 : 0;
  }
}
}  // namespace
}  // namespace clover

extern "C" int clover_gpu_quotient_selftest(const double* x, const double* b, double* q, int* fast,
                                            long long n) {
  using namespace clover;
  if (n <= 0) return 0;
  double *dx = nullptr, *db = nullptr, *dq = nullptr;
  int* df = nullptr;
  const size_t bytes = (size_t)n * sizeof(double);
  bool ok = cudaMalloc(&dx, bytes) == cudaSuccess && cudaMalloc(&db, bytes) == cudaSuccess &&
            cudaMalloc(&dq, bytes) == cudaSuccess &&
            cudaMalloc(&df, (size_t)n * sizeof(int)) == cudaSuccess;
  ok = ok && cudaMemcpy(dx, x, bytes, cudaMemcpyHostToDevice) == cudaSuccess &&
       cudaMemcpy(db, b, bytes, cudaMemcpyHostToDevice) == cudaSuccess;
  if (ok) {
    k_quotient_selftest<<<4 * 148, 256>>>(dx, db, dq, df, n);
    ok = cudaGetLastError() == cudaSuccess &&
         cudaMemcpy(q, dq, bytes, cudaMemcpyDeviceToHost) == cudaSuccess &&
         cudaMemcpy(fast, df, (size_t)n * sizeof(int), cudaMemcpyDeviceToHost) == cudaSuccess;
  }
  cudaFree(dx);
  cudaFree(db);
  cudaFree(dq);
  cudaFree(df);
  if (!ok) cudaGetLastError();
  return ok ? 0 : CLOVER_STATUS_CUDA_ERROR;
}
