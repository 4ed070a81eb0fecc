// Device helpers shared by the fused stencils (clover_fused.cu) and their
// shared-memory staged forms (clover_tma.cu): storage conversions, the
// comparisons the reference's MIN/MAX make, and the momentum advection's
// per-node terms and flux (advec_mom_kernel.f90), written once so that both
// forms run the same operations in the same order.
#pragma once

#include <cuda_runtime.h>

#include "clover_div.cuh"
#include "clover_layout.cuh"

namespace clover {

// A marching kernel's threads cover j in [jlo, jhi] and the cross axis c in
// [clo, chi] and walk the sweep axis p over [plo, phi] (cell sweeps: faces
// from the sweep axis minimum to its maximum+2, cells updated for c <= cmax).
struct MarchRange {
  int jlo, jhi, clo, chi, plo, phi, cmax;
};
// advec_mom y/z node pass: node fluxes from min-2 to max+2 along the sweep
template <int DIR>
__host__ __device__ inline MarchRange mom_node_range(const Geom& g) {
  const int pmin = DIR == 2 ? g.y_min : g.z_min, pmax = DIR == 2 ? g.y_max : g.z_max;
  const int cmin = DIR == 2 ? g.z_min : g.y_min, cmx = DIR == 2 ? g.z_max : g.y_max;
  return MarchRange{g.x_min, g.x_max + 1, cmin, cmx + 1, pmin - 2, pmax + 2, cmx + 1};
}
// advec_mom y/z velocity pass: nodes min..max+1 along the sweep
template <int DIR>
__host__ __device__ inline MarchRange mom_vel_range(const Geom& g) {
  const int pmin = DIR == 2 ? g.y_min : g.z_min, pmax = DIR == 2 ? g.y_max : g.z_max;
  const int cmin = DIR == 2 ? g.z_min : g.y_min, cmx = DIR == 2 ? g.z_max : g.y_max;
  return MarchRange{g.x_min, g.x_max + 1, cmin, cmx + 1, pmin, pmax + 1, cmx + 1};
}
// advec_cell y sweep: columns l in [z_min, z_max+2] (the reference's y face
// range), cells updated for l <= z_max; z sweep: rows k in [y_min, y_max]
template <int DIR>
__host__ __device__ inline MarchRange cell_sweep_range(const Geom& g) {
  if (DIR == 2)
    return MarchRange{g.x_min, g.x_max, g.z_min, g.z_max + 2, g.y_min, g.y_max + 2, g.z_max};
  return MarchRange{g.x_min, g.x_max, g.y_min, g.y_max, g.z_min, g.z_max + 2, g.y_max};
}

// a value in storage type T, converted once from the arithmetic it was
// formed in (no detour through double for an FP32 value stored as FP32)
template <class T, class U>
__device__ __forceinline__ T st(U v) { return (T)v; }

__device__ __forceinline__ double fmin2(double a, double b) { return b < a ? b : a; }
__device__ __forceinline__ double fmax2(double a, double b) { return b > a ? b : a; }
__device__ __forceinline__ float fmin2(float a, float b) { return b < a ? b : a; }
__device__ __forceinline__ float fmax2(float a, float b) { return b > a ? b : a; }
// a value of the momentum arithmetic type A from storage
template <class A>
__device__ __forceinline__ A lda(const double* p) { return (A)__ldg(p); }
template <class A>
__device__ __forceinline__ A lda(const float* p) { return (A)__ldg(p); }

// vertexd(j) / vertexd(dif) of the limiter: exactly 1 where the two widths
// are equal (every face of a uniform mesh), without the division
__device__ __forceinline__ double width_ratio(double a, double b) {
  return (a == b && a != 0.0 && fabs(a) <= DBL_MAX) ? 1.0 : a / b;
}

// advec_cell_kernel.f90:141-151 in the limiter's arithmetic A (FP64, or FP32
// in the mixed path: the limiter shapes a face flux that both cells of the
// face take, so its rounding does not touch conservation; the flux itself and
// the cell update stay FP64)
template <class A>
__device__ __forceinline__ A cell_limiter(A sig, A sigma3, A sigma4, A diffuw, A diffdw) {
  const A one_by_six = A(1.0) / A(6.0);
  if (diffuw * diffdw > A(0.0))
    return (A(1.0) - sig) * copysign(A(1.0), diffdw) *
           fmin2(fmin2(fabs(diffuw), fabs(diffdw)),
                 one_by_six * (sigma3 * fabs(diffuw) + sigma4 * fabs(diffdw)));
  return A(0.0);
}

// The per-chunk quotients of Geom in the arithmetic type A.
template <class A>
__device__ __forceinline__ A geo_rvol(const Geom& g) { return sizeof(A) == 4 ? (A)g.rvol_f : (A)g.rvol; }
template <class A>
__device__ __forceinline__ A geo_ds(const Geom& g) { return sizeof(A) == 4 ? (A)g.ds_f : (A)g.ds; }

// Node mass post (reference order of the eight cells) from cell products P.
__device__ __forceinline__ double node_mass_sum(double p_0m0, double p_000, double p_mm0,
                                                double p_m00, double p_0mm, double p_00m,
                                                double p_mmm, double p_m0m) {
  return 0.125 * (p_0m0 + p_000 + p_mm0 + p_m00 + p_0mm + p_00m + p_mmm + p_m0m);
}

// Momentum flux at node i (advec_mom_kernel.f90:211-242 and the y/z forms)
// from the velocity window v(i-1..i+2). The donor side, the Courant number
// sigma and the limiter's cell widths depend on the node only, so they are
// formed once per node (MomNodeTerms) for the three velocity components.
template <class A>
struct MomNodeTerms {
  bool neg;  // node flux < 0: the donor is node i+1
  A nf, sigma, width, cd_dif;
};

template <class A>
__device__ __forceinline__ MomNodeTerms<A> mom_node_terms(A nf, A nmpre_i, A nmpre_ip1, A width,
                                                          A cd_m1, A cd_p1) {
  MomNodeTerms<A> t;
  t.neg = nf < A(0.0);
  t.nf = nf;
  t.sigma = div_rn(fabs(nf), t.neg ? nmpre_ip1 : nmpre_i);
  t.width = width;
  t.cd_dif = t.neg ? cd_p1 : cd_m1;
  return t;
}

template <class A>
__device__ __forceinline__ A mom_flux_v(const MomNodeTerms<A>& t, A vm1, A v0, A vp1, A vp2) {
  const A v_upwind = t.neg ? vp2 : vm1;
  const A v_donor = t.neg ? vp1 : v0;
  const A v_downwind = t.neg ? v0 : vp1;
  const A vdiffuw = v_donor - v_upwind;
  const A vdiffdw = v_downwind - v_donor;
  A limiter = A(0.0);
  if (vdiffuw * vdiffdw > A(0.0)) {
    const A auw = fabs(vdiffuw);
    const A adw = fabs(vdiffdw);
    A wind = A(1.0);
    if (vdiffdw <= A(0.0)) wind = A(-1.0);
    const A width = t.width, sigma = t.sigma;
    // ... / 6.0_8 correctly rounded by div6 (clover_div.cuh)
    limiter = wind * fmin2(fmin2(div6(width * ((A(2.0) - sigma) * adw / width +
                                               (A(1.0) + sigma) * auw / t.cd_dif)),
                                 auw),
                           adw);
  }
  const A advec_vel_s = v_donor + (A(1.0) - t.sigma) * limiter;
  return advec_vel_s * t.nf;
}

template <class A>
__device__ __forceinline__ A mom_flux_at(A nf, A nmpre_i, A nmpre_ip1, A vm1, A v0, A vp1, A vp2,
                                         A width, A cd_m1, A cd_p1) {
  return mom_flux_v<A>(mom_node_terms<A>(nf, nmpre_i, nmpre_ip1, width, cd_m1, cd_p1), vm1, v0,
                       vp1, vp2);
}

}  // namespace clover
