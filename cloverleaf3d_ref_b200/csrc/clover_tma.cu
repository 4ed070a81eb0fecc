// Kernels of the native step whose inputs are staged plane by plane into
// shared memory with bulk-tensor copies (clover_tma.cuh), and the host-side
// encoding of their tensor maps.
//
//  k_visc_dt_tma  viscosity_kernel.f90:71-134, calc_dt_kernel.f90:102-149
//                 and ideal_gas_kernel.f90:47-58 on every interior cell, as
//                 k_visc_dt (clover_fused.cu) forms them, operation for
//                 operation. A block owns 32 x 8 columns (j, k) and marches
//                 a segment of planes l; a ring of plane buffers holds, for
//                 plane p, the node velocities of node plane p (9 rows x
//                 32+2H columns) and density0 / energy0 of cell plane p (10
//                 rows x 32+2H columns). Cell l reads node planes l, l+1 and
//                 cell planes l-1, l, l+1; one thread refills the buffer of
//                 plane l-1 with plane l-1+R once the block is done with l.
#include <cfloat>
#include <cstdio>

#include <cudaTypedefs.h>

#include "../../include/clover_kernels.h"
#include "clover_launch.h"
#include "clover_stencil.cuh"
#include "clover_tma.cuh"

namespace clover {

bool encode_plane_map(CUtensorMap* map, const void* base, int elem_bytes, const Geom& g,
                      int box_rows, bool rows_along_z) {
  static PFN_cuTensorMapEncodeTiled encode = nullptr;
  if (!encode) {
    void* fn = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &fn, cudaEnableDefault, &q) !=
            cudaSuccess ||
        q != cudaDriverEntryPointSuccess || !fn) {
      cudaGetLastError();
      return false;
    }
    encode = (PFN_cuTensorMapEncodeTiled)fn;
  }
  const int halo = 16 / elem_bytes;
  // the map starts halo columns before x_min (16-byte aligned: x_min is
  // 128-byte aligned); base points at column x_min - 2
  const char* start = (const char*)base - (long long)(halo - 2) * elem_bytes;
  const cuuint64_t dims[3] = {(cuuint64_t)g.px, (cuuint64_t)(g.pxy / g.px),
                              (cuuint64_t)(g.z_max - g.z_min + 6)};
  const cuuint64_t strides[2] = {(cuuint64_t)g.px * elem_bytes, (cuuint64_t)g.pxy * elem_bytes};
  // a box is one plane of box_rows rows: rows along y (x-y planes), or along
  // z (x-z slices, for sweeps that march along y)
  const cuuint32_t box[3] = {(cuuint32_t)(32 + 2 * halo), rows_along_z ? 1u : (cuuint32_t)box_rows,
                             rows_along_z ? (cuuint32_t)box_rows : 1u};
  const cuuint32_t estr[3] = {1, 1, 1};
  const CUresult r =
      encode(map, elem_bytes == 8 ? CU_TENSOR_MAP_DATA_TYPE_FLOAT64 : CU_TENSOR_MAP_DATA_TYPE_FLOAT32,
             3, (void*)start, dims, strides, box, estr, CU_TENSOR_MAP_INTERLEAVE_NONE,
             CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
             CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  return r == CUDA_SUCCESS;
}

namespace {

constexpr int TX = 32, TY = 8;

constexpr int round128(int b) { return (b + 127) / 128 * 128; }

// Byte layout of one plane buffer of the viscosity ring.
template <class S>
struct ViscPlane {
  using V = typename S::vel_t;
  using R = typename S::rho_t;
  using En = typename S::ene_t;
  static constexpr int WV = kTmaWidth<V>, WR = kTmaWidth<R>, WE = kTmaWidth<En>;
  static constexpr int HV = kTmaHalo<V>, HR = kTmaHalo<R>, HE = kTmaHalo<En>;
  static constexpr int kNodeRows = TY + 1, kCellRows = TY + 2;
  static constexpr int kVel = round128(kNodeRows * WV * (int)sizeof(V));
  static constexpr int kRho = round128(kCellRows * WR * (int)sizeof(R));
  static constexpr int kEne = round128(kCellRows * WE * (int)sizeof(En));
  static constexpr int kBytes = 3 * kVel + kRho + kEne;  // one plane buffer
  // bytes the five boxes of a plane deliver
  static constexpr unsigned kTx = 3 * box_bytes<V>(kNodeRows) + box_bytes<R>(kCellRows) +
                                  box_bytes<En>(kCellRows);
  __device__ static V* vel(unsigned char* p, int q) { return (V*)(p + q * kVel); }
  __device__ static R* rho(unsigned char* p) { return (R*)(p + 3 * kVel); }
  __device__ static En* ene(unsigned char* p) { return (En*)(p + 3 * kVel + kRho); }
};

template <class S, int RING, int MINB>
__global__ void __launch_bounds__(TX * TY, MINB)
k_visc_dt_tma(Geom g, int seg, GeomArrays ga, double g_small, double dtc_safe, double dtu_safe,
              double dtv_safe, double dtw_safe, double dtdiv_safe,
              const __grid_constant__ ViscMaps maps, typename S::cs_t* __restrict__ pressure,
              typename S::cs_t* __restrict__ viscosity, typename S::cs_t* __restrict__ soundspeed,
              unsigned long long* __restrict__ min_key, int* __restrict__ status) {
  using P = ViscPlane<S>;
  using A = typename S::arith_t;
  using C = typename S::cs_t;
  extern __shared__ __align__(128) unsigned char ring[];
  __shared__ unsigned long long full[RING];
  __shared__ unsigned long long wmin[TX * TY / 32];
  __shared__ int stop;
  const int tx = threadIdx.x, ty = threadIdx.y, tid = ty * TX + tx;
  const int j0 = g.x_min + TX * (int)blockIdx.x, k0 = g.y_min + TY * (int)blockIdx.y;
  const int l0 = g.z_min + seg * (int)blockIdx.z;
  const int l1 = l0 + seg - 1 < g.z_max ? l0 + seg - 1 : g.z_max;
  const int j = j0 + tx, k = k0 + ty;
  const bool in_jk = j <= g.x_max && k <= g.y_max;
  const int pfirst = l0 - 1, plast = l1 + 1;  // cell planes the segment reads
  if (tid == 0) {
    for (int r = 0; r < RING; r++) mbar_init(&full[r], 1);
    mbar_init_fence();
    stop = 0;
  }
  __syncthreads();
  int issued_hi = pfirst - 1;  // thread 0: the last plane whose copies it issued
  // plane p (node plane p and cell plane p) into its buffer
  auto issue = [&](int p) {
    issued_hi = p;
    const int s = (p - pfirst) % RING;
    unsigned char* b = ring + s * P::kBytes;
    mbar_arrive_expect_tx(&full[s], P::kTx);
    const int x = TX * (int)blockIdx.x, z = p - g.z_min + 2;
    const int yn = k0 - g.y_min + 2, yc = yn - 1;
    tma_load_box(P::vel(b, 0), &maps.u, &full[s], x, yn, z);
    tma_load_box(P::vel(b, 1), &maps.v, &full[s], x, yn, z);
    tma_load_box(P::vel(b, 2), &maps.w, &full[s], x, yn, z);
    tma_load_box(P::rho(b), &maps.d, &full[s], x, yc, z);
    tma_load_box(P::ene(b), &maps.e, &full[s], x, yc, z);
  };
  if (tid == 0)
    for (int p = pfirst; p <= plast && p < pfirst + RING; p++) issue(p);
  auto buf = [&](int p) { return ring + ((p - pfirst) % RING) * P::kBytes; };
  auto wait = [&](int p) {
    const int u = p - pfirst;
    if (!mbar_wait_bounded(&full[u % RING], (unsigned)(u / RING) & 1u)) stop = 1;
  };
  const A a_gs = (A)g_small, a_dtc = (A)dtc_safe, a_dtu = (A)dtu_safe, a_dtv = (A)dtv_safe;
  const A a_dtw = (A)dtw_safe, a_dtdiv = (A)dtdiv_safe;
  // calc_dt's four velocity quotients where the denominator is its floor
  // (1.0e-5 * volume: every cell at rest), formed once: the same operands give
  // the same quotient, so those cells skip the division (FP64 only: the FP32
  // division of the mixed path costs less than the test, measured)
  constexpr bool kFloor = sizeof(A) == 8;
  const A a_vol = (A)g.vol, a_flo = A(1.0e-5) * a_vol, a_flo_div = a_vol * A(1.0e-05);
  const A q_u = a_dtu * A(4.0) * a_vol / a_flo, q_v = a_dtv * A(4.0) * a_vol / a_flo;
  const A q_w = a_dtw * A(4.0) * a_vol / a_flo, q_div = a_dtdiv * A(4.0) * a_vol / a_flo_div;
  constexpr int WV = P::WV, WR = P::WR, WE = P::WE, HV = P::HV, HR = P::HR, HE = P::HE;
  unsigned long long key = ~0ull;
  wait(pfirst);
  wait(pfirst + 1);
  int l = l0;
  for (; l <= l1; l++) {
    wait(l + 1);
    if (in_jk && !stop) {
      unsigned char* bl = buf(l);
      unsigned char* bu = buf(l + 1);
      unsigned char* bd = buf(l - 1);
      // node (j+a, k+b) of a node plane buffer, cell (j+a, k+b) of a cell plane buffer
#define NV(bb, q, a, b) ((A)P::vel(bb, q)[(ty + (b)) * WV + tx + HV + (a)])
#define DN(bb, a, b) ((A)P::rho(bb)[(ty + 1 + (b)) * WR + tx + HR + (a)])
#define EN(bb, a, b) ((A)P::ene(bb)[(ty + 1 + (b)) * WE + tx + HE + (a)])
      const A u000 = NV(bl, 0, 0, 0), u100 = NV(bl, 0, 1, 0), u010 = NV(bl, 0, 0, 1), u110 = NV(bl, 0, 1, 1);
      const A v000 = NV(bl, 1, 0, 0), v100 = NV(bl, 1, 1, 0), v010 = NV(bl, 1, 0, 1), v110 = NV(bl, 1, 1, 1);
      const A w000 = NV(bl, 2, 0, 0), w100 = NV(bl, 2, 1, 0), w010 = NV(bl, 2, 0, 1), w110 = NV(bl, 2, 1, 1);
      const A u001 = NV(bu, 0, 0, 0), u101 = NV(bu, 0, 1, 0), u011 = NV(bu, 0, 0, 1), u111 = NV(bu, 0, 1, 1);
      const A v001 = NV(bu, 1, 0, 0), v101 = NV(bu, 1, 1, 0), v011 = NV(bu, 1, 0, 1), v111 = NV(bu, 1, 1, 1);
      const A w001 = NV(bu, 2, 0, 0), w101 = NV(bu, 2, 1, 0), w011 = NV(bu, 2, 0, 1), w111 = NV(bu, 2, 1, 1);
      const A ugradx1 = u000 + u010 + u001 + u011;
      const A ugradx2 = u100 + u110 + u101 + u111;
      const A vgrady1 = v000 + v100 + v001 + v101;
      const A vgrady2 = v010 + v110 + v011 + v111;
      const A wgradz1 = w000 + w100 + w010 + w110;
      const A wgradz2 = w001 + w101 + w011 + w111;
      const A xa = (A)g.xa, ya = (A)g.ya, za = (A)g.za;
      const A div = (xa * (ugradx2 - ugradx1) + ya * (vgrady2 - vgrady1)) + za * (wgradz2 - wgradz1);
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
        const A cdx = (A)ga.celldx[g.o1 + j - g.x_min + 2];
        const A cdy = (A)ga.celldy[g.o1 + k - g.y_min + 2];
        const A cdz = (A)ga.celldz[g.o1 + l - g.z_min + 2];
        const A xx = A(0.25) * (ugradx2 - ugradx1) / cdx;
        const A yy = A(0.25) * (vgrady2 - vgrady1) / cdy;
        const A zz = A(0.25) * (wgradz2 - wgradz1) / cdz;
        const A xy = A(0.25) * (ugrady2 - ugrady1) / cdy + A(0.25) * (vgradx2 - vgradx1) / cdx;
        const A xz = A(0.25) * (ugradz2 - ugradz1) / cdz + A(0.25) * (wgradx2 - wgradx1) / cdx;
        const A yz = A(0.25) * (vgradz2 - vgradz1) / cdz + A(0.25) * (wgrady2 - wgrady1) / cdy;
        // the neighbours' pressures as ideal_gas stores them
#define PN(bb, a, b) ((A)st<C>(((A(1.4) - A(1.0)) * DN(bb, a, b) * EN(bb, a, b))))
        A pgradx = (PN(bl, 1, 0) - PN(bl, -1, 0)) /
                   (cdx + (A)ga.celldx[g.o1 + j + 1 - g.x_min + 2]);
        A pgrady = (PN(bl, 0, 1) - PN(bl, 0, -1)) /
                   (cdy + (A)ga.celldy[g.o1 + k + 1 - g.y_min + 2]);
        A pgradz = (PN(bu, 0, 0) - PN(bd, 0, 0)) /
                   (cdz + (A)ga.celldz[g.o1 + l + 1 - g.z_min + 2]);
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
          q = A(2.0) * DN(bl, 0, 0) * grad2 * limiter * limiter;
        }
      }
      const long long o = off3(g, j, k, l);
      viscosity[o] = st<C>(q);
      // calc_dt_kernel.f90:102-149 (the viscosity as stored)
      const A visc = (A)st<C>(q);
      const A d0 = DN(bl, 0, 0);
      const A ds = geo_ds<A>(g);
      A ss;
      {
        const A v_eos = A(1.0) / d0;
        const A p_eos = (A(1.4) - A(1.0)) * d0 * EN(bl, 0, 0);
        const A pbe = (A(1.4) - A(1.0)) * d0;
        const A pbv = -d0 * p_eos;
        const A ss2 = v_eos * v_eos * (p_eos * pbe - pbv);
        pressure[o] = st<C>(p_eos);
        const C ss_st = st<C>(sqrt(ss2));
        soundspeed[o] = ss_st;
        ss = (A)ss_st;
      }
      A cc = ss * ss;
      // a zero viscosity over a positive density adds a zero to ss*ss (>= +0):
      // cc is unchanged, without the division
      if (!kFloor || visc != A(0.0) || !(d0 > A(0.0))) cc = cc + A(2.0) * visc / d0;
      A dtct = ds * cc;
      dtct = a_dtc * A(1.0) / fmax2(sqrt(dtct), a_gs);
      const A vol = a_vol;
      const A du1 = ugradx1 * xa, du2 = ugradx2 * xa;
      const A mu = fmax2(fmax2(fabs(du1), fabs(du2)), a_flo);
      const A dtut = kFloor && mu == a_flo ? q_u : a_dtu * A(4.0) * vol / mu;
      const A dv1 = vgrady1 * ya, dv2 = vgrady2 * ya;
      const A mv = fmax2(fmax2(fabs(dv1), fabs(dv2)), a_flo);
      const A dtvt = kFloor && mv == a_flo ? q_v : a_dtv * A(4.0) * vol / mv;
      // both z faces use zarea(j,k,l); its sums add (j,k+1) before (j+1,k)
      const A dw1 = (w000 + w010 + w100 + w110) * za;
      const A dw2 = (w001 + w011 + w101 + w111) * za;
      const A mw = fmax2(fmax2(fabs(dw1), fabs(dw2)), a_flo);
      const A dtwt = kFloor && mw == a_flo ? q_w : a_dtw * A(4.0) * vol / mw;
      const A dvg = du2 - du1 + dv2 - dv1 + dw2 - dw1;
      const A mdv = fmax2(a_flo_div, fabs(dvg));
      const A dtdivt = kFloor && mdv == a_flo_div ? q_div : a_dtdiv * A(4.0) * vol / mdv;
      const A mn = fmin2(fmin2(fmin2(fmin2(dtct, dtut), dtvt), dtwt), dtdivt);
      if (!(mn != mn)) {
        const unsigned long long kc = key_of(mn);
        key = kc < key ? kc : key;
      }
#undef EN
#undef DN
#undef NV
    }
    // every thread is done with plane l-1: its buffer takes plane l-1+RING
    __syncthreads();
    if (stop) break;
    if (tid == 0 && l - 1 + RING <= plast) issue(l - 1 + RING);
  }
  if (stop) {
    // a plane's copies did not arrive in time: report it, and give the copies
    // still in flight (planes from the one waited for last to the last one
    // issued) a bounded wait before the block's shared memory is released
    if (tid == 0) {
      atomicOr(status, CLOVER_STATUS_TIMEOUT);
      for (int p = (l < l1 ? l : l1) + 1; p <= issued_hi; p++) {
        const int u = p - pfirst;
        mbar_wait_bounded(&full[u % RING], (unsigned)(u / RING) & 1u);
      }
    }
    return;
  }
  // warp then block minimum, one atomic per block
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    unsigned long long other = __shfl_xor_sync(0xffffffffu, key, o);
    key = other < key ? other : key;
  }
  if (tx == 0) wmin[ty] = key;
  __syncthreads();
  if (ty == 0) {
    key = tx < TY ? wmin[tx] : ~0ull;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
      unsigned long long other = __shfl_xor_sync(0xffffffffu, key, o);
      key = other < key ? other : key;
    }
    if (tx == 0 && key != ~0ull) atomicMin(min_key, key);
  }
}

// ---------------------------------------------------------------------------
// The x momentum sweep (advec_mom_kernel.f90:166-252 for the three
// velocities) of k_mom_sweep_x (clover_fused.cu), with its inputs staged in
// shared memory. The lane layout stays: lane L of a warp holds node
// j = x_min-2+29t+L of row k, neighbouring nodes' node values come by
// shuffles, lanes 1..30 form momentum fluxes and lanes 2..30 update (29
// nodes per warp), the plane l-1 terms are carried in registers; what
// changes is where the values come from: every mass flux, density, volume
// flux and velocity of plane p arrives with plane p's boxes. Box columns
// start on the 16-byte boundary at or before the block's first node, so a
// lane's node sits `shift` columns into each box (shift depends on the
// element type). Plane p holds mass_flux_x and density1 of rows k0-1..k0+7,
// vol_flux_y of rows k0-1..k0+8 and vol_flux_z of rows k0-1..k0+7 (the post
// volumes of sweep 1; sweep 3 reads none), and the three velocities of rows
// k0..k0+7. Node plane l reads planes l and l+1 (vol_flux_z).
template <class S, int VAR>
struct MomXPlane {
  using MF = typename S::mf_t;
  using R = typename S::rho_t;
  using VF = typename S::vf_t;
  using V = typename S::vel_t;
  static constexpr bool kVf = VAR == 0;
  static constexpr int kMf = round128(9 * kTmaWidth<MF> * (int)sizeof(MF));
  static constexpr int kRho = round128(9 * kTmaWidth<R> * (int)sizeof(R));
  static constexpr int kVfy = kVf ? round128(10 * kTmaWidth<VF> * (int)sizeof(VF)) : 0;
  static constexpr int kVfz = kVf ? round128(9 * kTmaWidth<VF> * (int)sizeof(VF)) : 0;
  static constexpr int kVel = round128(8 * kTmaWidth<V> * (int)sizeof(V));
  static constexpr int kBytes = kMf + kRho + kVfy + kVfz + 3 * kVel;
  static constexpr unsigned kTx = box_bytes<MF>(9) + box_bytes<R>(9) +
                                  (kVf ? box_bytes<VF>(10) + box_bytes<VF>(9) : 0u) +
                                  3 * box_bytes<V>(8);
  __device__ static MF* mf(unsigned char* p) { return (MF*)p; }
  __device__ static R* rho(unsigned char* p) { return (R*)(p + kMf); }
  __device__ static VF* vfy(unsigned char* p) { return (VF*)(p + kMf + kRho); }
  __device__ static VF* vfz(unsigned char* p) { return (VF*)(p + kMf + kRho + kVfy); }
  __device__ static V* vel(unsigned char* p, int q) {
    return (V*)(p + kMf + kRho + kVfy + kVfz + q * kVel);
  }
};

// Box x coordinate of element type T for a block whose first node is
// x_min-2+29t, and the column of that node in the box.
template <class T>
__device__ __forceinline__ void x_box(int t, int& x, int& shift) {
  constexpr int H = kTmaHalo<T>;
  const int c = 29 * t + H - 2;  // the first node's column, counted from the map's base
  x = c / H * H;
  shift = c - x;
}

template <class S, int VAR, int RING, int MINB>
__global__ void __launch_bounds__(TX * TY, MINB)
k_mom_sweep_x_tma(Geom g, int seg, GeomArrays ga, const __grid_constant__ MomXMaps maps,
                  typename S::vel_t* __restrict__ u_out, typename S::vel_t* __restrict__ v_out,
                  typename S::vel_t* __restrict__ w_out, Level0<S> lz, int* __restrict__ status) {
  using P = MomXPlane<S, VAR>;
  using A = typename S::arith_t;
  using V = typename S::vel_t;
  using MF = typename S::mf_t;
  using R = typename S::rho_t;
  using VF = typename S::vf_t;
  extern __shared__ __align__(128) unsigned char ring[];
  __shared__ unsigned long long full[RING];
  __shared__ int stop;
  const int lane = threadIdx.x, ty = threadIdx.y, tid = ty * TX + lane;
  const unsigned fullmask = 0xffffffffu;
  const int j = g.x_min - 2 + 29 * (int)blockIdx.x + lane;  // node of this lane
  const int k0 = g.y_min + TY * (int)blockIdx.y, k = k0 + ty;
  const int l0 = g.z_min + seg * (int)blockIdx.z;
  const int l1 = l0 + seg - 1 < g.z_max + 1 ? l0 + seg - 1 : g.z_max + 1;
  const int pfirst = l0 - 1, plast = l1 + 1;
  const bool row = k <= g.y_max + 1;              // the whole warp: k depends on the row only
  const bool has_nf = row && j <= g.x_max + 2;    // node_flux range j in [x_min-2, x_max+2]
  const bool has_mf = row && lane >= 1 && lane <= 30 && j >= g.x_min - 1 && j <= g.x_max + 1;
  const bool has_up = row && lane >= 2 && lane <= 30 && j >= g.x_min && j <= g.x_max + 1;
  int xm, cm, xr, cr, xf, cf, xv, cv;
  x_box<MF>(blockIdx.x, xm, cm);
  x_box<R>(blockIdx.x, xr, cr);
  x_box<VF>(blockIdx.x, xf, cf);
  x_box<V>(blockIdx.x, xv, cv);
  cm += lane; cr += lane; cf += lane; cv += lane;  // this lane's node in each box
  constexpr int WM = kTmaWidth<MF>, WR = kTmaWidth<R>, WF = kTmaWidth<VF>, WV = kTmaWidth<V>;
  if (tid == 0) {
    for (int r = 0; r < RING; r++) mbar_init(&full[r], 1);
    mbar_init_fence();
    stop = 0;
  }
  __syncthreads();
  int issued_hi = pfirst - 1;
  auto issue = [&](int p) {
    issued_hi = p;
    const int s = (p - pfirst) % RING;
    unsigned char* b = ring + s * P::kBytes;
    mbar_arrive_expect_tx(&full[s], P::kTx);
    const int z = p - g.z_min + 2, y1 = k0 - g.y_min + 1, y0 = y1 + 1;  // rows k0-1.., k0..
    tma_load_box(P::mf(b), &maps.mf, &full[s], xm, y1, z);
    tma_load_box(P::rho(b), &maps.d, &full[s], xr, y1, z);
    if (P::kVf) {
      tma_load_box(P::vfy(b), &maps.vfy, &full[s], xf, y1, z);
      tma_load_box(P::vfz(b), &maps.vfz, &full[s], xf, y1, z);
    }
    tma_load_box(P::vel(b, 0), &maps.u, &full[s], xv, y0, z);
    tma_load_box(P::vel(b, 1), &maps.v, &full[s], xv, y0, z);
    tma_load_box(P::vel(b, 2), &maps.w, &full[s], xv, y0, z);
  };
  if (tid == 0)
    for (int p = pfirst; p <= plast && p < pfirst + RING; p++) issue(p);
  auto buf = [&](int p) { return ring + ((p - pfirst) % RING) * P::kBytes; };
  auto wait = [&](int p) {
    const int u = p - pfirst;
    if (!mbar_wait_bounded(&full[u % RING], (unsigned)(u / RING) & 1u)) stop = 1;
  };
  // values of plane p: mass flux at (j + a, row r) (r = 0 for k-1, 1 for k),
  // and the cell product density1 * post_vol of cell (j, k-1+r)
  auto MFv = [&](unsigned char* b, int r, int a) { return (double)P::mf(b)[(ty + r) * WM + cm + a]; };
  auto prod = [&](unsigned char* b, unsigned char* bz1, int r) {
    const double d = (double)P::rho(b)[(ty + r) * WR + cr];
    double pv = g.vol;
    if (VAR == 0)  // mom_post_vol variant 0, the reference's order
      pv = pv + (double)P::vfy(b)[(ty + r + 1) * WF + cf] - (double)P::vfy(b)[(ty + r) * WF + cf] +
           (double)P::vfz(bz1)[(ty + r) * WF + cf] - (double)P::vfz(b)[(ty + r) * WF + cf];
    return d * pv;
  };
  const double cd_0 = has_nf ? ga.celldx[g.o1 + j - g.x_min + 2] : 1.0;
  const double cd_m1 = has_mf ? ga.celldx[g.o1 + j - 1 - g.x_min + 2] : 1.0;
  const double cd_p1 = has_mf ? ga.celldx[g.o1 + j + 1 - g.x_min + 2] : 1.0;
  typename S::vel_t* out[3] = {u_out, v_out, w_out};
  typename S::vel_t* lev0[3] = {lz.xvel0, lz.yvel0, lz.zvel0};
  // plane l0-1 terms: mass fluxes at (j, k-1), (j, k), (j+1, k-1), (j+1, k);
  // cell products at (j, k-1), (j, k)
  wait(pfirst);
  wait(pfirst + 1);
  double fm_a = 0.0, fm_b = 0.0, fm_c = 0.0, fm_d = 0.0, pm_a = 0.0, pm_b = 0.0;
  if (has_nf && !stop) {
    unsigned char* b = buf(pfirst);
    fm_a = MFv(b, 0, 0); fm_b = MFv(b, 1, 0); fm_c = MFv(b, 0, 1); fm_d = MFv(b, 1, 1);
    pm_a = prod(b, buf(pfirst + 1), 0); pm_b = prod(b, buf(pfirst + 1), 1);
  }
  int l = l0;
  for (; l <= l1; l++) {
    wait(l + 1);
    if (row && !stop) {
      unsigned char* b = buf(l);
      unsigned char* bz = buf(l + 1);
      double f_a = 0.0, f_b = 0.0, f_c = 0.0, f_d = 0.0, p_a = 0.0, p_b = 0.0;
      if (has_nf) {
        f_a = MFv(b, 0, 0); f_b = MFv(b, 1, 0); f_c = MFv(b, 0, 1); f_d = MFv(b, 1, 1);
        p_a = prod(b, bz, 0); p_b = prod(b, bz, 1);
      }
      const double nf = 0.125 * (f_a + f_b + f_c + f_d + fm_a + fm_b + fm_c + fm_d);
      const double q_a = __shfl_up_sync(fullmask, p_a, 1);
      const double q_b = __shfl_up_sync(fullmask, p_b, 1);
      const double qm_a = __shfl_up_sync(fullmask, pm_a, 1);
      const double qm_b = __shfl_up_sync(fullmask, pm_b, 1);
      const double nmp = node_mass_sum(p_a, p_b, q_a, q_b, pm_a, pm_b, qm_a, qm_b);
      const double nf_m = __shfl_up_sync(fullmask, nf, 1);
      const double nmpre = nmp - nf_m + nf;
      const double nmpre_p = __shfl_down_sync(fullmask, nmpre, 1);
      const MomNodeTerms<A> nt =
          mom_node_terms<A>((A)nf, (A)nmpre, (A)nmpre_p, (A)cd_0, (A)cd_m1, (A)cd_p1);
      A vn[3];
#pragma unroll
      for (int q = 0; q < 3; q++) {
        const V* vr = P::vel(b, q) + ty * WV + cv;
        A mf = A(0.0), v0 = A(0.0);
        if (has_mf) {
          v0 = (A)vr[0];
          mf = mom_flux_v<A>(nt, (A)vr[-1], v0, (A)vr[1], (A)vr[2]);
        }
        const A mf_m = __shfl_up_sync(fullmask, mf, 1);
        vn[q] = v0 * (A)nmpre + mf_m - mf;
      }
      if (has_up) {
        div3_rn(vn, (A)nmp);  // the three updates share node_mass_post
        const long long o = off3(g, j, k, l);
#pragma unroll
        for (int q = 0; q < 3; q++) {
          const V vn1 = st<V>(vn[q]);
          out[q][o] = vn1;
          if (lz.xvel0) lev0[q][o] = vn1;  // last sweep of the step: reset_field
        }
      }
      fm_a = f_a; fm_b = f_b; fm_c = f_c; fm_d = f_d;
      pm_a = p_a; pm_b = p_b;
    }
    // every thread is done with plane l-1 (l0-1: read before the loop): its
    // buffer takes plane l-1+RING
    __syncthreads();
    if (stop) break;
    if (tid == 0 && l - 1 + RING <= plast) issue(l - 1 + RING);
  }
  if (stop && tid == 0) {
    atomicOr(status, CLOVER_STATUS_TIMEOUT);
    for (int p = (l < l1 ? l : l1) + 1; p <= issued_hi; p++) {
      const int u = p - pfirst;
      mbar_wait_bounded(&full[u % RING], (unsigned)(u / RING) & 1u);
    }
  }
}

// ---------------------------------------------------------------------------
// The march of a staged block over planes l in [l0, l1]: body(l) reads the
// buffers of planes l-BACK .. l+AHEAD; thread 0 starts plane p's copies with
// issue(p) (which arms the plane's barrier). Plane l-BACK's buffer takes plane
// l-BACK+RING once every thread is done with plane l. A wait that runs out
// stops the block: CLOVER_STATUS_TIMEOUT in *status, and the copies still in
// flight (the last RING planes issued) get a bounded wait before the block's
// shared memory is released. full[RING] and *stop are shared memory.
template <int RING, int BACK, int AHEAD>
struct PlaneMarch {
  unsigned char* ring;
  int bytes;
  unsigned long long* full;
  int* stop;
  int pfirst, plast;
  __device__ unsigned char* buf(int p) const { return ring + ((p - pfirst) % RING) * bytes; }
  __device__ unsigned long long* bar(int p) const { return &full[(p - pfirst) % RING]; }
  __device__ void wait(int p) const {
    const int u = p - pfirst;
    if (!mbar_wait_bounded(&full[u % RING], (unsigned)(u / RING) & 1u)) *stop = 1;
  }
  template <class Issue, class Body>
  __device__ void run(int l0, int l1, int* status, Issue issue, Body body) const {
    const int tid = threadIdx.y * blockDim.x + threadIdx.x;
    if (tid == 0) {
      for (int r = 0; r < RING; r++) mbar_init(&full[r], 1);
      mbar_init_fence();
      *stop = 0;
    }
    __syncthreads();
    int issued_hi = pfirst - 1;
    if (tid == 0)
      for (int p = pfirst; p <= plast && p < pfirst + RING; p++) issue(p), issued_hi = p;
    for (int p = pfirst; p < l0 + AHEAD; p++) wait(p);
    for (int l = l0; l <= l1; l++) {
      wait(l + AHEAD);
      if (!*stop) body(l);
      __syncthreads();
      if (*stop) break;
      const int np = l - BACK + RING;
      if (tid == 0 && np <= plast) issue(np), issued_hi = np;
    }
    if (*stop && tid == 0) {
      atomicOr(status, CLOVER_STATUS_TIMEOUT);
      for (int p = issued_hi - RING + 1 > pfirst ? issued_hi - RING + 1 : pfirst; p <= issued_hi; p++) {
        const int u = p - pfirst;
        mbar_wait_bounded(&full[u % RING], (unsigned)(u / RING) & 1u);
      }
    }
  }
};

// ---------------------------------------------------------------------------
// PdV_kernel.f90:72-118 (predict) + ideal_gas_kernel.f90:47-58 on the predicted
// state, as k_pdv_predict_eos (clover_fused.cu) forms them. Plane p: the
// three node velocities of node plane p (rows k0..k0+8) and density0,
// energy0, pressure and viscosity of cell plane p (rows k0..k0+7). Cell l
// reads node planes l, l+1 and cell plane l.
template <class S>
struct PdvPlane {
  using V = typename S::vel_t;
  using R = typename S::rho_t;
  using En = typename S::ene_t;
  using C = typename S::cs_t;
  static constexpr int kVel = round128(9 * kTmaWidth<V> * (int)sizeof(V));
  static constexpr int kRho = round128(8 * kTmaWidth<R> * (int)sizeof(R));
  static constexpr int kEne = round128(8 * kTmaWidth<En> * (int)sizeof(En));
  static constexpr int kCs = round128(8 * kTmaWidth<C> * (int)sizeof(C));
  static constexpr int kBytes = 3 * kVel + kRho + kEne + 2 * kCs;
  static constexpr unsigned kTx = 3 * box_bytes<V>(9) + box_bytes<R>(8) + box_bytes<En>(8) +
                                  2 * box_bytes<C>(8);
  __device__ static V* vel(unsigned char* p, int q) { return (V*)(p + q * kVel); }
  __device__ static R* rho(unsigned char* p) { return (R*)(p + 3 * kVel); }
  __device__ static En* ene(unsigned char* p) { return (En*)(p + 3 * kVel + kRho); }
  __device__ static C* cs(unsigned char* p, int q) { return (C*)(p + 3 * kVel + kRho + kEne + q * kCs); }
};

template <class S, int RING, int MINB>
__global__ void __launch_bounds__(TX * TY, MINB)
k_pdv_predict_eos_tma(Geom g, int seg, const double* __restrict__ dt_ptr,
                      const __grid_constant__ PdvMaps maps, typename S::cs_t* __restrict__ pressure,
                      int* __restrict__ status) {
  using P = PdvPlane<S>;
  using A = typename S::arith_t;
  using V = typename S::vel_t;
  using R = typename S::rho_t;
  using En = typename S::ene_t;
  using C = typename S::cs_t;
  extern __shared__ __align__(128) unsigned char ring[];
  __shared__ unsigned long long full[RING];
  __shared__ int stop;
  const int tx = threadIdx.x, ty = threadIdx.y;
  const int j = g.x_min + TX * (int)blockIdx.x + tx, k0 = g.y_min + TY * (int)blockIdx.y;
  const int k = k0 + ty;
  const int l0 = g.z_min + seg * (int)blockIdx.z;
  const int l1 = l0 + seg - 1 < g.z_max ? l0 + seg - 1 : g.z_max;
  const bool in_jk = j <= g.x_max && k <= g.y_max;
  const PlaneMarch<RING, 0, 1> pm{ring, P::kBytes, full, &stop, l0, l1 + 1};
  const A dt = (A)dt_ptr[0];
  constexpr int WV = kTmaWidth<V>, HV = kTmaHalo<V>, WR = kTmaWidth<R>, HR = kTmaHalo<R>;
  constexpr int WE = kTmaWidth<En>, HE = kTmaHalo<En>, WC = kTmaWidth<C>, HC = kTmaHalo<C>;
  auto issue = [&](int p) {
    unsigned char* b = pm.buf(p);
    unsigned long long* bar = pm.bar(p);
    mbar_arrive_expect_tx(bar, P::kTx);
    const int x = TX * (int)blockIdx.x, y = k0 - g.y_min + 2, z = p - g.z_min + 2;
    tma_load_box(P::vel(b, 0), &maps.u, bar, x, y, z);
    tma_load_box(P::vel(b, 1), &maps.v, bar, x, y, z);
    tma_load_box(P::vel(b, 2), &maps.w, bar, x, y, z);
    tma_load_box(P::rho(b), &maps.d, bar, x, y, z);
    tma_load_box(P::ene(b), &maps.e, bar, x, y, z);
    tma_load_box(P::cs(b, 0), &maps.p, bar, x, y, z);
    tma_load_box(P::cs(b, 1), &maps.q, bar, x, y, z);
  };
  pm.run(l0, l1, status, issue, [&](int l) {
    if (!in_jk) return;
    unsigned char* bl = pm.buf(l);
    unsigned char* bu = pm.buf(l + 1);
    // velocity q of node (j+a, k+b) of a node plane buffer
#define NV(bb, q, a, b) ((A)P::vel(bb, q)[(ty + (b)) * WV + tx + HV + (a)])
#define XS(a) (NV(bl, 0, a, 0) + NV(bl, 0, a, 1) + NV(bu, 0, a, 0) + NV(bu, 0, a, 1))
#define YS(b) (NV(bl, 1, 0, b) + NV(bl, 1, 1, b) + NV(bu, 1, 0, b) + NV(bu, 1, 1, b))
#define ZS(bb) (NV(bb, 2, 0, 0) + NV(bb, 2, 1, 0) + NV(bb, 2, 0, 1) + NV(bb, 2, 1, 1))
    // the predictor sums the same four node values twice (vel0 + vel0)
    A sm;
    sm = XS(0);
    const A left_flux = ((A)g.xa * (sm + NV(bl, 0, 0, 0) + NV(bl, 0, 0, 1) + NV(bu, 0, 0, 0) +
                                    NV(bu, 0, 0, 1))) * A(0.125) * dt * A(0.5);
    sm = XS(1);
    const A right_flux = ((A)g.xa * (sm + NV(bl, 0, 1, 0) + NV(bl, 0, 1, 1) + NV(bu, 0, 1, 0) +
                                     NV(bu, 0, 1, 1))) * A(0.125) * dt * A(0.5);
    sm = YS(0);
    const A bottom_flux = ((A)g.ya * (sm + NV(bl, 1, 0, 0) + NV(bl, 1, 1, 0) + NV(bu, 1, 0, 0) +
                                      NV(bu, 1, 1, 0))) * A(0.125) * dt * A(0.5);
    sm = YS(1);
    const A top_flux = ((A)g.ya * (sm + NV(bl, 1, 0, 1) + NV(bl, 1, 1, 1) + NV(bu, 1, 0, 1) +
                                   NV(bu, 1, 1, 1))) * A(0.125) * dt * A(0.5);
    sm = ZS(bl);
    const A back_flux = ((A)g.za * (sm + NV(bl, 2, 0, 0) + NV(bl, 2, 1, 0) + NV(bl, 2, 0, 1) +
                                    NV(bl, 2, 1, 1))) * A(0.125) * dt * A(0.5);
    sm = ZS(bu);
    const A front_flux = ((A)g.za * (sm + NV(bu, 2, 0, 0) + NV(bu, 2, 1, 0) + NV(bu, 2, 0, 1) +
                                     NV(bu, 2, 1, 1))) * A(0.125) * dt * A(0.5);
#undef ZS
#undef YS
#undef XS
#undef NV
    const A total_flux = right_flux - left_flux + top_flux - bottom_flux + front_flux - back_flux;
    const A vol = (A)g.vol;
    const A vol_change_s = div_rn(vol, vol + total_flux);
    const A recip_volume = geo_rvol<A>(g);  // 1/volume
    const A d0 = (A)P::rho(bl)[ty * WR + tx + HR];
    const A energy_change = quot_pair_sum((A)P::cs(bl, 0)[ty * WC + tx + HC],
                                          (A)P::cs(bl, 1)[ty * WC + tx + HC], d0) *
                            total_flux * recip_volume;
    // the predicted state goes through the storage types, as it would in memory
    const A e1 = (A)st<En>(((A)P::ene(bl)[ty * WE + tx + HE] - energy_change));
    const A d1 = (A)st<R>((d0 * vol_change_s));
    pressure[off3(g, j, k, l)] = st<C>(((A(1.4) - A(1.0)) * d1 * e1));
  });
}

// ---------------------------------------------------------------------------
// accelerate_kernel.f90:61-109 on the uniform mesh, as k_accelerate
// (clover_kernels.cu) forms it. Plane p: density0, pressure and viscosity of
// cell plane p (rows k0-1..k0+7) and the three node velocities of node plane
// p (rows k0..k0+7). Node l reads cell planes l-1, l and node plane l.
template <class S>
struct AccPlane {
  using V = typename S::vel_t;
  using R = typename S::rho_t;
  using C = typename S::cs_t;
  static constexpr int kRho = round128(9 * kTmaWidth<R> * (int)sizeof(R));
  static constexpr int kCs = round128(9 * kTmaWidth<C> * (int)sizeof(C));
  static constexpr int kVel = round128(8 * kTmaWidth<V> * (int)sizeof(V));
  static constexpr int kBytes = kRho + 2 * kCs + 3 * kVel;
  static constexpr unsigned kTx = box_bytes<R>(9) + 2 * box_bytes<C>(9) + 3 * box_bytes<V>(8);
  __device__ static R* rho(unsigned char* p) { return (R*)p; }
  __device__ static C* cs(unsigned char* p, int q) { return (C*)(p + kRho + q * kCs); }
  __device__ static V* vel(unsigned char* p, int q) { return (V*)(p + kRho + 2 * kCs + q * kVel); }
};

template <class S, int RING, int MINB>
__global__ void __launch_bounds__(TX * TY, MINB)
k_accelerate_tma(Geom g, int seg, const double* __restrict__ dt_ptr,
                 const __grid_constant__ AccMaps maps, typename S::vel_t* __restrict__ xvel1,
                 typename S::vel_t* __restrict__ yvel1, typename S::vel_t* __restrict__ zvel1,
                 int* __restrict__ status) {
  using P = AccPlane<S>;
  using A = typename S::arith_t;
  using V = typename S::vel_t;
  using R = typename S::rho_t;
  using C = typename S::cs_t;
  extern __shared__ __align__(128) unsigned char ring[];
  __shared__ unsigned long long full[RING];
  __shared__ int stop;
  const int tx = threadIdx.x, ty = threadIdx.y;
  const int j = g.x_min + TX * (int)blockIdx.x + tx, k0 = g.y_min + TY * (int)blockIdx.y;
  const int k = k0 + ty;
  const int l0 = g.z_min + seg * (int)blockIdx.z;
  const int l1 = l0 + seg - 1 < g.z_max + 1 ? l0 + seg - 1 : g.z_max + 1;
  const bool in_jk = j <= g.x_max + 1 && k <= g.y_max + 1;
  const PlaneMarch<RING, 1, 0> pm{ring, P::kBytes, full, &stop, l0 - 1, l1};
  const double dt = dt_ptr[0];
  constexpr int WV = kTmaWidth<V>, HV = kTmaHalo<V>, WR = kTmaWidth<R>, HR = kTmaHalo<R>;
  constexpr int WC = kTmaWidth<C>, HC = kTmaHalo<C>;
  auto issue = [&](int p) {
    unsigned char* b = pm.buf(p);
    unsigned long long* bar = pm.bar(p);
    mbar_arrive_expect_tx(bar, P::kTx);
    const int x = TX * (int)blockIdx.x, y1 = k0 - g.y_min + 1, z = p - g.z_min + 2;
    tma_load_box(P::rho(b), &maps.d, bar, x, y1, z);
    tma_load_box(P::cs(b, 0), &maps.p, bar, x, y1, z);
    tma_load_box(P::cs(b, 1), &maps.q, bar, x, y1, z);
    tma_load_box(P::vel(b, 0), &maps.u, bar, x, y1 + 1, z);
    tma_load_box(P::vel(b, 1), &maps.v, bar, x, y1 + 1, z);
    tma_load_box(P::vel(b, 2), &maps.w, bar, x, y1 + 1, z);
  };
  pm.run(l0, l1, status, issue, [&](int l) {
    if (!in_jk) return;
    unsigned char* bl = pm.buf(l);
    unsigned char* bd = pm.buf(l - 1);
    // cell (j+a, k+b) of the cell plane buffer bb (a, b in {-1, 0})
#define DC(bb, a, b) ((double)P::rho(bb)[(ty + 1 + (b)) * WR + tx + HR + (a)])
#define DV(a, b, c) (DC((c) ? bd : bl, a, b) * g.vol)
    const double nodal_mass = (DV(-1, -1, 0) + DV(0, -1, 0) + DV(0, 0, 0) + DV(-1, 0, 0) +
                               DV(-1, -1, -1) + DV(0, -1, -1) + DV(0, 0, -1) + DV(-1, 0, -1)) * 0.125;
#undef DV
#undef DC
    const double stepbymass_d = 0.25 * dt / nodal_mass;
    const A stepbymass_s = (A)stepbymass_d;
#define CS(bb, q, a, b) ((A)P::cs(bb, q)[(ty + 1 + (b)) * WC + tx + HC + (a)])
    const A p000 = CS(bl, 0, 0, 0), p100 = CS(bl, 0, -1, 0);
    const A p010 = CS(bl, 0, 0, -1), p110 = CS(bl, 0, -1, -1);
    const A p001 = CS(bd, 0, 0, 0), p101 = CS(bd, 0, -1, 0);
    const A p011 = CS(bd, 0, 0, -1), p111 = CS(bd, 0, -1, -1);
    const A q000 = CS(bl, 1, 0, 0), q100 = CS(bl, 1, -1, 0);
    const A q010 = CS(bl, 1, 0, -1), q110 = CS(bl, 1, -1, -1);
    const A q001 = CS(bd, 1, 0, 0), q101 = CS(bd, 1, -1, 0);
    const A q011 = CS(bd, 1, 0, -1), q111 = CS(bd, 1, -1, -1);
#undef CS
    const A xa0 = (A)g.xa, xa1 = (A)g.xa, xa2 = (A)g.xa, xa3 = (A)g.xa;
    const A ya0 = (A)g.ya, ya1 = (A)g.ya, ya2 = (A)g.ya, ya3 = (A)g.ya;
    const A za0 = (A)g.za, za1 = (A)g.za, za2 = (A)g.za, za3 = (A)g.za;
    const int c = ty * WV + tx + HV;
    const A xvel1_s = (A)P::vel(bl, 0)[c] -
        stepbymass_s * (xa0 * (p000 - p100) + xa1 * (p010 - p110) + xa2 * (p001 - p101) +
                        xa3 * (p011 - p111));
    const A yvel1_s = (A)P::vel(bl, 1)[c] -
        stepbymass_s * (ya0 * (p000 - p010) + ya1 * (p100 - p110) + ya2 * (p001 - p011) +
                        ya3 * (p101 - p111));
    const A zvel1_s = (A)P::vel(bl, 2)[c] -
        stepbymass_s * (za0 * (p000 - p001) + za1 * (p010 - p011) + za2 * (p100 - p101) +
                        za3 * (p110 - p111));
    const long long o = off3(g, j, k, l);
    xvel1[o] = st<V>(xvel1_s -
        stepbymass_s * (xa0 * (q000 - q100) + xa1 * (q010 - q110) + xa2 * (q001 - q101) +
                        xa3 * (q011 - q111)));
    yvel1[o] = st<V>(yvel1_s -
        stepbymass_s * (ya0 * (q000 - q010) + ya1 * (q100 - q110) + ya2 * (q001 - q011) +
                        ya3 * (q101 - q111)));
    zvel1[o] = st<V>(zvel1_s -
        stepbymass_s * (za0 * (q000 - q001) + za1 * (q010 - q011) + za2 * (q100 - q101) +
                        za3 * (q110 - q111)));
  });
}

// ---------------------------------------------------------------------------
// PdV_kernel.f90:120-166 (corrector) + flux_calc_kernel.f90:58-91 over the
// node box [min, max+1]^3, as k_pdv_flux (clover_fused.cu) forms them. Plane p:
// the time level 0 and 1 velocities of node plane p (rows k0..k0+8); the
// cell's own density0, energy0, pressure and viscosity are read directly.
template <class S>
struct FluxPlane {
  using V = typename S::vel_t;
  static constexpr int kVel = round128(9 * kTmaWidth<V> * (int)sizeof(V));
  static constexpr int kBytes = 6 * kVel;
  static constexpr unsigned kTx = 6 * box_bytes<V>(9);
  __device__ static V* vel(unsigned char* p, int q) { return (V*)(p + q * kVel); }
};

template <class S, int RING, int MINB>
__global__ void __launch_bounds__(TX * TY, MINB)
k_pdv_flux_tma(Geom g, int seg, const double* __restrict__ dt_ptr,
               const __grid_constant__ FluxMaps maps, const typename S::rho_t* __restrict__ density0,
               typename S::rho_t* __restrict__ density1, const typename S::ene_t* __restrict__ energy0,
               typename S::ene_t* __restrict__ energy1, const typename S::cs_t* __restrict__ pressure,
               const typename S::cs_t* __restrict__ viscosity, typename S::vf_t* __restrict__ vol_flux_x,
               typename S::vf_t* __restrict__ vol_flux_y, typename S::vf_t* __restrict__ vol_flux_z,
               int* __restrict__ status) {
  using P = FluxPlane<S>;
  using A = typename S::arith_t;
  using V = typename S::vel_t;
  using F = typename S::vf_t;
  extern __shared__ __align__(128) unsigned char ring[];
  __shared__ unsigned long long full[RING];
  __shared__ int stop;
  const int tx = threadIdx.x, ty = threadIdx.y;
  const int j = g.x_min + TX * (int)blockIdx.x + tx, k0 = g.y_min + TY * (int)blockIdx.y;
  const int k = k0 + ty;
  const int l0 = g.z_min + seg * (int)blockIdx.z;
  const int l1 = l0 + seg - 1 < g.z_max + 1 ? l0 + seg - 1 : g.z_max + 1;
  const bool in_jk = j <= g.x_max + 1 && k <= g.y_max + 1;
  const PlaneMarch<RING, 0, 1> pm{ring, P::kBytes, full, &stop, l0, l1 + 1};
  const double dt = dt_ptr[0];
  constexpr int WV = kTmaWidth<V>, HV = kTmaHalo<V>;
  // the cell's own density0, energy0, pressure and viscosity, loaded one plane
  // ahead (in flight across the block's barrier)
  using R = typename S::rho_t;
  using En = typename S::ene_t;
  using Cs = typename S::cs_t;
  const bool in_cell = j <= g.x_max && k <= g.y_max;
  R c_d = R(0);
  En c_e = En(0);
  Cs c_p = Cs(0), c_q = Cs(0);
  auto fetch = [&](int l) {
    if (in_cell && l <= g.z_max) {
      const long long o = off3(g, j, k, l);
      c_d = __ldg(&density0[o]);
      c_e = __ldg(&energy0[o]);
      c_p = __ldg(&pressure[o]);
      c_q = __ldg(&viscosity[o]);
    }
  };
  fetch(l0);
  auto issue = [&](int p) {
    unsigned char* b = pm.buf(p);
    unsigned long long* bar = pm.bar(p);
    mbar_arrive_expect_tx(bar, P::kTx);
    const int x = TX * (int)blockIdx.x, y = k0 - g.y_min + 2, z = p - g.z_min + 2;
    tma_load_box(P::vel(b, 0), &maps.u0, bar, x, y, z);
    tma_load_box(P::vel(b, 1), &maps.v0, bar, x, y, z);
    tma_load_box(P::vel(b, 2), &maps.w0, bar, x, y, z);
    tma_load_box(P::vel(b, 3), &maps.u1, bar, x, y, z);
    tma_load_box(P::vel(b, 4), &maps.v1, bar, x, y, z);
    tma_load_box(P::vel(b, 5), &maps.w1, bar, x, y, z);
  };
  pm.run(l0, l1, status, issue, [&](int l) {
    if (!in_jk) return;
    const R d0_s = c_d;
    const En e0_s = c_e;
    const Cs p_s = c_p, q_s = c_q;
    fetch(l + 1);
    const bool jin = j <= g.x_max, kin = k <= g.y_max, lin = l <= g.z_max;
    unsigned char* bl = pm.buf(l);
    unsigned char* bu = pm.buf(l + 1);
    // velocity q (0-2 time level 0, 3-5 time level 1) of node (j+a, k+b) of buffer bb
#define NV(bb, q, a, b) ((A)P::vel(bb, q)[(ty + (b)) * WV + tx + HV + (a)])
    auto xsum = [&](int a) {
      return (double)(NV(bl, 0, a, 0) + NV(bl, 0, a, 1) + NV(bu, 0, a, 0) + NV(bu, 0, a, 1) +
                      NV(bl, 3, a, 0) + NV(bl, 3, a, 1) + NV(bu, 3, a, 0) + NV(bu, 3, a, 1));
    };
    auto ysum = [&](int b) {
      return (double)(NV(bl, 1, 0, b) + NV(bl, 1, 1, b) + NV(bu, 1, 0, b) + NV(bu, 1, 1, b) +
                      NV(bl, 4, 0, b) + NV(bl, 4, 1, b) + NV(bu, 4, 0, b) + NV(bu, 4, 1, b));
    };
    auto zsum = [&](unsigned char* bb) {
      return (double)(NV(bb, 2, 0, 0) + NV(bb, 2, 1, 0) + NV(bb, 2, 0, 1) + NV(bb, 2, 1, 1) +
                      NV(bb, 5, 0, 0) + NV(bb, 5, 1, 0) + NV(bb, 5, 0, 1) + NV(bb, 5, 1, 1));
    };
    const long long o = off3(g, j, k, l);
    double sx = 0, sy = 0, sz = 0;
    F vfx0 = F(0), vfy0 = F(0);
    if (kin && lin) {
      sx = xsum(0);
      vfx0 = st<F>(0.125 * dt * g.xa * sx);
      vol_flux_x[o] = vfx0;
    }
    if (jin && lin) {
      sy = ysum(0);
      vfy0 = st<F>(0.125 * dt * g.ya * sy);
      vol_flux_y[o] = vfy0;
    }
    if (jin && kin) {
      // flux_calc_kernel.f90:86 repeats zvel0(j+1,k,l) and omits zvel0(j,k+1,l)
      const double bz = (double)(NV(bl, 2, 0, 0) + NV(bl, 2, 1, 0) + NV(bl, 2, 1, 0) +
                                 NV(bl, 2, 1, 1) + NV(bl, 5, 0, 0) + NV(bl, 5, 1, 0) +
                                 NV(bl, 5, 0, 1) + NV(bl, 5, 1, 1));
      vol_flux_z[o] = st<F>(0.125 * dt * g.za * bz);
      sz = zsum(bl);
    }
#undef NV
    if (!(jin && kin && lin)) return;
    double left_flux, right_flux, bottom_flux, top_flux, back_flux, front_flux;
    if (sizeof(F) == 8) {  // PdV_kernel.f90:120-131 order
      left_flux = (g.xa * sx) * 0.125 * dt;
      right_flux = (g.xa * xsum(1)) * 0.125 * dt;
      bottom_flux = (g.ya * sy) * 0.125 * dt;
      top_flux = (g.ya * ysum(1)) * 0.125 * dt;
      back_flux = (g.za * sz) * 0.125 * dt;
      front_flux = (g.za * zsum(bu)) * 0.125 * dt;
    } else {
      // FP32 volume fluxes: the corrector's face fluxes as the volume fluxes
      // are stored (the z faces from the corrector's own node sums)
      auto stored = [&](double area, double s) { return (double)st<F>(0.125 * dt * area * s); };
      left_flux = (double)vfx0;
      right_flux = stored(g.xa, xsum(1));
      bottom_flux = (double)vfy0;
      top_flux = stored(g.ya, ysum(1));
      back_flux = stored(g.za, sz);
      front_flux = stored(g.za, zsum(bu));
    }
    const double total_flux = right_flux - left_flux + top_flux - bottom_flux + front_flux - back_flux;
    const double vol = g.vol;
    const double vol_change_s = vol / (vol + total_flux);
    const double d0 = (double)d0_s;
    const A ad0 = (A)d0;
    const A energy_change = ((A)p_s / ad0 + (A)q_s / ad0) * (A)total_flux * geo_rvol<A>(g);
    energy1[o] = st<typename S::ene_t>(((A)e0_s - energy_change));
    density1[o] = st<typename S::rho_t>(d0 * vol_change_s);
  });
}

// ---------------------------------------------------------------------------
// PdV_kernel.f90:72-166 over the drop-in caller's arrays (the face areas and
// the volume are arrays there, not the uniform mesh's constants), as k_pdv
// (clover_kernels.cu) forms it. Plane p: the time level 0 node velocities of
// node plane p (rows k0..k0+8; the corrector also the time level 1
// velocities), xarea and zarea of plane p (rows k0..k0+7) and yarea (rows
// k0..k0+8). Cell l reads node and z-face planes l, l+1 and the x/y-face
// plane l; its own volume, density0, energy0, pressure and viscosity are
// loaded one plane ahead into registers.
template <bool PRED>
struct PdvDropPlane {
  static constexpr int kNv = PRED ? 3 : 6;
  static constexpr int W = kTmaWidth<double>;
  static constexpr int k9 = round128(9 * W * 8);
  static constexpr int k8 = round128(8 * W * 8);
  static constexpr int kBytes = kNv * k9 + k9 + 2 * k8;
  static constexpr unsigned kTx = kNv * box_bytes<double>(9) + box_bytes<double>(9) +
                                  2 * box_bytes<double>(8);
  __device__ static double* vel(unsigned char* p, int q) { return (double*)(p + q * k9); }
  __device__ static double* ya(unsigned char* p) { return (double*)(p + kNv * k9); }
  __device__ static double* xa(unsigned char* p) { return (double*)(p + (kNv + 1) * k9); }
  __device__ static double* za(unsigned char* p) { return (double*)(p + (kNv + 1) * k9 + k8); }
};

template <bool PRED, int RING, int MINB>
__global__ void __launch_bounds__(TX * TY, MINB)
k_pdv_dropin_tma(Geom g, int seg, double dt, const __grid_constant__ PdvDropMaps maps,
                 const double* __restrict__ volume, const double* __restrict__ density0,
                 double* __restrict__ density1, const double* __restrict__ energy0,
                 double* __restrict__ energy1, const double* __restrict__ pressure,
                 const double* __restrict__ viscosity, int* __restrict__ status) {
  using P = PdvDropPlane<PRED>;
  extern __shared__ __align__(128) unsigned char ring[];
  __shared__ unsigned long long full[RING];
  __shared__ int stop;
  const int tx = threadIdx.x, ty = threadIdx.y;
  const int j = g.x_min + TX * (int)blockIdx.x + tx, k0 = g.y_min + TY * (int)blockIdx.y;
  const int k = k0 + ty;
  const int l0 = g.z_min + seg * (int)blockIdx.z;
  const int l1 = l0 + seg - 1 < g.z_max ? l0 + seg - 1 : g.z_max;
  const bool in_jk = j <= g.x_max && k <= g.y_max;
  const PlaneMarch<RING, 0, 1> pm{ring, P::kBytes, full, &stop, l0, l1 + 1};
  constexpr int W = P::W, H = kTmaHalo<double>;
  double c_v = 0, c_d = 0, c_e = 0, c_p = 0, c_q = 0;
  auto fetch = [&](int l) {
    if (in_jk && l <= l1) {
      const long long o = off3(g, j, k, l);
      c_v = __ldg(&volume[o]);
      c_d = __ldg(&density0[o]);
      c_e = __ldg(&energy0[o]);
      c_p = __ldg(&pressure[o]);
      c_q = __ldg(&viscosity[o]);
    }
  };
  fetch(l0);
  auto issue = [&](int p) {
    unsigned char* b = pm.buf(p);
    unsigned long long* bar = pm.bar(p);
    mbar_arrive_expect_tx(bar, P::kTx);
    const int x = TX * (int)blockIdx.x, y = k0 - g.y_min + 2, z = p - g.z_min + 2;
    tma_load_box(P::vel(b, 0), &maps.u0, bar, x, y, z);
    tma_load_box(P::vel(b, 1), &maps.v0, bar, x, y, z);
    tma_load_box(P::vel(b, 2), &maps.w0, bar, x, y, z);
    if (!PRED) {
      tma_load_box(P::vel(b, 3), &maps.u1, bar, x, y, z);
      tma_load_box(P::vel(b, 4), &maps.v1, bar, x, y, z);
      tma_load_box(P::vel(b, 5), &maps.w1, bar, x, y, z);
    }
    tma_load_box(P::ya(b), &maps.ya, bar, x, y, z);
    tma_load_box(P::xa(b), &maps.xa, bar, x, y, z);
    tma_load_box(P::za(b), &maps.za, bar, x, y, z);
  };
  pm.run(l0, l1, status, issue, [&](int l) {
    if (!in_jk) return;
    const double vol = c_v, d0 = c_d, e0 = c_e, pr = c_p, vi = c_q;
    fetch(l + 1);
    unsigned char* bl = pm.buf(l);
    unsigned char* bu = pm.buf(l + 1);
    // velocity q of node (j+a, k+b) of a node plane buffer; the predictor's
    // second set is time level 0 again
#define NV(bb, q, a, b) (P::vel(bb, q)[(ty + (b)) * W + tx + H + (a)])
    constexpr int q1 = PRED ? 0 : 3;
    auto xsum = [&](int a) {
      return NV(bl, 0, a, 0) + NV(bl, 0, a, 1) + NV(bu, 0, a, 0) + NV(bu, 0, a, 1) +
             NV(bl, q1, a, 0) + NV(bl, q1, a, 1) + NV(bu, q1, a, 0) + NV(bu, q1, a, 1);
    };
    auto ysum = [&](int b) {
      return NV(bl, 1, 0, b) + NV(bl, 1, 1, b) + NV(bu, 1, 0, b) + NV(bu, 1, 1, b) +
             NV(bl, q1 + 1, 0, b) + NV(bl, q1 + 1, 1, b) + NV(bu, q1 + 1, 0, b) +
             NV(bu, q1 + 1, 1, b);
    };
    auto zsum = [&](unsigned char* bb) {
      return NV(bb, 2, 0, 0) + NV(bb, 2, 1, 0) + NV(bb, 2, 0, 1) + NV(bb, 2, 1, 1) +
             NV(bb, q1 + 2, 0, 0) + NV(bb, q1 + 2, 1, 0) + NV(bb, q1 + 2, 0, 1) +
             NV(bb, q1 + 2, 1, 1);
    };
#undef NV
    const double xa0 = P::xa(bl)[ty * W + tx + H], xa1 = P::xa(bl)[ty * W + tx + H + 1];
    const double ya0 = P::ya(bl)[ty * W + tx + H], ya1 = P::ya(bl)[(ty + 1) * W + tx + H];
    const double za0 = P::za(bl)[ty * W + tx + H], za1 = P::za(bu)[ty * W + tx + H];
    double left_flux, right_flux, bottom_flux, top_flux, back_flux, front_flux;
    if (PRED) {
      left_flux = (xa0 * xsum(0)) * 0.125 * dt * 0.5;
      right_flux = (xa1 * xsum(1)) * 0.125 * dt * 0.5;
      bottom_flux = (ya0 * ysum(0)) * 0.125 * dt * 0.5;
      top_flux = (ya1 * ysum(1)) * 0.125 * dt * 0.5;
      back_flux = (za0 * zsum(bl)) * 0.125 * dt * 0.5;
      front_flux = (za1 * zsum(bu)) * 0.125 * dt * 0.5;
    } else {
      left_flux = (xa0 * xsum(0)) * 0.125 * dt;
      right_flux = (xa1 * xsum(1)) * 0.125 * dt;
      bottom_flux = (ya0 * ysum(0)) * 0.125 * dt;
      top_flux = (ya1 * ysum(1)) * 0.125 * dt;
      back_flux = (za0 * zsum(bl)) * 0.125 * dt;
      front_flux = (za1 * zsum(bu)) * 0.125 * dt;
    }
    const double total_flux = right_flux - left_flux + top_flux - bottom_flux + front_flux - back_flux;
    const double vol_change_s = div_rn(vol, vol + total_flux);
    const double recip_volume = div_rn(1.0, vol);
    const double energy_change = quot_pair_sum(pr, vi, d0) * total_flux * recip_volume;
    const long long o = off3(g, j, k, l);
    energy1[o] = e0 - energy_change;
    density1[o] = d0 * vol_change_s;
  });
}

// ---------------------------------------------------------------------------
// The other one-cell-per-thread stencils of the drop-in over the caller's
// arrays, staged the same way (FP64, one chunk): a box per array and plane,
// the boxes a plane's cells or nodes do not read left out (their bytes are
// not expected on the plane's barrier).
constexpr int kDropW = kTmaWidth<double>, kDropH = kTmaHalo<double>;
constexpr int kBox8 = round128(8 * kDropW * 8), kBox9 = round128(9 * kDropW * 8);
constexpr int kBox10 = round128(10 * kDropW * 8);

// calc_dt_kernel.f90:102-149 as k_calc_dt forms it. Plane p: the node
// velocities of node plane p (rows k0..k0+8) and, for cell plane p, the sound
// speed, viscosity, density0, volume and the three face areas (rows
// k0..k0+7; not on the last node plane). Cell l reads planes l and l+1.
struct DtDropPlane {
  static constexpr int kBytes = 3 * kBox9 + 7 * kBox8;
  static constexpr unsigned kTxVel = 3 * box_bytes<double>(9);
  static constexpr unsigned kTxCell = 7 * box_bytes<double>(8);
  __device__ static double* vel(unsigned char* p, int q) { return (double*)(p + q * kBox9); }
  // 0 soundspeed, 1 viscosity, 2 density0, 3 volume, 4 xarea, 5 yarea, 6 zarea
  __device__ static double* cell(unsigned char* p, int q) {
    return (double*)(p + 3 * kBox9 + q * kBox8);
  }
};

template <int RING, int MINB>
__global__ void __launch_bounds__(TX * TY, MINB)
k_calc_dt_dropin_tma(Geom g, int seg, GeomArrays ga, double g_small, double dtc_safe,
                     double dtu_safe, double dtv_safe, double dtw_safe, double dtdiv_safe,
                     const __grid_constant__ DtDropMaps maps, double* __restrict__ dt_min,
                     unsigned long long* __restrict__ min_key, int* __restrict__ status) {
  using P = DtDropPlane;
  extern __shared__ __align__(128) unsigned char ring[];
  __shared__ unsigned long long full[RING];
  __shared__ unsigned long long wmin[TX * TY / 32];
  __shared__ int stop;
  const int tx = threadIdx.x, ty = threadIdx.y;
  const int j = g.x_min + TX * (int)blockIdx.x + tx, k0 = g.y_min + TY * (int)blockIdx.y;
  const int k = k0 + ty;
  const int l0 = g.z_min + seg * (int)blockIdx.z;
  const int l1 = l0 + seg - 1 < g.z_max ? l0 + seg - 1 : g.z_max;
  const bool in_jk = j <= g.x_max && k <= g.y_max;
  const PlaneMarch<RING, 0, 1> pm{ring, P::kBytes, full, &stop, l0, l1 + 1};
  constexpr int W = kDropW, H = kDropH;
  auto issue = [&](int p) {
    unsigned char* b = pm.buf(p);
    unsigned long long* bar = pm.bar(p);
    const bool cells = p <= l1;
    mbar_arrive_expect_tx(bar, P::kTxVel + (cells ? P::kTxCell : 0u));
    const int x = TX * (int)blockIdx.x, y = k0 - g.y_min + 2, z = p - g.z_min + 2;
    tma_load_box(P::vel(b, 0), &maps.u, bar, x, y, z);
    tma_load_box(P::vel(b, 1), &maps.v, bar, x, y, z);
    tma_load_box(P::vel(b, 2), &maps.w, bar, x, y, z);
    if (cells) {
      tma_load_box(P::cell(b, 0), &maps.ss, bar, x, y, z);
      tma_load_box(P::cell(b, 1), &maps.q, bar, x, y, z);
      tma_load_box(P::cell(b, 2), &maps.d, bar, x, y, z);
      tma_load_box(P::cell(b, 3), &maps.vol, bar, x, y, z);
      tma_load_box(P::cell(b, 4), &maps.xa, bar, x, y, z);
      tma_load_box(P::cell(b, 5), &maps.ya, bar, x, y, z);
      tma_load_box(P::cell(b, 6), &maps.za, bar, x, y, z);
    }
  };
  unsigned long long key = ~0ull;
  const double cdx = in_jk ? ga.celldx[g.o1 + j - g.x_min + 2] : 1.0;
  const double cdy = in_jk ? ga.celldy[g.o1 + k - g.y_min + 2] : 1.0;
  pm.run(l0, l1, status, issue, [&](int l) {
    if (!in_jk) return;
    unsigned char* bl = pm.buf(l);
    unsigned char* bu = pm.buf(l + 1);
    const int c = ty * W + tx + H;
#define NV(bb, q, a, b) (P::vel(bb, q)[(ty + (b)) * W + tx + H + (a)])
    const double m = fmin2(fmin2(cdx, cdy), ga.celldz[g.o1 + l - g.z_min + 2]);
    const double ds = 1.0 / (m * m);
    const double ss = P::cell(bl, 0)[c];
    double cc = ss * ss;
    cc = cc + 2.0 * P::cell(bl, 1)[c] / P::cell(bl, 2)[c];
    double dtct = ds * cc;
    dtct = dtc_safe * 1.0 / fmax2(sqrt(dtct), g_small);
    const double vol = P::cell(bl, 3)[c];
    const double xa = P::cell(bl, 4)[c];
    const double du1 = (NV(bl, 0, 0, 0) + NV(bl, 0, 0, 1) + NV(bu, 0, 0, 0) + NV(bu, 0, 0, 1)) * xa;
    const double du2 = (NV(bl, 0, 1, 0) + NV(bl, 0, 1, 1) + NV(bu, 0, 1, 0) + NV(bu, 0, 1, 1)) * xa;
    const double dtut = dtu_safe * 4.0 * vol / fmax2(fmax2(fabs(du1), fabs(du2)), 1.0e-5 * vol);
    const double ya = P::cell(bl, 5)[c];
    const double dv1 = (NV(bl, 1, 0, 0) + NV(bl, 1, 1, 0) + NV(bu, 1, 0, 0) + NV(bu, 1, 1, 0)) * ya;
    const double dv2 = (NV(bl, 1, 0, 1) + NV(bl, 1, 1, 1) + NV(bu, 1, 0, 1) + NV(bu, 1, 1, 1)) * ya;
    const double dtvt = dtv_safe * 4.0 * vol / fmax2(fmax2(fabs(dv1), fabs(dv2)), 1.0e-5 * vol);
    const double za = P::cell(bl, 6)[c];  // both z faces use zarea(j,k,l)
    const double dw1 = (NV(bl, 2, 0, 0) + NV(bl, 2, 0, 1) + NV(bl, 2, 1, 0) + NV(bl, 2, 1, 1)) * za;
    const double dw2 = (NV(bu, 2, 0, 0) + NV(bu, 2, 0, 1) + NV(bu, 2, 1, 0) + NV(bu, 2, 1, 1)) * za;
    const double dtwt = dtw_safe * 4.0 * vol / fmax2(fmax2(fabs(dw1), fabs(dw2)), 1.0e-5 * vol);
#undef NV
    const double div = du2 - du1 + dv2 - dv1 + dw2 - dw1;
    const double dtdivt = dtdiv_safe * 4.0 * vol / fmax2(vol * 1.0e-05, fabs(div));
    const double mn = fmin2(fmin2(fmin2(fmin2(dtct, dtut), dtvt), dtwt), dtdivt);
    if (dt_min) dt_min[off3(g, j, k, l)] = mn;
    if (!(mn != mn)) {
      const unsigned long long kc = key_of(mn);
      key = kc < key ? kc : key;
    }
  });
  if (stop) return;
  // warp then block minimum, one atomic per block
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    unsigned long long other = __shfl_xor_sync(0xffffffffu, key, o);
    key = other < key ? other : key;
  }
  if (tx == 0) wmin[ty] = key;
  __syncthreads();
  if (ty == 0) {
    key = tx < TY ? wmin[tx] : ~0ull;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
      unsigned long long other = __shfl_xor_sync(0xffffffffu, key, o);
      key = other < key ? other : key;
    }
    if (tx == 0 && key != ~0ull) atomicMin(min_key, key);
  }
}

// viscosity_kernel.f90:71-134 as k_viscosity forms it (the strain terms,
// pressure gradients and limiter of compressing cells only). Plane p: the node
// velocities of node plane p (rows k0..k0+8), the pressure of cell plane p
// (rows k0-1..k0+8), and for cell plane p the three face areas and density0
// (rows k0..k0+7). Cell l reads node planes l, l+1 and pressure planes
// l-1..l+1; plane l0-1 carries the pressure only, plane l1+1 no cell boxes.
struct ViscDropPlane {
  static constexpr int kBytes = 3 * kBox9 + kBox10 + 4 * kBox8;
  __device__ static double* vel(unsigned char* p, int q) { return (double*)(p + q * kBox9); }
  __device__ static double* pres(unsigned char* p) { return (double*)(p + 3 * kBox9); }
  // 0 xarea, 1 yarea, 2 zarea, 3 density0
  __device__ static double* cell(unsigned char* p, int q) {
    return (double*)(p + 3 * kBox9 + kBox10 + q * kBox8);
  }
};

template <int RING, int MINB>
__global__ void __launch_bounds__(TX * TY, MINB)
k_viscosity_dropin_tma(Geom g, int seg, GeomArrays ga, const __grid_constant__ ViscDropMaps maps,
                       double* __restrict__ viscosity, int* __restrict__ status) {
  using P = ViscDropPlane;
  extern __shared__ __align__(128) unsigned char ring[];
  __shared__ unsigned long long full[RING];
  __shared__ int stop;
  const int tx = threadIdx.x, ty = threadIdx.y;
  const int j = g.x_min + TX * (int)blockIdx.x + tx, k0 = g.y_min + TY * (int)blockIdx.y;
  const int k = k0 + ty;
  const int l0 = g.z_min + seg * (int)blockIdx.z;
  const int l1 = l0 + seg - 1 < g.z_max ? l0 + seg - 1 : g.z_max;
  const bool in_jk = j <= g.x_max && k <= g.y_max;
  const PlaneMarch<RING, 1, 1> pm{ring, P::kBytes, full, &stop, l0 - 1, l1 + 1};
  constexpr int W = kDropW, H = kDropH;
  auto issue = [&](int p) {
    unsigned char* b = pm.buf(p);
    unsigned long long* bar = pm.bar(p);
    const bool vel = p >= l0, cells = p >= l0 && p <= l1;
    mbar_arrive_expect_tx(bar, box_bytes<double>(10) + (vel ? 3 * box_bytes<double>(9) : 0u) +
                                   (cells ? 4 * box_bytes<double>(8) : 0u));
    const int x = TX * (int)blockIdx.x, y = k0 - g.y_min + 2, z = p - g.z_min + 2;
    tma_load_box(P::pres(b), &maps.p, bar, x, y - 1, z);
    if (vel) {
      tma_load_box(P::vel(b, 0), &maps.u, bar, x, y, z);
      tma_load_box(P::vel(b, 1), &maps.v, bar, x, y, z);
      tma_load_box(P::vel(b, 2), &maps.w, bar, x, y, z);
    }
    if (cells) {
      tma_load_box(P::cell(b, 0), &maps.xa, bar, x, y, z);
      tma_load_box(P::cell(b, 1), &maps.ya, bar, x, y, z);
      tma_load_box(P::cell(b, 2), &maps.za, bar, x, y, z);
      tma_load_box(P::cell(b, 3), &maps.d, bar, x, y, z);
    }
  };
  pm.run(l0, l1, status, issue, [&](int l) {
    if (!in_jk) return;
    unsigned char* bd = pm.buf(l - 1);
    unsigned char* bl = pm.buf(l);
    unsigned char* bu = pm.buf(l + 1);
    const int c = ty * W + tx + H;
#define NV(bb, q, a, b) (P::vel(bb, q)[(ty + (b)) * W + tx + H + (a)])
    const double u000 = NV(bl, 0, 0, 0), u100 = NV(bl, 0, 1, 0), u010 = NV(bl, 0, 0, 1);
    const double u110 = NV(bl, 0, 1, 1), u001 = NV(bu, 0, 0, 0), u101 = NV(bu, 0, 1, 0);
    const double u011 = NV(bu, 0, 0, 1), u111 = NV(bu, 0, 1, 1);
    const double v000 = NV(bl, 1, 0, 0), v100 = NV(bl, 1, 1, 0), v010 = NV(bl, 1, 0, 1);
    const double v110 = NV(bl, 1, 1, 1), v001 = NV(bu, 1, 0, 0), v101 = NV(bu, 1, 1, 0);
    const double v011 = NV(bu, 1, 0, 1), v111 = NV(bu, 1, 1, 1);
    const double w000 = NV(bl, 2, 0, 0), w100 = NV(bl, 2, 1, 0), w010 = NV(bl, 2, 0, 1);
    const double w110 = NV(bl, 2, 1, 1), w001 = NV(bu, 2, 0, 0), w101 = NV(bu, 2, 1, 0);
    const double w011 = NV(bu, 2, 0, 1), w111 = NV(bu, 2, 1, 1);
#undef NV
    const double ugradx1 = u000 + u010 + u001 + u011;
    const double ugradx2 = u100 + u110 + u101 + u111;
    const double vgrady1 = v000 + v100 + v001 + v101;
    const double vgrady2 = v010 + v110 + v011 + v111;
    const double wgradz1 = w000 + w100 + w010 + w110;
    const double wgradz2 = w001 + w101 + w011 + w111;
    const double div = (P::cell(bl, 0)[c] * (ugradx2 - ugradx1) +
                        P::cell(bl, 1)[c] * (vgrady2 - vgrady1)) +
                       P::cell(bl, 2)[c] * (wgradz2 - wgradz1);
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
      const double* cx = ga.celldx + g.o1 + 2 - g.x_min;
      const double* cy = ga.celldy + g.o1 + 2 - g.y_min;
      const double* cz = ga.celldz + g.o1 + 2 - g.z_min;
      const double cdx = cx[j], cdy = cy[k], cdz = cz[l];
      const double xx = 0.25 * (ugradx2 - ugradx1) / cdx;
      const double yy = 0.25 * (vgrady2 - vgrady1) / cdy;
      const double zz = 0.25 * (wgradz2 - wgradz1) / cdz;
      const double xy = 0.25 * (ugrady2 - ugrady1) / cdy + 0.25 * (vgradx2 - vgradx1) / cdx;
      const double xz = 0.25 * (ugradz2 - ugradz1) / cdz + 0.25 * (wgradx2 - wgradx1) / cdx;
      const double yz = 0.25 * (vgradz2 - vgradz1) / cdz + 0.25 * (wgrady2 - wgrady1) / cdy;
      // pressure (j+a, k+b) of a pressure buffer (rows from k0-1)
#define PR(bb, a, b) (P::pres(bb)[(ty + 1 + (b)) * W + tx + H + (a)])
      double pgradx = (PR(bl, 1, 0) - PR(bl, -1, 0)) / (cdx + cx[j + 1]);
      double pgrady = (PR(bl, 0, 1) - PR(bl, 0, -1)) / (cdy + cy[k + 1]);
      double pgradz = (PR(bu, 0, 0) - PR(bd, 0, 0)) / (cdz + cz[l + 1]);
#undef PR
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
        q = 2.0 * P::cell(bl, 3)[c] * grad2 * limiter * limiter;
      }
    }
    viscosity[off3(g, j, k, l)] = q;
  });
}

// accelerate_kernel.f90:61-109 as k_accelerate forms it over the caller's
// arrays. Plane p: density0, volume, pressure, viscosity, xarea and zarea of
// cell plane p (rows k0-1..k0+7), yarea (rows k0..k0+7) and the node
// velocities of node plane p (rows k0..k0+7). Node l reads cell planes l-1
// and l (zarea and the velocities of plane l only).
struct AccDropPlane {
  static constexpr int kBytes = 6 * kBox9 + 4 * kBox8;
  // 0 density0, 1 volume, 2 pressure, 3 viscosity, 4 xarea, 5 zarea
  __device__ static double* c9(unsigned char* p, int q) { return (double*)(p + q * kBox9); }
  __device__ static double* ya(unsigned char* p) { return (double*)(p + 6 * kBox9); }
  __device__ static double* vel(unsigned char* p, int q) {
    return (double*)(p + 6 * kBox9 + (1 + q) * kBox8);
  }
};

template <int RING, int MINB>
__global__ void __launch_bounds__(TX * TY, MINB)
k_accelerate_dropin_tma(Geom g, int seg, double dt, const __grid_constant__ AccDropMaps maps,
                        double* __restrict__ xvel1, double* __restrict__ yvel1,
                        double* __restrict__ zvel1, int* __restrict__ status) {
  using P = AccDropPlane;
  extern __shared__ __align__(128) unsigned char ring[];
  __shared__ unsigned long long full[RING];
  __shared__ int stop;
  const int tx = threadIdx.x, ty = threadIdx.y;
  const int j = g.x_min + TX * (int)blockIdx.x + tx, k0 = g.y_min + TY * (int)blockIdx.y;
  const int k = k0 + ty;
  const int l0 = g.z_min + seg * (int)blockIdx.z;
  const int l1 = l0 + seg - 1 < g.z_max + 1 ? l0 + seg - 1 : g.z_max + 1;
  const bool in_jk = j <= g.x_max + 1 && k <= g.y_max + 1;
  const PlaneMarch<RING, 1, 0> pm{ring, P::kBytes, full, &stop, l0 - 1, l1};
  constexpr int W = kDropW, H = kDropH;
  auto issue = [&](int p) {
    unsigned char* b = pm.buf(p);
    unsigned long long* bar = pm.bar(p);
    const bool node = p >= l0;  // zarea and the velocities: the nodes' own plane only
    mbar_arrive_expect_tx(bar, 5 * box_bytes<double>(9) + box_bytes<double>(8) +
                                   (node ? box_bytes<double>(9) + 3 * box_bytes<double>(8) : 0u));
    const int x = TX * (int)blockIdx.x, y = k0 - g.y_min + 2, z = p - g.z_min + 2;
    tma_load_box(P::c9(b, 0), &maps.d, bar, x, y - 1, z);
    tma_load_box(P::c9(b, 1), &maps.vol, bar, x, y - 1, z);
    tma_load_box(P::c9(b, 2), &maps.p, bar, x, y - 1, z);
    tma_load_box(P::c9(b, 3), &maps.q, bar, x, y - 1, z);
    tma_load_box(P::c9(b, 4), &maps.xa, bar, x, y - 1, z);
    tma_load_box(P::ya(b), &maps.ya, bar, x, y, z);
    if (node) {
      tma_load_box(P::c9(b, 5), &maps.za, bar, x, y - 1, z);
      tma_load_box(P::vel(b, 0), &maps.u, bar, x, y, z);
      tma_load_box(P::vel(b, 1), &maps.v, bar, x, y, z);
      tma_load_box(P::vel(b, 2), &maps.w, bar, x, y, z);
    }
  };
  pm.run(l0, l1, status, issue, [&](int l) {
    if (!in_jk) return;
    unsigned char* bd = pm.buf(l - 1);
    unsigned char* bl = pm.buf(l);
    // cell (j+a, k+b) of a 9-row buffer (rows from k0-1), of yarea (rows from k0)
#define C9(bb, q, a, b) (P::c9(bb, q)[(ty + 1 + (b)) * W + tx + H + (a)])
#define YA(bb, a) (P::ya(bb)[ty * W + tx + H + (a)])
#define DV(bb, a, b) (C9(bb, 0, a, b) * C9(bb, 1, a, b))
    const double nodal_mass = (DV(bl, -1, -1) + DV(bl, 0, -1) + DV(bl, 0, 0) + DV(bl, -1, 0) +
                               DV(bd, -1, -1) + DV(bd, 0, -1) + DV(bd, 0, 0) + DV(bd, -1, 0)) * 0.125;
#undef DV
    const double stepbymass_s = 0.25 * dt / nodal_mass;
    const double p000 = C9(bl, 2, 0, 0), p100 = C9(bl, 2, -1, 0);
    const double p010 = C9(bl, 2, 0, -1), p110 = C9(bl, 2, -1, -1);
    const double p001 = C9(bd, 2, 0, 0), p101 = C9(bd, 2, -1, 0);
    const double p011 = C9(bd, 2, 0, -1), p111 = C9(bd, 2, -1, -1);
    const double q000 = C9(bl, 3, 0, 0), q100 = C9(bl, 3, -1, 0);
    const double q010 = C9(bl, 3, 0, -1), q110 = C9(bl, 3, -1, -1);
    const double q001 = C9(bd, 3, 0, 0), q101 = C9(bd, 3, -1, 0);
    const double q011 = C9(bd, 3, 0, -1), q111 = C9(bd, 3, -1, -1);
    const double xa0 = C9(bl, 4, 0, 0), xa1 = C9(bl, 4, 0, -1);
    const double xa2 = C9(bd, 4, 0, 0), xa3 = C9(bd, 4, 0, -1);
    const double ya0 = YA(bl, 0), ya1 = YA(bl, -1);
    const double ya2 = YA(bd, 0), ya3 = YA(bd, -1);
    const double za0 = C9(bl, 5, 0, 0), za1 = C9(bl, 5, 0, -1);
    const double za2 = C9(bl, 5, -1, 0), za3 = C9(bl, 5, -1, -1);
#undef YA
#undef C9
    const int c = ty * W + tx + H;
    const double xvel1_s = P::vel(bl, 0)[c] -
        stepbymass_s * (xa0 * (p000 - p100) + xa1 * (p010 - p110) + xa2 * (p001 - p101) +
                        xa3 * (p011 - p111));
    const double yvel1_s = P::vel(bl, 1)[c] -
        stepbymass_s * (ya0 * (p000 - p010) + ya1 * (p100 - p110) + ya2 * (p001 - p011) +
                        ya3 * (p101 - p111));
    const double zvel1_s = P::vel(bl, 2)[c] -
        stepbymass_s * (za0 * (p000 - p001) + za1 * (p010 - p011) + za2 * (p100 - p101) +
                        za3 * (p110 - p111));
    const long long o = off3(g, j, k, l);
    xvel1[o] = xvel1_s - stepbymass_s * (xa0 * (q000 - q100) + xa1 * (q010 - q110) +
                                         xa2 * (q001 - q101) + xa3 * (q011 - q111));
    yvel1[o] = yvel1_s - stepbymass_s * (ya0 * (q000 - q010) + ya1 * (q100 - q110) +
                                         ya2 * (q001 - q011) + ya3 * (q101 - q111));
    zvel1[o] = zvel1_s - stepbymass_s * (za0 * (q000 - q001) + za1 * (q010 - q011) +
                                         za2 * (q100 - q101) + za3 * (q110 - q111));
  });
}

// ---------------------------------------------------------------------------
// The drop-in advec_mom node pass of the y (DIR 2) or z (DIR 3) sweep
// (advec_mom_kernel.f90:254-288 y, :339-374 z, as k_mom_node forms it over
// the caller's arrays): node flux over nodes min-2..max+2 along the sweep,
// node_mass_post and node_mass_pre (the lower neighbour's node flux formed
// again) over min-1..max+2. The block marches the sweep axis p (z for the z
// sweep; y for the y sweep, whose boxes are x-z slices) over rows r (y; z).
// Plane p: the sweep's mass flux, density1 and post_vol, rows r0-1..r0+7.
// Node p reads planes p-1..p+1 (mass flux) and p-1, p (cells); the mass-flux
// plane below min-2 lies outside the array, reads as zeros and is not used.
struct NodeDropPlane {
  static constexpr int kBytes = 3 * kBox9;
  static constexpr unsigned kTx = 3 * box_bytes<double>(9);
  __device__ static double* arr(unsigned char* p, int q) { return (double*)(p + q * kBox9); }
};

template <int DIR, int RING, int MINB>
__global__ void __launch_bounds__(TX * TY, MINB)
k_mom_node_dropin_tma(Geom g, int seg, const __grid_constant__ NodeDropMaps maps,
                      double* __restrict__ node_flux, double* __restrict__ node_mass_post,
                      double* __restrict__ node_mass_pre, int* __restrict__ status) {
  using P = NodeDropPlane;
  extern __shared__ __align__(128) unsigned char ring[];
  __shared__ unsigned long long full[RING];
  __shared__ int stop;
  const int tx = threadIdx.x, ty = threadIdx.y;
  const int pmin = DIR == 2 ? g.y_min : g.z_min, pmax = DIR == 2 ? g.y_max : g.z_max;
  const int rmin = DIR == 2 ? g.z_min : g.y_min, rmax = DIR == 2 ? g.z_max : g.y_max;
  const int j = g.x_min + TX * (int)blockIdx.x + tx, r0 = rmin + TY * (int)blockIdx.y;
  const int r = r0 + ty;
  const int q0 = pmin - 2 + seg * (int)blockIdx.z;
  const int q1 = q0 + seg - 1 < pmax + 2 ? q0 + seg - 1 : pmax + 2;
  const bool in_jr = j <= g.x_max + 1 && r <= rmax + 1;
  const PlaneMarch<RING, 1, 1> pm{ring, P::kBytes, full, &stop, q0 - 1, q1 + 1};
  constexpr int W = kDropW, H = kDropH;
  auto issue = [&](int p) {
    unsigned char* b = pm.buf(p);
    unsigned long long* bar = pm.bar(p);
    mbar_arrive_expect_tx(bar, P::kTx);
    const int x = TX * (int)blockIdx.x;
    const int rr = r0 - 1 - rmin + 2, pp = p - pmin + 2;
    const int y = DIR == 2 ? pp : rr, z = DIR == 2 ? rr : pp;
    tma_load_box(P::arr(b, 0), &maps.mf, bar, x, y, z);
    tma_load_box(P::arr(b, 1), &maps.d, bar, x, y, z);
    tma_load_box(P::arr(b, 2), &maps.pv, bar, x, y, z);
  };
  pm.run(q0, q1, status, issue, [&](int p) {
    if (!in_jr) return;
    unsigned char* bd = pm.buf(p - 1);
    unsigned char* bl = pm.buf(p);
    unsigned char* bu = pm.buf(p + 1);
    // array q at column j+a, row r+b of a plane buffer (rows from r0-1)
#define AT(bb, q, a, b) (P::arr(bb, q)[(ty + 1 + (b)) * W + tx + H + (a)])
    // the node flux of node (j, r, p) from mass-flux planes lo (p) and hi (p+1)
    auto nflux = [&](unsigned char* lo, unsigned char* hi) {
      if (DIR == 3)  // mf(j-1,k,l) + mf(j,k,l) + mf(j-1,k,l+1) + mf(j,k,l+1) + the k-1 row
        return 0.125 * (AT(lo, 0, -1, 0) + AT(lo, 0, 0, 0) + AT(hi, 0, -1, 0) + AT(hi, 0, 0, 0) +
                        AT(lo, 0, -1, -1) + AT(lo, 0, 0, -1) + AT(hi, 0, -1, -1) + AT(hi, 0, 0, -1));
      // mf(j-1,k,l) + mf(j,k,l) + mf(j-1,k+1,l) + mf(j,k+1,l) + the l-1 row
      return 0.125 * (AT(lo, 0, -1, 0) + AT(lo, 0, 0, 0) + AT(hi, 0, -1, 0) + AT(hi, 0, 0, 0) +
                      AT(lo, 0, -1, -1) + AT(lo, 0, 0, -1) + AT(hi, 0, -1, -1) + AT(hi, 0, 0, -1));
    };
    const double nf = nflux(bl, bu);
    const long long o = DIR == 2 ? off3(g, j, p, r) : off3(g, j, r, p);
    node_flux[o] = nf;
    if (p >= pmin - 1) {
      // cell (j+a, r+b) of cell plane p+c: the reference's order of the eight
      // cells, (a, p-offset, r-offset) in DIR 3's (j, k, l) terms
#define DP(a, b, bb) (AT(bb, 1, a, b) * AT(bb, 2, a, b))
      double nm;
      if (DIR == 3)  // DP(0,-1,0) DP(0,0,0) DP(-1,-1,0) DP(-1,0,0) then the l-1 plane
        nm = 0.125 * (DP(0, -1, bl) + DP(0, 0, bl) + DP(-1, -1, bl) + DP(-1, 0, bl) +
                      DP(0, -1, bd) + DP(0, 0, bd) + DP(-1, -1, bd) + DP(-1, 0, bd));
      else  // (j, k-1, l) (j, k, l) (j-1, k-1, l) (j-1, k, l) then the l-1 row
        nm = 0.125 * (DP(0, 0, bd) + DP(0, 0, bl) + DP(-1, 0, bd) + DP(-1, 0, bl) +
                      DP(0, -1, bd) + DP(0, -1, bl) + DP(-1, -1, bd) + DP(-1, -1, bl));
#undef DP
      node_mass_post[o] = nm;
      node_mass_pre[o] = nm - nflux(bd, bl) + nf;
    }
#undef AT
  });
}

// ---------------------------------------------------------------------------
// The drop-in advec_mom node pass of the x sweep (advec_mom_kernel.f90:166-202
// as k_mom_node forms it over the caller's arrays): node flux over nodes
// x_min-2..x_max+2, node_mass_post and node_mass_pre (the left neighbour's
// node flux formed again) over x_min-1..x_max+2, rows y_min..y_max+1, planes
// z_min..z_max+1. Lane m of tile t takes node x_min-2+32t+m, whose box
// starts two columns before it. Plane p: mass_flux_x, density1 and post_vol,
// rows k0-1..k0+7; node l reads planes l-1 and l.
template <int RING, int MINB>
__global__ void __launch_bounds__(TX * TY, MINB)
k_mom_node_x_dropin_tma(Geom g, int seg, const __grid_constant__ NodeDropMaps maps,
                        double* __restrict__ node_flux, double* __restrict__ node_mass_post,
                        double* __restrict__ node_mass_pre, int* __restrict__ status) {
  using P = NodeDropPlane;
  extern __shared__ __align__(128) unsigned char ring[];
  __shared__ unsigned long long full[RING];
  __shared__ int stop;
  const int tx = threadIdx.x, ty = threadIdx.y;
  const int j = g.x_min - 2 + TX * (int)blockIdx.x + tx, k0 = g.y_min + TY * (int)blockIdx.y;
  const int k = k0 + ty;
  const int l0 = g.z_min + seg * (int)blockIdx.z;
  const int l1 = l0 + seg - 1 < g.z_max + 1 ? l0 + seg - 1 : g.z_max + 1;
  const bool in_jk = j <= g.x_max + 2 && k <= g.y_max + 1;
  const PlaneMarch<RING, 1, 0> pm{ring, P::kBytes, full, &stop, l0 - 1, l1};
  constexpr int W = kDropW, H = kDropH;
  auto issue = [&](int p) {
    unsigned char* b = pm.buf(p);
    unsigned long long* bar = pm.bar(p);
    mbar_arrive_expect_tx(bar, P::kTx);
    const int x = TX * (int)blockIdx.x - H, y = k0 - 1 - g.y_min + 2, z = p - g.z_min + 2;
    tma_load_box(P::arr(b, 0), &maps.mf, bar, x, y, z);
    tma_load_box(P::arr(b, 1), &maps.d, bar, x, y, z);
    tma_load_box(P::arr(b, 2), &maps.pv, bar, x, y, z);
  };
  pm.run(l0, l1, status, issue, [&](int l) {
    if (!in_jk) return;
    unsigned char* bd = pm.buf(l - 1);
    unsigned char* bl = pm.buf(l);
    // array q at column j+a, row k+b of a plane buffer (rows from k0-1; the
    // box starts H columns before this tile's first node)
#define AT(bb, q, a, b) (P::arr(bb, q)[(ty + 1 + (b)) * W + tx + H + (a)])
    // mf(j,k-1,l) + mf(j,k,l) + mf(j+1,k-1,l) + mf(j+1,k,l) + the l-1 plane, at node j+a
    auto nflux = [&](int a) {
      return 0.125 * (AT(bl, 0, a, -1) + AT(bl, 0, a, 0) + AT(bl, 0, a + 1, -1) + AT(bl, 0, a + 1, 0) +
                      AT(bd, 0, a, -1) + AT(bd, 0, a, 0) + AT(bd, 0, a + 1, -1) + AT(bd, 0, a + 1, 0));
    };
    const double nf = nflux(0);
    const long long o = off3(g, j, k, l);
    node_flux[o] = nf;
    if (j >= g.x_min - 1) {
#define DP(a, b, bb) (AT(bb, 1, a, b) * AT(bb, 2, a, b))
      // the reference's order: (j,k-1,l) (j,k,l) (j-1,k-1,l) (j-1,k,l), then plane l-1
      const double nm = 0.125 * (DP(0, -1, bl) + DP(0, 0, bl) + DP(-1, -1, bl) + DP(-1, 0, bl) +
                                 DP(0, -1, bd) + DP(0, 0, bd) + DP(-1, -1, bd) + DP(-1, 0, bd));
#undef DP
      node_mass_post[o] = nm;
      node_mass_pre[o] = nm - nflux(-1) + nf;
    }
#undef AT
  });
}

// ---------------------------------------------------------------------------
// The node pass of the y or z momentum sweep (advec_mom_kernel.f90:254-293 for
// y, :339-379 for z), as k_mom_node_march (clover_fused.cu) forms it, with the
// inputs staged in shared memory. The lane layout stays: lane L of a warp holds
// column j = x_min-1+31t+L, the values at column j-1 come from lane L-1 (lane 0
// only serves lane 1), rows c = c0..c0+7 are the warps; the sweep axis p is
// marched. Plane p holds the sweep direction's mass flux and density1 of rows
// c0-1..c0+7 and the volume fluxes of the post volume (variant 1: vol_flux_x
// and vol_flux_y; 2: vol_flux_z; 3: vol_flux_x; 4: none), rows along y for
// the z sweep (p = l, c = k) and along z for the y sweep (p = k, c = l). Node p
// reads planes p-1 (node flux p-1, the cell products below), p and p+1.
template <class S, int VAR>
struct NodePlane {
  using MF = typename S::mf_t;
  using R = typename S::rho_t;
  using VF = typename S::vf_t;
  static constexpr bool kX = VAR == 1 || VAR == 3;  // vol_flux_x, columns j, j+1
  static constexpr bool kR = VAR == 1 || VAR == 2;  // the row-direction volume flux, rows c, c+1
  static constexpr int kMf = round128(9 * kTmaWidth<MF> * (int)sizeof(MF));
  static constexpr int kRho = round128(9 * kTmaWidth<R> * (int)sizeof(R));
  static constexpr int kVfx = kX ? round128(9 * kTmaWidth<VF> * (int)sizeof(VF)) : 0;
  static constexpr int kVfr = kR ? round128(10 * kTmaWidth<VF> * (int)sizeof(VF)) : 0;
  static constexpr int kBytes = kMf + kRho + kVfx + kVfr;
  static constexpr unsigned kTx = box_bytes<MF>(9) + box_bytes<R>(9) +
                                  (kX ? box_bytes<VF>(9) : 0u) + (kR ? box_bytes<VF>(10) : 0u);
  __device__ static MF* mf(unsigned char* p) { return (MF*)p; }
  __device__ static R* rho(unsigned char* p) { return (R*)(p + kMf); }
  __device__ static VF* vfx(unsigned char* p) { return (VF*)(p + kMf + kRho); }
  __device__ static VF* vfr(unsigned char* p) { return (VF*)(p + kMf + kRho + kVfx); }
};

// Box x coordinate of element type T for a block whose first column is
// x_min-1+31t, and the column of that node in the box.
template <class T>
__device__ __forceinline__ void x_box31(int t, int& x, int& shift) {
  constexpr int H = kTmaHalo<T>;
  const int c = 31 * t + H - 1;  // the first column, counted from the map's base
  x = c / H * H;
  shift = c - x;
}

template <class S, int DIR, int VAR, int RING, int MINB>
__global__ void __launch_bounds__(TX * TY, MINB)
k_mom_node_tma(Geom g, int seg, const __grid_constant__ NodeMaps maps,
               typename S::nd_t* __restrict__ node_flux, typename S::nd_t* __restrict__ node_mass_post,
               typename S::nd_t* __restrict__ node_mass_pre, int* __restrict__ status) {
  using P = NodePlane<S, VAR>;
  using MF = typename S::mf_t;
  using R = typename S::rho_t;
  using VF = typename S::vf_t;
  using W = typename S::nd_t;
  extern __shared__ __align__(128) unsigned char ring[];
  __shared__ unsigned long long full[RING];
  __shared__ int stop;
  const unsigned fullmask = 0xffffffffu;
  const MarchRange r = mom_node_range<DIR>(g);
  const int lane = threadIdx.x, ty = threadIdx.y;
  const int j = r.jlo - 1 + 31 * (int)blockIdx.x + lane;
  const int c0 = r.clo + TY * (int)blockIdx.y, c = c0 + ty;
  const bool row = c <= r.chi;      // the whole warp: c depends on the row only
  const bool lds = row && j <= r.jhi;
  const bool own = lds && lane >= 1;
  const int p0 = r.plo + seg * (int)blockIdx.z;
  const int p1 = p0 + seg - 1 < r.phi ? p0 + seg - 1 : r.phi;
  const PlaneMarch<RING, 1, 1> pm{ring, P::kBytes, full, &stop, p0 - 1, p1 + 1};
  int xm, cm, xr, cr, xf, cf;
  x_box31<MF>(blockIdx.x, xm, cm);
  x_box31<R>(blockIdx.x, xr, cr);
  x_box31<VF>(blockIdx.x, xf, cf);
  cm += lane; cr += lane; cf += lane;
  constexpr int WM = kTmaWidth<MF>, WR = kTmaWidth<R>, WF = kTmaWidth<VF>;
  auto issue = [&](int p) {
    unsigned char* b = pm.buf(p);
    unsigned long long* bar = pm.bar(p);
    mbar_arrive_expect_tx(bar, P::kTx);
    // rows from c0-1: along y (z sweep) or along z (y sweep)
    const int y = DIR == 3 ? c0 - 1 - g.y_min + 2 : p - g.y_min + 2;
    const int z = DIR == 3 ? p - g.z_min + 2 : c0 - 1 - g.z_min + 2;
    tma_load_box(P::mf(b), &maps.mf, bar, xm, y, z);
    tma_load_box(P::rho(b), &maps.d, bar, xr, y, z);
    if (P::kX) tma_load_box(P::vfx(b), &maps.vfx, bar, xf, y, z);
    if (P::kR) tma_load_box(P::vfr(b), &maps.vfr, bar, xf, y, z);
  };
  auto up = [&](double v) { return __shfl_up_sync(fullmask, v, 1); };
  // mass fluxes of plane b at (j, c) and (j, c-1), and of column j-1
  struct Mf { double a, b, am, bm; };
  auto mfs = [&](unsigned char* b) {
    Mf f{0.0, 0.0, 0.0, 0.0};
    if (lds) {
      f.a = (double)P::mf(b)[(ty + 1) * WM + cm];
      f.b = (double)P::mf(b)[ty * WM + cm];
    }
    f.am = up(f.a);
    f.bm = up(f.b);
    return f;
  };
  // the node-flux sum of the reference from the mass fluxes of two planes
  auto nflux = [](const Mf& lo, const Mf& hi) {
    return 0.125 * (lo.am + lo.a + hi.am + hi.a + lo.bm + lo.b + hi.bm + hi.b);
  };
  // cell product density1 * post_vol of cell (j, box row rr) of plane b
  auto prod = [&](unsigned char* b, int rr) {
    const double d = (double)P::rho(b)[rr * WR + cr];
    double pv = g.vol;
    if (VAR == 1)
      pv = pv + (double)P::vfx(b)[rr * WF + cf + 1] - (double)P::vfx(b)[rr * WF + cf] +
           (double)P::vfr(b)[(rr + 1) * WF + cf] - (double)P::vfr(b)[rr * WF + cf];
    else if (VAR == 2)
      pv = pv + (double)P::vfr(b)[(rr + 1) * WF + cf] - (double)P::vfr(b)[rr * WF + cf];
    else if (VAR == 3)
      pv = pv + (double)P::vfx(b)[rr * WF + cf + 1] - (double)P::vfx(b)[rr * WF + cf];
    return d * pv;
  };
  // the four products of the node's plane-b cells in the order the node-mass
  // sum takes them (a, b: this column; c, d: column j-1)
  struct Pq { double a, b, c, d; };
  auto prods = [&](unsigned char* b) {
    Pq u;
    double x0 = 0.0, x1 = 0.0;
    if (DIR == 3) {  // plane l: P(j,k-1,l), P(j,k,l), P(j-1,k-1,l), P(j-1,k,l)
      if (lds) { x0 = prod(b, ty); x1 = prod(b, ty + 1); }
      u.a = x0; u.b = x1; u.c = up(x0); u.d = up(x1);
    } else {  // plane k: P(j,k,l), P(j-1,k,l), P(j,k,l-1), P(j-1,k,l-1)
      if (lds) { x0 = prod(b, ty + 1); x1 = prod(b, ty); }
      u.a = x0; u.b = up(x0); u.c = x1; u.d = up(x1);
    }
    return u;
  };
  pm.run(p0, p1, status, issue, [&](int p) {
    if (!row) return;
    unsigned char* bm = pm.buf(p - 1);
    unsigned char* b0 = pm.buf(p);
    unsigned char* b1 = pm.buf(p + 1);
    const Mf fm = mfs(bm), f0 = mfs(b0), f1 = mfs(b1);
    const double nf_prev = nflux(fm, f0);
    const double nf = nflux(f0, f1);
    const long long o = DIR == 3 ? off3(g, j, c, p) : off3(g, j, p, c);
    if (own) node_flux[o] = st<W>(nf);
    const Pq q = prods(bm), u = prods(b0);
    double nmp;
    if (DIR == 3)
      nmp = node_mass_sum(u.a, u.b, u.c, u.d, q.a, q.b, q.c, q.d);
    else  // P(j,k-1,l) P(j,k,l) P(j-1,k-1,l) P(j-1,k,l) P(j,k-1,l-1) P(j,k,l-1) P(j-1,k-1,l-1) P(j-1,k,l-1)
      nmp = node_mass_sum(q.a, u.a, q.b, u.b, q.c, u.c, q.d, u.d);
    if (own && p >= r.plo + 1) {  // node masses run from one node after the flux range start
      node_mass_post[o] = st<W>(nmp);
      node_mass_pre[o] = st<W>(nmp - nf_prev + nf);
    }
  });
}

// ---------------------------------------------------------------------------
// The velocity pass of the y or z momentum sweep (advec_mom_kernel.f90:295-337
// for y, :381-423 for z), as k_mom_vel3_march (clover_fused.cu) forms it: each
// thread walks a segment of its (j, c) column with the velocity window and the
// previous momentum fluxes in registers. The segment's start (the window
// v(p0-2..p0+1) and the node values at p0-1, p0) is read from global memory;
// in the loop, node p reads the node flux and node masses of plane p (and the
// node mass pre of plane p+1) and the three velocities of plane p+2 from
// staged planes (rows c0..c0+7, along y for the z sweep, along z for the y
// sweep).
template <class S>
struct VelPlane {
  using W = typename S::nd_t;
  using V = typename S::vel_t;
  static constexpr int kNd = round128(8 * kTmaWidth<W> * (int)sizeof(W));
  static constexpr int kVel = round128(8 * kTmaWidth<V> * (int)sizeof(V));
  static constexpr int kBytes = 3 * kNd + 3 * kVel;
  static constexpr unsigned kTx = 3 * box_bytes<W>(8) + 3 * box_bytes<V>(8);
  __device__ static W* nd(unsigned char* p, int q) { return (W*)(p + q * kNd); }
  __device__ static V* vel(unsigned char* p, int q) { return (V*)(p + 3 * kNd + q * kVel); }
};

template <class S, int DIR, int RING, int MINB>
__global__ void __launch_bounds__(TX * TY, MINB)
k_mom_vel_tma(Geom g, int seg, GeomArrays ga, const __grid_constant__ VelMaps maps,
              const typename S::nd_t* __restrict__ node_flux,
              const typename S::nd_t* __restrict__ node_mass_pre,
              const typename S::vel_t* __restrict__ u_in, const typename S::vel_t* __restrict__ v_in,
              const typename S::vel_t* __restrict__ w_in, typename S::vel_t* __restrict__ u_out,
              typename S::vel_t* __restrict__ v_out, typename S::vel_t* __restrict__ w_out,
              Level0<S> lz, int* __restrict__ status) {
  using P = VelPlane<S>;
  using W = typename S::nd_t;
  using V = typename S::vel_t;
  using A = typename S::arith_t;  // arithmetic of the flux and update
  extern __shared__ __align__(128) unsigned char ring[];
  __shared__ unsigned long long full[RING];
  __shared__ int stop;
  const MarchRange r = mom_vel_range<DIR>(g);
  const int tx = threadIdx.x, ty = threadIdx.y;
  const int j = r.jlo + TX * (int)blockIdx.x + tx;
  const int c0 = r.clo + TY * (int)blockIdx.y, c = c0 + ty;
  const bool in_jc = j <= r.jhi && c <= r.chi;
  const int p0 = r.plo + seg * (int)blockIdx.z;
  const int p1 = p0 + seg - 1 < r.phi ? p0 + seg - 1 : r.phi;
  const PlaneMarch<RING, 0, 2> pm{ring, P::kBytes, full, &stop, p0, p1 + 2};
  constexpr int WW = kTmaWidth<W>, HW = kTmaHalo<W>, WV = kTmaWidth<V>, HV = kTmaHalo<V>;
  const int cw = ty * WW + tx + HW, cv = ty * WV + tx + HV;  // this node in the boxes
#define IDX(p) j, (DIR == 2 ? (p) : c), (DIR == 2 ? c : (p))
  const double* cd = DIR == 2 ? ga.celldy : ga.celldz;
  const int cdlo = DIR == 2 ? g.y_min : g.z_min;
#define CD(p) cd[g.o1 + (p) - cdlo + 2]
#define LA(a, idx) lda<A>(&EI_(a, idx))
#define EI_(a, jj, kk, ll) (a)[off3(g, (jj), (kk), (ll))]
  const typename S::vel_t* in[3] = {u_in, v_in, w_in};
  typename S::vel_t* out[3] = {u_out, v_out, w_out};
  typename S::vel_t* lev0[3] = {lz.xvel0, lz.yvel0, lz.zvel0};
  // window v(p-2), v(p-1), v(p), v(p+1) and the momentum flux of node p-1, from
  // global memory at the segment's start
  A vw[3][4];
  A mf_prev[3];
  A pre_0 = A(0.0);
  if (in_jc) {
    const A nf_m = LA(node_flux, IDX(p0 - 1));
    const A pre_m = LA(node_mass_pre, IDX(p0 - 1));
    pre_0 = LA(node_mass_pre, IDX(p0));
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
  auto issue = [&](int p) {
    unsigned char* b = pm.buf(p);
    unsigned long long* bar = pm.bar(p);
    mbar_arrive_expect_tx(bar, P::kTx);
    const int x = TX * (int)blockIdx.x;
    const int y = DIR == 3 ? c0 - g.y_min + 2 : p - g.y_min + 2;
    const int z = DIR == 3 ? p - g.z_min + 2 : c0 - g.z_min + 2;
    tma_load_box(P::nd(b, 0), &maps.nf, bar, x, y, z);
    tma_load_box(P::nd(b, 1), &maps.pre, bar, x, y, z);
    tma_load_box(P::nd(b, 2), &maps.post, bar, x, y, z);
    tma_load_box(P::vel(b, 0), &maps.u, bar, x, y, z);
    tma_load_box(P::vel(b, 1), &maps.v, bar, x, y, z);
    tma_load_box(P::vel(b, 2), &maps.w, bar, x, y, z);
  };
  pm.run(p0, p1, status, issue, [&](int p) {
    if (!in_jc) return;
    unsigned char* b0 = pm.buf(p);
    unsigned char* b1 = pm.buf(p + 1);
    unsigned char* b2 = pm.buf(p + 2);
    const A nf_0 = (A)P::nd(b0, 0)[cw];
    const A pre_p = (A)P::nd(b1, 1)[cw];
    const A post_0 = (A)P::nd(b0, 2)[cw];
    const MomNodeTerms<A> nt =
        mom_node_terms<A>(nf_0, pre_0, pre_p, (A)CD(p), (A)CD(p - 1), (A)CD(p + 1));
    const long long o = off3(g, IDX(p));
    A vn[3];
#pragma unroll
    for (int q = 0; q < 3; q++) {
      const A vp2 = (A)P::vel(b2, q)[cv];
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
      out[q][o] = vn1;
      if (lz.xvel0) lev0[q][o] = vn1;  // last sweep of the step: reset_field
    }
    pre_0 = pre_p;
  });
#undef EI_
#undef LA
#undef CD
#undef IDX
}

// ---------------------------------------------------------------------------
// The y or z cell sweep (advec_cell_kernel.f90:190-281 for y, :287-376 for z)
// out of place, its inputs staged in shared memory: the old density1/energy1
// come from one buffer of the pair and the updated cells go to the other, so
// segments of the sweep axis need no ordering between them (every interior
// cell is written; the depth-2 halo update that follows rewrites the shell).
// The arithmetic is k_cell_sweep_march's (clover_fused.cu), face by face: the
// window of old values of cells p-2..p+1 and the pre-volumes of cells p-1, p
// in registers, face p, then cell p-1. A segment's start (cells q0-2..q0 and
// the pre-volume of cell q0-1) is read from global memory; at face p the loop
// reads plane p (the sweep direction's volume flux at face p, the cross fluxes
// of cell p's pre-volume) and plane p+1 (the volume flux at face p+1, density1
// and energy1 of cell p+1). Rows c0..c0+7 (c0..c0+8 for the cross flux along
// the rows) run along y for the z sweep and along z for the y sweep. Pre-volume
// variants: y sweep 2 (after x: vol_flux_y and vol_flux_z) and 3 (after z:
// vol_flux_y and vol_flux_x); z sweep 4 (first: all three) and 5 (last:
// vol_flux_z).
template <class S, int DIR, int VAR>
struct CellPlane {
  using R = typename S::rho_t;
  using En = typename S::ene_t;
  using VF = typename S::vf_t;
  static constexpr bool kX = VAR == 3 || VAR == 4;  // vol_flux_x, columns j, j+1
  static constexpr bool kR = VAR == 2 || VAR == 4;  // the flux along the rows, rows c, c+1
  static constexpr int kRho = round128(8 * kTmaWidth<R> * (int)sizeof(R));
  static constexpr int kEne = round128(8 * kTmaWidth<En> * (int)sizeof(En));
  static constexpr int kVfd = round128(8 * kTmaWidth<VF> * (int)sizeof(VF));
  static constexpr int kVfx = kX ? round128(8 * kTmaWidth<VF> * (int)sizeof(VF)) : 0;
  static constexpr int kVfr = kR ? round128(9 * kTmaWidth<VF> * (int)sizeof(VF)) : 0;
  static constexpr int kBytes = kRho + kEne + kVfd + kVfx + kVfr;
  static constexpr unsigned kTx = box_bytes<R>(8) + box_bytes<En>(8) + box_bytes<VF>(8) +
                                  (kX ? box_bytes<VF>(8) : 0u) + (kR ? box_bytes<VF>(9) : 0u);
  __device__ static R* rho(unsigned char* p) { return (R*)p; }
  __device__ static En* ene(unsigned char* p) { return (En*)(p + kRho); }
  __device__ static VF* vfd(unsigned char* p) { return (VF*)(p + kRho + kEne); }
  __device__ static VF* vfx(unsigned char* p) { return (VF*)(p + kRho + kEne + kVfd); }
  __device__ static VF* vfr(unsigned char* p) { return (VF*)(p + kRho + kEne + kVfd + kVfx); }
};

template <class S, int DIR, int VAR, int RING, int MINB>
__global__ void __launch_bounds__(TX * TY, MINB)
k_cell_sweep_tma(Geom g, int seg, GeomArrays ga, const __grid_constant__ CellMaps maps,
                 const typename S::rho_t* __restrict__ d_in, const typename S::ene_t* __restrict__ e_in,
                 typename S::rho_t* __restrict__ d_out, typename S::ene_t* __restrict__ e_out,
                 const typename S::vf_t* __restrict__ vfx, const typename S::vf_t* __restrict__ vfy,
                 const typename S::vf_t* __restrict__ vfz, typename S::mf_t* __restrict__ mass_flux,
                 Level0<S> lz, int* __restrict__ status) {
  using P = CellPlane<S, DIR, VAR>;
  using R = typename S::rho_t;
  using En = typename S::ene_t;
  using VF = typename S::vf_t;
  using MF = typename S::mf_t;
  using AL = typename S::arith_t;  // the limiters' arithmetic
  extern __shared__ __align__(128) unsigned char ring[];
  __shared__ unsigned long long full[RING];
  __shared__ int stop;
  const MarchRange r = cell_sweep_range<DIR>(g);
  const int tx = threadIdx.x, ty = threadIdx.y;
  const int j = r.jlo + TX * (int)blockIdx.x + tx;
  const int c0 = r.clo + TY * (int)blockIdx.y, c = c0 + ty;
  const bool col = j <= r.jhi && c <= r.chi;
  const bool update = c <= r.cmax;
  const int pmin = DIR == 2 ? g.y_min : g.z_min;
  const int pmax = DIR == 2 ? g.y_max : g.z_max;
  const int top = pmax + 2;
  const int q0 = pmin + seg * (int)blockIdx.z;  // cells of this segment: [q0, q1]
  const int q1 = q0 + seg - 1 < pmax ? q0 + seg - 1 : pmax;
  const bool last = q1 == pmax;  // this segment also walks the faces pmax+1, pmax+2
  const int pend = last ? top : q1 + 1;
  const PlaneMarch<RING, 0, 1> pm{ring, P::kBytes, full, &stop, q0, pend + 1};
  constexpr int WR = kTmaWidth<R>, HR = kTmaHalo<R>, WE = kTmaWidth<En>, HE = kTmaHalo<En>;
  constexpr int WF = kTmaWidth<VF>, HF = kTmaHalo<VF>;
  const int cr = ty * WR + tx + HR, ce = ty * WE + tx + HE, cf = ty * WF + tx + HF;
#define IDX(p) j, (DIR == 2 ? (p) : c), (DIR == 2 ? c : (p))
#define LI(a, p) ((double)__ldg(&(a)[off3(g, IDX(p))]))
  const typename S::vf_t* vf_d = DIR == 2 ? vfy : vfz;
  const double* vd = DIR == 2 ? ga.vertexdy : ga.vertexdz;
#define VD(p) vd[g.o1 + (p) - pmin + 2]
  // pre_vol of cell p from global memory (the segment's start), the variant's order
  auto prevol_g = [&](int p) {
    const double vol = g.vol;
    const int jj = j, kk = DIR == 2 ? p : c, ll = DIR == 2 ? c : p;
    auto ld = [&](const VF* a, int dj, int dk, int dl) {
      return (double)__ldg(&a[off3(g, jj + dj, kk + dk, ll + dl)]);
    };
    switch (VAR) {
      case 4: {
        const double fx1 = ld(vfx, 1, 0, 0), fx0 = ld(vfx, 0, 0, 0);
        const double fy1 = ld(vfy, 0, 1, 0), fy0 = ld(vfy, 0, 0, 0);
        const double fz1 = ld(vfz, 0, 0, 1), fz0 = ld(vfz, 0, 0, 0);
        return vol + (fx1 - fx0 + fy1 - fy0 + fz1 - fz0);
      }
      case 2:
        return vol + ld(vfy, 0, 1, 0) - ld(vfy, 0, 0, 0) + ld(vfz, 0, 0, 1) - ld(vfz, 0, 0, 0);
      case 3:
        return vol + ld(vfy, 0, 1, 0) - ld(vfy, 0, 0, 0) + ld(vfx, 1, 0, 0) - ld(vfx, 0, 0, 0);
      default:
        return vol + ld(vfz, 0, 0, 1) - ld(vfz, 0, 0, 0);
    }
  };
  // pre_vol of cell p from the staged planes p (b0) and p+1 (b1), the same order
  auto prevol_s = [&](unsigned char* b0, unsigned char* b1) {
    const double vol = g.vol;
    const double d1 = (double)P::vfd(b1)[cf], d0 = (double)P::vfd(b0)[cf];
    switch (VAR) {
      case 4: {  // z sweep: x, y (the rows), z (the sweep)
        const double fx1 = (double)P::vfx(b0)[cf + 1], fx0 = (double)P::vfx(b0)[cf];
        const double fy1 = (double)P::vfr(b0)[cf + WF], fy0 = (double)P::vfr(b0)[cf];
        return vol + (fx1 - fx0 + fy1 - fy0 + d1 - d0);
      }
      case 2:  // y sweep: y (the sweep), z (the rows)
        return vol + d1 - d0 + (double)P::vfr(b0)[cf + WF] - (double)P::vfr(b0)[cf];
      case 3:  // y sweep: y (the sweep), x
        return vol + d1 - d0 + (double)P::vfx(b0)[cf + 1] - (double)P::vfx(b0)[cf];
      default:  // z sweep: z only
        return vol + d1 - d0;
    }
  };
  // window: d0..d3 = density1(p-2..p+1), e0..e3 = energy1(p-2..p+1), old values
  double d0 = 0.0, d1 = 0.0, d2 = 0.0, d3 = 0.0, e0 = 0.0, e1 = 0.0, e2 = 0.0, e3 = 0.0;
  double pv_m = 0.0, pv_0 = 0.0;  // pre_vol(p-1), pre_vol(p)
  double vf_prev = 0.0, mf_prev = 0.0, ef_prev = 0.0;
  if (col) {
    d0 = LI(d_in, q0 - 2); d1 = LI(d_in, q0 - 1); d2 = LI(d_in, q0);
    e0 = LI(e_in, q0 - 2); e1 = LI(e_in, q0 - 1); e2 = LI(e_in, q0);
    pv_m = prevol_g(q0 - 1);
  }
  auto issue = [&](int p) {
    unsigned char* b = pm.buf(p);
    unsigned long long* bar = pm.bar(p);
    mbar_arrive_expect_tx(bar, P::kTx);
    const int x = TX * (int)blockIdx.x;
    const int y = DIR == 3 ? c0 - g.y_min + 2 : p - g.y_min + 2;
    const int z = DIR == 3 ? p - g.z_min + 2 : c0 - g.z_min + 2;
    tma_load_box(P::rho(b), &maps.d, bar, x, y, z);
    tma_load_box(P::ene(b), &maps.e, bar, x, y, z);
    tma_load_box(P::vfd(b), &maps.vfd, bar, x, y, z);
    if (P::kX) tma_load_box(P::vfx(b), &maps.vfx, bar, x, y, z);
    if (P::kR) tma_load_box(P::vfr(b), &maps.vfr, bar, x, y, z);
  };
  using MFT = MF;
  pm.run(q0, pend, status, issue, [&](int p) {
    if (!col) return;
    unsigned char* b0 = pm.buf(p);
    unsigned char* b1 = pm.buf(p + 1);
    // cell p+1 is read by face p (the upwind index clamps to pmax+2 at the top)
    unsigned char* bn = p + 1 <= top ? b1 : b0;
    d3 = (double)P::rho(bn)[cr];
    e3 = (double)P::ene(bn)[ce];
    pv_0 = prevol_s(b0, b1);
    const double vf = (double)P::vfd(b0)[cf];
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
    const AL sigmat = div_rn((AL)fabs(vf), (AL)pv_don);
    const AL sigma3 = (AL(1.0) + sigmat) * (AL)width_ratio(VD(p), VD(dif));
    const AL sigma4 = AL(2.0) - sigmat;
    AL diffuw = (AL)(d_don - d_up);
    AL diffdw = (AL)(d_dn - d_don);
    AL limiter = cell_limiter<AL>(sigmat, sigma3, sigma4, diffuw, diffdw);
    const double mflux = vf * (d_don + (double)limiter);
    if (p <= q1 || last) mass_flux[off3(g, IDX(p))] = st<MFT>(mflux);
    const double mf_stored = mflux;  // FP64 in the cell update; mf_t storage feeds the momentum sweep
    const AL sigmam = div_rn((AL)fabs(mflux), (AL)d_don * (AL)pv_don);
    diffuw = (AL)(e_don - e_up);
    diffdw = (AL)(e_dn - e_don);
    limiter = cell_limiter<AL>(sigmam, sigma3, sigma4, diffuw, diffdw);
    const double eflux = mflux * (e_don + (double)limiter);
    // advec_cell_kernel.f90:270-281 (y) / :365-376 (z) for cell p-1
    if (update && p - 1 >= q0 && p - 1 <= q1) {
      const double pmass = d1 * pv_m;
      const double pom = pmass + mf_prev - mf_stored;
      const double poe = (e1 * pmass + ef_prev - eflux) / pom;
      const double av = pv_m + vf_prev - vf;
      const R dn = st<R>(pom / av);
      const En en = st<En>(poe);
      const long long o = off3(g, IDX(p - 1));
      d_out[o] = dn;
      e_out[o] = en;
      if (lz.density0) {  // last sweep of the step: reset_field
        lz.density0[o] = dn;
        lz.energy0[o] = en;
      }
    }
    vf_prev = vf;
    mf_prev = mf_stored;
    ef_prev = eflux;
    d0 = d1; d1 = d2; d2 = d3;
    e0 = e1; e1 = e2; e2 = e3;
    pv_m = pv_0;
  });
#undef VD
#undef LI
#undef IDX
}

// The x cell sweep (advec_cell_kernel.f90:97-186) out of place, its inputs
// staged in shared memory, as k_cell_sweep_x (clover_fused.cu) forms it. Lane
// m of a warp takes face and cell c = x_min+31t+m of one row: it forms the
// fluxes at face c from cells c-2..c+1 of the row's box, and lanes 0..30
// update cell c from faces c and c+1 (lane m+1's) into the output pair, so
// 31 cells per warp and no thread reads what another writes. Plane p:
// density1, energy1 and vol_flux_x (rows k0..k0+7) and, for pre-volume
// variant 0, vol_flux_y (rows k0..k0+8) and vol_flux_z (rows k0..k0+7);
// cell l reads planes l and l+1 (vol_flux_z).
constexpr int kCellXLanes = 31;

// The box x coordinate (from the map's base, H columns before x_min) of tile
// t and the column of the tile's first cell x_min+31t in the box: the box
// starts two cells before it, rounded down to 16 bytes.
template <class T>
__device__ __forceinline__ void cell_x_box(int t, int& x, int& col) {
  constexpr int H = kTmaHalo<T>;
  const int c = kCellXLanes * t + H - 2;  // the column of cell x_min+31t-2
  x = c / H * H;
  col = c - x + 2;
}

template <class S, int VAR>
struct CellXPlane {
  using R = typename S::rho_t;
  using En = typename S::ene_t;
  using VF = typename S::vf_t;
  static constexpr bool kVf = VAR == 0;
  static constexpr int kRho = round128(8 * kTmaWidth<R> * (int)sizeof(R));
  static constexpr int kEne = round128(8 * kTmaWidth<En> * (int)sizeof(En));
  static constexpr int kVf8 = round128(8 * kTmaWidth<VF> * (int)sizeof(VF));
  static constexpr int kVf9 = round128(9 * kTmaWidth<VF> * (int)sizeof(VF));
  static constexpr int kBytes = kRho + kEne + kVf8 + (kVf ? kVf9 + kVf8 : 0);
  static constexpr unsigned kTx = box_bytes<R>(8) + box_bytes<En>(8) + box_bytes<VF>(8) +
                                  (kVf ? box_bytes<VF>(9) + box_bytes<VF>(8) : 0u);
  __device__ static R* rho(unsigned char* p) { return (R*)p; }
  __device__ static En* ene(unsigned char* p) { return (En*)(p + kRho); }
  __device__ static VF* vfx(unsigned char* p) { return (VF*)(p + kRho + kEne); }
  __device__ static VF* vfy(unsigned char* p) { return (VF*)(p + kRho + kEne + kVf8); }
  __device__ static VF* vfz(unsigned char* p) { return (VF*)(p + kRho + kEne + kVf8 + kVf9); }
};

template <class S, int VAR, int RING, int MINB>
__global__ void __launch_bounds__(TX * TY, MINB)
k_cell_sweep_x_tma(Geom g, int seg, GeomArrays ga, const __grid_constant__ CellXMaps maps,
                   typename S::rho_t* __restrict__ d_out, typename S::ene_t* __restrict__ e_out,
                   typename S::mf_t* __restrict__ mass_flux, Level0<S> lz,
                   int* __restrict__ status) {
  using P = CellXPlane<S, VAR>;
  using R = typename S::rho_t;
  using En = typename S::ene_t;
  using VF = typename S::vf_t;
  using MF = typename S::mf_t;
  using AL = typename S::arith_t;  // the limiters' arithmetic
  extern __shared__ __align__(128) unsigned char ring[];
  __shared__ unsigned long long full[RING];
  __shared__ int stop;
  const int lane = threadIdx.x, ty = threadIdx.y;
  const int c = g.x_min + kCellXLanes * (int)blockIdx.x + lane;  // this lane's face and cell
  const int k0 = g.y_min + TY * (int)blockIdx.y, k = k0 + ty;
  const int l0 = g.z_min + seg * (int)blockIdx.z;
  const int l1 = l0 + seg - 1 < g.z_max ? l0 + seg - 1 : g.z_max;
  const bool row = k <= g.y_max;  // the whole warp: k is the row's
  const int top = g.x_max + 2;
  const bool face = row && c <= top;
  const bool upd = row && lane < kCellXLanes && c <= g.x_max;
  const PlaneMarch<RING, 0, 1> pm{ring, P::kBytes, full, &stop, l0, l1 + 1};
  int xr, cr, xe, ce, xf, cf;
  cell_x_box<R>(blockIdx.x, xr, cr);
  cell_x_box<En>(blockIdx.x, xe, ce);
  cell_x_box<VF>(blockIdx.x, xf, cf);
  cr += lane; ce += lane; cf += lane;  // cell c in each box
  constexpr int WR = kTmaWidth<R>, WE = kTmaWidth<En>, WF = kTmaWidth<VF>;
  // vertexdx at c-1, c and MIN(c+1, x_max+2)
  const double* vdx = ga.vertexdx + g.o1 + 2 - g.x_min;
  const double vd_0 = face ? vdx[c] : 1.0;
  const double vd_m1 = face ? vdx[c - 1] : 1.0;
  const double vd_p1 = face && c + 1 <= top ? vdx[c + 1] : vd_0;
  auto issue = [&](int p) {
    unsigned char* b = pm.buf(p);
    unsigned long long* bar = pm.bar(p);
    mbar_arrive_expect_tx(bar, P::kTx);
    const int y = k0 - g.y_min + 2, z = p - g.z_min + 2;
    tma_load_box(P::rho(b), &maps.d, bar, xr, y, z);
    tma_load_box(P::ene(b), &maps.e, bar, xe, y, z);
    tma_load_box(P::vfx(b), &maps.vfx, bar, xf, y, z);
    if (P::kVf) {
      tma_load_box(P::vfy(b), &maps.vfy, bar, xf, y, z);
      tma_load_box(P::vfz(b), &maps.vfz, bar, xf, y, z);
    }
  };
  pm.run(l0, l1, status, issue, [&](int l) {
    if (!row) return;
    unsigned char* b = pm.buf(l);
    unsigned char* bz = pm.buf(l + 1);
    const R* dr = P::rho(b) + ty * WR + cr;
    const En* er = P::ene(b) + ty * WE + ce;
    const VF* fx = P::vfx(b) + ty * WF + cf;
    // the pre-volume of cell c+a (a = -1, 0): cell_pre_vol's variants 0 and 1
    auto pre_vol = [&](int a) {
      const double vol = g.vol;
      const double fx1 = (double)fx[a + 1], fx0 = (double)fx[a];
      if (VAR == 0) {
        const VF* fy = P::vfy(b) + ty * WF + cf + a;
        const double fy1 = (double)fy[WF], fy0 = (double)fy[0];
        const double fz1 = (double)(P::vfz(bz) + ty * WF + cf)[a];
        const double fz0 = (double)(P::vfz(b) + ty * WF + cf)[a];
        return vol + (fx1 - fx0 + fy1 - fy0 + fz1 - fz0);
      }
      return vol + fx1 - fx0;
    };
    double mf_st = 0.0, ef = 0.0;
    const double d = (double)dr[0], e = (double)er[0], vf = (double)fx[0];
    const double pv = pre_vol(0);
    if (face && c >= g.x_min) {
      // advec_cell_kernel.f90:131-169 at face c; the upwind index clamps to x_max+2
      const double d_m2 = (double)dr[-2], d_m1 = (double)dr[-1];
      const double e_m2 = (double)er[-2], e_m1 = (double)er[-1];
      double d_up, d_don, d_dn, e_up, e_don, e_dn, pv_don, vd_dif;
      if (vf > 0.0) {  // upwind c-2, donor c-1, downwind c
        d_up = d_m2; d_don = d_m1; d_dn = d; e_up = e_m2; e_don = e_m1; e_dn = e;
        pv_don = pre_vol(-1); vd_dif = vd_m1;
      } else {  // upwind min(c+1, x_max+2), donor c, downwind c-1
        const bool clamp = c + 1 > top;
        d_up = clamp ? d : (double)dr[1]; d_don = d; d_dn = d_m1;
        e_up = clamp ? e : (double)er[1]; e_don = e; e_dn = e_m1;
        pv_don = pv; vd_dif = clamp ? vd_0 : vd_p1;
      }
      const AL sigmat = div_rn((AL)fabs(vf), (AL)pv_don);
      const AL sigma3 = (AL(1.0) + sigmat) * (AL)width_ratio(vd_0, vd_dif);
      const AL sigma4 = AL(2.0) - sigmat;
      AL diffuw = (AL)(d_don - d_up);
      AL diffdw = (AL)(d_dn - d_don);
      AL limiter = cell_limiter<AL>(sigmat, sigma3, sigma4, diffuw, diffdw);
      const double mflux = vf * (d_don + (double)limiter);
      // the cell update takes the FP64 face fluxes; the stored mass flux
      // (mf_t) feeds only the momentum sweep
      mf_st = mflux;
      if (lane < kCellXLanes) mass_flux[off3(g, c, k, l)] = st<MF>(mflux);
      const AL sigmam = div_rn((AL)fabs(mflux), (AL)d_don * (AL)pv_don);
      diffuw = (AL)(e_don - e_up);
      diffdw = (AL)(e_dn - e_don);
      limiter = cell_limiter<AL>(sigmam, sigma3, sigma4, diffuw, diffdw);
      ef = mflux * (e_don + (double)limiter);
    }
    // advec_cell_kernel.f90:173-185 for cell c from faces c and c+1
    const double mf_p = __shfl_down_sync(0xffffffffu, mf_st, 1);
    const double ef_p = __shfl_down_sync(0xffffffffu, ef, 1);
    if (upd) {
      const double vf_p = (double)fx[1];
      const double pm_ = d * pv;
      const double pom = pm_ + mf_st - mf_p;
      const double poe = (e * pm_ + ef - ef_p) / pom;
      const double av = pv + vf - vf_p;
      const R dn = st<R>(pom / av);
      const En en = st<En>(poe);
      const long long o = off3(g, c, k, l);
      d_out[o] = dn;
      e_out[o] = en;
      if (lz.density0) {  // last sweep of the step: reset_field
        lz.density0[o] = dn;
        lz.energy0[o] = en;
      }
    }
  });
}

constexpr int kViscRing = 4;
constexpr int kViscSeg = 32;

}  // namespace

template <class S>
bool visc_dt_tma_maps(const Geom& g, const typename S::vel_t* xvel0, const typename S::vel_t* yvel0,
                      const typename S::vel_t* zvel0, const typename S::rho_t* density0,
                      const typename S::ene_t* energy0, ViscMaps* m) {
  using V = typename S::vel_t;
  return encode_plane_map(&m->u, xvel0, sizeof(V), g, TY + 1) &&
         encode_plane_map(&m->v, yvel0, sizeof(V), g, TY + 1) &&
         encode_plane_map(&m->w, zvel0, sizeof(V), g, TY + 1) &&
         encode_plane_map(&m->d, density0, sizeof(typename S::rho_t), g, TY + 2) &&
         encode_plane_map(&m->e, energy0, sizeof(typename S::ene_t), g, TY + 2);
}

// blocks per SM (measured at 512^3: FP64 2.90 ms at 3 against 3.15 ms at 2,
// where the FP64 form spills no register)
template <class S>
constexpr int kViscMinBlocks = sizeof(typename S::arith_t) == 4 ? 4 : 3;

template <class S>
bool visc_dt_tma_prepare() {
  return cudaFuncSetAttribute(k_visc_dt_tma<S, kViscRing, kViscMinBlocks<S>>,
                              cudaFuncAttributeMaxDynamicSharedMemorySize,
                              kViscRing * ViscPlane<S>::kBytes) == cudaSuccess;
}

template <class S>
void launch_visc_dt_tma(const Geom& g, cudaStream_t s, const ViscMaps& maps, const GeomArrays& ga,
                        double g_small, double dtc_safe, double dtu_safe, double dtv_safe,
                        double dtw_safe, double dtdiv_safe, typename S::cs_t* pressure,
                        typename S::cs_t* viscosity, typename S::cs_t* soundspeed,
                        unsigned long long* min_key, int* status) {
  auto kern = k_visc_dt_tma<S, kViscRing, kViscMinBlocks<S>>;
  const int smem = kViscRing * ViscPlane<S>::kBytes;
  const dim3 grid((g.x_max - g.x_min + TX) / TX, (g.y_max - g.y_min + TY) / TY,
                  (g.z_max - g.z_min + kViscSeg) / kViscSeg);
  kern<<<grid, dim3(TX, TY), smem, s>>>(g, kViscSeg, ga, g_small, dtc_safe, dtu_safe, dtv_safe,
                                         dtw_safe, dtdiv_safe, maps, pressure,
                                         viscosity, soundspeed, min_key, status);
}

constexpr int kMomXRing = 4;
template <class S>
constexpr int kMomXMinBlocks = sizeof(typename S::arith_t) == 4 ? 4 : 3;

template <class S>
bool mom_x_tma_prepare() {
  return cudaFuncSetAttribute(k_mom_sweep_x_tma<S, 0, kMomXRing, kMomXMinBlocks<S>>,
                              cudaFuncAttributeMaxDynamicSharedMemorySize,
                              kMomXRing * MomXPlane<S, 0>::kBytes) == cudaSuccess &&
         cudaFuncSetAttribute(k_mom_sweep_x_tma<S, 4, kMomXRing, kMomXMinBlocks<S>>,
                              cudaFuncAttributeMaxDynamicSharedMemorySize,
                              kMomXRing * MomXPlane<S, 4>::kBytes) == cudaSuccess;
}

template <class S>
void launch_mom_x_tma(const Geom& g, cudaStream_t s, int sweep, int seg, const MomXMaps& maps,
                      const GeomArrays& ga, typename S::vel_t* const* vel_out,
                      const Level0<S>& level0, int* status) {
  const dim3 grid((g.x_max + 1 - g.x_min + 1 + 28) / 29, (g.y_max + 1 - g.y_min + 1 + TY - 1) / TY,
                  (g.z_max + 1 - g.z_min + 1 + seg - 1) / seg);
  // post_vol variant: 0 on sweep 1, 4 (the cell volume) on sweep 3
  if (sweep == 1)
    k_mom_sweep_x_tma<S, 0, kMomXRing, kMomXMinBlocks<S>>
        <<<grid, dim3(TX, TY), kMomXRing * MomXPlane<S, 0>::kBytes, s>>>(
            g, seg, ga, maps, vel_out[0], vel_out[1], vel_out[2], level0, status);
  else
    k_mom_sweep_x_tma<S, 4, kMomXRing, kMomXMinBlocks<S>>
        <<<grid, dim3(TX, TY), kMomXRing * MomXPlane<S, 4>::kBytes, s>>>(
            g, seg, ga, maps, vel_out[0], vel_out[1], vel_out[2], level0, status);
}

// The bounded wait of the staged kernels, made to run out: one block arms a
// barrier phase for 16 bytes of copies that nothing issues, waits with the
// same mbar_wait_bounded the kernels use (limit `cycles`), and reports the
// failure as they do. Nothing else happens on the GPU, so the context stays
// usable.
__global__ void k_wait_selftest(long long cycles, int* status) {
  __shared__ unsigned long long bar;
  if (threadIdx.x == 0) {
    mbar_init(&bar, 1);
    mbar_init_fence();
  }
  __syncthreads();
  if (threadIdx.x == 0) mbar_arrive_expect_tx(&bar, 16);
  __syncthreads();
  const bool done = mbar_wait_bounded(&bar, 0u, cycles);
  if (!done && threadIdx.x == 0) atomicOr(status, CLOVER_STATUS_TIMEOUT);
}

constexpr int kStencilRing = 4, kStencilSeg = 32;
// blocks per SM: FP64 holds three (56-72 registers, 60-69 KB of plane
// buffers), the mixed forms four
template <class S>
constexpr int kStencilMinBlocks = sizeof(typename S::arith_t) == 4 ? 4 : 3;

template <class S>
bool stencils_tma_prepare() {
  return cudaFuncSetAttribute(k_pdv_predict_eos_tma<S, kStencilRing, kStencilMinBlocks<S>>,
                              cudaFuncAttributeMaxDynamicSharedMemorySize,
                              kStencilRing * PdvPlane<S>::kBytes) == cudaSuccess &&
         cudaFuncSetAttribute(k_accelerate_tma<S, kStencilRing, kStencilMinBlocks<S>>,
                              cudaFuncAttributeMaxDynamicSharedMemorySize,
                              kStencilRing * AccPlane<S>::kBytes) == cudaSuccess &&
         cudaFuncSetAttribute(k_pdv_flux_tma<S, kStencilRing, kStencilMinBlocks<S>>,
                              cudaFuncAttributeMaxDynamicSharedMemorySize,
                              kStencilRing * FluxPlane<S>::kBytes) == cudaSuccess;
}

// Planes per block of a staged drop-in stencil over nz planes with xy blocks
// per plane: 32 where that leaves at least eight blocks per SM (148 SMs),
// fewer on small chunks (down to 4), whose blocks would otherwise each march
// a long column of planes with most SMs idle.
int drop_seg(int nz, int xy) {
  const long long want = 148LL * 8;
  long long seg = ((long long)nz * xy + want - 1) / want;
  if (seg > kStencilSeg) seg = kStencilSeg;
  if (seg < 4) seg = 4;
  return (int)seg;
}

// blocks per SM of the drop-in PdV: the corrector's plane (six velocity
// boxes and three area boxes, 23 KB) leaves room for two blocks of a
// four-plane ring, the predictor's for three
template <bool PRED>
constexpr int kPdvDropMinBlocks = PRED ? 3 : 2;

bool pdv_dropin_tma_prepare() {
  return cudaFuncSetAttribute(k_pdv_dropin_tma<true, kStencilRing, kPdvDropMinBlocks<true>>,
                              cudaFuncAttributeMaxDynamicSharedMemorySize,
                              kStencilRing * PdvDropPlane<true>::kBytes) == cudaSuccess &&
         cudaFuncSetAttribute(k_pdv_dropin_tma<false, kStencilRing, kPdvDropMinBlocks<false>>,
                              cudaFuncAttributeMaxDynamicSharedMemorySize,
                              kStencilRing * PdvDropPlane<false>::kBytes) == cudaSuccess;
}

void launch_pdv_dropin_tma(const Geom& g, cudaStream_t s, bool predict, double dt,
                           const PdvDropMaps& maps, const double* volume, const double* density0,
                           double* density1, const double* energy0, double* energy1,
                           const double* pressure, const double* viscosity, int* status) {
  const int gx = (g.x_max - g.x_min + TX) / TX, gy = (g.y_max - g.y_min + TY) / TY;
  const int nz = g.z_max - g.z_min + 1, seg = drop_seg(nz, gx * gy);
  const dim3 grid(gx, gy, (nz + seg - 1) / seg);
  if (predict)
    k_pdv_dropin_tma<true, kStencilRing, kPdvDropMinBlocks<true>>
        <<<grid, dim3(TX, TY), kStencilRing * PdvDropPlane<true>::kBytes, s>>>(
            g, seg, dt, maps, volume, density0, density1, energy0, energy1, pressure, viscosity,
            status);
  else
    k_pdv_dropin_tma<false, kStencilRing, kPdvDropMinBlocks<false>>
        <<<grid, dim3(TX, TY), kStencilRing * PdvDropPlane<false>::kBytes, s>>>(
            g, seg, dt, maps, volume, density0, density1, energy0, energy1, pressure, viscosity,
            status);
}

constexpr int kDropMinBlocks = 2;


bool stencils_dropin_tma_prepare() {
  return cudaFuncSetAttribute(k_calc_dt_dropin_tma<kStencilRing, kDropMinBlocks>,
                              cudaFuncAttributeMaxDynamicSharedMemorySize,
                              kStencilRing * DtDropPlane::kBytes) == cudaSuccess &&
         cudaFuncSetAttribute(k_viscosity_dropin_tma<kStencilRing, kDropMinBlocks>,
                              cudaFuncAttributeMaxDynamicSharedMemorySize,
                              kStencilRing * ViscDropPlane::kBytes) == cudaSuccess &&
         cudaFuncSetAttribute(k_accelerate_dropin_tma<kStencilRing, kDropMinBlocks>,
                              cudaFuncAttributeMaxDynamicSharedMemorySize,
                              kStencilRing * AccDropPlane::kBytes) == cudaSuccess;
}

void launch_calc_dt_dropin_tma(const Geom& g, cudaStream_t s, const GeomArrays& ga, double g_small,
                               double dtc_safe, double dtu_safe, double dtv_safe, double dtw_safe,
                               double dtdiv_safe, const DtDropMaps& maps, double* dt_min,
                               unsigned long long* min_key, int* status) {
  const int gx = (g.x_max - g.x_min + TX) / TX, gy = (g.y_max - g.y_min + TY) / TY;
  const int nz = g.z_max - g.z_min + 1, seg = drop_seg(nz, gx * gy);
  const dim3 grid(gx, gy, (nz + seg - 1) / seg);
  k_calc_dt_dropin_tma<kStencilRing, kDropMinBlocks>
      <<<grid, dim3(TX, TY), kStencilRing * DtDropPlane::kBytes, s>>>(
          g, seg, ga, g_small, dtc_safe, dtu_safe, dtv_safe, dtw_safe, dtdiv_safe, maps,
          dt_min, min_key, status);
}

void launch_viscosity_dropin_tma(const Geom& g, cudaStream_t s, const GeomArrays& ga,
                                 const ViscDropMaps& maps, double* viscosity, int* status) {
  const int gx = (g.x_max - g.x_min + TX) / TX, gy = (g.y_max - g.y_min + TY) / TY;
  const int nz = g.z_max - g.z_min + 1, seg = drop_seg(nz, gx * gy);
  const dim3 grid(gx, gy, (nz + seg - 1) / seg);
  k_viscosity_dropin_tma<kStencilRing, kDropMinBlocks>
      <<<grid, dim3(TX, TY), kStencilRing * ViscDropPlane::kBytes, s>>>(g, seg, ga, maps,
                                                                         viscosity, status);
}

void launch_accelerate_dropin_tma(const Geom& g, cudaStream_t s, double dt,
                                  const AccDropMaps& maps, double* xvel1, double* yvel1,
                                  double* zvel1, int* status) {
  const int gx = (g.x_max + 1 - g.x_min + TX) / TX, gy = (g.y_max + 1 - g.y_min + TY) / TY;
  const int nz = g.z_max - g.z_min + 2, seg = drop_seg(nz, gx * gy);
  const dim3 grid(gx, gy, (nz + seg - 1) / seg);
  k_accelerate_dropin_tma<kStencilRing, kDropMinBlocks>
      <<<grid, dim3(TX, TY), kStencilRing * AccDropPlane::kBytes, s>>>(g, seg, dt, maps, xvel1,
                                                                        yvel1, zvel1, status);
}

bool mom_node_dropin_tma_prepare() {
  return cudaFuncSetAttribute(k_mom_node_x_dropin_tma<kStencilRing, 4>,
                              cudaFuncAttributeMaxDynamicSharedMemorySize,
                              kStencilRing * NodeDropPlane::kBytes) == cudaSuccess &&
         cudaFuncSetAttribute(k_mom_node_dropin_tma<2, kStencilRing, 4>,
                              cudaFuncAttributeMaxDynamicSharedMemorySize,
                              kStencilRing * NodeDropPlane::kBytes) == cudaSuccess &&
         cudaFuncSetAttribute(k_mom_node_dropin_tma<3, kStencilRing, 4>,
                              cudaFuncAttributeMaxDynamicSharedMemorySize,
                              kStencilRing * NodeDropPlane::kBytes) == cudaSuccess;
}

void launch_mom_node_dropin_tma(const Geom& g, cudaStream_t s, int dir, const NodeDropMaps& maps,
                                double* node_flux, double* node_mass_post, double* node_mass_pre,
                                int* status) {
  const int smem = kStencilRing * NodeDropPlane::kBytes;
  if (dir == 1) {  // nodes x_min-2..x_max+2, 32 per tile
    const int gx = (g.x_max - g.x_min + 5 + TX - 1) / TX, gy = (g.y_max - g.y_min + 2 + TY - 1) / TY;
    const int nz = g.z_max - g.z_min + 2, seg = drop_seg(nz, gx * gy);
    k_mom_node_x_dropin_tma<kStencilRing, 4><<<dim3(gx, gy, (nz + seg - 1) / seg), dim3(TX, TY),
                                               smem, s>>>(g, seg, maps, node_flux, node_mass_post,
                                                          node_mass_pre, status);
    return;
  }
  const int nr = (dir == 2 ? g.z_max - g.z_min : g.y_max - g.y_min) + 2;
  const int np = (dir == 2 ? g.y_max - g.y_min : g.z_max - g.z_min) + 5;
  const int gx = (g.x_max + 1 - g.x_min + TX) / TX, gy = (nr + TY - 1) / TY;
  const int seg = drop_seg(np, gx * gy);
  const dim3 grid(gx, gy, (np + seg - 1) / seg);
  if (dir == 2)
    k_mom_node_dropin_tma<2, kStencilRing, 4><<<grid, dim3(TX, TY), smem, s>>>(
        g, seg, maps, node_flux, node_mass_post, node_mass_pre, status);
  else
    k_mom_node_dropin_tma<3, kStencilRing, 4><<<grid, dim3(TX, TY), smem, s>>>(
        g, seg, maps, node_flux, node_mass_post, node_mass_pre, status);
}

// four blocks per SM in both precisions (FP64 at 64 registers, 4 bytes spilled: 1.85 -> 1.76 ms at 512^3
// against three; the y/z cell sweeps measured slower at four)
template <class S>
constexpr int kCellXMinBlocks = 4;

template <class S>
bool cell_sweep_x_tma_prepare() {
  return cudaFuncSetAttribute(k_cell_sweep_x_tma<S, 0, kStencilRing, kCellXMinBlocks<S>>,
                              cudaFuncAttributeMaxDynamicSharedMemorySize,
                              kStencilRing * CellXPlane<S, 0>::kBytes) == cudaSuccess &&
         cudaFuncSetAttribute(k_cell_sweep_x_tma<S, 1, kStencilRing, kCellXMinBlocks<S>>,
                              cudaFuncAttributeMaxDynamicSharedMemorySize,
                              kStencilRing * CellXPlane<S, 1>::kBytes) == cudaSuccess;
}

template <class S>
void launch_cell_sweep_x_tma(const Geom& g, cudaStream_t s, int sweep, const CellXMaps& maps,
                             const GeomArrays& ga, typename S::rho_t* d_out,
                             typename S::ene_t* e_out, typename S::mf_t* mass_flux_x,
                             const Level0<S>& level0, int* status) {
  // faces x_min..x_max+2, 31 per warp
  const dim3 grid((g.x_max - g.x_min + 3 + kCellXLanes - 1) / kCellXLanes,
                  (g.y_max - g.y_min + TY) / TY, (g.z_max - g.z_min + kStencilSeg) / kStencilSeg);
  if (sweep == 1)
    k_cell_sweep_x_tma<S, 0, kStencilRing, kCellXMinBlocks<S>>
        <<<grid, dim3(TX, TY), kStencilRing * CellXPlane<S, 0>::kBytes, s>>>(
            g, kStencilSeg, ga, maps, d_out, e_out, mass_flux_x, level0, status);
  else
    k_cell_sweep_x_tma<S, 1, kStencilRing, kCellXMinBlocks<S>>
        <<<grid, dim3(TX, TY), kStencilRing * CellXPlane<S, 1>::kBytes, s>>>(
            g, kStencilSeg, ga, maps, d_out, e_out, mass_flux_x, level0, status);
}

template <class S>
void launch_pdv_predict_eos_tma(const Geom& g, cudaStream_t s, const double* dt_ptr,
                                const PdvMaps& maps, typename S::cs_t* pressure, int* status) {
  const dim3 grid((g.x_max - g.x_min + TX) / TX, (g.y_max - g.y_min + TY) / TY,
                  (g.z_max - g.z_min + kStencilSeg) / kStencilSeg);
  k_pdv_predict_eos_tma<S, kStencilRing, kStencilMinBlocks<S>>
      <<<grid, dim3(TX, TY), kStencilRing * PdvPlane<S>::kBytes, s>>>(g, kStencilSeg, dt_ptr, maps,
                                                                       pressure, status);
}

template <class S>
void launch_accelerate_tma(const Geom& g, cudaStream_t s, const double* dt_ptr, const AccMaps& maps,
                           typename S::vel_t* xvel1, typename S::vel_t* yvel1,
                           typename S::vel_t* zvel1, int* status) {
  const dim3 grid((g.x_max + 1 - g.x_min + TX) / TX, (g.y_max + 1 - g.y_min + TY) / TY,
                  (g.z_max + 1 - g.z_min + kStencilSeg) / kStencilSeg);
  k_accelerate_tma<S, kStencilRing, kStencilMinBlocks<S>>
      <<<grid, dim3(TX, TY), kStencilRing * AccPlane<S>::kBytes, s>>>(g, kStencilSeg, dt_ptr, maps,
                                                                      xvel1, yvel1, zvel1, status);
}

template <class S>
void launch_pdv_flux_tma(const Geom& g, cudaStream_t s, const double* dt_ptr, const FluxMaps& maps,
                         const typename S::rho_t* density0, typename S::rho_t* density1,
                         const typename S::ene_t* energy0, typename S::ene_t* energy1,
                         const typename S::cs_t* pressure, const typename S::cs_t* viscosity,
                         typename S::vf_t* vol_flux_x, typename S::vf_t* vol_flux_y,
                         typename S::vf_t* vol_flux_z, int* status) {
  const dim3 grid((g.x_max + 1 - g.x_min + TX) / TX, (g.y_max + 1 - g.y_min + TY) / TY,
                  (g.z_max + 1 - g.z_min + kStencilSeg) / kStencilSeg);
  k_pdv_flux_tma<S, kStencilRing, kStencilMinBlocks<S>>
      <<<grid, dim3(TX, TY), kStencilRing * FluxPlane<S>::kBytes, s>>>(
          g, kStencilSeg, dt_ptr, maps, density0, density1, energy0, energy1, pressure, viscosity,
          vol_flux_x, vol_flux_y, vol_flux_z, status);
}

template <class S>
constexpr int kNodeMinBlocks = sizeof(typename S::arith_t) == 4 ? 5 : 5;

template <class S>
bool mom_node_tma_prepare() {
  bool ok = true;
  auto set = [&](auto kern, int bytes) {
    ok = ok && cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                    kStencilRing * bytes) == cudaSuccess;
  };
  set(k_mom_node_tma<S, 3, 1, kStencilRing, kNodeMinBlocks<S>>, NodePlane<S, 1>::kBytes);
  set(k_mom_node_tma<S, 3, 4, kStencilRing, kNodeMinBlocks<S>>, NodePlane<S, 4>::kBytes);
  set(k_mom_node_tma<S, 2, 2, kStencilRing, kNodeMinBlocks<S>>, NodePlane<S, 2>::kBytes);
  set(k_mom_node_tma<S, 2, 3, kStencilRing, kNodeMinBlocks<S>>, NodePlane<S, 3>::kBytes);
  return ok;
}

template <class S>
void launch_mom_node_tma(const Geom& g, cudaStream_t s, int dir, int var, const NodeMaps& maps,
                         typename S::nd_t* node_flux, typename S::nd_t* node_mass_post,
                         typename S::nd_t* node_mass_pre, int* status) {
  auto go = [&](auto kern, int bytes, const MarchRange& r) {
    const dim3 grid((r.jhi - r.jlo + 1 + 30) / 31, (r.chi - r.clo + 1 + TY - 1) / TY,
                    (r.phi - r.plo + 1 + kStencilSeg - 1) / kStencilSeg);
    kern<<<grid, dim3(TX, TY), kStencilRing * bytes, s>>>(g, kStencilSeg, maps, node_flux,
                                                          node_mass_post, node_mass_pre, status);
  };
  if (dir == 3) {
    const MarchRange r = mom_node_range<3>(g);
    if (var == 1) go(k_mom_node_tma<S, 3, 1, kStencilRing, kNodeMinBlocks<S>>, NodePlane<S, 1>::kBytes, r);
    else go(k_mom_node_tma<S, 3, 4, kStencilRing, kNodeMinBlocks<S>>, NodePlane<S, 4>::kBytes, r);
  } else {
    const MarchRange r = mom_node_range<2>(g);
    if (var == 2) go(k_mom_node_tma<S, 2, 2, kStencilRing, kNodeMinBlocks<S>>, NodePlane<S, 2>::kBytes, r);
    else go(k_mom_node_tma<S, 2, 3, kStencilRing, kNodeMinBlocks<S>>, NodePlane<S, 3>::kBytes, r);
  }
}

template <class S>
constexpr int kVelMinBlocks = sizeof(typename S::arith_t) == 4 ? 5 : 3;
// five plane buffers: two planes in flight beyond the three a node reads
// (advec_mom_yz 6.97 -> 6.85 ms at 512^3 FP64 against four)
constexpr int kVelRing = 5;

template <class S>
bool mom_vel_tma_prepare() {
  return cudaFuncSetAttribute(k_mom_vel_tma<S, 2, kVelRing, kVelMinBlocks<S>>,
                              cudaFuncAttributeMaxDynamicSharedMemorySize,
                              kVelRing * VelPlane<S>::kBytes) == cudaSuccess &&
         cudaFuncSetAttribute(k_mom_vel_tma<S, 3, kVelRing, kVelMinBlocks<S>>,
                              cudaFuncAttributeMaxDynamicSharedMemorySize,
                              kVelRing * VelPlane<S>::kBytes) == cudaSuccess;
}

template <class S>
void launch_mom_vel_tma(const Geom& g, cudaStream_t s, int dir, const VelMaps& maps,
                        const GeomArrays& ga, const typename S::nd_t* node_flux,
                        const typename S::nd_t* node_mass_pre, typename S::vel_t* const* vel_in,
                        typename S::vel_t* const* vel_out, const Level0<S>& level0, int* status) {
  auto go = [&](auto kern, const MarchRange& r) {
    const dim3 grid((r.jhi - r.jlo + TX) / TX, (r.chi - r.clo + TY) / TY,
                    (r.phi - r.plo + kStencilSeg) / kStencilSeg);
    kern<<<grid, dim3(TX, TY), kVelRing * VelPlane<S>::kBytes, s>>>(
        g, kStencilSeg, ga, maps, node_flux, node_mass_pre, vel_in[0], vel_in[1], vel_in[2],
        vel_out[0], vel_out[1], vel_out[2], level0, status);
  };
  if (dir == 2) go(k_mom_vel_tma<S, 2, kVelRing, kVelMinBlocks<S>>, mom_vel_range<2>(g));
  else go(k_mom_vel_tma<S, 3, kVelRing, kVelMinBlocks<S>>, mom_vel_range<3>(g));
}

template <class S>
constexpr int kCellMinBlocks = sizeof(typename S::arith_t) == 4 ? 4 : 3;

template <class S>
bool cell_sweep_tma_prepare() {
  bool ok = true;
  auto set = [&](auto kern, int bytes) {
    ok = ok && cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                    kStencilRing * bytes) == cudaSuccess;
  };
  set(k_cell_sweep_tma<S, 2, 2, kStencilRing, kCellMinBlocks<S>>, CellPlane<S, 2, 2>::kBytes);
  set(k_cell_sweep_tma<S, 2, 3, kStencilRing, kCellMinBlocks<S>>, CellPlane<S, 2, 3>::kBytes);
  set(k_cell_sweep_tma<S, 3, 4, kStencilRing, kCellMinBlocks<S>>, CellPlane<S, 3, 4>::kBytes);
  set(k_cell_sweep_tma<S, 3, 5, kStencilRing, kCellMinBlocks<S>>, CellPlane<S, 3, 5>::kBytes);
  return ok;
}

template <class S>
void launch_cell_sweep_tma(const Geom& g, cudaStream_t s, int dir, int var, const CellMaps& maps,
                           const GeomArrays& ga, const typename S::rho_t* d_in,
                           const typename S::ene_t* e_in, typename S::rho_t* d_out,
                           typename S::ene_t* e_out, const typename S::vf_t* vfx,
                           const typename S::vf_t* vfy, const typename S::vf_t* vfz,
                           typename S::mf_t* mass_flux, const Level0<S>& level0, int* status) {
  auto go = [&](auto kern, int bytes, const MarchRange& r, int pcells) {
    const dim3 grid((r.jhi - r.jlo + TX) / TX, (r.chi - r.clo + TY) / TY,
                    (pcells + kStencilSeg - 1) / kStencilSeg);
    kern<<<grid, dim3(TX, TY), kStencilRing * bytes, s>>>(g, kStencilSeg, ga, maps, d_in, e_in,
                                                          d_out, e_out, vfx, vfy, vfz, mass_flux,
                                                          level0, status);
  };
  const int ny = g.y_max - g.y_min + 1, nz = g.z_max - g.z_min + 1;
  if (dir == 2) {
    const MarchRange r = cell_sweep_range<2>(g);
    if (var == 2) go(k_cell_sweep_tma<S, 2, 2, kStencilRing, kCellMinBlocks<S>>, CellPlane<S, 2, 2>::kBytes, r, ny);
    else go(k_cell_sweep_tma<S, 2, 3, kStencilRing, kCellMinBlocks<S>>, CellPlane<S, 2, 3>::kBytes, r, ny);
  } else {
    const MarchRange r = cell_sweep_range<3>(g);
    if (var == 4) go(k_cell_sweep_tma<S, 3, 4, kStencilRing, kCellMinBlocks<S>>, CellPlane<S, 3, 4>::kBytes, r, nz);
    else go(k_cell_sweep_tma<S, 3, 5, kStencilRing, kCellMinBlocks<S>>, CellPlane<S, 3, 5>::kBytes, r, nz);
  }
}

#define INST_TMA(S)                                                                              \
  template bool visc_dt_tma_maps<S>(const Geom&, const S::vel_t*, const S::vel_t*,              \
                                    const S::vel_t*, const S::rho_t*, const S::ene_t*,          \
                                    ViscMaps*);                                                  \
  template bool visc_dt_tma_prepare<S>();                                                        \
  template bool mom_x_tma_prepare<S>();                                                          \
  template bool stencils_tma_prepare<S>();                                                       \
  template bool mom_node_tma_prepare<S>();                                                       \
  template bool mom_vel_tma_prepare<S>();                                                        \
  template bool cell_sweep_tma_prepare<S>();                                                     \
  template void launch_cell_sweep_tma<S>(const Geom&, cudaStream_t, int, int, const CellMaps&,   \
                                         const GeomArrays&, const S::rho_t*, const S::ene_t*,    \
                                         S::rho_t*, S::ene_t*, const S::vf_t*, const S::vf_t*,   \
                                         const S::vf_t*, S::mf_t*, const Level0<S>&, int*);      \
  template void launch_mom_vel_tma<S>(const Geom&, cudaStream_t, int, const VelMaps&,            \
                                      const GeomArrays&, const S::nd_t*, const S::nd_t*,         \
                                      S::vel_t* const*, S::vel_t* const*, const Level0<S>&, int*); \
  template void launch_mom_node_tma<S>(const Geom&, cudaStream_t, int, int, const NodeMaps&,     \
                                       S::nd_t*, S::nd_t*, S::nd_t*, int*);                      \
  template bool cell_sweep_x_tma_prepare<S>();                                                   \
  template void launch_cell_sweep_x_tma<S>(const Geom&, cudaStream_t, int, const CellXMaps&,     \
                                           const GeomArrays&, S::rho_t*, S::ene_t*, S::mf_t*,    \
                                           const Level0<S>&, int*);                              \
  template void launch_pdv_predict_eos_tma<S>(const Geom&, cudaStream_t, const double*,         \
                                              const PdvMaps&, S::cs_t*, int*);                   \
  template void launch_accelerate_tma<S>(const Geom&, cudaStream_t, const double*,               \
                                         const AccMaps&, S::vel_t*, S::vel_t*, S::vel_t*, int*); \
  template void launch_pdv_flux_tma<S>(const Geom&, cudaStream_t, const double*, const FluxMaps&, \
                                       const S::rho_t*, S::rho_t*, const S::ene_t*, S::ene_t*,   \
                                       const S::cs_t*, const S::cs_t*, S::vf_t*, S::vf_t*,       \
                                       S::vf_t*, int*);                                          \
  template void launch_mom_x_tma<S>(const Geom&, cudaStream_t, int, int, const MomXMaps&,        \
                                    const GeomArrays&, S::vel_t* const*, const Level0<S>&, int*); \
  template void launch_visc_dt_tma<S>(const Geom&, cudaStream_t, const ViscMaps&, const GeomArrays&, \
                                      double, double, double, double, double, double, S::cs_t*,  \
                                      S::cs_t*, S::cs_t*, unsigned long long*, int*);
INST_TMA(F64)
INST_TMA(F32Mixed)

void launch_wait_selftest(cudaStream_t s, long long cycles, int* status) {
  k_wait_selftest<<<1, 32, 0, s>>>(cycles, status);
}

}  // namespace clover

using namespace clover;

extern "C" int clover_gpu_wait_selftest(long long cycles) {
  int* d = nullptr;
  int h = 0;
  if (cudaMalloc(&d, sizeof(int)) != cudaSuccess) {
    cudaGetLastError();
    return CLOVER_STATUS_CUDA_ERROR;
  }
  cudaMemset(d, 0, sizeof(int));
  k_wait_selftest<<<1, 32>>>(cycles, d);
  const cudaError_t e1 = cudaGetLastError();
  const cudaError_t e2 = cudaMemcpy(&h, d, sizeof(int), cudaMemcpyDeviceToHost);
  cudaFree(d);
  if (e1 != cudaSuccess || e2 != cudaSuccess) return CLOVER_STATUS_CUDA_ERROR;
  return h;
}
