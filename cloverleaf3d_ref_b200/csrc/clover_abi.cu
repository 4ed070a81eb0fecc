// Drop-in C ABI (include/clover_kernels.h): host-pointer mirrors and the
// extern "C" entry points that replace the reference's *_kernel procedures.
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <mutex>
#include <string>
#include <unordered_map>

#include "../../include/clover_kernels.h"
#include "clover_launch.h"

namespace clover {
namespace {

// Host-side extents of a reference array argument (Fortran declared shape).
struct HostShape {
  int hx, hy, hz;  // 1D arrays: hy = hz = 1
  bool one_d;
};

struct Mirror {
  void* raw = nullptr;      // cudaMalloc'd base
  double* dev = nullptr;    // element (min-2, min-2, min-2)
  HostShape shape{};        // largest declared shape seen
  int planes = 0;           // host planes copied up so far
  bool pinned = false;
};

struct Context {
  bool ready = false;
  Geom g{};
  cudaStream_t stream = nullptr;
  std::unordered_map<const void*, Mirror> mirrors;
  unsigned long long* d_key = nullptr;
  double* d_partials = nullptr;
  double* d_sum = nullptr;
  double* stage = nullptr;  // contiguous copy of host planes on their way up or down
  size_t stage_bytes = 0;
  int status = 0;
  std::string err;
  bool pin_host = true;
};

Context& ctx() {
  static Context c;
  return c;
}

void set_error(int bit, const std::string& msg) {
  Context& c = ctx();
  c.status |= bit;
  if (c.err.empty()) c.err = msg;
}

bool check(cudaError_t e, const char* what) {
  if (e == cudaSuccess) return true;
  set_error(CLOVER_STATUS_CUDA_ERROR, std::string(what) + ": " + cudaGetErrorString(e));
  return false;
}

void check_launch(const char* what) { check(cudaGetLastError(), what); }

// Create the context on first use; every call must pass the same bounds.
bool enter(const int* x_min, const int* x_max, const int* y_min, const int* y_max,
           const int* z_min, const int* z_max) {
  Context& c = ctx();
  if (!c.ready) {
    int n = 0;
    if (cudaGetDeviceCount(&n) != cudaSuccess || n == 0) {
      set_error(CLOVER_STATUS_NO_DEVICE, "no CUDA device");
      return false;
    }
    c.g = make_geom(*x_min, *x_max, *y_min, *y_max, *z_min, *z_max);
    if (!check(cudaStreamCreateWithFlags(&c.stream, cudaStreamNonBlocking), "stream")) return false;
    if (!check(cudaMalloc(&c.d_key, sizeof(unsigned long long)), "malloc")) return false;
    if (!check(cudaMalloc(&c.d_partials, summary_partials_len() * sizeof(double)), "malloc"))
      return false;
    if (!check(cudaMalloc(&c.d_sum, 5 * sizeof(double)), "malloc")) return false;
    const char* pin = getenv("CLOVER_GPU_PIN_HOST");
    c.pin_host = !(pin && pin[0] == '0');
    c.ready = true;
    return true;
  }
  const Geom& g = c.g;
  if (g.x_min != *x_min || g.x_max != *x_max || g.y_min != *y_min || g.y_max != *y_max ||
      g.z_min != *z_min || g.z_max != *z_max) {
    set_error(CLOVER_STATUS_BOUNDS, "call with bounds of another chunk");
    return false;
  }
  return true;
}

bool is_device_pointer(const void* p) {
  cudaPointerAttributes a;
  if (cudaPointerGetAttributes(&a, p) != cudaSuccess) {
    cudaGetLastError();
    return false;
  }
  return a.type == cudaMemoryTypeDevice || a.type == cudaMemoryTypeManaged;
}

}  // namespace

// Rows of hx elements between the host's contiguous planes (hy rows each) and
// the mirror's pitched layout (row pitch px, plane pitch pxy): one block per
// row, grid-strided.
__global__ void k_rows_to_pitched(const double* __restrict__ src, double* __restrict__ dst, int hx,
                                  int hy, long long rows, int px, long long pxy) {
  for (long long r = blockIdx.x; r < rows; r += gridDim.x) {
    const double* s = src + r * hx;
    double* d = dst + (r / hy) * pxy + (r % hy) * px;
    for (int i = threadIdx.x; i < hx; i += blockDim.x) d[i] = s[i];
  }
}
__global__ void k_pitched_to_rows(const double* __restrict__ src, double* __restrict__ dst, int hx,
                                  int hy, long long rows, int px, long long pxy) {
  for (long long r = blockIdx.x; r < rows; r += gridDim.x) {
    const double* s = src + (r / hy) * pxy + (r % hy) * px;
    double* d = dst + r * hx;
    for (int i = threadIdx.x; i < hx; i += blockDim.x) d[i] = s[i];
  }
}

// Host <-> device copy of planes [p0,p1) of a 3D mirror: one contiguous DMA
// of the host planes to or from a staging buffer, and a kernel that moves the
// rows between the staging buffer and the pitched mirror (a strided copy of
// ~4 KB rows runs at a fraction of the link's rate).
static void xfer3d(const void* host, Mirror& m, int p0, int p1, bool up) {
  Context& c = ctx();
  if (p1 <= p0) return;
  const HostShape& s = m.shape;
  const size_t host_plane = (size_t)s.hx * s.hy * 8;
  const size_t bytes = host_plane * (size_t)(p1 - p0);
  if (bytes > c.stage_bytes) {
    cudaStreamSynchronize(c.stream);
    cudaFree(c.stage);
    c.stage = nullptr;
    c.stage_bytes = 0;
    if (!check(cudaMalloc(&c.stage, bytes), "staging malloc")) return;
    c.stage_bytes = bytes;
  }
  char* hp = (char*)host + host_plane * p0;
  double* dp = m.dev + c.g.pxy * p0;
  const long long rows = (long long)s.hy * (p1 - p0);
  if (up) {
    check(cudaMemcpyAsync(c.stage, hp, bytes, cudaMemcpyHostToDevice, c.stream), "upload");
    k_rows_to_pitched<<<148 * 8, 256, 0, c.stream>>>(c.stage, dp, s.hx, s.hy, rows, c.g.px,
                                                     c.g.pxy);
    check_launch("upload rows");
  } else {
    k_pitched_to_rows<<<148 * 8, 256, 0, c.stream>>>(dp, c.stage, s.hx, s.hy, rows, c.g.px,
                                                     c.g.pxy);
    check_launch("download rows");
    check(cudaMemcpyAsync(hp, c.stage, bytes, cudaMemcpyDeviceToHost, c.stream), "download");
  }
}

// Resolve a 3D array argument to its device copy.
static double* dev3(double* host, int hx, int hy, int hz) {
  Context& c = ctx();
  if (!host) return nullptr;
  auto it = c.mirrors.find(host);
  if (it == c.mirrors.end()) {
    if (is_device_pointer(host)) return host;
    Mirror m;
    const long long elems = array_elems(c.g) + kFrontPad<double>;
    if (!check(cudaMalloc(&m.raw, (size_t)elems * 8), "mirror malloc")) return nullptr;
    m.dev = (double*)m.raw + kFrontPad<double>;
    check(cudaMemsetAsync(m.raw, 0, (size_t)elems * 8, c.stream), "mirror clear");
    m.shape = HostShape{hx, hy, hz, false};
    // Page-lock large host arrays for full-bandwidth copies. Only arrays of
    // 64 MiB and more: those are mapped on pages of their own, whereas small
    // heap arrays share pages with their neighbours, and a copy that
    // straddles the end of a locked range is rejected.
    const size_t bytes = (size_t)hx * hy * hz * 8;
    if (c.pin_host && bytes >= ((size_t)64 << 20)) {
      m.pinned = cudaHostRegister(host, bytes, cudaHostRegisterDefault) == cudaSuccess;
      if (!m.pinned) cudaGetLastError();
    }
    it = c.mirrors.emplace(host, m).first;
  }
  Mirror& m = it->second;
  if (hz > m.shape.hz) {
    // A later declaration covers more planes (e.g. post_ener is declared to
    // z_max+2, the same work array elsewhere to z_max+3): a copy may not
    // straddle the end of a page-locked range, so lock the larger range.
    if (m.pinned) {
      cudaHostUnregister(host);
      m.pinned = cudaHostRegister(host, (size_t)hx * hy * hz * 8, cudaHostRegisterDefault) ==
                 cudaSuccess;
      if (!m.pinned) cudaGetLastError();
    }
    m.shape.hz = hz;
  }
  if (hz > m.planes) {
    xfer3d(host, m, m.planes, hz, true);
    m.planes = hz;
  }
  return m.dev;
}

// Resolve a 1D coordinate array argument (n elements from min-2).
static double* dev1(double* host, int n) {
  Context& c = ctx();
  if (!host) return nullptr;
  auto it = c.mirrors.find(host);
  if (it == c.mirrors.end()) {
    if (is_device_pointer(host)) return host;
    Mirror m;
    if (!check(cudaMalloc(&m.raw, (size_t)(n + 32) * 8), "mirror malloc")) return nullptr;
    m.dev = (double*)m.raw;
    m.shape = HostShape{n, 1, 1, true};
    it = c.mirrors.emplace(host, m).first;
  }
  Mirror& m = it->second;
  if (m.planes == 0 || n > m.shape.hx) {
    m.shape.hx = n > m.shape.hx ? n : m.shape.hx;
    check(cudaMemcpyAsync(m.dev, host, (size_t)m.shape.hx * 8, cudaMemcpyHostToDevice, c.stream),
          "upload");
    m.planes = 1;
  }
  return m.dev;
}

}  // namespace clover

using namespace clover;

#define BOUNDS x_min, x_max, y_min, y_max, z_min, z_max
#define ENTER()                                   \
  if (!enter(BOUNDS)) return;                     \
  Context& c = ctx();                             \
  const Geom& g = c.g;                            \
  const int nx = *x_max - *x_min + 1, ny = *y_max - *y_min + 1, nz = *z_max - *z_min + 1; \
  (void)nx; (void)ny; (void)nz; (void)g
// declared shapes (build_field.f90:41-146)
#define CELL(p) dev3(p, nx + 4, ny + 4, nz + 4)
#define VERT(p) dev3(p, nx + 5, ny + 5, nz + 5)
#define VERTZ2(p) dev3(p, nx + 5, ny + 5, nz + 4) /* z declared to z_max+2 */
#define XF(p) dev3(p, nx + 5, ny + 4, nz + 4)
#define YF(p) dev3(p, nx + 4, ny + 5, nz + 4)
#define ZF(p) dev3(p, nx + 4, ny + 4, nz + 5)
#define CX(p) dev1(p, nx + 4)
#define CY(p) dev1(p, ny + 4)
#define CZ(p) dev1(p, nz + 4)
#define VX(p) dev1(p, nx + 5)
#define VY(p) dev1(p, ny + 5)
#define VZ(p) dev1(p, nz + 5)

static GeomArrays no_geom() {
  GeomArrays ga;
  memset(&ga, 0, sizeof(ga));
  return ga;
}

extern "C" {

void clover_ideal_gas_kernel(const int* x_min, const int* x_max, const int* y_min,
                             const int* y_max, const int* z_min, const int* z_max,
                             double* density, double* energy, double* pressure,
                             double* soundspeed) {
  ENTER();
  launch_ideal_gas<F64>(g, c.stream, CELL(density), CELL(energy), CELL(pressure), CELL(soundspeed));
  check_launch("ideal_gas");
}

void clover_viscosity_kernel(const int* x_min, const int* x_max, const int* y_min,
                             const int* y_max, const int* z_min, const int* z_max,
                             double* xarea, double* yarea, double* zarea, double* celldx,
                             double* celldy, double* celldz, double* density0,
                             double* pressure, double* viscosity, double* xvel0,
                             double* yvel0, double* zvel0) {
  ENTER();
  GeomArrays ga = no_geom();
  ga.xarea = XF(xarea); ga.yarea = YF(yarea); ga.zarea = ZF(zarea);
  ga.celldx = CX(celldx); ga.celldy = CY(celldy); ga.celldz = CZ(celldz);
  launch_viscosity<F64>(g, c.stream, ga, CELL(density0), CELL(pressure), CELL(viscosity),
                        VERT(xvel0), VERT(yvel0), VERT(zvel0));
  check_launch("viscosity");
}

void clover_calc_dt_kernel(const int* x_min, const int* x_max, const int* y_min,
                           const int* y_max, const int* z_min, const int* z_max,
                           const double* g_small, const double* g_big, const double* dtmin,
                           const double* dtc_safe, const double* dtu_safe,
                           const double* dtv_safe, const double* dtw_safe,
                           const double* dtdiv_safe, double* xarea, double* yarea,
                           double* zarea, double* cellx, double* celly, double* cellz,
                           double* celldx, double* celldy, double* celldz, double* volume,
                           double* density0, double* energy0, double* pressure,
                           double* viscosity_a, double* soundspeed, double* xvel0,
                           double* yvel0, double* zvel0, double* dt_min, double* dt_min_val,
                           int* dtl_control, double* xl_pos, double* yl_pos, double* zl_pos,
                           int* jldt, int* kldt, int* lldt, int* small) {
  ENTER();
  (void)energy0;
  (void)pressure;
  GeomArrays ga = no_geom();
  ga.xarea = XF(xarea); ga.yarea = YF(yarea); ga.zarea = ZF(zarea);
  ga.celldx = CX(celldx); ga.celldy = CY(celldy); ga.celldz = CZ(celldz);
  ga.volume = CELL(volume);
  const unsigned long long init = min_key_of(*g_big);
  check(cudaMemcpyAsync(c.d_key, &init, sizeof(init), cudaMemcpyHostToDevice, c.stream), "key");
  launch_calc_dt<F64>(g, c.stream, ga, *g_small, *dtc_safe, *dtu_safe, *dtv_safe, *dtw_safe,
                      *dtdiv_safe, CELL(density0), CELL(viscosity_a), CELL(soundspeed),
                      VERT(xvel0), VERT(yvel0), VERT(zvel0), VERT(dt_min), c.d_key);
  check_launch("calc_dt");
  unsigned long long key = init;
  check(cudaMemcpyAsync(&key, c.d_key, sizeof(key), cudaMemcpyDeviceToHost, c.stream), "key");
  check(cudaStreamSynchronize(c.stream), "calc_dt sync");
  *dt_min_val = min_key_value(key);
  // calc_dt_kernel.f90:154-161: jkl_control is the constant 1.1 (a default
  // REAL), so these outputs never depend on the field.
  double jkl_control = (double)1.1f;
  *dtl_control = (int)((double)10.01f * (jkl_control - (double)(int)jkl_control));
  jkl_control = jkl_control - (jkl_control - (double)(int)jkl_control);
  *jldt = ((int)jkl_control) % (*x_max);
  *kldt = (int)(1.0 + (jkl_control / (double)(*x_max)));
  *lldt = (int)(1.0 + (jkl_control / (double)(*x_max)));
  const double* px = is_device_pointer(cellx) ? nullptr : cellx;
  const double* py = is_device_pointer(celly) ? nullptr : celly;
  const double* pz = is_device_pointer(cellz) ? nullptr : cellz;
  *xl_pos = px ? px[*jldt - *x_min + 2] : 0.0;
  *yl_pos = py ? py[*kldt - *y_min + 2] : 0.0;
  *zl_pos = pz ? pz[*lldt - *z_min + 2] : 0.0;
  *small = *dt_min_val < *dtmin ? 1 : 0;
  if (*small) {
    c.status |= CLOVER_STATUS_SMALL_DT;
    fprintf(stderr, "Timestep information:\n timestep : %.17g\n", *dt_min_val);
  }
}

void clover_pdv_kernel(const int32_t* predict, const int* x_min, const int* x_max,
                       const int* y_min, const int* y_max, const int* z_min, const int* z_max,
                       const double* dt, double* xarea, double* yarea, double* zarea,
                       double* volume, double* density0, double* density1, double* energy0,
                       double* energy1, double* pressure, double* viscosity, double* xvel0,
                       double* xvel1, double* yvel0, double* yvel1, double* zvel0,
                       double* zvel1) {
  ENTER();
  GeomArrays ga = no_geom();
  ga.xarea = XF(xarea); ga.yarea = YF(yarea); ga.zarea = ZF(zarea); ga.volume = CELL(volume);
  launch_pdv<F64>(g, c.stream, *predict != 0, *dt, nullptr, ga, CELL(density0), CELL(density1),
                  CELL(energy0), CELL(energy1), CELL(pressure), CELL(viscosity), VERT(xvel0),
                  VERT(xvel1), VERT(yvel0), VERT(yvel1), VERT(zvel0), VERT(zvel1));
  check_launch("PdV");
}

void clover_revert_kernel(const int* x_min, const int* x_max, const int* y_min,
                          const int* y_max, const int* z_min, const int* z_max,
                          double* density0, double* density1, double* energy0,
                          double* energy1) {
  ENTER();
  launch_revert<F64>(g, c.stream, CELL(density0), CELL(density1), CELL(energy0), CELL(energy1));
  check_launch("revert");
}

void clover_accelerate_kernel(const int* x_min, const int* x_max, const int* y_min,
                              const int* y_max, const int* z_min, const int* z_max,
                              const double* dt, double* xarea, double* yarea, double* zarea,
                              double* volume, double* density0, double* pressure,
                              double* viscosity, double* xvel0, double* yvel0, double* zvel0,
                              double* xvel1, double* yvel1, double* zvel1) {
  ENTER();
  GeomArrays ga = no_geom();
  ga.xarea = XF(xarea); ga.yarea = YF(yarea); ga.zarea = ZF(zarea); ga.volume = CELL(volume);
  launch_accelerate<F64>(g, c.stream, *dt, nullptr, ga, CELL(density0), CELL(pressure),
                         CELL(viscosity), VERT(xvel0), VERT(yvel0), VERT(zvel0), VERT(xvel1),
                         VERT(yvel1), VERT(zvel1));
  check_launch("accelerate");
}

void clover_flux_calc_kernel(const int* x_min, const int* x_max, const int* y_min,
                             const int* y_max, const int* z_min, const int* z_max,
                             const double* dt, double* xarea, double* yarea, double* zarea,
                             double* xvel0, double* yvel0, double* zvel0, double* xvel1,
                             double* yvel1, double* zvel1, double* vol_flux_x,
                             double* vol_flux_y, double* vol_flux_z) {
  ENTER();
  GeomArrays ga = no_geom();
  ga.xarea = XF(xarea); ga.yarea = YF(yarea); ga.zarea = ZF(zarea);
  launch_flux_calc<F64>(g, c.stream, *dt, nullptr, ga, VERT(xvel0), VERT(yvel0), VERT(zvel0),
                        VERT(xvel1), VERT(yvel1), VERT(zvel1), XF(vol_flux_x), YF(vol_flux_y),
                        ZF(vol_flux_z));
  check_launch("flux_calc");
}

void clover_advec_cell_kernel(const int* x_min, const int* x_max, const int* y_min,
                              const int* y_max, const int* z_min, const int* z_max,
                              const int32_t* advect_x, const int* dir, const int* sweep_number,
                              double* vertexdx, double* vertexdy, double* vertexdz,
                              double* volume, double* density1, double* energy1,
                              double* mass_flux_x, double* vol_flux_x, double* mass_flux_y,
                              double* vol_flux_y, double* mass_flux_z, double* vol_flux_z,
                              double* pre_vol, double* post_vol, double* pre_mass,
                              double* post_mass, double* advec_vol, double* post_ener,
                              double* ener_flux) {
  ENTER();
  GeomArrays ga = no_geom();
  ga.vertexdx = VX(vertexdx); ga.vertexdy = VY(vertexdy); ga.vertexdz = VZ(vertexdz);
  ga.volume = CELL(volume);
  double* work[7] = {VERT(pre_vol), VERT(post_vol), VERT(pre_mass), VERT(post_mass),
                     VERT(advec_vol), VERTZ2(post_ener), VERTZ2(ener_flux)};
  launch_advec_cell<F64>(g, c.stream, *advect_x != 0, *dir, *sweep_number, ga, CELL(density1),
                         CELL(energy1), XF(mass_flux_x), XF(vol_flux_x), YF(mass_flux_y),
                         YF(vol_flux_y), ZF(mass_flux_z), ZF(vol_flux_z), work);
  check_launch("advec_cell");
}

void clover_advec_mom_kernel(const int* x_min, const int* x_max, const int* y_min,
                             const int* y_max, const int* z_min, const int* z_max,
                             double* vel1, double* mass_flux_x, double* vol_flux_x,
                             double* mass_flux_y, double* vol_flux_y, double* mass_flux_z,
                             double* vol_flux_z, double* volume, double* density1,
                             double* node_flux, double* node_mass_post, double* node_mass_pre,
                             double* advec_vel, double* mom_flux, double* pre_vol,
                             double* post_vol, double* celldx, double* celldy, double* celldz,
                             const int32_t* advect_x, const int* which_vel,
                             const int* sweep_number, const int* direction) {
  ENTER();
  GeomArrays ga = no_geom();
  ga.volume = CELL(volume);
  ga.celldx = CX(celldx); ga.celldy = CY(celldy); ga.celldz = CZ(celldz);
  double* work[7] = {VERT(node_flux), VERT(node_mass_post), VERT(node_mass_pre),
                     VERT(advec_vel), VERT(mom_flux), VERT(pre_vol), VERT(post_vol)};
  launch_advec_mom<F64>(g, c.stream, VERT(vel1), XF(mass_flux_x), XF(vol_flux_x),
                        YF(mass_flux_y), YF(vol_flux_y), ZF(mass_flux_z), ZF(vol_flux_z), ga,
                        CELL(density1), work, *advect_x != 0, *which_vel, *sweep_number,
                        *direction);
  check_launch("advec_mom");
}

void clover_reset_field_kernel(const int* x_min, const int* x_max, const int* y_min,
                               const int* y_max, const int* z_min, const int* z_max,
                               double* density0, double* density1, double* energy0,
                               double* energy1, double* xvel0, double* xvel1, double* yvel0,
                               double* yvel1, double* zvel0, double* zvel1) {
  ENTER();
  launch_reset_field<F64>(g, c.stream, CELL(density0), CELL(density1), CELL(energy0),
                          CELL(energy1), VERT(xvel0), VERT(xvel1), VERT(yvel0), VERT(yvel1),
                          VERT(zvel0), VERT(zvel1));
  check_launch("reset_field");
}

void clover_field_summary_kernel(const int* x_min, const int* x_max, const int* y_min,
                                 const int* y_max, const int* z_min, const int* z_max,
                                 double* volume, double* density0, double* energy0,
                                 double* pressure, double* xvel0, double* yvel0, double* zvel0,
                                 double* vol, double* mass, double* ie, double* ke,
                                 double* press) {
  ENTER();
  launch_field_summary<F64>(g, c.stream, CELL(volume), CELL(density0), CELL(energy0),
                            CELL(pressure), VERTZ2(xvel0), VERTZ2(yvel0), VERTZ2(zvel0),
                            c.d_partials, c.d_sum);
  check_launch("field_summary");
  double s[5] = {0, 0, 0, 0, 0};
  check(cudaMemcpyAsync(s, c.d_sum, sizeof(s), cudaMemcpyDeviceToHost, c.stream), "summary");
  check(cudaStreamSynchronize(c.stream), "summary sync");
  *vol = s[0]; *mass = s[1]; *ie = s[2]; *ke = s[3]; *press = s[4];
}

void clover_update_halo_kernel(const int* x_min, const int* x_max, const int* y_min,
                               const int* y_max, const int* z_min, const int* z_max,
                               const int* chunk_neighbours, const int* tile_neighbours,
                               double* density0, double* energy0, double* pressure,
                               double* viscosity, double* soundspeed, double* density1,
                               double* energy1, double* xvel0, double* yvel0, double* zvel0,
                               double* xvel1, double* yvel1, double* zvel1,
                               double* vol_flux_x, double* vol_flux_y, double* vol_flux_z,
                               double* mass_flux_x, double* mass_flux_y, double* mass_flux_z,
                               const int* fields, const int* depth) {
  ENTER();
  if (*depth < 1 || *depth > 2) {  // the halo is two cells deep
    set_error(CLOVER_STATUS_BAD_ARG, "update_halo depth must be 1 or 2");
    return;
  }
  int ext[6];
  for (int f = 0; f < 6; f++) ext[f] = chunk_neighbours[f] == -1 && tile_neighbours[f] == -1;
  HaloFields hf;
  double* host[19] = {density0, density1, energy0, energy1, pressure, viscosity, soundspeed,
                      xvel0, xvel1, yvel0, yvel1, zvel0, zvel1, vol_flux_x, vol_flux_y,
                      vol_flux_z, mass_flux_x, mass_flux_y, mass_flux_z};
  for (int i = 0; i < 19; i++) {
    hf.f[i] = nullptr;
    if (fields[i] != 1) continue;
    if (i < 7) hf.f[i] = CELL(host[i]);
    else if (i < 13) hf.f[i] = VERT(host[i]);
    else if (i == 13 || i == 16) hf.f[i] = XF(host[i]);
    else if (i == 14 || i == 17) hf.f[i] = YF(host[i]);
    else hf.f[i] = ZF(host[i]);
  }
  launch_update_halo<F64>(g, c.stream, hf, fields, *depth, ext);
  check_launch("update_halo");
}

void clover_initialise_chunk_kernel(const int* x_min, const int* x_max, const int* y_min,
                                    const int* y_max, const int* z_min, const int* z_max,
                                    const double* xmin, const double* ymin, const double* zmin,
                                    const double* dx, const double* dy, const double* dz,
                                    double* vertexx, double* vertexdx, double* vertexy,
                                    double* vertexdy, double* vertexz, double* vertexdz,
                                    double* cellx, double* celldx, double* celly,
                                    double* celldy, double* cellz, double* celldz,
                                    double* volume, double* xarea, double* yarea,
                                    double* zarea) {
  ENTER();
  launch_initialise_chunk(g, c.stream, *xmin, *ymin, *zmin, *dx, *dy, *dz, VX(vertexx),
                          VX(vertexdx), VY(vertexy), VY(vertexdy), VZ(vertexz), VZ(vertexdz),
                          CX(cellx), CX(celldx), CY(celly), CY(celldy), CZ(cellz), CZ(celldz),
                          CELL(volume), XF(xarea), YF(yarea), ZF(zarea));
  check_launch("initialise_chunk");
}

void clover_generate_chunk_kernel(const int* x_min, const int* x_max, const int* y_min,
                                  const int* y_max, const int* z_min, const int* z_max,
                                  double* vertexx, double* vertexy, double* vertexz,
                                  double* cellx, double* celly, double* cellz,
                                  double* density0, double* energy0, double* xvel0,
                                  double* yvel0, double* zvel0, const int* number_of_states,
                                  const double* state_density, const double* state_energy,
                                  const double* state_xvel, const double* state_yvel,
                                  const double* state_zvel, const double* state_xmin,
                                  const double* state_xmax, const double* state_ymin,
                                  const double* state_ymax, const double* state_zmin,
                                  const double* state_zmax, const double* state_radius,
                                  const int* state_geometry, const int* g_rect,
                                  const int* g_circ, const int* g_point) {
  ENTER();
  if (*number_of_states < 1 || *number_of_states > 16) {
    set_error(CLOVER_STATUS_BAD_ARG, "generate_chunk supports 1..16 states");
    return;
  }
  StateTable st;
  st.n = *number_of_states;
  for (int i = 0; i < st.n; i++) {
    st.density[i] = state_density[i]; st.energy[i] = state_energy[i];
    st.xvel[i] = state_xvel[i]; st.yvel[i] = state_yvel[i]; st.zvel[i] = state_zvel[i];
    st.xmin[i] = state_xmin[i]; st.xmax[i] = state_xmax[i];
    st.ymin[i] = state_ymin[i]; st.ymax[i] = state_ymax[i];
    st.zmin[i] = state_zmin[i]; st.zmax[i] = state_zmax[i];
    st.radius[i] = state_radius[i];
    // map the caller's geometry codes onto 1 cuboid, 2 sphere, 3 point
    const int gc = state_geometry[i];
    st.geometry[i] = gc == *g_rect ? 1 : gc == *g_circ ? 2 : gc == *g_point ? 3 : 0;
  }
  GeomArrays ga = no_geom();
  ga.vertexx = VX(vertexx); ga.vertexy = VY(vertexy); ga.vertexz = VZ(vertexz);
  ga.cellx = CX(cellx); ga.celly = CY(celly); ga.cellz = CZ(cellz);
  launch_generate_chunk<F64>(g, c.stream, ga, CELL(density0), CELL(energy0), VERT(xvel0),
                             VERT(yvel0), VERT(zvel0), st);
  check_launch("generate_chunk");
}

int clover_gpu_status(void) { return ctx().status; }

const char* clover_gpu_error_string(void) { return ctx().err.c_str(); }

void clover_gpu_clear_status(void) {
  ctx().status = 0;
  ctx().err.clear();
}

void clover_gpu_sync_to_host(void) {
  Context& c = ctx();
  if (!c.ready) return;
  for (auto& kv : c.mirrors) {
    Mirror& m = kv.second;
    if (m.shape.one_d)
      check(cudaMemcpyAsync((void*)kv.first, m.dev, (size_t)m.shape.hx * 8,
                            cudaMemcpyDeviceToHost, c.stream), "download");
    else
      xfer3d(kv.first, m, 0, m.planes, false);
  }
  check(cudaStreamSynchronize(c.stream), "sync_to_host");
}

void clover_gpu_invalidate(const void* host_array) {
  Context& c = ctx();
  auto it = c.mirrors.find(host_array);
  if (it != c.mirrors.end()) it->second.planes = 0;
}

void clover_gpu_invalidate_all(void) {
  Context& c = ctx();
  for (auto& kv : c.mirrors) kv.second.planes = 0;
}

void clover_gpu_synchronize(void) {
  Context& c = ctx();
  if (c.ready) check(cudaStreamSynchronize(c.stream), "synchronize");
}

void clover_gpu_release(void) {
  Context& c = ctx();
  if (!c.ready) return;
  cudaStreamSynchronize(c.stream);
  for (auto& kv : c.mirrors) {
    if (kv.second.pinned) cudaHostUnregister((void*)kv.first);
    cudaFree(kv.second.raw);
  }
  c.mirrors.clear();
  cudaFree(c.d_key);
  cudaFree(c.d_partials);
  cudaFree(c.d_sum);
  cudaFree(c.stage);
  c.stage = nullptr;
  c.stage_bytes = 0;
  cudaStreamDestroy(c.stream);
  c.ready = false;
}

void clover_gpu_layout(const int* x_min, const int* x_max, const int* y_min, const int* y_max,
                       const int* z_min, const int* z_max, int* px, long long* pxy,
                       long long* elems) {
  const Geom g = make_geom(*x_min, *x_max, *y_min, *y_max, *z_min, *z_max);
  *px = g.px;
  *pxy = g.pxy;
  *elems = array_elems(g);
}

void clover_gpu_mirror_stats(int* arrays, long long* bytes) {
  Context& c = ctx();
  long long b = 0;
  for (auto& kv : c.mirrors)
    b += kv.second.shape.one_d ? (long long)(kv.second.shape.hx + 32) * 8
                               : (array_elems(c.g) + kFrontPad<double>) * 8;
  *arrays = (int)c.mirrors.size();
  *bytes = b;
}

}  // extern "C"
