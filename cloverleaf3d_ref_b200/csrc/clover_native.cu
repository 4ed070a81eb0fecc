// Native chunk: the whole hydro cycle resident in HBM, dt/time/step on the
// device, one step replayed from a CUDA graph (one graph per sweep order).
// Also the deck reader (parse.f90 + read_input.f90 semantics).
#include <cctype>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <vector>

#include "../../include/clover_b200.h"
#include "../../include/clover_kernels.h"
#include "clover_launch.h"

namespace clover {
namespace {

std::string g_last_error;

// data.f90:30-31 -- default-REAL literals assigned to REAL(8)
const double kGSmall = (double)1.0e-16f;
const double kGBig = (double)1.0e+21f;

// Device-resident step state.
struct DevScalars {
  double dt, dtold, time;
  unsigned long long key;
  int step;
  int status;
  int dt_cap;
  int pad;
};

__global__ void k_dt_prepare(DevScalars* sc, unsigned long long init) { sc->key = init; }

// timestep.f90:90-126 after the calc_dt reduction
__global__ void k_dt_finalize(DevScalars* sc, double* dt_hist, double dtrise, double dtmax,
                              double dtmin) {
  unsigned long long key = sc->key;
  unsigned long long b = (key >> 63) ? (key & 0x7fffffffffffffffull) : ~key;
  const double dtlp = __longlong_as_double((long long)b);
  double dt = kGBig;
  if (dtlp <= dt) dt = dtlp;
  double m = dt;
  const double r = sc->dtold * dtrise;
  if (r < m) m = r;
  if (dtmax < m) m = dtmax;
  dt = m;
  if (dt < dtmin) sc->status |= CLOVER_STATUS_SMALL_DT;
  sc->dt = dt;
  sc->dtold = dt;
  const int s = sc->step;
  if (s < sc->dt_cap) dt_hist[s] = dt;
  sc->step = s + 1;
}

// hydro.f90:68
__global__ void k_step_end(DevScalars* sc) { sc->time = sc->time + sc->dt; }

template <class T>
T* alloc_field(const Geom& g, std::vector<void*>& owned, long long& bytes, cudaStream_t s) {
  void* raw = nullptr;
  const size_t n = (size_t)(array_elems(g) + kFrontPad<T>) * sizeof(T);
  if (cudaMalloc(&raw, n) != cudaSuccess) return nullptr;
  cudaMemsetAsync(raw, 0, n, s);
  owned.push_back(raw);
  bytes += (long long)n;
  return (T*)raw + kFrontPad<T>;
}

double* alloc_1d(int n, std::vector<void*>& owned, long long& bytes, cudaStream_t s) {
  void* raw = nullptr;
  const size_t sz = (size_t)(n + 32) * sizeof(double);
  if (cudaMalloc(&raw, sz) != cudaSuccess) return nullptr;
  cudaMemsetAsync(raw, 0, sz, s);
  owned.push_back(raw);
  bytes += (long long)sz;
  return (double*)raw;
}

}  // namespace

struct ChunkBase {
  virtual ~ChunkBase() {}
};

template <class S>
struct Chunk : ChunkBase {
  using R = typename S::rho_t;
  using En = typename S::ene_t;
  using C = typename S::cs_t;
  using V = typename S::vel_t;
  using VF = typename S::vf_t;
  using MF = typename S::mf_t;
  using W = typename S::wk_t;

  clover_deck deck;
  Geom g;
  cudaStream_t stream = nullptr;
  std::vector<void*> owned;
  long long bytes = 0;

  R *density0, *density1;
  En *energy0, *energy1;
  C *pressure, *viscosity, *soundspeed;
  V *xvel0, *xvel1, *yvel0, *yvel1, *zvel0, *zvel1;
  V* vel1b[3];  // second buffer of each time-level-1 velocity (fused step)
  VF *vol_flux_x, *vol_flux_y, *vol_flux_z;
  MF *mass_flux_x, *mass_flux_y, *mass_flux_z;
  W* work[7];
  double *volume, *xarea, *yarea, *zarea;
  double *cellx, *celly, *cellz, *celldx, *celldy, *celldz;
  double *vertexx, *vertexy, *vertexz, *vertexdx, *vertexdy, *vertexdz;
  GeomArrays ga;

  DevScalars* sc = nullptr;
  double* dt_hist = nullptr;
  int dt_cap = 0;
  double* sum_hist = nullptr;
  int sum_cap = 0;
  std::vector<int> sum_steps;  // host: step of each recorded summary
  double* partials = nullptr;

  double cell_volume = 0.0;  // dx*dy*dz, the volume of every cell (initialise_chunk)
  int host_step = 0;     // steps enqueued
  bool advect_x = true;  // start.f90:99
  bool use_graphs = true;
  bool fused = true;  // fused kernels (clover_fused.cu) instead of one kernel per reference pass
  cudaGraphExec_t graph[2] = {nullptr, nullptr};
  int launches_per_step = 0;
  int ext[6] = {1, 1, 1, 1, 1, 1};

  // Per-kernel-group timing with events on the chunk stream (profile mode,
  // direct launches only). bytes = algorithmic bytes of the group's launch:
  // distinct 3D arrays read + written over the cells it covers.
  struct ProfRec { const char* name; cudaEvent_t a, b; double bytes; };
  struct ProfAcc { std::string name; double ms = 0, bytes = 0; int launches = 0; };
  bool profile = false;
  std::vector<ProfRec> prof_pending;
  std::vector<cudaEvent_t> ev_pool;
  std::vector<ProfAcc> prof_acc;
  cudaEvent_t cur_a = nullptr;

  cudaEvent_t get_event() {
    if (!ev_pool.empty()) { cudaEvent_t e = ev_pool.back(); ev_pool.pop_back(); return e; }
    cudaEvent_t e;
    cudaEventCreate(&e);
    return e;
  }
  void pbeg() {
    if (!profile) return;
    cur_a = get_event();
    cudaEventRecord(cur_a, stream);
  }
  void pend(const char* name, double bytes) {
    if (!profile) return;
    cudaEvent_t b = get_event();
    cudaEventRecord(b, stream);
    prof_pending.push_back(ProfRec{name, cur_a, b, bytes});
  }
  void prof_collect() {
    cudaStreamSynchronize(stream);
    for (auto& r : prof_pending) {
      float ms = 0;
      cudaEventElapsedTime(&ms, r.a, r.b);
      ProfAcc* acc = nullptr;
      for (auto& x : prof_acc) if (x.name == r.name) acc = &x;
      if (!acc) { prof_acc.push_back(ProfAcc{r.name}); acc = &prof_acc.back(); }
      acc->ms += ms;
      acc->bytes += r.bytes;
      acc->launches += 1;
      ev_pool.push_back(r.a);
      ev_pool.push_back(r.b);
    }
    prof_pending.clear();
  }
  double cells() const {
    return (double)(g.x_max - g.x_min + 1) * (g.y_max - g.y_min + 1) * (g.z_max - g.z_min + 1);
  }

  // time-level-1 velocity c (0 x, 1 y, 2 z) in buffer b of its pair
  V* vel1(int c, int b) const {
    V* a[3] = {xvel1, yvel1, zvel1};
    return b ? vel1b[c] : a[c];
  }
  // the buffer holding time level 1 velocities after `steps` fused steps:
  // each step flips the pair three times (one per sweep)
  int vel1_buffer(int steps) const { return fused ? steps % 2 : 0; }

  HaloFields halo_fields(int vb) {
    HaloFields h;
    void* f[19] = {density0, density1, energy0, energy1, pressure, viscosity, soundspeed,
                   xvel0, vel1(0, vb), yvel0, vel1(1, vb), zvel0, vel1(2, vb), vol_flux_x,
                   vol_flux_y, vol_flux_z, mass_flux_x, mass_flux_y, mass_flux_z};
    for (int i = 0; i < 19; i++) h.f[i] = f[i];
    return h;
  }

  void halo(std::initializer_list<int> ids, int depth, int vb = 0) {
    int fields[19] = {0};
    for (int id : ids) fields[id - 1] = 1;
    launch_update_halo<S>(g, stream, halo_fields(vb), fields, depth, ext);
  }

  bool create(const clover_deck& d) {
    deck = d;
    g = make_geom(1, d.x_cells, 1, d.y_cells, 1, d.z_cells);
    if (cudaStreamCreateWithFlags(&stream, cudaStreamNonBlocking) != cudaSuccess) return false;
    bool ok = true;
    auto chk = [&](const void* p) { ok = ok && p != nullptr; };
    chk(density0 = alloc_field<R>(g, owned, bytes, stream));
    chk(density1 = alloc_field<R>(g, owned, bytes, stream));
    chk(energy0 = alloc_field<En>(g, owned, bytes, stream));
    chk(energy1 = alloc_field<En>(g, owned, bytes, stream));
    chk(pressure = alloc_field<C>(g, owned, bytes, stream));
    chk(viscosity = alloc_field<C>(g, owned, bytes, stream));
    chk(soundspeed = alloc_field<C>(g, owned, bytes, stream));
    chk(xvel0 = alloc_field<V>(g, owned, bytes, stream));
    chk(xvel1 = alloc_field<V>(g, owned, bytes, stream));
    chk(yvel0 = alloc_field<V>(g, owned, bytes, stream));
    chk(yvel1 = alloc_field<V>(g, owned, bytes, stream));
    chk(zvel0 = alloc_field<V>(g, owned, bytes, stream));
    chk(zvel1 = alloc_field<V>(g, owned, bytes, stream));
    for (int c3 = 0; c3 < 3; c3++) chk(vel1b[c3] = alloc_field<V>(g, owned, bytes, stream));
    chk(vol_flux_x = alloc_field<VF>(g, owned, bytes, stream));
    chk(vol_flux_y = alloc_field<VF>(g, owned, bytes, stream));
    chk(vol_flux_z = alloc_field<VF>(g, owned, bytes, stream));
    chk(mass_flux_x = alloc_field<MF>(g, owned, bytes, stream));
    chk(mass_flux_y = alloc_field<MF>(g, owned, bytes, stream));
    chk(mass_flux_z = alloc_field<MF>(g, owned, bytes, stream));
    for (int i = 0; i < 7; i++) chk(work[i] = alloc_field<W>(g, owned, bytes, stream));
    chk(volume = alloc_field<double>(g, owned, bytes, stream));
    chk(xarea = alloc_field<double>(g, owned, bytes, stream));
    chk(yarea = alloc_field<double>(g, owned, bytes, stream));
    chk(zarea = alloc_field<double>(g, owned, bytes, stream));
    const int nx = d.x_cells, ny = d.y_cells, nz = d.z_cells;
    chk(cellx = alloc_1d(nx + 4, owned, bytes, stream));
    chk(celly = alloc_1d(ny + 4, owned, bytes, stream));
    chk(cellz = alloc_1d(nz + 4, owned, bytes, stream));
    chk(celldx = alloc_1d(nx + 4, owned, bytes, stream));
    chk(celldy = alloc_1d(ny + 4, owned, bytes, stream));
    chk(celldz = alloc_1d(nz + 4, owned, bytes, stream));
    chk(vertexx = alloc_1d(nx + 5, owned, bytes, stream));
    chk(vertexy = alloc_1d(ny + 5, owned, bytes, stream));
    chk(vertexz = alloc_1d(nz + 5, owned, bytes, stream));
    chk(vertexdx = alloc_1d(nx + 5, owned, bytes, stream));
    chk(vertexdy = alloc_1d(ny + 5, owned, bytes, stream));
    chk(vertexdz = alloc_1d(nz + 5, owned, bytes, stream));
    if (!ok) {
      g_last_error = "device allocation failed";
      return false;
    }
    ga = GeomArrays{volume, xarea, yarea, zarea, cellx, celly, cellz, celldx, celldy, celldz,
                    vertexx, vertexy, vertexz, vertexdx, vertexdy, vertexdz};

    dt_cap = d.end_step < (1 << 22) ? d.end_step + 16 : (1 << 22);
    sum_cap = dt_cap / (d.summary_frequency > 0 ? d.summary_frequency : dt_cap) + 8;
    void* p = nullptr;
    ok = cudaMalloc(&p, sizeof(DevScalars)) == cudaSuccess;
    sc = (DevScalars*)p;
    ok = ok && cudaMalloc(&p, (size_t)dt_cap * sizeof(double)) == cudaSuccess;
    dt_hist = (double*)p;
    ok = ok && cudaMalloc(&p, (size_t)sum_cap * 5 * sizeof(double)) == cudaSuccess;
    sum_hist = (double*)p;
    ok = ok && cudaMalloc(&p, (size_t)summary_partials_len() * sizeof(double)) == cudaSuccess;
    partials = (double*)p;
    if (!ok) {
      g_last_error = "device allocation failed";
      return false;
    }
    DevScalars h{};
    h.dt = d.initial_timestep;     // start.f90:51-52
    h.dtold = d.initial_timestep;
    h.time = 0.0;
    h.step = 0;
    h.dt_cap = dt_cap;
    cudaMemcpyAsync(sc, &h, sizeof(h), cudaMemcpyHostToDevice, stream);

    // initialise_chunk.f90:38-46
    const double dx = (d.xmax - d.xmin) / (double)(float)d.x_cells;
    const double dy = (d.ymax - d.ymin) / (double)(float)d.y_cells;
    const double dz = (d.zmax - d.zmin) / (double)(float)d.z_cells;
    const double xmin = d.xmin + dx * (double)(float)0;
    const double ymin = d.ymin + dy * (double)(float)0;
    const double zmin = d.zmin + dz * (double)(float)0;
    cell_volume = dx * dy * dz;  // initialise_chunk_kernel.f90:155
    launch_initialise_chunk(g, stream, xmin, ymin, zmin, dx, dy, dz, vertexx, vertexdx, vertexy,
                            vertexdy, vertexz, vertexdz, cellx, celldx, celly, celldy, cellz,
                            celldz, volume, xarea, yarea, zarea);
    // read_input.f90:293-303 nudge, then generate_chunk
    StateTable st;
    st.n = d.number_of_states;
    for (int i = 0; i < st.n; i++) {
      st.density[i] = d.state_density[i]; st.energy[i] = d.state_energy[i];
      st.xvel[i] = d.state_xvel[i]; st.yvel[i] = d.state_yvel[i]; st.zvel[i] = d.state_zvel[i];
      st.xmin[i] = d.state_xmin[i]; st.xmax[i] = d.state_xmax[i];
      st.ymin[i] = d.state_ymin[i]; st.ymax[i] = d.state_ymax[i];
      st.zmin[i] = d.state_zmin[i]; st.zmax[i] = d.state_zmax[i];
      st.radius[i] = d.state_radius[i];
      st.geometry[i] = d.state_geometry[i];
      if (i >= 1) {
        st.xmin[i] = st.xmin[i] + (dx / 100.0);
        st.ymin[i] = st.ymin[i] + (dy / 100.0);
        st.zmin[i] = st.zmin[i] + (dz / 100.0);
        st.xmax[i] = st.xmax[i] - (dx / 100.0);
        st.ymax[i] = st.ymax[i] - (dy / 100.0);
        st.zmax[i] = st.zmax[i] - (dz / 100.0);
      }
    }
    launch_generate_chunk<S>(g, stream, ga, density0, energy0, xvel0, yvel0, zvel0, st);
    // start.f90:109-136
    launch_ideal_gas<S>(g, stream, density0, energy0, pressure, soundspeed);
    halo({1, 3, 5, 6, 2, 4, 8, 10, 12, 9, 11, 13}, 2);
    summary(0);
    if (cudaStreamSynchronize(stream) != cudaSuccess || cudaGetLastError() != cudaSuccess) {
      g_last_error = "chunk set-up failed on the device";
      return false;
    }
    return true;
  }

  // field_summary.f90:55-108, recorded at the given step
  void summary(int step) {
    const int idx = (int)sum_steps.size();
    if (idx >= sum_cap) return;
    pbeg();
    launch_ideal_gas<S>(g, stream, density0, energy0, pressure, soundspeed);
    launch_field_summary<S>(g, stream, volume, density0, energy0, pressure, xvel0, yvel0, zvel0,
                            partials, sum_hist + 5 * idx);
    pend("field_summary", cells() * (2 * sizeof(R) + 2 * sizeof(En) + 3 * sizeof(C) +
                                     sizeof(double) + 3 * sizeof(V)));
    sum_steps.push_back(step);
  }

  // One hydro step with the fused kernels (same results, bit for bit).
  void enqueue_step_fused(bool ax) {
    const double* dtp = &sc->dt;
    const double n = cells();
    const double R8 = sizeof(R), E8 = sizeof(En), C8 = sizeof(C), V8 = sizeof(V),
                 VF8 = sizeof(VF), MF8 = sizeof(MF), W8 = sizeof(W), G8 = sizeof(double);
    int vc = ax ? 0 : 1;  // buffer of the velocity pairs at the start of this step
    // timestep.f90:56-126
    k_dt_prepare<<<1, 1, 0, stream>>>(sc, min_key_of(kGBig));
    pbeg();
    launch_ideal_gas<S>(g, stream, density0, energy0, pressure, soundspeed);
    pend("ideal_gas", n * (R8 + E8 + 2 * C8));
    pbeg();
    halo({5, 3, 1, 8, 10}, 1, vc);
    pend("update_halo", 0);
    pbeg();
    launch_timestep_visc<S>(g, stream, ga, density0, pressure, viscosity, xvel0, yvel0, zvel0);
    pend("viscosity", n * (3 * V8 + 3 * G8 + C8));
    pbeg();
    halo({6}, 1, vc);
    pend("update_halo", 0);
    pbeg();
    launch_calc_dt<S>(g, stream, ga, kGSmall, deck.dtc_safe, deck.dtu_safe, deck.dtv_safe,
                      deck.dtw_safe, deck.dtdiv_safe, density0, viscosity, soundspeed, xvel0,
                      yvel0, zvel0, (W*)nullptr, &sc->key);
    k_dt_finalize<<<1, 1, 0, stream>>>(sc, dt_hist, deck.timestep_rise, deck.max_timestep,
                                       deck.dtmin);
    pend("calc_dt", n * (4 * G8 + R8 + 2 * C8 + 3 * V8));
    // PdV.f90:50-107: predictor + EOS on the predicted state; revert is implied
    pbeg();
    launch_pdv_predict_eos<S>(g, stream, dtp, ga, density0, energy0, pressure, viscosity, xvel0,
                              yvel0, zvel0);
    pend("pdv", n * (4 * G8 + R8 + E8 + 3 * C8 + 3 * V8));
    pbeg();
    halo({5}, 1, vc);
    pend("update_halo", 0);
    pbeg();
    launch_accelerate<S>(g, stream, 0.0, dtp, ga, density0, pressure, viscosity, xvel0, yvel0,
                         zvel0, vel1(0, vc), vel1(1, vc), vel1(2, vc));
    pend("accelerate", n * (4 * G8 + R8 + 2 * C8 + 6 * V8));
    pbeg();
    launch_pdv_flux<S>(g, stream, dtp, ga, density0, density1, energy0, energy1, pressure,
                       viscosity, xvel0, vel1(0, vc), yvel0, vel1(1, vc), zvel0, vel1(2, vc),
                       vol_flux_x, vol_flux_y, vol_flux_z);
    pend("pdv_flux", n * (4 * G8 + 2 * R8 + 2 * E8 + 2 * C8 + 6 * V8 + 3 * VF8));
    // advection.f90:43-179
    const int axi = ax ? 1 : 0;
    auto sweep = [&](int sweep_number, int dir, bool pre_halo) {
      if (pre_halo) {
        pbeg();
        halo({4, 2, 14, 15, 16}, 2, vc);
        pend("update_halo", 0);
      }
      // volume fluxes read for pre_vol: all three on sweep 1, two on the y sweep,
      // the sweep direction only on sweep 3
      const double nvf = sweep_number == 1 ? 3 : sweep_number == 2 ? 2 : 1;
      pbeg();
      launch_advec_cell_fused<S>(g, stream, axi, dir, sweep_number, ga, density1, energy1,
                                 mass_flux_x, vol_flux_x, mass_flux_y, vol_flux_y, mass_flux_z,
                                 vol_flux_z, work[6]);
      // x: face pass + update pass; y, z: one marching pass (in place)
      if (dir == 1)
        pend("advec_cell_x", n * ((G8 + nvf * VF8 + R8 + E8 + MF8 + W8) +
                                  (G8 + nvf * VF8 + 2 * R8 + 2 * E8 + MF8 + W8)));
      else
        pend("advec_cell_yz", n * (G8 + nvf * VF8 + 2 * R8 + 2 * E8 + MF8));
      pbeg();
      halo({2, 4, 9, 11, 13, 17, 18, 19}, 2, vc);
      pend("update_halo", 0);
      // post_vol reads two volume fluxes on sweep 1, one on sweep 2, none on sweep 3
      const double npv = sweep_number == 1 ? 2 : sweep_number == 2 ? 1 : 0;
      V* vin[3] = {vel1(0, vc), vel1(1, vc), vel1(2, vc)};
      V* vout[3] = {vel1(0, vc ^ 1), vel1(1, vc ^ 1), vel1(2, vc ^ 1)};
      pbeg();
      launch_advec_mom_fused<S>(g, stream, axi, sweep_number, dir, cell_volume, ga, density1, mass_flux_x,
                                mass_flux_y, mass_flux_z, vol_flux_x, vol_flux_y, vol_flux_z,
                                work[0], work[1], work[2], vin, vout);
      // x: node pass + velocity pass; y, z: one marching pass
      if (dir == 1)  // one pass
        pend("advec_mom_x", n * (MF8 + R8 + G8 + npv * VF8 + 6 * V8));
      else  // node pass + velocity pass
        pend("advec_mom_yz", n * ((MF8 + R8 + G8 + npv * VF8 + 3 * W8) + (3 * W8 + 6 * V8)));
      vc ^= 1;
    };
    sweep(1, ax ? 1 : 3, true);
    sweep(2, 2, true);
    sweep(3, ax ? 3 : 1, false);
    pbeg();
    launch_reset_field<S>(g, stream, density0, density1, energy0, energy1, xvel0, vel1(0, vc),
                          yvel0, vel1(1, vc), zvel0, vel1(2, vc));
    pend("reset_field", n * (2 * R8 + 2 * E8 + 6 * V8));
    k_step_end<<<1, 1, 0, stream>>>(sc);
  }

  // One hydro step, hydro.f90:52-68 (timestep .. time = time + dt).
  void enqueue_step(bool ax) {
    if (fused) {
      enqueue_step_fused(ax);
      return;
    }
    const double* dtp = &sc->dt;
    const double n = cells();
    const double R8 = sizeof(R), E8 = sizeof(En), C8 = sizeof(C), V8 = sizeof(V),
                 VF8 = sizeof(VF), MF8 = sizeof(MF), W8 = sizeof(W), G8 = sizeof(double);
    // timestep.f90:56-126
    k_dt_prepare<<<1, 1, 0, stream>>>(sc, min_key_of(kGBig));
    pbeg();
    launch_ideal_gas<S>(g, stream, density0, energy0, pressure, soundspeed);
    pend("ideal_gas", n * (R8 + E8 + 2 * C8));
    pbeg();
    halo({5, 3, 1, 8, 10}, 1);
    pend("update_halo", 0);
    pbeg();
    launch_viscosity<S>(g, stream, ga, density0, pressure, viscosity, xvel0, yvel0, zvel0);
    pend("viscosity", n * (3 * G8 + R8 + 2 * C8 + 3 * V8));
    pbeg();
    halo({6}, 1);
    pend("update_halo", 0);
    pbeg();
    launch_calc_dt<S>(g, stream, ga, kGSmall, deck.dtc_safe, deck.dtu_safe, deck.dtv_safe,
                      deck.dtw_safe, deck.dtdiv_safe, density0, viscosity, soundspeed, xvel0,
                      yvel0, zvel0, (W*)nullptr, &sc->key);
    k_dt_finalize<<<1, 1, 0, stream>>>(sc, dt_hist, deck.timestep_rise, deck.max_timestep,
                                       deck.dtmin);
    pend("calc_dt", n * (4 * G8 + R8 + 2 * C8 + 3 * V8));
    // PdV.f90:50-107 (predictor), accelerate, PdV (corrector), flux_calc
    pbeg();
    launch_pdv<S>(g, stream, 1, 0.0, dtp, ga, density0, density1, energy0, energy1, pressure,
                  viscosity, xvel0, xvel1, yvel0, yvel1, zvel0, zvel1);
    pend("pdv", n * (4 * G8 + 2 * R8 + 2 * E8 + 2 * C8 + 3 * V8));
    pbeg();
    launch_ideal_gas<S>(g, stream, density1, energy1, pressure, soundspeed);
    pend("ideal_gas", n * (R8 + E8 + 2 * C8));
    pbeg();
    halo({5}, 1);
    pend("update_halo", 0);
    pbeg();
    launch_revert<S>(g, stream, density0, density1, energy0, energy1);
    pend("revert", n * (2 * R8 + 2 * E8));
    pbeg();
    launch_accelerate<S>(g, stream, 0.0, dtp, ga, density0, pressure, viscosity, xvel0, yvel0,
                         zvel0, xvel1, yvel1, zvel1);
    pend("accelerate", n * (4 * G8 + R8 + 2 * C8 + 6 * V8));
    pbeg();
    launch_pdv<S>(g, stream, 0, 0.0, dtp, ga, density0, density1, energy0, energy1, pressure,
                  viscosity, xvel0, xvel1, yvel0, yvel1, zvel0, zvel1);
    pend("pdv", n * (4 * G8 + 2 * R8 + 2 * E8 + 2 * C8 + 6 * V8));
    pbeg();
    launch_flux_calc<S>(g, stream, 0.0, dtp, ga, xvel0, yvel0, zvel0, xvel1, yvel1, zvel1,
                        vol_flux_x, vol_flux_y, vol_flux_z);
    pend("flux_calc", n * (3 * G8 + 6 * V8 + 3 * VF8));
    // advection.f90:43-179
    const int axi = ax ? 1 : 0;
    V* vel[3] = {xvel1, yvel1, zvel1};
    auto sweep = [&](int sweep_number, int dir, bool pre_halo) {
      if (pre_halo) {
        pbeg();
        halo({4, 2, 14, 15, 16}, 2);
        pend("update_halo", 0);
      }
      pbeg();
      launch_advec_cell<S>(g, stream, axi, dir, sweep_number, ga, density1, energy1,
                           mass_flux_x, vol_flux_x, mass_flux_y, vol_flux_y, mass_flux_z,
                           vol_flux_z, work);
      // volumes: volume + 3 fluxes -> pre, post; flux: vf, rho1, e1, pre -> mf, ener_flux;
      // update: rho1, e1, pre, mf, ener_flux, vf -> pre_mass, post_mass, post_ener,
      // advec_vol, rho1, e1
      pend("advec_cell", n * ((G8 + 3 * VF8 + 2 * W8) + (VF8 + R8 + E8 + W8 + MF8 + W8) +
                              (R8 + E8 + W8 + MF8 + W8 + VF8 + 4 * W8 + R8 + E8)));
      pbeg();
      halo({2, 4, 9, 11, 13, 17, 18, 19}, 2);
      pend("update_halo", 0);
      for (int v = 1; v <= 3; v++) {
        pbeg();
        launch_advec_mom<S>(g, stream, vel[v - 1], mass_flux_x, vol_flux_x, mass_flux_y,
                            vol_flux_y, mass_flux_z, vol_flux_z, ga, density1, work, axi, v,
                            sweep_number, dir);
        // volumes (6) + [node flux/mass (5) + node_mass_pre (3) when v == 1] +
        // mom_flux (4) + velocity update (5)
        double b = (G8 + 3 * VF8 + 2 * W8) + (2 * V8 + 2 * W8) + (2 * V8 + 3 * W8);
        if (v == 1) b += (MF8 + R8 + 3 * W8) + 3 * W8;
        pend("advec_mom", n * b);
      }
    };
    sweep(1, ax ? 1 : 3, true);
    sweep(2, 2, true);
    sweep(3, ax ? 3 : 1, false);
    pbeg();
    launch_reset_field<S>(g, stream, density0, density1, energy0, energy1, xvel0, xvel1, yvel0,
                          yvel1, zvel0, zvel1);
    pend("reset_field", n * (2 * R8 + 2 * E8 + 6 * V8));
    k_step_end<<<1, 1, 0, stream>>>(sc);
  }

  bool capture_graphs() {
    for (int i = 0; i < 2; i++) {
      if (graph[i]) continue;
      cudaGraph_t gr;
      if (cudaStreamBeginCapture(stream, cudaStreamCaptureModeThreadLocal) != cudaSuccess)
        return false;
      const bool prof = profile;
      profile = false;
      enqueue_step(i == 0);
      profile = prof;
      if (cudaStreamEndCapture(stream, &gr) != cudaSuccess) return false;
      size_t n = 0;
      cudaGraphGetNodes(gr, nullptr, &n);
      launches_per_step = (int)n;
      if (cudaGraphInstantiate(&graph[i], gr, 0) != cudaSuccess) return false;
      cudaGraphDestroy(gr);
    }
    return true;
  }

  int step(int n) {
    const bool graphs = use_graphs && !profile;
    if (graphs && !capture_graphs()) {
      cudaGetLastError();
      use_graphs = false;
    }
    for (int i = 0; i < n; i++) {
      if (graphs && use_graphs)
        cudaGraphLaunch(graph[advect_x ? 0 : 1], stream);
      else
        enqueue_step(advect_x);
      advect_x = !advect_x;
      host_step++;
      if (deck.summary_frequency != 0 && host_step % deck.summary_frequency == 0)
        summary(host_step);
    }
    return cudaGetLastError() == cudaSuccess ? 0 : -1;
  }

  DevScalars scalars() {
    DevScalars h{};
    cudaMemcpyAsync(&h, sc, sizeof(h), cudaMemcpyDeviceToHost, stream);
    cudaStreamSynchronize(stream);
    return h;
  }

  // hydro.f90:46-98 with the end test; runs in batches that cannot overshoot
  // end_time, since dt <= max_timestep.
  int run() {
    for (;;) {
      DevScalars h = scalars();
      if (h.status & CLOVER_STATUS_SMALL_DT) return -host_step;
      if (host_step > 0 && (h.time + kGSmall > deck.end_time || host_step >= deck.end_step)) {
        summary(host_step);  // the final summary (hydro.f90:87)
        cudaStreamSynchronize(stream);
        return host_step;
      }
      int batch = deck.end_step - host_step;
      const double room = deck.end_time - kGSmall - h.time;
      const int safe = (int)std::floor(room / deck.max_timestep) - 1;
      if (safe < batch) batch = safe;
      if (batch < 1) batch = 1;
      if (step(batch) != 0) return -1000000000;
    }
  }

  int read_field(int id, double* host, bool write) {
    if (id < 1 || id > 19) return -1;
    const int vb = vel1_buffer(host_step);
    void* f[19] = {density0, density1, energy0, energy1, pressure, viscosity, soundspeed,
                   xvel0, vel1(0, vb), yvel0, vel1(1, vb), zvel0, vel1(2, vb), vol_flux_x,
                   vol_flux_y, vol_flux_z, mass_flux_x, mass_flux_y, mass_flux_z};
    const int eb[19] = {(int)sizeof(R), (int)sizeof(R), (int)sizeof(En), (int)sizeof(En),
                        (int)sizeof(C), (int)sizeof(C), (int)sizeof(C), (int)sizeof(V),
                        (int)sizeof(V), (int)sizeof(V), (int)sizeof(V), (int)sizeof(V),
                        (int)sizeof(V), (int)sizeof(VF), (int)sizeof(VF), (int)sizeof(VF),
                        (int)sizeof(MF), (int)sizeof(MF), (int)sizeof(MF)};
    const int nx = g.x_max - g.x_min + 1, ny = g.y_max - g.y_min + 1, nz = g.z_max - g.z_min + 1;
    int hx = nx + 4, hy = ny + 4, hz = nz + 4;
    if (id >= 8 && id <= 13) { hx = nx + 5; hy = ny + 5; hz = nz + 5; }
    if (id == 14 || id == 17) hx = nx + 5;
    if (id == 15 || id == 18) hy = ny + 5;
    if (id == 16 || id == 19) hz = nz + 5;
    const int e = eb[id - 1];
    std::vector<char> stage((size_t)hx * hy * hz * e);
    cudaMemcpy3DParms q = {};
    cudaPitchedPtr hp = make_cudaPitchedPtr(stage.data(), (size_t)hx * e, (size_t)hx * e, hy);
    cudaPitchedPtr dp = make_cudaPitchedPtr(f[id - 1], (size_t)g.px * e, (size_t)hx * e,
                                            (size_t)(g.pxy / g.px));
    q.extent = make_cudaExtent((size_t)hx * e, hy, hz);
    if (write) {
      for (size_t i = 0; i < (size_t)hx * hy * hz; i++) {
        if (e == 8) ((double*)stage.data())[i] = host[i];
        else ((float*)stage.data())[i] = (float)host[i];
      }
      q.srcPtr = hp; q.dstPtr = dp; q.kind = cudaMemcpyHostToDevice;
    } else {
      q.srcPtr = dp; q.dstPtr = hp; q.kind = cudaMemcpyDeviceToHost;
    }
    if (cudaMemcpy3DAsync(&q, stream) != cudaSuccess) return -1;
    if (cudaStreamSynchronize(stream) != cudaSuccess) return -1;
    if (!write)
      for (size_t i = 0; i < (size_t)hx * hy * hz; i++)
        host[i] = e == 8 ? ((double*)stage.data())[i] : (double)((float*)stage.data())[i];
    return 0;
  }

  ~Chunk() {
    if (stream) cudaStreamSynchronize(stream);
    prof_collect();
    for (auto e : ev_pool) cudaEventDestroy(e);
    for (int i = 0; i < 2; i++)
      if (graph[i]) cudaGraphExecDestroy(graph[i]);
    for (void* p : owned) cudaFree(p);
    cudaFree(sc);
    cudaFree(dt_hist);
    cudaFree(sum_hist);
    cudaFree(partials);
    if (stream) cudaStreamDestroy(stream);
  }
};

}  // namespace clover

using namespace clover;

struct clover_chunk {
  int precision;
  Chunk<F64>* f64 = nullptr;
  Chunk<F32Mixed>* mixed = nullptr;
};

#define DISPATCH(c, expr) ((c)->f64 ? (c)->f64->expr : (c)->mixed->expr)

// ---------------------------------------------------------------------------
// Deck reader: parse.f90:118-379 + read_input.f90:38-277
namespace {

std::vector<std::string> deck_lines(const char* text) {
  // parse_getline: control characters to blanks, '!' and ';' start comments,
  // lower case, '=' and ',' are blanks; only lines inside *clover..*endclover.
  std::vector<std::string> out;
  std::string cur;
  bool inside = false;
  const char* p = text;
  while (true) {
    const char ch = *p;
    if (ch == '\n' || ch == '\0') {
      std::string l = cur;
      cur.clear();
      for (auto& x : l)
        if ((unsigned char)x < 32 || (unsigned char)x > 128) x = ' ';
      size_t s = l.find('!');
      if (s != std::string::npos) l = l.substr(0, s);
      s = l.find(';');
      if (s != std::string::npos) l = l.substr(0, s);
      for (auto& x : l) {
        x = (char)std::tolower((unsigned char)x);
        if (x == '=' || x == ',') x = ' ';
      }
      size_t b = l.find_first_not_of(' ');
      l = b == std::string::npos ? std::string() : l.substr(b);
      if (!l.empty() && l[0] == '*') {
        std::string word = l.substr(0, l.find(' '));
        if (word == "*clover") inside = true;
        else if (word == "*endclover") inside = false;
      } else if (inside && !l.empty()) {
        out.push_back(l);
      }
      if (ch == '\0') break;
    } else {
      cur.push_back(ch);
    }
    p++;
  }
  return out;
}

std::vector<std::string> split(const std::string& l) {
  std::vector<std::string> w;
  size_t i = 0;
  while (i < l.size()) {
    while (i < l.size() && l[i] == ' ') i++;
    size_t j = i;
    while (j < l.size() && l[j] != ' ') j++;
    if (j > i) w.push_back(l.substr(i, j - i));
    i = j;
  }
  return w;
}

// parse_getrval: an integer word gains '.0'; Fortran list-directed read
bool to_real(std::string w, double* v) {
  for (auto& x : w)
    if (x == 'd') x = 'e';
  char* end = nullptr;
  *v = strtod(w.c_str(), &end);
  return end && *end == '\0' && !w.empty();
}

// parse_getival: READ(word,'(I7)') reads the first 7 characters
bool to_int(const std::string& w, int* v) {
  std::string s = w.substr(0, 7);
  char* end = nullptr;
  long x = strtol(s.c_str(), &end, 10);
  if (!end || *end != '\0' || s.empty()) return false;
  *v = (int)x;
  return true;
}

}  // namespace

extern "C" {

void clover_deck_defaults(clover_deck* d) {
  memset(d, 0, sizeof(*d));
  d->xmin = 0.0; d->ymin = 0.0; d->zmin = 0.0;
  d->xmax = 100.0; d->ymax = 100.0; d->zmax = 100.0;
  d->x_cells = 10; d->y_cells = 10; d->z_cells = 10;
  d->end_time = 10.0;
  d->end_step = 640000;  // g_ibig
  d->visit_frequency = 0;
  d->summary_frequency = 10;
  d->tiles_per_chunk = 1;
  d->initial_timestep = 0.1;
  d->max_timestep = 1.0;
  d->dtmin = 0.0000001;
  d->timestep_rise = 1.05;
  d->dtc_safe = 0.75;
  d->dtu_safe = 0.5;
  d->dtv_safe = 0.5;
  d->dtw_safe = 0.5;
  d->dtdiv_safe = 0.5;
  for (int i = 0; i < CLOVER_MAX_STATES; i++) d->state_geometry[i] = 1;
}

int clover_deck_parse(const char* text, clover_deck* d, char* err, int errlen) {
  auto fail = [&](int code, const char* msg) {
    if (err && errlen > 0) snprintf(err, (size_t)errlen, "%s", msg);
    return code;
  };
  clover_deck_defaults(d);
  std::vector<std::string> words;
  std::vector<std::vector<std::string>> lines;
  for (auto& l : deck_lines(text)) lines.push_back(split(l));
  // first pass: number of states = largest state index (read_input.f90:112-123)
  int state_max = 0;
  for (auto& w : lines)
    for (size_t i = 0; i < w.size(); i++)
      if (w[i] == "state" && i + 1 < w.size()) {
        int s = 0;
        if (!to_int(w[i + 1], &s)) return fail(3, "bad state number");
        if (s > state_max) state_max = s;
        break;
      }
  if (state_max < 1) return fail(1, "No states defined.");
  if (state_max > CLOVER_MAX_STATES) return fail(4, "too many states");
  d->number_of_states = state_max;
  // flatten the words so a value may sit on the next line (parse_getword(.TRUE.))
  struct Tok { std::string w; int line; };
  std::vector<Tok> toks;
  for (size_t li = 0; li < lines.size(); li++)
    for (auto& w : lines[li]) toks.push_back({w, (int)li});
  size_t i = 0;
  auto next_val = [&](std::string* out) {
    if (i + 1 >= toks.size()) return false;
    *out = toks[++i].w;
    return true;
  };
  while (i < toks.size()) {
    const std::string& w = toks[i].w;
    std::string v;
    double r;
    int n;
    auto real_key = [&](double* dst) {
      if (!next_val(&v) || !to_real(v, &r)) return false;
      *dst = r;
      return true;
    };
    auto int_key = [&](int* dst) {
      if (!next_val(&v) || !to_int(v, &n)) return false;
      *dst = n;
      return true;
    };
    bool ok = true;
    if (w == "initial_timestep") ok = real_key(&d->initial_timestep);
    else if (w == "max_timestep") ok = real_key(&d->max_timestep);
    else if (w == "timestep_rise") ok = real_key(&d->timestep_rise);
    else if (w == "end_time") ok = real_key(&d->end_time);
    else if (w == "end_step") ok = int_key(&d->end_step);
    else if (w == "xmin") ok = real_key(&d->xmin);
    else if (w == "xmax") ok = real_key(&d->xmax);
    else if (w == "ymin") ok = real_key(&d->ymin);
    else if (w == "ymax") ok = real_key(&d->ymax);
    else if (w == "zmin") ok = real_key(&d->zmin);
    else if (w == "zmax") ok = real_key(&d->zmax);
    else if (w == "x_cells") ok = int_key(&d->x_cells);
    else if (w == "y_cells") ok = int_key(&d->y_cells);
    else if (w == "z_cells") ok = int_key(&d->z_cells);
    else if (w == "visit_frequency") ok = int_key(&d->visit_frequency);
    else if (w == "summary_frequency") ok = int_key(&d->summary_frequency);
    else if (w == "tiles_per_chunk" || w == "tiles_per_problem") ok = int_key(&d->tiles_per_chunk);
    else if (w == "profiler_on") d->profiler_on = 1;
    else if (w == "test_problem") ok = int_key(&d->test_problem);
    else if (w == "state") {
      int s = 0;
      if (!next_val(&v) || !to_int(v, &s) || s < 1 || s > state_max) return fail(3, "bad state number");
      const int si = s - 1;
      if (d->state_defined[si]) return fail(2, "State defined twice.");
      d->state_defined[si] = 1;
      const int line = toks[i].line;
      // the rest of the line holds the state's keys (parse_getword(.FALSE.))
      while (i + 1 < toks.size() && toks[i + 1].line == line) {
        const std::string k = toks[++i].w;
        double* dst = nullptr;
        if (k == "xvel") dst = &d->state_xvel[si];
        else if (k == "yvel") dst = &d->state_yvel[si];
        else if (k == "zvel") dst = &d->state_zvel[si];
        else if (k == "xmin") dst = &d->state_xmin[si];
        else if (k == "ymin") dst = &d->state_ymin[si];
        else if (k == "zmin") dst = &d->state_zmin[si];
        else if (k == "xmax") dst = &d->state_xmax[si];
        else if (k == "ymax") dst = &d->state_ymax[si];
        else if (k == "zmax") dst = &d->state_zmax[si];
        else if (k == "radius") dst = &d->state_radius[si];
        else if (k == "density") dst = &d->state_density[si];
        else if (k == "energy") dst = &d->state_energy[si];
        if (dst) {
          if (!next_val(&v) || !to_real(v, &r)) return fail(3, "bad real");
          *dst = r;
        } else if (k == "geometry") {
          if (!next_val(&v)) return fail(3, "missing geometry");
          if (v == "cuboid") d->state_geometry[si] = 1;
          else if (v == "sphere") d->state_geometry[si] = 2;
          else if (v == "point") d->state_geometry[si] = 3;
        }
      }
    }
    if (!ok) return fail(3, "bad number");
    i++;
  }
  return 0;
}

const char* clover_last_error(void) { return g_last_error.c_str(); }

clover_chunk* clover_chunk_create(const clover_deck* deck, int precision) {
  g_last_error.clear();
  if (deck->number_of_states < 1 || deck->number_of_states > CLOVER_MAX_STATES) {
    g_last_error = "deck needs 1..16 states";
    return nullptr;
  }
  clover_chunk* c = new clover_chunk;
  c->precision = precision;
  bool ok;
  if (precision == CLOVER_PRECISION_MIXED) {
    c->mixed = new Chunk<F32Mixed>;
    ok = c->mixed->create(*deck);
  } else {
    c->f64 = new Chunk<F64>;
    ok = c->f64->create(*deck);
  }
  if (!ok) {
    if (g_last_error.empty()) g_last_error = "chunk creation failed";
    clover_chunk_destroy(c);
    return nullptr;
  }
  return c;
}

void clover_chunk_destroy(clover_chunk* c) {
  if (!c) return;
  delete c->f64;
  delete c->mixed;
  delete c;
}

int clover_chunk_step(clover_chunk* c, int n) { return DISPATCH(c, step(n)); }
int clover_chunk_run(clover_chunk* c) { return DISPATCH(c, run()); }
int clover_chunk_sync(clover_chunk* c) {
  cudaStream_t s = c->f64 ? c->f64->stream : c->mixed->stream;
  return cudaStreamSynchronize(s) == cudaSuccess ? 0 : -1;
}
void clover_chunk_use_graphs(clover_chunk* c, int on) {
  if (c->f64) c->f64->use_graphs = on != 0;
  else c->mixed->use_graphs = on != 0;
}
int clover_chunk_steps(clover_chunk* c) { return DISPATCH(c, scalars()).step; }
double clover_chunk_time(clover_chunk* c) { return DISPATCH(c, scalars()).time; }
int clover_chunk_status(clover_chunk* c) { return DISPATCH(c, scalars()).status; }

int clover_chunk_dt_history(clover_chunk* c, double* out, int cap) {
  DevScalars h = DISPATCH(c, scalars());
  int n = h.step < cap ? h.step : cap;
  const double* src = c->f64 ? c->f64->dt_hist : c->mixed->dt_hist;
  const int dcap = c->f64 ? c->f64->dt_cap : c->mixed->dt_cap;
  if (n > dcap) n = dcap;
  if (n > 0 && cudaMemcpy(out, src, (size_t)n * sizeof(double), cudaMemcpyDeviceToHost) != cudaSuccess)
    return -1;
  return n;
}

int clover_chunk_summaries(clover_chunk* c, double* out5, int* steps, int cap) {
  clover_chunk_sync(c);
  const std::vector<int>& ss = c->f64 ? c->f64->sum_steps : c->mixed->sum_steps;
  const double* src = c->f64 ? c->f64->sum_hist : c->mixed->sum_hist;
  int n = (int)ss.size() < cap ? (int)ss.size() : cap;
  if (n > 0 && cudaMemcpy(out5, src, (size_t)n * 5 * sizeof(double), cudaMemcpyDeviceToHost) != cudaSuccess)
    return -1;
  for (int i = 0; i < n; i++) steps[i] = ss[i];
  return n;
}

int clover_chunk_read_field(clover_chunk* c, int id, double* host) {
  return DISPATCH(c, read_field(id, host, false));
}
int clover_chunk_write_field(clover_chunk* c, int id, const double* host) {
  return DISPATCH(c, read_field(id, const_cast<double*>(host), true));
}
uintptr_t clover_chunk_stream(clover_chunk* c) {
  return (uintptr_t)(c->f64 ? c->f64->stream : c->mixed->stream);
}
long long clover_chunk_device_bytes(clover_chunk* c) { return DISPATCH(c, bytes); }
void clover_chunk_use_fused(clover_chunk* c, int on) {
  // only between runs: the velocity buffers of a fused step alternate per step
  if (c->f64) {
    if (c->f64->host_step == 0) { c->f64->fused = on != 0; for (auto& gr : c->f64->graph) if (gr) { cudaGraphExecDestroy(gr); gr = nullptr; } }
  } else if (c->mixed->host_step == 0) {
    c->mixed->fused = on != 0;
    for (auto& gr : c->mixed->graph) if (gr) { cudaGraphExecDestroy(gr); gr = nullptr; }
  }
}

void clover_chunk_profile(clover_chunk* c, int on) {
  if (c->f64) { c->f64->prof_collect(); c->f64->profile = on != 0; if (!on) c->f64->prof_acc.clear(); }
  else { c->mixed->prof_collect(); c->mixed->profile = on != 0; if (!on) c->mixed->prof_acc.clear(); }
}

int clover_chunk_profile_report(clover_chunk* c, char* names, int name_len, double* ms,
                                double* bytes, int* launches, int cap) {
  auto report = [&](auto* ch) {
    ch->prof_collect();
    int n = 0;
    for (auto& a : ch->prof_acc) {
      if (n >= cap) break;
      snprintf(names + (size_t)n * name_len, (size_t)name_len, "%s", a.name.c_str());
      ms[n] = a.ms;
      bytes[n] = a.bytes;
      launches[n] = a.launches;
      n++;
    }
    ch->prof_acc.clear();
    return n;
  };
  return c->f64 ? report(c->f64) : report(c->mixed);
}

int clover_chunk_launches_per_step(clover_chunk* c) {
  if (c->f64) { c->f64->capture_graphs(); return c->f64->launches_per_step; }
  c->mixed->capture_graphs();
  return c->mixed->launches_per_step;
}

}  // extern "C"
