// Host driver over the drop-in ABI: the reference's own control flow
// (start.f90, hydro.f90, timestep.f90, PdV.f90, advection.f90,
// field_summary.f90) calling the clover_*_kernel entry points with host
// arrays allocated as build_field.f90 allocates them. This is what the
// unchanged Fortran drivers do once relinked against the ABI; the arrays
// stay resident on the GPU and only scalars cross back per step.
#include <cuda_runtime.h>

#include <cstdlib>
#include <cstring>
#include <vector>

#include "../../include/clover_b200.h"
#include "../../include/clover_kernels.h"

namespace {

const double kGSmall = (double)1.0e-16f;  // data.f90:30
const double kGBig = (double)1.0e+21f;    // data.f90:31

enum {
  F_DENSITY0 = 1, F_DENSITY1, F_ENERGY0, F_ENERGY1, F_PRESSURE, F_VISCOSITY, F_SOUNDSPEED,
  F_XVEL0, F_XVEL1, F_YVEL0, F_YVEL1, F_ZVEL0, F_ZVEL1, F_VOL_FLUX_X, F_VOL_FLUX_Y,
  F_VOL_FLUX_Z, F_MASS_FLUX_X, F_MASS_FLUX_Y, F_MASS_FLUX_Z
};

}  // namespace

struct clover_dropin {
  clover_deck deck;
  int x_min = 1, x_max, y_min = 1, y_max, z_min = 1, z_max;
  int left = 1, bottom = 1, back = 1;  // global index of the chunk's first cell per axis
  std::vector<double> density0, density1, energy0, energy1, pressure, viscosity, soundspeed;
  std::vector<double> xvel0, xvel1, yvel0, yvel1, zvel0, zvel1;
  std::vector<double> vol_flux_x, vol_flux_y, vol_flux_z, mass_flux_x, mass_flux_y, mass_flux_z;
  std::vector<double> wa[7];
  std::vector<double> cellx, celly, cellz, vertexx, vertexy, vertexz;
  std::vector<double> celldx, celldy, celldz, vertexdx, vertexdy, vertexdz;
  std::vector<double> volume, xarea, yarea, zarea;
  int neighbours[6] = {-1, -1, -1, -1, -1, -1};
  double dt = 0, dtold = 0, time = 0;
  int step = 0;
  bool advect_x = true;
  std::vector<double> dt_hist, sum_hist;
  std::vector<int> sum_steps;

#define B &x_min, &x_max, &y_min, &y_max, &z_min, &z_max

  // build_field.f90:41-229
  void build() {
    const size_t nx = x_max, ny = y_max, nz = z_max;
    const size_t cell = (nx + 4) * (ny + 4) * (nz + 4), vert = (nx + 5) * (ny + 5) * (nz + 5);
    const size_t xf = (nx + 5) * (ny + 4) * (nz + 4), yf = (nx + 4) * (ny + 5) * (nz + 4),
                 zf = (nx + 4) * (ny + 4) * (nz + 5);
    for (auto* v : {&density0, &density1, &energy0, &energy1, &pressure, &viscosity,
                    &soundspeed, &volume})
      v->assign(cell, 0.0);
    for (auto* v : {&xvel0, &xvel1, &yvel0, &yvel1, &zvel0, &zvel1}) v->assign(vert, 0.0);
    for (int i = 0; i < 7; i++) wa[i].assign(vert, 0.0);
    vol_flux_x.assign(xf, 0.0); mass_flux_x.assign(xf, 0.0); xarea.assign(xf, 0.0);
    vol_flux_y.assign(yf, 0.0); mass_flux_y.assign(yf, 0.0); yarea.assign(yf, 0.0);
    vol_flux_z.assign(zf, 0.0); mass_flux_z.assign(zf, 0.0); zarea.assign(zf, 0.0);
    cellx.assign(nx + 4, 0.0); celldx.assign(nx + 4, 0.0);
    celly.assign(ny + 4, 0.0); celldy.assign(ny + 4, 0.0);
    cellz.assign(nz + 4, 0.0); celldz.assign(nz + 4, 0.0);
    vertexx.assign(nx + 5, 0.0); vertexdx.assign(nx + 5, 0.0);
    vertexy.assign(ny + 5, 0.0); vertexdy.assign(ny + 5, 0.0);
    vertexz.assign(nz + 5, 0.0); vertexdz.assign(nz + 5, 0.0);
  }

  void update_halo(std::initializer_list<int> ids, int depth) {
    update_halo(std::vector<int>(ids), depth);
  }
  void update_halo(const std::vector<int>& ids, int depth) {
    int fields[19] = {0};
    for (int id : ids) fields[id - 1] = 1;
    clover_update_halo_kernel(B, neighbours, neighbours, density0.data(), energy0.data(),
                              pressure.data(), viscosity.data(), soundspeed.data(),
                              density1.data(), energy1.data(), xvel0.data(), yvel0.data(),
                              zvel0.data(), xvel1.data(), yvel1.data(), zvel1.data(),
                              vol_flux_x.data(), vol_flux_y.data(), vol_flux_z.data(),
                              mass_flux_x.data(), mass_flux_y.data(), mass_flux_z.data(),
                              fields, &depth);
  }

  void ideal_gas(bool predict) {  // ideal_gas.f90:38-66
    if (!predict)
      clover_ideal_gas_kernel(B, density0.data(), energy0.data(), pressure.data(), soundspeed.data());
    else
      clover_ideal_gas_kernel(B, density1.data(), energy1.data(), pressure.data(), soundspeed.data());
  }

  void field_summary() {  // field_summary.f90:55-113
    ideal_gas(false);
    double s[5];
    summary_kernel(s);
    sum_hist.insert(sum_hist.end(), s, s + 5);
    sum_steps.push_back(step);
  }

  bool start(const clover_deck& d) {  // start.f90:49-136
    const int ext[6] = {1, d.x_cells, 1, d.y_cells, 1, d.z_cells};
    generate(d, ext);
    update_halo({F_DENSITY0, F_ENERGY0, F_PRESSURE, F_VISCOSITY, F_DENSITY1, F_ENERGY1, F_XVEL0,
                 F_YVEL0, F_ZVEL0, F_XVEL1, F_YVEL1, F_ZVEL1}, 2);
    field_summary();
    return clover_gpu_status() == 0;
  }

  // start.f90:49-98 for the chunk of global cells ext = left, right, bottom,
  // top, back, front (clover_decompose): build_field, initialise_chunk (its
  // mesh origin shifted to the chunk's first cell, initialise_chunk.f90:38-46),
  // generate_chunk and ideal_gas.
  void generate(const clover_deck& d, const int* ext) {
    deck = d;
    left = ext[0]; bottom = ext[2]; back = ext[4];
    x_max = ext[1] - ext[0] + 1; y_max = ext[3] - ext[2] + 1; z_max = ext[5] - ext[4] + 1;
    time = 0.0;
    step = 0;
    dtold = d.initial_timestep;
    dt = d.initial_timestep;
    build();
    // initialise_chunk.f90:38-46
    double dx = (d.xmax - d.xmin) / (double)(float)d.x_cells;
    double dy = (d.ymax - d.ymin) / (double)(float)d.y_cells;
    double dz = (d.zmax - d.zmin) / (double)(float)d.z_cells;
    double xmin = d.xmin + dx * (double)(float)(left - 1),
           ymin = d.ymin + dy * (double)(float)(bottom - 1),
           zmin = d.zmin + dz * (double)(float)(back - 1);
    clover_initialise_chunk_kernel(B, &xmin, &ymin, &zmin, &dx, &dy, &dz, vertexx.data(),
                                   vertexdx.data(), vertexy.data(), vertexdy.data(),
                                   vertexz.data(), vertexdz.data(), cellx.data(), celldx.data(),
                                   celly.data(), celldy.data(), cellz.data(), celldz.data(),
                                   volume.data(), xarea.data(), yarea.data(), zarea.data());
    // read_input.f90:293-303
    clover_deck s = d;
    for (int n = 1; n < s.number_of_states; n++) {
      s.state_xmin[n] = s.state_xmin[n] + (dx / 100.0);
      s.state_ymin[n] = s.state_ymin[n] + (dy / 100.0);
      s.state_zmin[n] = s.state_zmin[n] + (dz / 100.0);
      s.state_xmax[n] = s.state_xmax[n] - (dx / 100.0);
      s.state_ymax[n] = s.state_ymax[n] - (dy / 100.0);
      s.state_zmax[n] = s.state_zmax[n] - (dz / 100.0);
    }
    const int g_rect = 1, g_circ = 2, g_point = 3;
    clover_generate_chunk_kernel(B, vertexx.data(), vertexy.data(), vertexz.data(), cellx.data(),
                                 celly.data(), cellz.data(), density0.data(), energy0.data(),
                                 xvel0.data(), yvel0.data(), zvel0.data(), &s.number_of_states,
                                 s.state_density, s.state_energy, s.state_xvel, s.state_yvel,
                                 s.state_zvel, s.state_xmin, s.state_xmax, s.state_ymin,
                                 s.state_ymax, s.state_zmin, s.state_zmax, s.state_radius,
                                 s.state_geometry, &g_rect, &g_circ, &g_point);
    advect_x = true;
    ideal_gas(false);
  }

  // ---- the kernel calls of the drivers, one chunk each (the brick driver
  // makes each call on every brick before the next) ----
  void viscosity_kernel() {
    clover_viscosity_kernel(B, xarea.data(), yarea.data(), zarea.data(), celldx.data(),
                            celldy.data(), celldz.data(), density0.data(), pressure.data(),
                            viscosity.data(), xvel0.data(), yvel0.data(), zvel0.data());
  }
  double calc_dt() {  // calc_dt.f90:42-97 for this chunk: its dt_min
    double dtlp, xl, yl, zl;
    int ctl, jl, kl, ll, small = 0;
    const double g_small = kGSmall, g_big = kGBig;
    clover_calc_dt_kernel(B, &g_small, &g_big, &deck.dtmin, &deck.dtc_safe, &deck.dtu_safe,
                          &deck.dtv_safe, &deck.dtw_safe, &deck.dtdiv_safe, xarea.data(),
                          yarea.data(), zarea.data(), cellx.data(), celly.data(), cellz.data(),
                          celldx.data(), celldy.data(), celldz.data(), volume.data(),
                          density0.data(), energy0.data(), pressure.data(), viscosity.data(),
                          soundspeed.data(), xvel0.data(), yvel0.data(), zvel0.data(),
                          wa[0].data(), &dtlp, &ctl, &xl, &yl, &zl, &jl, &kl, &ll, &small);
    return dtlp;
  }
  void pdv_kernel(bool predict, double dt_) {
    const int32_t p = predict ? 1 : 0;
    clover_pdv_kernel(&p, B, &dt_, xarea.data(), yarea.data(), zarea.data(), volume.data(),
                      density0.data(), density1.data(), energy0.data(), energy1.data(),
                      pressure.data(), viscosity.data(), xvel0.data(), xvel1.data(),
                      yvel0.data(), yvel1.data(), zvel0.data(), zvel1.data());
  }
  void revert() {
    clover_revert_kernel(B, density0.data(), density1.data(), energy0.data(), energy1.data());
  }
  void accelerate(double dt_) {
    clover_accelerate_kernel(B, &dt_, xarea.data(), yarea.data(), zarea.data(), volume.data(),
                             density0.data(), pressure.data(), viscosity.data(), xvel0.data(),
                             yvel0.data(), zvel0.data(), xvel1.data(), yvel1.data(), zvel1.data());
  }
  void flux_calc(double dt_) {
    clover_flux_calc_kernel(B, &dt_, xarea.data(), yarea.data(), zarea.data(), xvel0.data(),
                            yvel0.data(), zvel0.data(), xvel1.data(), yvel1.data(), zvel1.data(),
                            vol_flux_x.data(), vol_flux_y.data(), vol_flux_z.data());
  }
  void reset_field() {
    clover_reset_field_kernel(B, density0.data(), density1.data(), energy0.data(), energy1.data(),
                              xvel0.data(), xvel1.data(), yvel0.data(), yvel1.data(),
                              zvel0.data(), zvel1.data());
  }
  void summary_kernel(double* s) {  // field_summary_kernel on this chunk (after ideal_gas)
    clover_field_summary_kernel(B, volume.data(), density0.data(), energy0.data(),
                                pressure.data(), xvel0.data(), yvel0.data(), zvel0.data(), &s[0],
                                &s[1], &s[2], &s[3], &s[4]);
  }
  void bounds(int* b6) const {
    b6[0] = x_min; b6[1] = x_max; b6[2] = y_min; b6[3] = y_max; b6[4] = z_min; b6[5] = z_max;
  }

  bool timestep() {  // timestep.f90:56-126
    dt = kGBig;
    ideal_gas(false);
    update_halo({F_PRESSURE, F_ENERGY0, F_DENSITY0, F_XVEL0, F_YVEL0}, 1);
    viscosity_kernel();
    update_halo({F_VISCOSITY}, 1);
    const double dtlp = calc_dt();
    if (dtlp <= dt) dt = dtlp;
    double m = dt;
    const double r = dtold * deck.timestep_rise;
    if (r < m) m = r;
    if (deck.max_timestep < m) m = deck.max_timestep;
    dt = m;
    const bool err = dt < deck.dtmin;
    dtold = dt;
    return !err;
  }

  void pdv(bool predict) {  // PdV.f90:50-107
    pdv_kernel(predict, dt);
    if (predict) {
      ideal_gas(true);
      update_halo({F_PRESSURE}, 1);
      revert();
    }
  }

  void advec_cell(int sweep, int dir) {
    const int32_t ax = advect_x ? 1 : 0;
    clover_advec_cell_kernel(B, &ax, &dir, &sweep, vertexdx.data(), vertexdy.data(),
                             vertexdz.data(), volume.data(), density1.data(), energy1.data(),
                             mass_flux_x.data(), vol_flux_x.data(), mass_flux_y.data(),
                             vol_flux_y.data(), mass_flux_z.data(), vol_flux_z.data(),
                             wa[0].data(), wa[1].data(), wa[2].data(), wa[3].data(),
                             wa[4].data(), wa[5].data(), wa[6].data());
  }

  void advec_mom(int which_vel, int dir, int sweep) {
    const int32_t ax = advect_x ? 1 : 0;
    double* vel = which_vel == 1 ? xvel1.data() : which_vel == 2 ? yvel1.data() : zvel1.data();
    clover_advec_mom_kernel(B, vel, mass_flux_x.data(), vol_flux_x.data(), mass_flux_y.data(),
                            vol_flux_y.data(), mass_flux_z.data(), vol_flux_z.data(),
                            volume.data(), density1.data(), wa[0].data(), wa[1].data(),
                            wa[2].data(), wa[3].data(), wa[4].data(), wa[5].data(),
                            wa[6].data(), celldx.data(), celldy.data(), celldz.data(), &ax,
                            &which_vel, &sweep, &dir);
  }

  void advection() {  // advection.f90:43-179
    auto pre = [&] { update_halo({F_ENERGY1, F_DENSITY1, F_VOL_FLUX_X, F_VOL_FLUX_Y, F_VOL_FLUX_Z}, 2); };
    auto post = [&] {
      update_halo({F_DENSITY1, F_ENERGY1, F_XVEL1, F_YVEL1, F_ZVEL1, F_MASS_FLUX_X,
                   F_MASS_FLUX_Y, F_MASS_FLUX_Z}, 2);
    };
    int dir = advect_x ? 1 : 3;
    pre();
    advec_cell(1, dir);
    post();
    for (int v = 1; v <= 3; v++) advec_mom(v, dir, 1);
    pre();
    advec_cell(2, 2);
    post();
    for (int v = 1; v <= 3; v++) advec_mom(v, 2, 2);
    dir = advect_x ? 3 : 1;
    advec_cell(3, dir);
    post();
    for (int v = 1; v <= 3; v++) advec_mom(v, dir, 3);
  }

  // hydro.f90:46-98; returns steps taken (negative on the small-dt error)
  int hydro(int max_steps) {
    for (;;) {
      step = step + 1;
      if (!timestep()) return -step;
      dt_hist.push_back(dt);
      pdv(true);
      accelerate(dt);
      pdv(false);
      flux_calc(dt);
      advection();
      reset_field();
      advect_x = !advect_x;
      time = time + dt;
      if (deck.summary_frequency != 0 && step % deck.summary_frequency == 0) field_summary();
      if (time + kGSmall > deck.end_time || step >= deck.end_step || step >= max_steps) {
        field_summary();
        return step;
      }
    }
  }

  double* field(int id) {
    std::vector<double>* f[19] = {&density0, &density1, &energy0, &energy1, &pressure,
                                  &viscosity, &soundspeed, &xvel0, &xvel1, &yvel0, &yvel1,
                                  &zvel0, &zvel1, &vol_flux_x, &vol_flux_y, &vol_flux_z,
                                  &mass_flux_x, &mass_flux_y, &mass_flux_z};
    return id >= 1 && id <= 19 ? f[id - 1]->data() : nullptr;
  }
#undef B
};

namespace {

// clover.f90:108-256 (clover_decompose): the chunk grid with the smallest
// surface-to-volume metric over the factorisations of n (the metric in
// default REAL, as the reference forms it: 1.0*x_cells is single precision),
// then each chunk's global cell range and its neighbours (chunk ids from 1 in
// x-fastest order, -1 for an external face).
void decompose(int x_cells, int y_cells, int z_cells, int n, int* cxyz, int* ext, int* nbr) {
  auto metric = [&](int cx, int cy, int cz) {
    const float ax = (1.0f * (float)x_cells) / (float)cx;
    const float ay = (1.0f * (float)y_cells) / (float)cy;
    const float az = (1.0f * (float)z_cells) / (float)cz;
    const double surface = (double)(ax * ay * 2.0f + ax * az * 2.0f + ay * az * 2.0f);
    const double volume = (double)(ax * ay * az);
    return surface / volume;
  };
  int chunk_x = 1, chunk_y = 1, chunk_z = n;
  double best = metric(1, 1, n);
  for (int c = 1; c <= n; c++) {
    if (n % c != 0) continue;
    const int div1 = n / c;
    for (int j = 1; j <= div1; j++) {
      if (div1 % j != 0) continue;
      if (n % (c * j) != 0) continue;
      const int cz = n / (c * j);
      const double m = metric(c, j, cz);
      if (m < best) {
        chunk_x = c; chunk_y = j; chunk_z = cz;
        best = m;
      }
    }
  }
  cxyz[0] = chunk_x; cxyz[1] = chunk_y; cxyz[2] = chunk_z;
  const int delta_x = x_cells / chunk_x, delta_y = y_cells / chunk_y, delta_z = z_cells / chunk_z;
  const int mod_x = x_cells % chunk_x, mod_y = y_cells % chunk_y, mod_z = z_cells % chunk_z;
  int add_x_prev = 0, add_y_prev = 0, add_z_prev = 0, id = 1;
  for (int cz = 1; cz <= chunk_z; cz++) {
    for (int cy = 1; cy <= chunk_y; cy++) {
      for (int cx = 1; cx <= chunk_x; cx++) {
        const int add_x = cx <= mod_x ? 1 : 0, add_y = cy <= mod_y ? 1 : 0,
                  add_z = cz <= mod_z ? 1 : 0;
        int* e = ext + 6 * (id - 1);
        int* nb = nbr + 6 * (id - 1);
        e[0] = (cx - 1) * delta_x + 1 + add_x_prev;
        e[1] = e[0] + delta_x - 1 + add_x;
        e[2] = (cy - 1) * delta_y + 1 + add_y_prev;
        e[3] = e[2] + delta_y - 1 + add_y;
        e[4] = (cz - 1) * delta_z + 1 + add_z_prev;
        e[5] = e[4] + delta_z - 1 + add_z;
        nb[0] = cx == 1 ? -1 : id - 1;
        nb[1] = cx == chunk_x ? -1 : id + 1;
        nb[2] = cy == 1 ? -1 : id - chunk_x;
        nb[3] = cy == chunk_y ? -1 : id + chunk_x;
        nb[4] = cz == 1 ? -1 : id - chunk_x * chunk_y;
        nb[5] = cz == chunk_z ? -1 : id + chunk_x * chunk_y;
        if (cx <= mod_x) add_x_prev++;
        id++;
      }
      add_x_prev = 0;
      if (cy <= mod_y) add_y_prev++;
    }
    add_x_prev = 0;
    add_y_prev = 0;
    if (cz <= mod_z) add_z_prev++;
  }
}

// pack_kernel.f90 field type of each field id (data.f90:55-74)
int field_type_of(int id) {
  if (id <= 7) return 1;                // cell
  if (id <= 13) return 2;               // vertex
  if (id == 14 || id == 17) return 3;   // x face
  if (id == 15 || id == 18) return 4;   // y face
  return 5;                             // z face
}

}  // namespace

// The reference's decomposed run (clover.f90 with its MPI exchange,
// update_halo.f90, timestep.f90's clover_min, field_summary.f90's clover_sum)
// over the bricks of one deck in this process: every driver call is made on
// each brick in turn, each update_halo exchanges the bricks' faces first
// (x, then y, then z messages, pack_kernel.f90's layers, on the device) and
// then applies the reflective rules on each brick's external faces.
struct clover_bricks {
  clover_deck deck;
  int grid[3] = {1, 1, 1};
  std::vector<clover_dropin*> b;
  double dt = 0, dtold = 0, time = 0;
  int step = 0;
  bool advect_x = true;
  std::vector<double> dt_hist, sum_hist;
  std::vector<int> sum_steps;
  // one brick per rank: this rank's chunk (id rank + 1) and the transport of
  // its messages and reductions; rank < 0: every brick in this process
  int rank = -1;
  clover_transport tr{};
  double* dmsg[4] = {nullptr, nullptr, nullptr, nullptr};  // send lo, recv lo, send hi, recv hi
  double* hmsg[4] = {nullptr, nullptr, nullptr, nullptr};  // their host copies (host_staged)
  long long msg_cap = 0;
  bool failed = false;

  ~clover_bricks() {
    for (clover_dropin* d : b) delete d;
    for (int q = 0; q < 4; q++) {
      if (dmsg[q]) cudaFree(dmsg[q]);
      if (hmsg[q]) cudaFreeHost(hmsg[q]);
    }
  }

  bool reserve(long long n) {
    if (n <= msg_cap) return true;
    for (int q = 0; q < 4; q++) {
      if (dmsg[q]) cudaFree(dmsg[q]);
      if (hmsg[q]) cudaFreeHost(hmsg[q]);
      dmsg[q] = hmsg[q] = nullptr;
      if (cudaMalloc(&dmsg[q], (size_t)n * 8) != cudaSuccess) return false;
      if (tr.host_staged && cudaMallocHost(&hmsg[q], (size_t)n * 8) != cudaSuccess) return false;
    }
    msg_cap = n;
    return true;
  }

  // clover_exchange for this rank's brick: per axis, the messages of every
  // field of the call packed one after another per side (clover.f90:474-713
  // packs them into one buffer per side), moved by the transport, unpacked
  void exchange_ranks(const std::vector<int>& ids, int depth) {
    clover_dropin* c = b[0];
    int bnd[6];
    c->bounds(bnd);
    for (int axis = 0; axis < 3; axis++) {
      const int nb[2] = {c->neighbours[2 * axis], c->neighbours[2 * axis + 1]};
      long long len[2] = {0, 0};
      for (int s2 = 0; s2 < 2; s2++)
        if (nb[s2] >= 0)
          for (int id : ids)
            len[s2] += clover_gpu_message_len(bnd, 2 * axis + s2, field_type_of(id), depth);
      if (!reserve(len[0] > len[1] ? len[0] : len[1])) {
        failed = true;
        return;
      }
      for (int s2 = 0; s2 < 2; s2++) {
        if (nb[s2] < 0) continue;
        long long off = 0;
        for (int id : ids) {
          const int t = field_type_of(id);
          clover_gpu_pack_device(bnd, c->field(id), 2 * axis + s2, t, depth, dmsg[2 * s2] + off, 0);
          off += clover_gpu_message_len(bnd, 2 * axis + s2, t, depth);
        }
      }
      clover_gpu_synchronize();
      double* io[4];
      for (int q = 0; q < 4; q++) io[q] = tr.host_staged ? hmsg[q] : dmsg[q];
      if (tr.host_staged)
        for (int s2 = 0; s2 < 2; s2++)
          if (nb[s2] >= 0)
            cudaMemcpy(hmsg[2 * s2], dmsg[2 * s2], (size_t)len[s2] * 8, cudaMemcpyDeviceToHost);
      if (tr.exchange(tr.ctx, axis, nb[0], io[0], io[1], len[0], nb[1], io[2], io[3], len[1]) != 0) {
        failed = true;
        return;
      }
      for (int s2 = 0; s2 < 2; s2++) {
        if (nb[s2] < 0) continue;
        if (tr.host_staged)
          cudaMemcpy(dmsg[2 * s2 + 1], hmsg[2 * s2 + 1], (size_t)len[s2] * 8,
                     cudaMemcpyHostToDevice);
        long long off = 0;
        for (int id : ids) {
          const int t = field_type_of(id);
          clover_gpu_pack_device(bnd, c->field(id), 2 * axis + s2, t, depth,
                                 dmsg[2 * s2 + 1] + off, 1);
          off += clover_gpu_message_len(bnd, 2 * axis + s2, t, depth);
        }
      }
    }
  }

  // clover_exchange (clover.f90:474-713): per axis, both messages of every
  // pair of neighbours along it, then the reflective halos
  void update_halo(const std::vector<int>& ids, int depth) {
    if (rank >= 0) {
      exchange_ranks(ids, depth);
      for (clover_dropin* d : b) d->update_halo(ids, depth);
      return;
    }
    // one launch per axis phase: every message of the phase (both directions
    // of every pair of neighbours along the axis, every field of the call)
    std::vector<int> sb, db, sides, types;
    std::vector<double*> src, dst;
    for (int axis = 0; axis < 3; axis++) {
      sb.clear(); db.clear(); sides.clear(); types.clear(); src.clear(); dst.clear();
      for (size_t i = 0; i < b.size(); i++) {
        const int hi = b[i]->neighbours[2 * axis + 1];
        if (hi < 0) continue;
        clover_dropin* lo_b = b[i];
        clover_dropin* hi_b = b[hi - 1];
        int lo_bounds[6], hi_bounds[6];
        lo_b->bounds(lo_bounds);
        hi_b->bounds(hi_bounds);
        for (int id : ids) {
          const int t = field_type_of(id);
          for (int dir = 0; dir < 2; dir++) {  // lo's hi side to hi, hi's lo side to lo
            const int* from = dir == 0 ? lo_bounds : hi_bounds;
            const int* to = dir == 0 ? hi_bounds : lo_bounds;
            sb.insert(sb.end(), from, from + 6);
            db.insert(db.end(), to, to + 6);
            src.push_back(dir == 0 ? lo_b->field(id) : hi_b->field(id));
            dst.push_back(dir == 0 ? hi_b->field(id) : lo_b->field(id));
            sides.push_back(dir == 0 ? 2 * axis + 1 : 2 * axis);
            types.push_back(t);
          }
        }
      }
      if (!sides.empty())
        clover_gpu_face_copy_many((int)sides.size(), sb.data(), src.data(), db.data(), dst.data(),
                                  sides.data(), types.data(), depth);
    }
    for (clover_dropin* d : b) d->update_halo(ids, depth);
  }

  void ideal_gas(bool predict) {
    for (clover_dropin* d : b) d->ideal_gas(predict);
  }

  void field_summary() {  // field_summary.f90:55-113 with clover_sum over the bricks
    ideal_gas(false);
    double t[5] = {0, 0, 0, 0, 0};
    for (clover_dropin* d : b) {
      double s[5];
      d->summary_kernel(s);
      for (int q = 0; q < 5; q++) t[q] += s[q];
    }
    if (rank >= 0 && tr.sum(tr.ctx, t, 5) != 0) failed = true;
    sum_hist.insert(sum_hist.end(), t, t + 5);
    sum_steps.push_back(step);
  }

  bool start(const clover_deck& d, int n) {
    deck = d;
    std::vector<int> ext(6 * n), nbr(6 * n);
    decompose(d.x_cells, d.y_cells, d.z_cells, n, grid, ext.data(), nbr.data());
    for (int i = 0; i < n; i++) {
      if (rank >= 0 && i != rank) continue;
      clover_dropin* c = new clover_dropin;
      b.push_back(c);
      for (int f = 0; f < 6; f++) c->neighbours[f] = nbr[6 * i + f];
      c->generate(d, &ext[6 * i]);
    }
    dt = dtold = d.initial_timestep;
    update_halo({F_DENSITY0, F_ENERGY0, F_PRESSURE, F_VISCOSITY, F_DENSITY1, F_ENERGY1, F_XVEL0,
                 F_YVEL0, F_ZVEL0, F_XVEL1, F_YVEL1, F_ZVEL1}, 2);
    field_summary();
    return clover_gpu_status() == 0;
  }

  bool timestep() {  // timestep.f90:56-126, the chunks' dt_min reduced by clover_min
    dt = kGBig;
    ideal_gas(false);
    update_halo({F_PRESSURE, F_ENERGY0, F_DENSITY0, F_XVEL0, F_YVEL0}, 1);
    for (clover_dropin* c : b) c->viscosity_kernel();
    update_halo({F_VISCOSITY}, 1);
    for (clover_dropin* c : b) {
      const double dtlp = c->calc_dt();
      if (dtlp <= dt) dt = dtlp;
    }
    if (rank >= 0 && tr.min(tr.ctx, &dt) != 0) failed = true;
    double m = dt;
    const double r = dtold * deck.timestep_rise;
    if (r < m) m = r;
    if (deck.max_timestep < m) m = deck.max_timestep;
    dt = m;
    const bool err = dt < deck.dtmin;
    dtold = dt;
    return !err;
  }

  void pdv(bool predict) {  // PdV.f90:50-107
    for (clover_dropin* c : b) c->pdv_kernel(predict, dt);
    if (predict) {
      ideal_gas(true);
      update_halo({F_PRESSURE}, 1);
      for (clover_dropin* c : b) c->revert();
    }
  }

  void advection() {  // advection.f90:43-179
    const std::vector<int> pre = {F_ENERGY1, F_DENSITY1, F_VOL_FLUX_X, F_VOL_FLUX_Y, F_VOL_FLUX_Z};
    const std::vector<int> post = {F_DENSITY1, F_ENERGY1, F_XVEL1, F_YVEL1, F_ZVEL1,
                                   F_MASS_FLUX_X, F_MASS_FLUX_Y, F_MASS_FLUX_Z};
    for (clover_dropin* c : b) c->advect_x = advect_x;
    int dir = advect_x ? 1 : 3;
    update_halo(pre, 2);
    for (clover_dropin* c : b) c->advec_cell(1, dir);
    update_halo(post, 2);
    for (clover_dropin* c : b)  // a brick's three velocity calls back to back
      for (int v = 1; v <= 3; v++) c->advec_mom(v, dir, 1);
    update_halo(pre, 2);
    for (clover_dropin* c : b) c->advec_cell(2, 2);
    update_halo(post, 2);
    for (clover_dropin* c : b)  // a brick's three velocity calls back to back
      for (int v = 1; v <= 3; v++) c->advec_mom(v, 2, 2);
    dir = advect_x ? 3 : 1;
    for (clover_dropin* c : b) c->advec_cell(3, dir);
    update_halo(post, 2);
    for (clover_dropin* c : b)  // a brick's three velocity calls back to back
      for (int v = 1; v <= 3; v++) c->advec_mom(v, dir, 3);
  }

  int hydro(int max_steps) {  // hydro.f90:46-98
    for (;;) {
      step = step + 1;
      if (!timestep()) return -step;
      if (failed) return -step;
      dt_hist.push_back(dt);
      pdv(true);
      for (clover_dropin* c : b) c->accelerate(dt);
      pdv(false);
      for (clover_dropin* c : b) c->flux_calc(dt);
      advection();
      for (clover_dropin* c : b) c->reset_field();
      advect_x = !advect_x;
      time = time + dt;
      if (deck.summary_frequency != 0 && step % deck.summary_frequency == 0) field_summary();
      if (time + kGSmall > deck.end_time || step >= deck.end_step || step >= max_steps) {
        field_summary();
        return step;
      }
    }
  }
};

extern "C" {

clover_dropin* clover_dropin_create(const clover_deck* deck) {
  clover_dropin* d = new clover_dropin;
  if (!d->start(*deck)) {
    delete d;
    return nullptr;
  }
  return d;
}

int clover_dropin_run(clover_dropin* d, int max_steps) { return d->hydro(max_steps); }

int clover_dropin_dt_history(clover_dropin* d, double* out, int cap) {
  int n = (int)d->dt_hist.size() < cap ? (int)d->dt_hist.size() : cap;
  memcpy(out, d->dt_hist.data(), (size_t)n * sizeof(double));
  return n;
}

int clover_dropin_summaries(clover_dropin* d, double* out5, int* steps, int cap) {
  int n = (int)d->sum_steps.size() < cap ? (int)d->sum_steps.size() : cap;
  memcpy(out5, d->sum_hist.data(), (size_t)n * 5 * sizeof(double));
  memcpy(steps, d->sum_steps.data(), (size_t)n * sizeof(int));
  return n;
}

int clover_dropin_read_field(clover_dropin* d, int id, double* out, long long n) {
  clover_gpu_sync_to_host();
  double* f = d->field(id);
  if (!f) return -1;
  memcpy(out, f, (size_t)n * sizeof(double));
  return clover_gpu_status() == 0 ? 0 : -1;
}

void clover_dropin_destroy(clover_dropin* d) {
  clover_gpu_release();
  delete d;
}

int clover_decompose(int x_cells, int y_cells, int z_cells, int n_chunks, int* chunks_xyz,
                     int* extents, int* neighbours) {
  if (x_cells < 1 || y_cells < 1 || z_cells < 1 || n_chunks < 1) return -1;
  decompose(x_cells, y_cells, z_cells, n_chunks, chunks_xyz, extents, neighbours);
  for (int i = 0; i < n_chunks; i++) {
    const int* e = extents + 6 * i;
    if (e[1] < e[0] || e[3] < e[2] || e[5] < e[4]) return -1;  // more chunks than cells
  }
  return 0;
}

clover_bricks* clover_bricks_create(const clover_deck* deck, int n_chunks) {
  if (n_chunks < 1 || n_chunks > deck->x_cells * deck->y_cells * deck->z_cells) return nullptr;
  clover_bricks* w = new clover_bricks;
  if (!w->start(*deck, n_chunks)) {
    delete w;
    return nullptr;
  }
  return w;
}

clover_bricks* clover_bricks_create_rank(const clover_deck* deck, int n_chunks, int rank,
                                         const clover_transport* t) {
  if (n_chunks < 1 || rank < 0 || rank >= n_chunks || !t || !t->exchange || !t->min || !t->sum)
    return nullptr;
  clover_bricks* w = new clover_bricks;
  w->rank = rank;
  w->tr = *t;
  if (!w->start(*deck, n_chunks) || w->failed) {
    delete w;
    return nullptr;
  }
  return w;
}

int clover_bricks_run(clover_bricks* w, int max_steps) {
  const int n = w->hydro(max_steps);
  return w->failed ? -1 : n;
}

int clover_bricks_count(clover_bricks* w, int* chunks_xyz) {
  for (int q = 0; q < 3; q++) chunks_xyz[q] = w->grid[q];
  return (int)w->b.size();
}

int clover_bricks_extent(clover_bricks* w, int brick, int* ext6, int* neighbours6) {
  if (brick < 0 || brick >= (int)w->b.size()) return -1;
  const clover_dropin* c = w->b[brick];
  ext6[0] = c->left; ext6[1] = c->left + c->x_max - 1;
  ext6[2] = c->bottom; ext6[3] = c->bottom + c->y_max - 1;
  ext6[4] = c->back; ext6[5] = c->back + c->z_max - 1;
  for (int f = 0; f < 6; f++) neighbours6[f] = c->neighbours[f];
  return 0;
}

int clover_bricks_dt_history(clover_bricks* w, double* out, int cap) {
  int n = (int)w->dt_hist.size() < cap ? (int)w->dt_hist.size() : cap;
  memcpy(out, w->dt_hist.data(), (size_t)n * sizeof(double));
  return n;
}

int clover_bricks_summaries(clover_bricks* w, double* out5, int* steps, int cap) {
  int n = (int)w->sum_steps.size() < cap ? (int)w->sum_steps.size() : cap;
  memcpy(out5, w->sum_hist.data(), (size_t)n * 5 * sizeof(double));
  memcpy(steps, w->sum_steps.data(), (size_t)n * sizeof(int));
  return n;
}

int clover_bricks_read_field(clover_bricks* w, int brick, int id, double* out, long long n) {
  if (brick < 0 || brick >= (int)w->b.size()) return -1;
  return clover_dropin_read_field(w->b[brick], id, out, n);
}

void clover_bricks_destroy(clover_bricks* w) {
  clover_gpu_release();
  delete w;
}

}  // extern "C"
