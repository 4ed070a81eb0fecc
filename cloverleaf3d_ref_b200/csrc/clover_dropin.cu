// Host driver over the drop-in ABI: the reference's own control flow
// (start.f90, hydro.f90, timestep.f90, PdV.f90, advection.f90,
// field_summary.f90) calling the clover_*_kernel entry points with host
// arrays allocated as build_field.f90 allocates them. This is what the
// unchanged Fortran drivers do once relinked against the ABI; the arrays
// stay resident on the GPU and only scalars cross back per step.
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
    clover_field_summary_kernel(B, volume.data(), density0.data(), energy0.data(),
                                pressure.data(), xvel0.data(), yvel0.data(), zvel0.data(), &s[0],
                                &s[1], &s[2], &s[3], &s[4]);
    sum_hist.insert(sum_hist.end(), s, s + 5);
    sum_steps.push_back(step);
  }

  bool start(const clover_deck& d) {  // start.f90:49-136
    deck = d;
    x_max = d.x_cells; y_max = d.y_cells; z_max = d.z_cells;
    time = 0.0;
    step = 0;
    dtold = d.initial_timestep;
    dt = d.initial_timestep;
    build();
    // initialise_chunk.f90:38-46
    double dx = (d.xmax - d.xmin) / (double)(float)d.x_cells;
    double dy = (d.ymax - d.ymin) / (double)(float)d.y_cells;
    double dz = (d.zmax - d.zmin) / (double)(float)d.z_cells;
    double xmin = d.xmin + dx * (double)(float)0, ymin = d.ymin + dy * (double)(float)0,
           zmin = d.zmin + dz * (double)(float)0;
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
    update_halo({F_DENSITY0, F_ENERGY0, F_PRESSURE, F_VISCOSITY, F_DENSITY1, F_ENERGY1, F_XVEL0,
                 F_YVEL0, F_ZVEL0, F_XVEL1, F_YVEL1, F_ZVEL1}, 2);
    field_summary();
    return clover_gpu_status() == 0;
  }

  bool timestep() {  // timestep.f90:56-126
    dt = kGBig;
    ideal_gas(false);
    update_halo({F_PRESSURE, F_ENERGY0, F_DENSITY0, F_XVEL0, F_YVEL0}, 1);
    clover_viscosity_kernel(B, xarea.data(), yarea.data(), zarea.data(), celldx.data(),
                            celldy.data(), celldz.data(), density0.data(), pressure.data(),
                            viscosity.data(), xvel0.data(), yvel0.data(), zvel0.data());
    update_halo({F_VISCOSITY}, 1);
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
    const int32_t p = predict ? 1 : 0;
    clover_pdv_kernel(&p, B, &dt, xarea.data(), yarea.data(), zarea.data(), volume.data(),
                      density0.data(), density1.data(), energy0.data(), energy1.data(),
                      pressure.data(), viscosity.data(), xvel0.data(), xvel1.data(),
                      yvel0.data(), yvel1.data(), zvel0.data(), zvel1.data());
    if (predict) {
      ideal_gas(true);
      update_halo({F_PRESSURE}, 1);
      clover_revert_kernel(B, density0.data(), density1.data(), energy0.data(), energy1.data());
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
      clover_accelerate_kernel(B, &dt, xarea.data(), yarea.data(), zarea.data(), volume.data(),
                               density0.data(), pressure.data(), viscosity.data(), xvel0.data(),
                               yvel0.data(), zvel0.data(), xvel1.data(), yvel1.data(),
                               zvel1.data());
      pdv(false);
      clover_flux_calc_kernel(B, &dt, xarea.data(), yarea.data(), zarea.data(), xvel0.data(),
                              yvel0.data(), zvel0.data(), xvel1.data(), yvel1.data(),
                              zvel1.data(), vol_flux_x.data(), vol_flux_y.data(),
                              vol_flux_z.data());
      advection();
      clover_reset_field_kernel(B, density0.data(), density1.data(), energy0.data(),
                                energy1.data(), xvel0.data(), xvel1.data(), yvel0.data(),
                                yvel1.data(), zvel0.data(), zvel1.data());
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

}  // extern "C"
