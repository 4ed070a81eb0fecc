// Native chunk: the whole hydro cycle resident in HBM, dt/time/step on the
// device, one step replayed from a CUDA graph (one graph per sweep order).
// The same object holds an ensemble: many independent decks whose arrays
// share one allocation per field (each deck at its own offset), every
// kernel of the step launched once over all decks through a BatchPlan
// schedule, each deck with its own dt, time and calc_dt reduction.
// Also the deck reader (parse.f90 + read_input.f90 semantics).
#include <cctype>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <map>
#include <string>
#include <vector>

#include "../../include/clover_b200.h"
#include "../../include/clover_kernels.h"
#include <thread>

#include "clover_batch.h"
#include "clover_launch.h"
#include "clover_tma.cuh"
#include "clover_visit.h"

namespace clover {
namespace {

std::string g_last_error;

// data.f90:30-31 -- default-REAL literals assigned to REAL(8)
const double kGSmall = (double)1.0e-16f;
const double kGBig = (double)1.0e+21f;

// One thread per deck: the key of the calc_dt reduction starts at g_big.
__global__ void k_dt_prepare(DevScalars* sc, int nd, unsigned long long init) {
  const int d = blockIdx.x * blockDim.x + threadIdx.x;
  if (d < nd) sc[d].key = init;
}

// timestep.f90:90-126 after the calc_dt reduction, one thread per deck
__global__ void k_dt_finalize(DevScalars* scs, int nd, double* dt_hist) {
  const int d = blockIdx.x * blockDim.x + threadIdx.x;
  if (d >= nd) return;
  DevScalars* sc = scs + d;
  unsigned long long key = sc->key;
  unsigned long long b = (key >> 63) ? (key & 0x7fffffffffffffffull) : ~key;
  const double dtlp = __longlong_as_double((long long)b);
  double dt = kGBig;
  if (dtlp <= dt) dt = dtlp;
  double m = dt;
  const double r = sc->dtold * sc->dtrise;
  if (r < m) m = r;
  if (sc->dtmax < m) m = sc->dtmax;
  dt = m;
  if (dt < sc->dtmin) sc->status |= CLOVER_STATUS_SMALL_DT;
  sc->dt = dt;
  sc->dtold = dt;
  const int s = sc->step;
  if (s < sc->dt_cap) dt_hist[(long long)d * sc->dt_cap + s] = dt;
  sc->step = s + 1;
}

// hydro.f90:68, one thread per deck
__global__ void k_step_end(DevScalars* sc, int nd) {
  const int d = blockIdx.x * blockDim.x + threadIdx.x;
  if (d < nd) sc[d].time = sc[d].time + sc[d].dt;
}

struct Owned {
  void* p;
  size_t bytes;
};

// One 3D array for all decks (elems after the front pad), zeroed.
template <class T>
T* alloc_field(long long elems, std::vector<Owned>& owned, long long& bytes, cudaStream_t s) {
  void* raw = nullptr;
  const size_t n = (size_t)(elems + kFrontPad<T>) * sizeof(T);
  if (cudaMalloc(&raw, n) != cudaSuccess) return nullptr;
  cudaMemsetAsync(raw, 0, n, s);
  owned.push_back(Owned{raw, n});
  bytes += (long long)n;
  return (T*)raw + kFrontPad<T>;
}

double* alloc_1d(long long n, std::vector<Owned>& owned, long long& bytes, cudaStream_t s) {
  void* raw = nullptr;
  const size_t sz = (size_t)(n + 32) * sizeof(double);
  if (cudaMalloc(&raw, sz) != cudaSuccess) return nullptr;
  cudaMemsetAsync(raw, 0, sz, s);
  owned.push_back(Owned{raw, sz});
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
  using ND = typename S::nd_t;

  clover_deck deck;                // deck 0: summary cadence and end step of all decks
  Geom g;                          // deck 0's geometry (the whole chunk when nd == 1)
  std::vector<clover_deck> decks;  // every deck
  std::vector<Geom> geoms;         // every deck, with its offsets in the shared arrays
  int nd = 1;
  BatchPlan* plan = nullptr;       // ensemble: the schedules of the batched launches
  Target tg{Geom{}};               // where the step's launchers run
  bool warm[2] = {false, false};   // a step of each sweep order ran since the schedules changed
  cudaStream_t stream = nullptr;
  std::vector<Owned> owned;
  long long bytes = 0;

  R *density0, *density1;
  En *energy0, *energy1;
  C *pressure, *viscosity, *soundspeed;
  V *xvel0, *xvel1, *yvel0, *yvel1, *zvel0, *zvel1;
  V* vel1b[3];  // second buffer of each time-level-1 velocity (fused step)
  R* rho1b;     // second buffer of density1 and energy1 (the fused x cell sweep
  En* e1b;      // writes out of place)
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
  int* plane_base = nullptr;  // ensemble: first summary plane of each deck (nd + 1)

  double cell_volume = 0.0;  // dx*dy*dz, the volume of every cell (initialise_chunk)
  int host_step = 0;     // steps enqueued
  bool advect_x = true;  // start.f90:99
  bool use_graphs = true;
  bool fused = true;  // fused kernels (clover_fused.cu) instead of one kernel per reference pass
  // one chunk: stencils staged through shared memory by bulk-tensor copies
  // (clover_tma.cu) where their tensor maps could be made; their
  // register-marching forms otherwise, and for ensembles
  bool tma = false;
  bool use_tma = true;
  ViscMaps visc_maps;
  // tensor maps of the arrays the staged kernels read, by (array, box rows
  // and orientation): both buffers of the density1 and velocity pairs occur
  std::map<std::pair<const void*, int>, CUtensorMap> tmaps;
  bool tmap(const void* base, int elem_bytes, int rows, CUtensorMap* out, bool zrows = false) {
    const auto key = std::make_pair(base, 2 * rows + (zrows ? 1 : 0));
    auto it = tmaps.find(key);
    if (it == tmaps.end()) {
      CUtensorMap m;
      if (!encode_plane_map(&m, base, elem_bytes, g, rows, zrows)) return false;
      it = tmaps.emplace(key, m).first;
    }
    *out = it->second;
    return true;
  }
  // the maps of the x momentum sweep reading density1 buffer rho and the
  // velocity buffers vin
  // the maps of the y (dir 2) or z (dir 3) node pass reading density1 buffer
  // rho, with the post-volume variant of the sweep
  bool mom_node_maps(int dir, int var, const R* rho, NodeMaps* m) {
    const bool zr = dir == 2;  // the y sweep's planes are x-z slices
    bool ok = tmap(dir == 2 ? (const void*)mass_flux_y : (const void*)mass_flux_z, sizeof(MF), 9,
                   &m->mf, zr) &&
              tmap(rho, sizeof(R), 9, &m->d, zr);
    if (ok && (var == 1 || var == 3)) ok = tmap(vol_flux_x, sizeof(VF), 9, &m->vfx, zr);
    if (ok && var == 1) ok = tmap(vol_flux_y, sizeof(VF), 10, &m->vfr, false);
    if (ok && var == 2) ok = tmap(vol_flux_z, sizeof(VF), 10, &m->vfr, true);
    return ok;
  }
  // the maps of the y (dir 2) or z (dir 3) velocity pass: the node arrays in
  // work[0..2] (as nd_t) and the velocity buffers vin
  bool mom_vel_maps(int dir, V* const* vin, VelMaps* m) {
    const bool zr = dir == 2;
    return tmap(nd_array<S>(work[0]), sizeof(ND), 8, &m->nf, zr) &&
           tmap(nd_array<S>(work[2]), sizeof(ND), 8, &m->pre, zr) &&
           tmap(nd_array<S>(work[1]), sizeof(ND), 8, &m->post, zr) &&
           tmap(vin[0], sizeof(V), 8, &m->u, zr) &&
           tmap(vin[1], sizeof(V), 8, &m->v, zr) && tmap(vin[2], sizeof(V), 8, &m->w, zr);
  }
  // the maps of the staged y (dir 2) or z (dir 3) cell sweep reading buffer cb
  // of the density1/energy1 pair, with pre-volume variant var
  // the maps of the staged x cell sweep of sweep 1 or 3 reading buffer cb of
  // the density1/energy1 pair
  bool cell_x_maps(int sweep, int cb, CellXMaps* m) {
    bool ok = tmap(rho1(cb), sizeof(R), 8, &m->d) && tmap(ene1(cb), sizeof(En), 8, &m->e) &&
              tmap(vol_flux_x, sizeof(VF), 8, &m->vfx);
    if (ok && sweep == 1)
      ok = tmap(vol_flux_y, sizeof(VF), 9, &m->vfy) && tmap(vol_flux_z, sizeof(VF), 8, &m->vfz);
    return ok;
  }
  bool cell_maps(int dir, int var, int cb, CellMaps* m) {
    const bool zr = dir == 2;
    bool ok = tmap(rho1(cb), sizeof(R), 8, &m->d, zr) && tmap(ene1(cb), sizeof(En), 8, &m->e, zr) &&
              tmap(dir == 2 ? (const void*)vol_flux_y : (const void*)vol_flux_z, sizeof(VF), 8,
                   &m->vfd, zr);
    if (ok && (var == 3 || var == 4)) ok = tmap(vol_flux_x, sizeof(VF), 8, &m->vfx, zr);
    if (ok && var == 2) ok = tmap(vol_flux_z, sizeof(VF), 9, &m->vfr, true);
    if (ok && var == 4) ok = tmap(vol_flux_y, sizeof(VF), 9, &m->vfr, false);
    return ok;
  }
  bool mom_x_maps(const R* rho, V* const* vin, MomXMaps* m) {
    return tmap(mass_flux_x, sizeof(MF), 9, &m->mf) && tmap(rho, sizeof(R), 9, &m->d) &&
           tmap(vol_flux_y, sizeof(VF), 10, &m->vfy) && tmap(vol_flux_z, sizeof(VF), 9, &m->vfz) &&
           tmap(vin[0], sizeof(V), 8, &m->u) && tmap(vin[1], sizeof(V), 8, &m->v) &&
           tmap(vin[2], sizeof(V), 8, &m->w);
  }
  // Every axis of every deck has at least three cells. A repeated halo update
  // of a cell field, a vertex velocity or a z-face flux, whose values have
  // not changed since its last update at the same depth, then rewrites every
  // halo cell with the value it holds (update_halo_kernel.f90 is idempotent
  // for those fields on such grids; not for the x- and y-face fluxes, whose
  // far halo corners keep values read before a later face pass wrote them),
  // so the fused step leaves such repeats out. A depth-2 update of those
  // fields also rewrites every halo cell from the interior whatever it held,
  // so the shell copies of the out-of-place sweeps are left out where one
  // follows before the shell is read.
  bool halo_repeat_free = false;
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
    double n = 0.0;
    for (const Geom& q : geoms)
      n += (double)(q.x_max - q.x_min + 1) * (q.y_max - q.y_min + 1) * (q.z_max - q.z_min + 1);
    return n;
  }

  // time-level-1 velocity c (0 x, 1 y, 2 z) in buffer b of its pair
  V* vel1(int c, int b) const {
    V* a[3] = {xvel1, yvel1, zvel1};
    return b ? vel1b[c] : a[c];
  }
  // the buffer holding time level 1 velocities after `steps` fused steps:
  // each step flips the pair three times (one per sweep)
  int vel1_buffer(int steps) const { return fused ? steps % 2 : 0; }
  // density1/energy1 pair b, and the buffer holding them after `steps` fused
  // steps: the out-of-place cell sweeps flip it an odd number of times per
  // step (the x sweep; with the staged y/z sweeps, all three)
  R* rho1(int b) const { return b ? rho1b : density1; }
  En* ene1(int b) const { return b ? e1b : energy1; }
  int cell_buffer(int steps) const { return fused ? steps % 2 : 0; }

  HaloFields halo_fields(int vb, int cb) {
    HaloFields h;
    void* f[19] = {density0, rho1(cb), energy0, ene1(cb), pressure, viscosity, soundspeed,
                   xvel0, vel1(0, vb), yvel0, vel1(1, vb), zvel0, vel1(2, vb), vol_flux_x,
                   vol_flux_y, vol_flux_z, mass_flux_x, mass_flux_y, mass_flux_z};
    for (int i = 0; i < 19; i++) h.f[i] = f[i];
    return h;
  }

  void halo(std::initializer_list<int> ids, int depth, int vb = 0, int cb = 0) {
    int fields[19] = {0};
    for (int id : ids) fields[id - 1] = 1;
    launch_update_halo<S>(tg, stream, halo_fields(vb, cb), fields, depth, ext);
  }

  int deck_blocks() const { return (nd + 127) / 128; }

  // Allocate the shared arrays of the decks (batched: launch every kernel
  // over all decks through a plan, even for one deck) and set them up.
  bool create(const clover_deck* ds, int n, bool batched) {
    decks.assign(ds, ds + n);
    nd = n;
    deck = decks[0];
    long long total3 = 0, total1 = 0;
    for (int d = 0; d < nd; d++) {
      const clover_deck& dk = decks[d];
      Geom q = make_geom(1, dk.x_cells, 1, dk.y_cells, 1, dk.z_cells);
      // initialise_chunk.f90:38-46 and initialise_chunk_kernel.f90:113-175
      const double dx = (dk.xmax - dk.xmin) / (double)(float)dk.x_cells;
      const double dy = (dk.ymax - dk.ymin) / (double)(float)dk.y_cells;
      const double dz = (dk.zmax - dk.zmin) / (double)(float)dk.z_cells;
      q.vol = dx * dy * dz;
      q.xa = dy * dz;
      q.ya = dx * dz;
      q.za = dx * dy;
      // the kernels' min(celldx, celldy, celldz) takes b when b < a
      auto mn = [](auto a, auto b) { return b < a ? b : a; };
      const double mcd = mn(mn(dx, dy), dz);
      const float mcd_f = mn(mn((float)dx, (float)dy), (float)dz);
      q.rvol = 1.0 / q.vol;
      q.rvol_f = 1.0f / (float)q.vol;
      q.ds = 1.0 / (mcd * mcd);
      q.ds_f = 1.0f / (mcd_f * mcd_f);
      q.o3 = total3;
      q.o1 = (int)total1;
      total3 += array_elems(q);
      total1 += array1d_elems(q);
      geoms.push_back(q);
    }
    g = geoms[0];
    halo_repeat_free = true;
    for (int d = 0; d < nd; d++)
      if (decks[d].x_cells < 3 || decks[d].y_cells < 3 || decks[d].z_cells < 3)
        halo_repeat_free = false;
    if (cudaStreamCreateWithFlags(&stream, cudaStreamNonBlocking) != cudaSuccess) return false;
    if (batched) {
      plan = new BatchPlan;
      if (!plan->init(geoms)) {
        g_last_error = "device allocation failed";
        return false;
      }
      tg = Target(plan);
      fused = true;  // the batched step is the fused one
    } else {
      tg = Target(g);
    }
    bool ok = true;
    auto chk = [&](const void* p) { ok = ok && p != nullptr; };
    const long long e3 = total3;
    chk(density0 = alloc_field<R>(e3, owned, bytes, stream));
    chk(density1 = alloc_field<R>(e3, owned, bytes, stream));
    chk(energy0 = alloc_field<En>(e3, owned, bytes, stream));
    chk(energy1 = alloc_field<En>(e3, owned, bytes, stream));
    chk(pressure = alloc_field<C>(e3, owned, bytes, stream));
    chk(viscosity = alloc_field<C>(e3, owned, bytes, stream));
    chk(soundspeed = alloc_field<C>(e3, owned, bytes, stream));
    chk(xvel0 = alloc_field<V>(e3, owned, bytes, stream));
    chk(xvel1 = alloc_field<V>(e3, owned, bytes, stream));
    chk(yvel0 = alloc_field<V>(e3, owned, bytes, stream));
    chk(yvel1 = alloc_field<V>(e3, owned, bytes, stream));
    chk(zvel0 = alloc_field<V>(e3, owned, bytes, stream));
    chk(zvel1 = alloc_field<V>(e3, owned, bytes, stream));
    for (int c3 = 0; c3 < 3; c3++) chk(vel1b[c3] = alloc_field<V>(e3, owned, bytes, stream));
    chk(rho1b = alloc_field<R>(e3, owned, bytes, stream));
    chk(e1b = alloc_field<En>(e3, owned, bytes, stream));
    chk(vol_flux_x = alloc_field<VF>(e3, owned, bytes, stream));
    chk(vol_flux_y = alloc_field<VF>(e3, owned, bytes, stream));
    chk(vol_flux_z = alloc_field<VF>(e3, owned, bytes, stream));
    chk(mass_flux_x = alloc_field<MF>(e3, owned, bytes, stream));
    chk(mass_flux_y = alloc_field<MF>(e3, owned, bytes, stream));
    chk(mass_flux_z = alloc_field<MF>(e3, owned, bytes, stream));
    for (int i = 0; i < 7; i++) chk(work[i] = alloc_field<W>(e3, owned, bytes, stream));
    chk(volume = alloc_field<double>(e3, owned, bytes, stream));
    chk(xarea = alloc_field<double>(e3, owned, bytes, stream));
    chk(yarea = alloc_field<double>(e3, owned, bytes, stream));
    chk(zarea = alloc_field<double>(e3, owned, bytes, stream));
    double** one_d[12] = {&cellx, &celly, &cellz, &celldx, &celldy, &celldz,
                          &vertexx, &vertexy, &vertexz, &vertexdx, &vertexdy, &vertexdz};
    for (double** a : one_d) chk(*a = alloc_1d(total1, owned, bytes, stream));
    if (!ok) {
      g_last_error = "device allocation failed";
      return false;
    }
    ga = GeomArrays{volume, xarea, yarea, zarea, cellx, celly, cellz, celldx, celldy, celldz,
                    vertexx, vertexy, vertexz, vertexdx, vertexdy, vertexdz};
    // one chunk: the stencils that stage their planes with bulk-tensor copies
    // get their tensor maps (the arrays they read never move)
    if (!batched)
      tma = visc_dt_tma_prepare<S>() && mom_x_tma_prepare<S>() && stencils_tma_prepare<S>() &&
            mom_node_tma_prepare<S>() && mom_vel_tma_prepare<S>() && cell_sweep_tma_prepare<S>() &&
            cell_sweep_x_tma_prepare<S>() &&
            visc_dt_tma_maps<S>(g, xvel0, yvel0, zvel0, density0, energy0, &visc_maps);
    // by default the staged forms only where a launch has blocks to fill the
    // GPU (32 x 8 columns by 32 planes each: at least four per SM); on smaller
    // chunks (the measured 24..128-cell decks) the register-marching forms are
    // faster. clover_chunk_use_tma chooses either way; both give the same bits.
    {
      const long long blocks = (long long)((g.x_max - g.x_min + 32) / 32) *
                               ((g.y_max - g.y_min + 8) / 8) * ((g.z_max - g.z_min + 32) / 32);
      use_tma = blocks >= 4 * 148;
    }

    dt_cap = deck.end_step < (1 << 22) ? deck.end_step + 16 : (1 << 22);
    sum_cap = dt_cap / (deck.summary_frequency > 0 ? deck.summary_frequency : dt_cap) + 8;
    int planes = 0;
    std::vector<int> pb(nd + 1, 0);
    for (int d = 0; d < nd; d++) {
      pb[d] = planes;
      planes += geoms[d].z_max - geoms[d].z_min + 1;
    }
    pb[nd] = planes;
    void* p = nullptr;
    ok = cudaMalloc(&p, (size_t)nd * sizeof(DevScalars)) == cudaSuccess;
    sc = (DevScalars*)p;
    ok = ok && cudaMalloc(&p, (size_t)nd * dt_cap * sizeof(double)) == cudaSuccess;
    dt_hist = (double*)p;
    ok = ok && cudaMalloc(&p, (size_t)nd * sum_cap * 5 * sizeof(double)) == cudaSuccess;
    sum_hist = (double*)p;
    // per plane (ensemble) or per block: five sums and their five compensations
    const size_t np = plan ? (size_t)planes * 10 : (size_t)summary_partials_len();
    ok = ok && cudaMalloc(&p, np * sizeof(double)) == cudaSuccess;
    partials = (double*)p;
    if (ok && plan) {
      ok = cudaMalloc(&p, pb.size() * sizeof(int)) == cudaSuccess;
      plane_base = (int*)p;
      // on the chunk's stream and waited for: pb is released at return
      ok = ok && cudaMemcpyAsync(plane_base, pb.data(), pb.size() * sizeof(int),
                                 cudaMemcpyHostToDevice, stream) == cudaSuccess &&
           cudaStreamSynchronize(stream) == cudaSuccess;
    }
    if (!ok) {
      g_last_error = "device allocation failed";
      return false;
    }
    const clover_deck& d = deck;
    const double dx = (d.xmax - d.xmin) / (double)(float)d.x_cells;
    const double dy = (d.ymax - d.ymin) / (double)(float)d.y_cells;
    const double dz = (d.zmax - d.zmin) / (double)(float)d.z_cells;
    cell_volume = dx * dy * dz;  // initialise_chunk_kernel.f90:155 (deck 0)
    return initial_state();
  }

  // start.f90:49-136 for every deck on the device: scalars, geometry,
  // generated state, EOS, halos and the step-0 summary. The arrays must hold
  // zeros (fresh allocation or reset()).
  bool initial_state() {
    std::vector<DevScalars> h(nd);
    for (int i = 0; i < nd; i++) {
      h[i] = DevScalars{};
      h[i].dt = decks[i].initial_timestep;     // start.f90:51-52
      h[i].dtold = decks[i].initial_timestep;
      h[i].time = 0.0;
      h[i].step = 0;
      h[i].dt_cap = dt_cap;
      h[i].dtrise = decks[i].timestep_rise;
      h[i].dtmax = decks[i].max_timestep;
      h[i].dtmin = decks[i].dtmin;
    }
    cudaMemcpyAsync(sc, h.data(), (size_t)nd * sizeof(DevScalars), cudaMemcpyHostToDevice, stream);
    cudaStreamSynchronize(stream);  // h is released at return
    for (int i = 0; i < nd; i++) {
      const clover_deck& d = decks[i];
      const Geom& q = geoms[i];
      // initialise_chunk.f90:38-46
      const double dx = (d.xmax - d.xmin) / (double)(float)d.x_cells;
      const double dy = (d.ymax - d.ymin) / (double)(float)d.y_cells;
      const double dz = (d.zmax - d.zmin) / (double)(float)d.z_cells;
      const double xmin = d.xmin + dx * (double)(float)0;
      const double ymin = d.ymin + dy * (double)(float)0;
      const double zmin = d.zmin + dz * (double)(float)0;
      launch_initialise_chunk(q, stream, xmin, ymin, zmin, dx, dy, dz, vertexx, vertexdx,
                              vertexy, vertexdy, vertexz, vertexdz, cellx, celldx, celly, celldy,
                              cellz, celldz, volume, xarea, yarea, zarea);
      // read_input.f90:293-303 nudge, then generate_chunk
      StateTable st;
      st.n = d.number_of_states;
      for (int k = 0; k < st.n; k++) {
        st.density[k] = d.state_density[k]; st.energy[k] = d.state_energy[k];
        st.xvel[k] = d.state_xvel[k]; st.yvel[k] = d.state_yvel[k]; st.zvel[k] = d.state_zvel[k];
        st.xmin[k] = d.state_xmin[k]; st.xmax[k] = d.state_xmax[k];
        st.ymin[k] = d.state_ymin[k]; st.ymax[k] = d.state_ymax[k];
        st.zmin[k] = d.state_zmin[k]; st.zmax[k] = d.state_zmax[k];
        st.radius[k] = d.state_radius[k];
        st.geometry[k] = d.state_geometry[k];
        if (k >= 1) {
          st.xmin[k] = st.xmin[k] + (dx / 100.0);
          st.ymin[k] = st.ymin[k] + (dy / 100.0);
          st.zmin[k] = st.zmin[k] + (dz / 100.0);
          st.xmax[k] = st.xmax[k] - (dx / 100.0);
          st.ymax[k] = st.ymax[k] - (dy / 100.0);
          st.zmax[k] = st.zmax[k] - (dz / 100.0);
        }
      }
      launch_generate_chunk<S>(q, stream, ga, density0, energy0, xvel0, yvel0, zvel0, st);
    }
    // start.f90:109-136
    launch_ideal_gas<S>(tg, stream, density0, energy0, pressure, soundspeed);
    halo({1, 3, 5, 6, 2, 4, 8, 10, 12, 9, 11, 13}, 2);
    host_step = 0;
    advect_x = true;
    sum_steps.clear();
    summary(0);
    // start.f90:138: written before the first step (so that the output
    // directory can be set after creation)
    visit_pending = deck.visit_frequency != 0;
    if (cudaStreamSynchronize(stream) != cudaSuccess || cudaGetLastError() != cudaSuccess ||
        (plan && plan->failed)) {
      g_last_error = "chunk set-up failed on the device";
      return false;
    }
    return true;
  }

  // Checkpoint file: a header (format tag, precision, decks, step state and
  // the sizes of every device allocation), the device scalars, dt and summary
  // histories, then every device allocation byte for byte. A restore needs a
  // chunk made from the same decks and precision; it replaces the whole
  // device state, so the continued run is bit-identical to an uninterrupted
  // one.
  struct CkptHeader {
    char tag[8];
    int version, precision, nd, host_step, advect_x, fused, n_owned, n_sum, dt_cap, sum_cap;
  };
  static constexpr const char* kCkptTag = "CLVCKPT";

  CkptHeader ckpt_header() const {
    CkptHeader h{};
    memcpy(h.tag, kCkptTag, 8);
    h.version = 1;
    h.precision = sizeof(V) == 8 ? CLOVER_PRECISION_FP64 : CLOVER_PRECISION_MIXED;
    h.nd = nd;
    h.host_step = host_step;
    h.advect_x = advect_x ? 1 : 0;
    h.fused = fused ? 1 : 0;
    h.n_owned = (int)owned.size();
    h.n_sum = (int)sum_steps.size();
    h.dt_cap = dt_cap;
    h.sum_cap = sum_cap;
    return h;
  }

  // device <-> file through a bounded host buffer
  static bool dev_to_file(FILE* f, const void* d, size_t n, std::vector<char>& buf) {
    for (size_t o = 0; o < n; o += buf.size()) {
      const size_t c = n - o < buf.size() ? n - o : buf.size();
      if (cudaMemcpy(buf.data(), (const char*)d + o, c, cudaMemcpyDeviceToHost) != cudaSuccess)
        return false;
      if (fwrite(buf.data(), 1, c, f) != c) return false;
    }
    return true;
  }
  static bool file_to_dev(FILE* f, void* d, size_t n, std::vector<char>& buf) {
    for (size_t o = 0; o < n; o += buf.size()) {
      const size_t c = n - o < buf.size() ? n - o : buf.size();
      if (fread(buf.data(), 1, c, f) != c) return false;
      if (cudaMemcpy((char*)d + o, buf.data(), c, cudaMemcpyHostToDevice) != cudaSuccess)
        return false;
    }
    return true;
  }

  int checkpoint(const char* path) {
    if (cudaStreamSynchronize(stream) != cudaSuccess) return -1;
    FILE* f = fopen(path, "wb");
    if (!f) return -2;
    const CkptHeader h = ckpt_header();
    bool ok = fwrite(&h, sizeof(h), 1, f) == 1;
    ok = ok && fwrite(decks.data(), sizeof(clover_deck), (size_t)nd, f) == (size_t)nd;
    for (const Owned& o : owned) ok = ok && fwrite(&o.bytes, sizeof(o.bytes), 1, f) == 1;
    if (h.n_sum > 0)
      ok = ok && fwrite(sum_steps.data(), sizeof(int), (size_t)h.n_sum, f) == (size_t)h.n_sum;
    std::vector<char> buf((size_t)64 << 20);
    ok = ok && dev_to_file(f, sc, (size_t)nd * sizeof(DevScalars), buf);
    ok = ok && dev_to_file(f, dt_hist, (size_t)nd * dt_cap * sizeof(double), buf);
    ok = ok && dev_to_file(f, sum_hist, (size_t)nd * sum_cap * 5 * sizeof(double), buf);
    for (const Owned& o : owned) ok = ok && dev_to_file(f, o.p, o.bytes, buf);
    ok = (fclose(f) == 0) && ok;
    return ok ? 0 : -3;
  }

  int restore(const char* path) {
    if (cudaStreamSynchronize(stream) != cudaSuccess) return -1;
    FILE* f = fopen(path, "rb");
    if (!f) return -2;
    CkptHeader h{};
    const CkptHeader mine = ckpt_header();
    bool ok = fread(&h, sizeof(h), 1, f) == 1 && memcmp(h.tag, kCkptTag, 8) == 0 &&
              h.version == 1 && h.precision == mine.precision && h.nd == nd &&
              h.n_owned == mine.n_owned && h.dt_cap == dt_cap && h.sum_cap == sum_cap &&
              h.n_sum >= 0 && h.n_sum <= sum_cap;
    std::vector<clover_deck> ds(ok ? (size_t)nd : 0);
    ok = ok && fread(ds.data(), sizeof(clover_deck), (size_t)nd, f) == (size_t)nd &&
         memcmp(ds.data(), decks.data(), (size_t)nd * sizeof(clover_deck)) == 0;
    for (const Owned& o : owned) {
      size_t b = 0;
      ok = ok && fread(&b, sizeof(b), 1, f) == 1 && b == o.bytes;
    }
    std::vector<int> ss(ok ? (size_t)h.n_sum : 0);
    if (ok && h.n_sum > 0) ok = fread(ss.data(), sizeof(int), (size_t)h.n_sum, f) == (size_t)h.n_sum;
    if (!ok) {
      fclose(f);
      g_last_error = "checkpoint does not match this chunk (decks, precision or sizes)";
      return -4;
    }
    std::vector<char> buf((size_t)64 << 20);
    ok = file_to_dev(f, sc, (size_t)nd * sizeof(DevScalars), buf);
    ok = ok && file_to_dev(f, dt_hist, (size_t)nd * dt_cap * sizeof(double), buf);
    ok = ok && file_to_dev(f, sum_hist, (size_t)nd * sum_cap * 5 * sizeof(double), buf);
    for (const Owned& o : owned) ok = ok && file_to_dev(f, o.p, o.bytes, buf);
    fclose(f);
    if (!ok) {
      g_last_error = "checkpoint read failed";
      return -5;
    }
    drop_graphs();
    host_step = h.host_step;
    advect_x = h.advect_x != 0;
    fused = h.fused != 0;
    sum_steps = ss;
    return 0;
  }

  // visit.f90: ideal_gas, the halos of pressure and the velocities, the
  // viscosity, then the fields of every deck copied to the host and written
  // as VTK by a writer thread (the previous frame's writer is joined first).
  // None of this changes the run: each step recomputes these fields.
  std::string visit_dir = ".";
  bool visit_pending = false;  // the step-0 frame is still to be written
  std::thread visit_writer;
  bool visit_first = true;
  std::string visit_error;
  bool visit_failed = false;

  void visit_join() {
    if (visit_writer.joinable()) visit_writer.join();
  }

  int visit() {
    launch_ideal_gas<S>(tg, stream, density0, energy0, pressure, soundspeed);
    halo({5, 8, 10, 12}, 1, vel1_buffer(host_step), cell_buffer(host_step));
    for (int d = 0; d < nd; d++)
      launch_viscosity<S>(geoms[d], stream, ga, density0, pressure, viscosity, xvel0, yvel0, zvel0);
    if (cudaStreamSynchronize(stream) != cudaSuccess) return -1;
    VisitFrame fr;
    fr.dir = visit_dir;
    fr.step = host_step;
    fr.first = visit_first;
    for (int d = 0; d < nd; d++) {
      const Geom& q = geoms[d];
      VisitChunk c;
      c.chunk = d + 1;
      c.nx = q.x_max - q.x_min + 1;
      c.ny = q.y_max - q.y_min + 1;
      c.nz = q.z_max - q.z_min + 1;
      const size_t nc = (size_t)(c.nx + 4) * (c.ny + 4) * (c.nz + 4);
      const size_t nv = (size_t)(c.nx + 5) * (c.ny + 5) * (c.nz + 5);
      std::vector<double>* f[7] = {&c.density0, &c.energy0, &c.pressure, &c.viscosity,
                                   &c.xvel0, &c.yvel0, &c.zvel0};
      const int ids[7] = {1, 3, 5, 6, 8, 10, 12};
      for (int i = 0; i < 7; i++) {
        f[i]->resize(i < 4 ? nc : nv);
        if (read_field(ids[i], f[i]->data(), false, d) != 0) return -1;
      }
      const int n1[3] = {c.nx + 1, c.ny + 1, c.nz + 1};
      const double* v1[3] = {vertexx, vertexy, vertexz};
      std::vector<double>* h1[3] = {&c.vertexx, &c.vertexy, &c.vertexz};
      for (int a = 0; a < 3; a++) {
        h1[a]->resize(n1[a]);
        // vertex j = min (index 2 from min-2) .. max+1
        if (cudaMemcpy(h1[a]->data(), v1[a] + q.o1 + 2, (size_t)n1[a] * sizeof(double),
                       cudaMemcpyDeviceToHost) != cudaSuccess)
          return -1;
      }
      fr.chunks.push_back(std::move(c));
    }
    visit_join();
    if (visit_failed) return -2;
    visit_first = false;
    visit_writer = std::thread([this, fr]() {
      std::string err;
      if (!write_visit_frame(fr, &err)) {
        visit_error = err;
        visit_failed = true;
      }
    });
    return 0;
  }

  bool drop_graphs() {
    cudaStreamSynchronize(stream);
    for (auto& gr : graph)
      if (gr) { cudaGraphExecDestroy(gr); gr = nullptr; }
    warm[0] = warm[1] = false;
    return true;
  }

  // Zero every array and set the decks up again (after autotuning, whose
  // trial steps advance the state). The schedules stay; the graphs are
  // captured again.
  bool reset() {
    cudaStreamSynchronize(stream);
    for (auto& gr : graph)
      if (gr) { cudaGraphExecDestroy(gr); gr = nullptr; }
    for (const Owned& o : owned) cudaMemsetAsync(o.p, 0, o.bytes, stream);
    warm[0] = warm[1] = false;
    return initial_state();
  }

  // The autotuner: per batched launch (key), the item order and grid size,
  // then the segment length of the marching kernels, that run fastest. Each
  // candidate runs one untimed and trial_steps timed eager steps with every
  // batched launch bracketed by events; the fastest candidate per key is
  // kept. Trial steps advance the decks, so the ensemble is reset to its
  // initial state afterwards. Results do not depend on the schedule.
  int autotune(int trial_steps) {
    if (!plan) return -1;
    if (trial_steps < 1) trial_steps = 1;
    const bool prof = profile;
    profile = false;
    plan->timing = true;
    std::map<unsigned, std::pair<double, SchedCfg>> best;
    auto trial = [&](SchedCfg c) {
      plan->trial = c;
      plan->trial_active = true;
      step(1);
      cudaStreamSynchronize(stream);
      plan->collect_marks();
      step(trial_steps);
      for (auto& kv : plan->collect_marks()) {
        const SchedCfg eff = plan->cfg_for(kv.first);
        auto it = best.find(kv.first);
        if (it == best.end() || kv.second < it->second.first) best[kv.first] = {kv.second, eff};
      }
    };
    const int orders[3] = {0, 1, 2}, divs[4] = {0, 1, 2, 4}, segs[4] = {8, 16, 32, 64};
    for (int o : orders)
      for (int dv : divs) trial(SchedCfg{o, dv, -1});
    for (auto& kv : best) plan->tuned[kv.first] = kv.second.second;
    for (int sg : segs) trial(SchedCfg{-1, -1, sg});
    for (auto& kv : best) plan->tuned[kv.first] = kv.second.second;
    plan->trial_active = false;
    plan->timing = false;
    profile = prof;
    const bool ok = reset() && !plan->failed;
    return ok ? (int)plan->tuned.size() : -1;
  }

  // One line per batched launch: key, order, grid divisor, segment, blocks,
  // items.
  std::string schedule_report() const {
    std::string out;
    if (!plan) return out;
    for (auto& kv : plan->seg_tunable) {
      const SchedCfg c = plan->cfg_for(kv.first);
      int grid = 0, n = 0, a = 0;
      for (auto& e : plan->cache)
        if ((unsigned)e.first[0] == kv.first && e.first[1] == c.order && e.first[2] == c.grid_div &&
            (!kv.second || c.seg <= 0 || e.first[3] == c.seg)) {
          grid = e.second.grid; n = e.second.n; a = e.second.aux;
        }
      char line[160];
      snprintf(line, sizeof(line), "%u %d %d %d %d %d\n", kv.first, c.order, c.grid_div,
               kv.second ? a : 0, grid, n);
      out += line;
    }
    return out;
  }

  // field_summary.f90:55-108, recorded at the given step
  void summary(int step) {
    const int idx = (int)sum_steps.size();
    if (idx >= sum_cap) return;
    pbeg();
    launch_ideal_gas<S>(tg, stream, density0, energy0, pressure, soundspeed);
    if (plan)
      launch_field_summary_batch<S>(plan, nd, stream, plane_base, volume, density0, energy0,
                                    pressure, xvel0, yvel0, zvel0, partials,
                                    sum_hist + (size_t)5 * nd * idx);
    else
      launch_field_summary<S>(g, stream, volume, density0, energy0, pressure, xvel0, yvel0,
                              zvel0, partials, sum_hist + 5 * idx);
    pend("field_summary", cells() * (2 * sizeof(R) + 2 * sizeof(En) + 3 * sizeof(C) +
                                     sizeof(double) + 3 * sizeof(V)));
    sum_steps.push_back(step);
  }

  // One hydro step with the fused kernels (same results, bit for bit).
  void enqueue_step_fused(bool ax) {
    const double* dtp = &sc->dt;
    const double n = cells();
    const double R8 = sizeof(R), E8 = sizeof(En), C8 = sizeof(C), V8 = sizeof(V),
                 VF8 = sizeof(VF), MF8 = sizeof(MF), N8 = sizeof(ND);
    int vc = ax ? 0 : 1;  // buffer of the velocity pairs at the start of this step
    int cb = ax ? 0 : 1;  // buffer of the density1/energy1 pair at the start of this step
    // timestep.f90:56-126
    k_dt_prepare<<<deck_blocks(), 128, 0, stream>>>(sc, nd, min_key_of(kGBig));
    // ideal_gas runs inside the viscosity/calc_dt kernel: it stores every
    // cell's pressure and sound speed and forms the neighbours' pressures
    // from density0/energy0, whose halo is updated first. The step-start
    // update of the pressure's halo is left out: the depth-1 update after the
    // predictor rewrites the same cells before anything reads them.
    pbeg();
    halo({3, 1, 8, 10}, 1, vc, cb);
    pend("update_halo", 0);
    pbeg();
    if (tma && use_tma)
      launch_visc_dt_tma<S>(g, stream, visc_maps, ga, kGSmall, deck.dtc_safe, deck.dtu_safe,
                            deck.dtv_safe, deck.dtw_safe, deck.dtdiv_safe, pressure, viscosity,
                            soundspeed, &sc->key, &sc->status);
    else
      launch_visc_dt<S>(tg, stream, ga, kGSmall, deck.dtc_safe, deck.dtu_safe, deck.dtv_safe,
                        deck.dtw_safe, deck.dtdiv_safe, density0, energy0, pressure, viscosity,
                        soundspeed, xvel0, yvel0, zvel0, &sc->key);
    k_dt_finalize<<<deck_blocks(), 128, 0, stream>>>(sc, nd, dt_hist);
    pend("eos_viscosity_calc_dt", n * (3 * V8 + R8 + E8 + 3 * C8));
    pbeg();
    halo({6}, 1, vc, cb);  // read by accelerate at its neighbours
    pend("update_halo", 0);
    // PdV.f90:50-107: predictor + EOS on the predicted state; revert is implied
    pbeg();
    PdvMaps pdv_m;
    if (tma && use_tma && tmap(xvel0, sizeof(V), 9, &pdv_m.u) && tmap(yvel0, sizeof(V), 9, &pdv_m.v) &&
        tmap(zvel0, sizeof(V), 9, &pdv_m.w) && tmap(density0, sizeof(R), 8, &pdv_m.d) &&
        tmap(energy0, sizeof(En), 8, &pdv_m.e) && tmap(pressure, sizeof(C), 8, &pdv_m.p) &&
        tmap(viscosity, sizeof(C), 8, &pdv_m.q))
      launch_pdv_predict_eos_tma<S>(g, stream, dtp, pdv_m, pressure, &sc->status);
    else
      launch_pdv_predict_eos<S>(tg, stream, dtp, ga, density0, energy0, pressure, viscosity, xvel0,
                                yvel0, zvel0);
    pend("pdv", n * (R8 + E8 + 3 * C8 + 3 * V8));
    pbeg();
    halo({5}, 1, vc, cb);
    pend("update_halo", 0);
    pbeg();
    AccMaps acc_m;
    if (tma && use_tma && tmap(density0, sizeof(R), 9, &acc_m.d) &&
        tmap(pressure, sizeof(C), 9, &acc_m.p) && tmap(viscosity, sizeof(C), 9, &acc_m.q) &&
        tmap(xvel0, sizeof(V), 8, &acc_m.u) && tmap(yvel0, sizeof(V), 8, &acc_m.v) &&
        tmap(zvel0, sizeof(V), 8, &acc_m.w))
      launch_accelerate_tma<S>(g, stream, dtp, acc_m, vel1(0, vc), vel1(1, vc), vel1(2, vc),
                               &sc->status);
    else
      launch_accelerate<S>(tg, stream, 0.0, dtp, ga, density0, pressure, viscosity, xvel0, yvel0,
                           zvel0, vel1(0, vc), vel1(1, vc), vel1(2, vc), true);
    pend("accelerate", n * (R8 + 2 * C8 + 6 * V8));
    pbeg();
    FluxMaps flux_m;
    if (tma && use_tma && tmap(xvel0, sizeof(V), 9, &flux_m.u0) &&
        tmap(yvel0, sizeof(V), 9, &flux_m.v0) && tmap(zvel0, sizeof(V), 9, &flux_m.w0) &&
        tmap(vel1(0, vc), sizeof(V), 9, &flux_m.u1) && tmap(vel1(1, vc), sizeof(V), 9, &flux_m.v1) &&
        tmap(vel1(2, vc), sizeof(V), 9, &flux_m.w1))
      launch_pdv_flux_tma<S>(g, stream, dtp, flux_m, density0, rho1(cb), energy0, ene1(cb),
                             pressure, viscosity, vol_flux_x, vol_flux_y, vol_flux_z, &sc->status);
    else
      launch_pdv_flux<S>(tg, stream, dtp, ga, density0, rho1(cb), energy0, ene1(cb), pressure,
                         viscosity, xvel0, vel1(0, vc), yvel0, vel1(1, vc), zvel0, vel1(2, vc),
                         vol_flux_x, vol_flux_y, vol_flux_z);
    pend("pdv_flux", n * (2 * R8 + 2 * E8 + 2 * C8 + 6 * V8 + 3 * VF8));
    // advection.f90:43-179. The last sweep also writes time level 0 (the
    // interior density/energy and node velocities reset_field copies), so
    // reset_field needs no pass of its own.
    const int axi = ax ? 1 : 0;
    const Level0<S> no_level0{nullptr, nullptr, nullptr, nullptr, nullptr};
    const Level0<S> level0{density0, energy0, xvel0, yvel0, zvel0};
    auto sweep = [&](int sweep_number, int dir, bool pre_halo) {
      const Level0<S>& l0 = sweep_number == 3 ? level0 : no_level0;
      const double nl0 = sweep_number == 3 ? 1 : 0;  // level 0 written by this sweep
      if (pre_halo) {
        pbeg();
        // before sweep 2, density1 and energy1 (updated after sweep 1) and
        // vol_flux_z (updated before sweep 1) have not changed since
        if (sweep_number == 2 && halo_repeat_free) halo({14, 15}, 2, vc, cb);
        else halo({4, 2, 14, 15, 16}, 2, vc, cb);
        pend("update_halo", 0);
      }
      // volume fluxes read for pre_vol: all three on sweep 1, two on the y sweep,
      // the sweep direction only on sweep 3
      const double nvf = sweep_number == 1 ? 3 : sweep_number == 2 ? 2 : 1;
      pbeg();
      if (dir == 1) {
        // one pass, out of place into the other buffer of the pair
        // the post-sweep depth-2 halo update rewrites the output pair's shell
        CellXMaps xm;
        const bool x_tma = tma && use_tma && cell_x_maps(sweep_number, cb, &xm);
        launch_advec_cell_x<S>(tg, stream, sweep_number, ga, rho1(cb), ene1(cb), rho1(cb ^ 1),
                               ene1(cb ^ 1), vol_flux_x, vol_flux_y, vol_flux_z, mass_flux_x,
                               !halo_repeat_free, l0, x_tma ? &xm : nullptr, &sc->status);
        cb ^= 1;
        pend("advec_cell_x", n * (nvf * VF8 + (2 + nl0) * (R8 + E8) + MF8));
      } else {
        // one marching pass: staged and out of place into the other buffer of
        // the pair where the depth-2 halo update that follows rewrites the
        // output's shell, in place otherwise
        const int cvar = dir == 2 ? (axi ? 2 : 3) : (sweep_number == 1 ? 4 : 5);
        CellMaps cm;
        if (tma && use_tma && halo_repeat_free && cell_maps(dir, cvar, cb, &cm)) {
          launch_cell_sweep_tma<S>(g, stream, dir, cvar, cm, ga, rho1(cb), ene1(cb), rho1(cb ^ 1),
                                   ene1(cb ^ 1), vol_flux_x, vol_flux_y, vol_flux_z,
                                   dir == 2 ? mass_flux_y : mass_flux_z, l0, &sc->status);
          cb ^= 1;
        } else {
          launch_advec_cell_fused<S>(tg, stream, axi, dir, sweep_number, ga, rho1(cb), ene1(cb),
                                     mass_flux_x, vol_flux_x, mass_flux_y, vol_flux_y,
                                     mass_flux_z, vol_flux_z, work[6], l0);
        }
        pend("advec_cell_yz", n * (nvf * VF8 + (2 + nl0) * (R8 + E8) + MF8));
      }
      pbeg();
      // mass_flux_z changes only in the z sweep and is updated right after it
      if (dir != 3 && halo_repeat_free) halo({2, 4, 9, 11, 13, 17, 18}, 2, vc, cb);
      else halo({2, 4, 9, 11, 13, 17, 18, 19}, 2, vc, cb);
      pend("update_halo", 0);
      // post_vol reads two volume fluxes on sweep 1, one on sweep 2, none on sweep 3
      const double npv = sweep_number == 1 ? 2 : sweep_number == 2 ? 1 : 0;
      V* vin[3] = {vel1(0, vc), vel1(1, vc), vel1(2, vc)};
      V* vout[3] = {vel1(0, vc ^ 1), vel1(1, vc ^ 1), vel1(2, vc ^ 1)};
      pbeg();
      // after sweeps 1 and 2 the next post-sweep depth-2 halo update rewrites
      // the velocities' shell before anything reads it; after sweep 3 the
      // shell carries the step's final halo values
      MomXMaps xm;
      NodeMaps nm;
      const bool x_tma = dir == 1 && tma && use_tma && mom_x_maps(rho1(cb), vin, &xm);
      const int node_var = dir == 2 ? (axi ? 2 : 3) : (sweep_number == 1 ? 1 : 4);
      const bool node_tma =
          dir != 1 && tma && use_tma && mom_node_maps(dir, node_var, rho1(cb), &nm);
      VelMaps vm;
      const bool vel_tma = dir != 1 && tma && use_tma && mom_vel_maps(dir, vin, &vm);
      launch_advec_mom_fused<S>(tg, stream, axi, sweep_number, dir, cell_volume, ga, rho1(cb),
                                mass_flux_x, mass_flux_y, mass_flux_z, vol_flux_x, vol_flux_y,
                                vol_flux_z, work[0], work[1], work[2], vin, vout,
                                sweep_number == 3 || !halo_repeat_free, l0,
                                x_tma ? &xm : nullptr, &sc->status, node_tma ? &nm : nullptr,
                                vel_tma ? &vm : nullptr);
      // x: one pass; y, z: node pass + velocity pass
      if (dir == 1)
        pend("advec_mom_x", n * (MF8 + R8 + npv * VF8 + (6 + 3 * nl0) * V8));
      else  // node pass + velocity pass
        pend("advec_mom_yz",
             n * ((MF8 + R8 + npv * VF8 + 3 * N8) + (3 * N8 + (6 + 3 * nl0) * V8)));
      vc ^= 1;
    };
    sweep(1, ax ? 1 : 3, true);
    sweep(2, 2, true);
    sweep(3, ax ? 3 : 1, false);
    k_step_end<<<deck_blocks(), 128, 0, stream>>>(sc, nd);
  }

  // One hydro step, hydro.f90:52-68 (timestep .. time = time + dt).
  void enqueue_step(bool ax) {
    if (fused || plan) {
      enqueue_step_fused(ax);
      return;
    }
    const double* dtp = &sc->dt;
    const double n = cells();
    const double R8 = sizeof(R), E8 = sizeof(En), C8 = sizeof(C), V8 = sizeof(V),
                 VF8 = sizeof(VF), MF8 = sizeof(MF), W8 = sizeof(W), G8 = sizeof(double);
    // timestep.f90:56-126
    k_dt_prepare<<<1, 128, 0, stream>>>(sc, 1, min_key_of(kGBig));
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
    k_dt_finalize<<<1, 128, 0, stream>>>(sc, 1, dt_hist);
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
    k_step_end<<<1, 128, 0, stream>>>(sc, 1);
  }

  // An ensemble's schedules are built by eager steps (one per sweep order)
  // before its graphs are captured: a capture cannot allocate them.
  bool capture_graphs() {
    if (plan && !(warm[0] && warm[1])) return false;
    for (int i = 0; i < 2; i++) {
      if (graph[i]) continue;
      cudaGraph_t gr;
      if (cudaStreamBeginCapture(stream, cudaStreamCaptureModeThreadLocal) != cudaSuccess)
        return false;
      const bool prof = profile;
      profile = false;
      if (plan) {
        plan->capturing = true;
        plan->missing = false;
      }
      enqueue_step(i == 0);
      profile = prof;
      if (plan) plan->capturing = false;
      if (cudaStreamEndCapture(stream, &gr) != cudaSuccess) return false;
      if (plan && plan->missing) {
        cudaGraphDestroy(gr);
        return false;
      }
      size_t n = 0;
      cudaGraphGetNodes(gr, nullptr, &n);
      launches_per_step = (int)n;
      if (cudaGraphInstantiate(&graph[i], gr, 0) != cudaSuccess) return false;
      cudaGraphDestroy(gr);
    }
    return true;
  }

  int step(int n) {
    if (visit_pending && n > 0) {
      visit_pending = false;
      if (visit() != 0) return -1;
    }
    for (int i = 0; i < n; i++) {
      bool graphs = use_graphs && !profile && !(plan && plan->timing);
      if (graphs && !graph[advect_x ? 0 : 1] && !capture_graphs()) {
        cudaGetLastError();
        if (!plan) use_graphs = false;  // an ensemble captures once it is warm
        graphs = false;
      }
      if (graphs)
        cudaGraphLaunch(graph[advect_x ? 0 : 1], stream);
      else
        enqueue_step(advect_x);
      if (plan && !plan->failed) warm[advect_x ? 0 : 1] = true;
      advect_x = !advect_x;
      host_step++;
      if (deck.summary_frequency != 0 && host_step % deck.summary_frequency == 0)
        summary(host_step);
      // hydro.f90:73-75
      if (deck.visit_frequency != 0 && host_step % deck.visit_frequency == 0) visit();
    }
    return cudaGetLastError() == cudaSuccess ? 0 : -1;
  }

  DevScalars scalars(int d = 0) {
    DevScalars h{};
    cudaMemcpyAsync(&h, sc + d, sizeof(h), cudaMemcpyDeviceToHost, stream);
    cudaStreamSynchronize(stream);
    return h;
  }

  // hydro.f90:46-98 with the end test; runs in batches that cannot overshoot
  // end_time, since dt <= max_timestep.
  int run() {
    if (plan) {
      // every deck advances deck 0's end_step steps (no per-deck end_time)
      if (host_step < deck.end_step && step(deck.end_step - host_step) != 0) return -1000000000;
      int bad = 0;
      for (int d = 0; d < nd; d++) bad |= scalars(d).status & CLOVER_STATUS_SMALL_DT;
      if (bad) return -host_step;
      summary(host_step);  // the final summary (hydro.f90:87)
      if (deck.visit_frequency != 0) visit();  // hydro.f90:88
      cudaStreamSynchronize(stream);
      visit_join();
      return host_step;
    }
    for (;;) {
      DevScalars h = scalars();
      if (h.status & CLOVER_STATUS_SMALL_DT) return -host_step;
      if (host_step > 0 && (h.time + kGSmall > deck.end_time || host_step >= deck.end_step)) {
        summary(host_step);  // the final summary (hydro.f90:87)
        if (deck.visit_frequency != 0) visit();  // hydro.f90:88
        cudaStreamSynchronize(stream);
        visit_join();
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

  int read_field(int id, double* host, bool write, int deck_index = 0) {
    if (id < 1 || id > 19 || deck_index < 0 || deck_index >= nd) return -1;
    const Geom& g = geoms[deck_index];
    const int vb = vel1_buffer(host_step), cb = cell_buffer(host_step);
    void* f[19] = {density0, rho1(cb), energy0, ene1(cb), pressure, viscosity, soundspeed,
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
    cudaPitchedPtr dp = make_cudaPitchedPtr((char*)f[id - 1] + g.o3 * e, (size_t)g.px * e,
                                            (size_t)hx * e, (size_t)(g.pxy / g.px));
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
    visit_join();
    if (stream) cudaStreamSynchronize(stream);
    prof_collect();
    for (auto e : ev_pool) cudaEventDestroy(e);
    for (int i = 0; i < 2; i++)
      if (graph[i]) cudaGraphExecDestroy(graph[i]);
    for (const Owned& o : owned) cudaFree(o.p);
    delete plan;
    cudaFree(plane_base);
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
    ok = c->mixed->create(deck, 1, false);
  } else {
    c->f64 = new Chunk<F64>;
    ok = c->f64->create(deck, 1, false);
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
  if (c->f64 ? c->f64->plan != nullptr : c->mixed->plan != nullptr)
    return clover_ensemble_summaries(c, 0, out5, steps, cap);
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

int clover_chunk_use_tma(clover_chunk* c, int on) {
  auto set = [&](auto* ch) {
    if (ch->use_tma != (on != 0)) {
      ch->use_tma = on != 0;
      ch->drop_graphs();  // the captured steps hold the other kernels
    }
    return ch->tma && ch->use_tma ? 1 : 0;
  };
  return c->f64 ? set(c->f64) : set(c->mixed);
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

// ---- ensembles ----
clover_chunk* clover_ensemble_create(const clover_deck* decks, int n_decks, int precision) {
  g_last_error.clear();
  if (!decks || n_decks < 1) {
    g_last_error = "an ensemble needs at least one deck";
    return nullptr;
  }
  for (int i = 0; i < n_decks; i++) {
    const clover_deck& d = decks[i];
    if (d.number_of_states < 1 || d.number_of_states > CLOVER_MAX_STATES) {
      g_last_error = "deck needs 1..16 states";
      return nullptr;
    }
    if (d.x_cells < 1 || d.y_cells < 1 || d.z_cells < 1) {
      g_last_error = "deck needs at least one cell per axis";
      return nullptr;
    }
    // one step sequence for all decks: calc_dt's safety factors, the step
    // count and the summary cadence are shared
    const clover_deck& a = decks[0];
    if (d.end_step != a.end_step || d.summary_frequency != a.summary_frequency ||
        d.dtc_safe != a.dtc_safe || d.dtu_safe != a.dtu_safe || d.dtv_safe != a.dtv_safe ||
        d.dtw_safe != a.dtw_safe || d.dtdiv_safe != a.dtdiv_safe) {
      g_last_error = "ensemble decks must share end_step, summary_frequency and the dt safety factors";
      return nullptr;
    }
  }
  clover_chunk* c = new clover_chunk;
  c->precision = precision;
  bool ok;
  if (precision == CLOVER_PRECISION_MIXED) {
    c->mixed = new Chunk<F32Mixed>;
    ok = c->mixed->create(decks, n_decks, true);
  } else {
    c->f64 = new Chunk<F64>;
    ok = c->f64->create(decks, n_decks, true);
  }
  if (!ok) {
    if (g_last_error.empty()) g_last_error = "ensemble creation failed";
    clover_chunk_destroy(c);
    return nullptr;
  }
  return c;
}

int clover_ensemble_decks(clover_chunk* c) { return DISPATCH(c, nd); }

int clover_ensemble_autotune(clover_chunk* c, int trial_steps) {
  return DISPATCH(c, autotune(trial_steps));
}

int clover_ensemble_reset(clover_chunk* c) { return DISPATCH(c, reset()) ? 0 : -1; }

int clover_ensemble_set_schedule(clover_chunk* c, int order, int grid_div, int seg) {
  BatchPlan* plan = c->f64 ? c->f64->plan : c->mixed->plan;
  if (!plan || order < 0 || order > 2 || grid_div < 0 || seg < 0) return -1;
  plan->tuned.clear();
  plan->fallback = SchedCfg{order, grid_div, seg};
  // the graphs hold the old schedule: capture again after eager steps
  return DISPATCH(c, drop_graphs()) ? 0 : -1;
}

int clover_ensemble_schedule(clover_chunk* c, char* buf, int len) {
  const std::string r = DISPATCH(c, schedule_report());
  if (buf && len > 0) snprintf(buf, (size_t)len, "%s", r.c_str());
  return (int)r.size();
}

int clover_ensemble_status(clover_chunk* c, int deck) {
  if (deck < 0 || deck >= DISPATCH(c, nd)) return -1;
  return DISPATCH(c, scalars(deck)).status;
}

double clover_ensemble_time(clover_chunk* c, int deck) {
  if (deck < 0 || deck >= DISPATCH(c, nd)) return -1.0;
  return DISPATCH(c, scalars(deck)).time;
}

int clover_ensemble_dt_history(clover_chunk* c, int deck, double* out, int cap) {
  const int nd = DISPATCH(c, nd);
  if (deck < 0 || deck >= nd) return -1;
  DevScalars h = DISPATCH(c, scalars(deck));
  const int dcap = c->f64 ? c->f64->dt_cap : c->mixed->dt_cap;
  int n = h.step < cap ? h.step : cap;
  if (n > dcap) n = dcap;
  const double* src = (c->f64 ? c->f64->dt_hist : c->mixed->dt_hist) + (size_t)deck * dcap;
  if (n > 0 && cudaMemcpy(out, src, (size_t)n * sizeof(double), cudaMemcpyDeviceToHost) != cudaSuccess)
    return -1;
  return n;
}

int clover_ensemble_summaries(clover_chunk* c, int deck, double* out5, int* steps, int cap) {
  const int nd = DISPATCH(c, nd);
  if (deck < 0 || deck >= nd) return -1;
  clover_chunk_sync(c);
  const std::vector<int>& ss = c->f64 ? c->f64->sum_steps : c->mixed->sum_steps;
  const double* src = c->f64 ? c->f64->sum_hist : c->mixed->sum_hist;
  const bool batched = c->f64 ? c->f64->plan != nullptr : c->mixed->plan != nullptr;
  int n = (int)ss.size() < cap ? (int)ss.size() : cap;
  for (int i = 0; i < n; i++) {
    // batched summaries hold all decks per record; a single chunk one deck
    const double* rec = src + (batched ? (size_t)5 * ((size_t)i * nd + deck) : (size_t)5 * i);
    if (cudaMemcpy(out5 + 5 * i, rec, 5 * sizeof(double), cudaMemcpyDeviceToHost) != cudaSuccess)
      return -1;
    steps[i] = ss[i];
  }
  return n;
}

int clover_ensemble_read_field(clover_chunk* c, int deck, int id, double* host) {
  return DISPATCH(c, read_field(id, host, false, deck));
}

int clover_chunk_set_visit_dir(clover_chunk* c, const char* dir) {
  if (!dir) return -1;
  if (c->f64) c->f64->visit_dir = dir;
  else c->mixed->visit_dir = dir;
  return 0;
}

int clover_chunk_visit(clover_chunk* c) {
  if (c->f64) c->f64->visit_pending = false; else c->mixed->visit_pending = false;
  const int rc = DISPATCH(c, visit());
  if (c->f64) c->f64->visit_join(); else c->mixed->visit_join();
  const bool failed = c->f64 ? c->f64->visit_failed : c->mixed->visit_failed;
  if (failed) g_last_error = c->f64 ? c->f64->visit_error : c->mixed->visit_error;
  return rc != 0 ? rc : (failed ? -2 : 0);
}

int clover_chunk_checkpoint(clover_chunk* c, const char* path) {
  return DISPATCH(c, checkpoint(path));
}

int clover_chunk_restore(clover_chunk* c, const char* path) {
  return DISPATCH(c, restore(path));
}

}  // extern "C"
