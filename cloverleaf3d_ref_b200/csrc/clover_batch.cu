// Schedules of the batched launches over the decks of an ensemble.
//
// A batched launch runs one kernel over every deck: its work is the list of
// (deck, tile) items obtained by asking the launch's grid function for each
// deck's tile grid, and a persistent grid of blocks walks that list
// (clover_sched.cuh). Three things are chosen per launch (key):
//   order     the order of the items: 0 deck by deck in deck order, 1 deck
//             by deck from the deck with the most tiles down, 2 round robin
//             over the decks (tile i of every deck before tile i+1)
//   grid_div  0: one block per item; n > 0: the blocks that fit on the GPU
//             at the kernel's occupancy, divided by n
//   seg       segment length of a marching kernel (planes per thread)
// Schedules are built on first use and cached by (key, order, grid_div,
// seg); building allocates and copies, so it runs outside stream capture.
// The autotuner (Chunk::autotune in clover_native.cu) times each key's
// launches under candidate settings through the marks below and keeps the
// fastest per key; the results do not depend on the schedule.
#include <algorithm>
#include <array>
#include <map>
#include <string>
#include <vector>

#include "clover_batch.h"

namespace clover {

BatchPlan::~BatchPlan() {
  for (auto& kv : cache) cudaFree(kv.second.items);
  for (auto& m : marks) {
    cudaEventDestroy(m.a);
    if (m.b) cudaEventDestroy(m.b);
  }
  for (auto e : ev_pool) cudaEventDestroy(e);
  cudaFree(d_decks);
}

bool BatchPlan::init(const std::vector<Geom>& geoms) {
  decks = geoms;
  int dev = 0;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  if (sms <= 0) sms = 148;
  if (cudaMalloc(&d_decks, decks.size() * sizeof(Geom)) != cudaSuccess) return false;
  // a copy from pageable memory may still be in flight when cudaMemcpy
  // returns, and the kernels run on non-blocking streams: wait for it
  if (cudaMemcpy(d_decks, decks.data(), decks.size() * sizeof(Geom), cudaMemcpyHostToDevice) !=
      cudaSuccess)
    return false;
  return cudaDeviceSynchronize() == cudaSuccess;
}

SchedCfg BatchPlan::cfg_for(unsigned key) const {
  auto it = tuned.find(key);
  SchedCfg c = it != tuned.end() ? it->second : fallback;
  if (trial_active) {
    // a trial overrides what it names (-1: keep the tuned or default value)
    if (trial.order >= 0) c.order = trial.order;
    if (trial.grid_div >= 0) c.grid_div = trial.grid_div;
    if (trial.seg >= 0) c.seg = trial.seg;
  }
  return c;
}

std::vector<int4> BatchPlan::make_items(GridFn grid_fn, int aux, int order) const {
  const int nd = (int)decks.size();
  std::vector<std::vector<int4>> per(nd);
  for (int d = 0; d < nd; d++) {
    const dim3 gr = grid_fn(decks[d], aux);
    if (!gr.x || !gr.y || !gr.z) continue;
    per[d].reserve((size_t)gr.x * gr.y * gr.z);
    for (unsigned z = 0; z < gr.z; z++)
      for (unsigned y = 0; y < gr.y; y++)
        for (unsigned x = 0; x < gr.x; x++) per[d].push_back(make_int4(d, (int)x, (int)y, (int)z));
  }
  std::vector<int4> items;
  std::vector<int> deck_order(nd);
  for (int d = 0; d < nd; d++) deck_order[d] = d;
  if (order == 1)
    std::stable_sort(deck_order.begin(), deck_order.end(),
                     [&](int a, int b) { return per[a].size() > per[b].size(); });
  if (order == 2) {
    size_t most = 0;
    for (auto& v : per) most = std::max(most, v.size());
    for (size_t i = 0; i < most; i++)
      for (int d = 0; d < nd; d++)
        if (i < per[d].size()) items.push_back(per[d][i]);
  } else {
    for (int d : deck_order) items.insert(items.end(), per[d].begin(), per[d].end());
  }
  return items;
}

BatchLaunch batch_launch(BatchPlan* plan, cudaStream_t s, unsigned key, GridFn grid_fn, int aux,
                         bool seg_tunable, const void* kernel, int threads) {
  BatchLaunch out{nullptr, plan->d_decks, 0, 0, aux};
  plan->seg_tunable[key] = seg_tunable;
  const SchedCfg c = plan->cfg_for(key);
  const int a = (seg_tunable && c.seg > 0) ? c.seg : aux;
  const std::array<int, 4> id{(int)key, c.order, c.grid_div, a};
  auto it = plan->cache.find(id);
  if (it == plan->cache.end()) {
    if (plan->capturing) {
      plan->missing = true;  // a schedule cannot be built inside a capture
      return out;
    }
    BatchPlan::Entry e{};
    std::vector<int4> items = plan->make_items(grid_fn, a, c.order);
    e.n = (int)items.size();
    int occ = 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, kernel, threads, 0) != cudaSuccess ||
        occ < 1)
      occ = 1;
    const long long resident = (long long)occ * plan->sms;
    long long grid = c.grid_div <= 0 ? e.n : resident / c.grid_div;
    if (grid < 1) grid = 1;
    if (grid > e.n) grid = e.n;
    e.grid = (int)grid;
    e.aux = a;
    if (e.n > 0) {
      if (cudaMalloc(&e.items, items.size() * sizeof(int4)) != cudaSuccess) {
        plan->failed = true;
        return out;
      }
      // ordered before the launch on its stream, and complete before the
      // host vector goes away
      if (cudaMemcpyAsync(e.items, items.data(), items.size() * sizeof(int4),
                          cudaMemcpyHostToDevice, s) != cudaSuccess ||
          cudaStreamSynchronize(s) != cudaSuccess) {
        cudaFree(e.items);
        plan->failed = true;
        return out;
      }
    }
    it = plan->cache.emplace(id, e).first;
  }
  out.items = it->second.items;
  out.n = it->second.n;
  out.grid = it->second.grid;
  out.aux = it->second.aux;
  return out;
}

cudaEvent_t BatchPlan::event() {
  if (!ev_pool.empty()) {
    cudaEvent_t e = ev_pool.back();
    ev_pool.pop_back();
    return e;
  }
  cudaEvent_t e;
  cudaEventCreate(&e);
  return e;
}

void batch_mark(BatchPlan* plan, unsigned key, cudaStream_t s, bool begin) {
  if (!plan->timing || plan->capturing) return;
  if (begin) {
    BatchPlan::Mark m{key, plan->event(), nullptr};
    cudaEventRecord(m.a, s);
    plan->marks.push_back(m);
  } else if (!plan->marks.empty() && plan->marks.back().key == key && !plan->marks.back().b) {
    plan->marks.back().b = plan->event();
    cudaEventRecord(plan->marks.back().b, s);
  }
}

std::map<unsigned, double> BatchPlan::collect_marks() {
  std::map<unsigned, double> ms;
  for (auto& m : marks) {
    if (m.b) {
      cudaEventSynchronize(m.b);
      float t = 0.f;
      cudaEventElapsedTime(&t, m.a, m.b);
      ms[m.key] += t;
      ev_pool.push_back(m.b);
    }
    ev_pool.push_back(m.a);
  }
  marks.clear();
  return ms;
}

}  // namespace clover
