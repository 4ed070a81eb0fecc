// Host side of the batched launches: the decks of an ensemble, the cached
// schedules of their launches and the per-launch settings the autotuner
// picks (clover_batch.cu).
#pragma once

#include <array>
#include <map>
#include <vector>

#include "clover_launch.h"

namespace clover {

// Settings of one batched launch; -1 in a trial keeps the current value.
struct SchedCfg {
  int order = 0;     // 0 deck order, 1 largest deck first, 2 round robin over decks
  int grid_div = 1;  // 0: one block per item; n: resident blocks / n
  int seg = 0;       // segment length of a marching kernel; 0: the launch's default
};

struct BatchPlan {
  struct Entry {
    int4* items;
    int n, grid, aux;
  };
  struct Mark {
    unsigned key;
    cudaEvent_t a, b;
  };

  std::vector<Geom> decks;
  Geom* d_decks = nullptr;
  int sms = 148;
  std::map<std::array<int, 4>, Entry> cache;  // (key, order, grid_div, seg)
  std::map<unsigned, SchedCfg> tuned;         // per launch key
  std::map<unsigned, bool> seg_tunable;       // keys seen, and whether seg applies
  SchedCfg fallback;                          // keys without a tuned entry
  SchedCfg trial;                             // the autotuner's candidate
  bool trial_active = false;
  bool capturing = false;  // a stream capture is open: no schedule may be built
  bool missing = false;    // a launch was skipped for want of a schedule
  bool failed = false;     // a schedule could not be allocated
  bool timing = false;     // record events around every batched launch
  std::vector<Mark> marks;
  std::vector<cudaEvent_t> ev_pool;

  ~BatchPlan();
  bool init(const std::vector<Geom>& geoms);
  SchedCfg cfg_for(unsigned key) const;
  std::vector<int4> make_items(GridFn grid_fn, int aux, int order) const;
  cudaEvent_t event();
  // milliseconds per key of the marked launches since the last call
  std::map<unsigned, double> collect_marks();
};

}  // namespace clover
