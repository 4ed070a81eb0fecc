// Block-to-work mapping of the hydro kernels.
//
// A kernel body runs once per tile: the geometry of the chunk it works on
// (which carries the chunk's offsets into the shared allocations), the
// chunk's deck index, and the tile's coordinates in that chunk's tile grid.
//
//   MapSingle  one chunk; the launch grid is the tile grid (tile = blockIdx).
//   MapBatch   the decks of an ensemble in one launch: a persistent grid of
//              blocks walks a schedule of (deck, tile) work items, block b
//              taking items b, b + gridDim.x, b + 2*gridDim.x, ...
//
// Both maps also carry the segment length of the marching kernels (the
// number of planes a thread walks), which is part of the tile shape.
#pragma once

#include <cuda_runtime.h>

#include "clover_layout.cuh"

namespace clover {

struct Tile {
  int d;        // deck index (0 for a single chunk)
  int x, y, z;  // tile coordinates in the deck's tile grid
};

struct MapSingle {
  static constexpr bool kFlat = false;  // box kernels use 32 x 8 tiles of (j, k)
  Geom g;
  int seg;
  template <class F>
  __device__ __forceinline__ void run(F&& f) const {
    f(g, Tile{0, (int)blockIdx.x, (int)blockIdx.y, (int)blockIdx.z});
  }
};

// kSync: a barrier after each item, for kernels whose threads share memory
// within an item (the next item may reuse it only when every thread is done);
// without it the warps of a block move on to their next item independently.
template <bool kSync>
struct MapBatchT {
  // box kernels take 256 consecutive cells of a deck's (j, k) plane per tile,
  // so that decks whose x extent is not a multiple of 32 fill every lane
  static constexpr bool kFlat = true;
  const int4* __restrict__ items;  // (deck, tile x, tile y, tile z)
  const Geom* __restrict__ decks;  // per deck geometry and offsets
  int n;                           // number of items
  int seg;
  template <class F>
  __device__ __forceinline__ void run(F&& f) const {
    for (int w = blockIdx.x; w < n; w += gridDim.x) {
      const int4 it = __ldg(items + w);
      const Geom g = decks[it.x];
      f(g, Tile{it.x, it.y, it.z, it.w});
      if (kSync) __syncthreads();
    }
  }
};
using MapBatch = MapBatchT<true>;       // kernels with shared memory or block barriers
using MapBatchFree = MapBatchT<false>;  // kernels whose warps work independently

}  // namespace clover
