// Device layout of a CloverLeaf3D chunk in HBM.
//
// Every 3D array of a chunk (cell, vertex, face and work arrays) shares one
// pitched layout: element (j,k,l), j in [x_min-2, x_max+3], k in
// [y_min-2, y_max+3], l in [z_min-2, z_max+3], sits at
//   (j - x_min + 2) + (k - y_min + 2) * px + (l - z_min + 2) * pxy
// with px a multiple of 32 elements and each allocation shifted so that the
// first interior column (j = x_min) of every row starts on a 128-byte
// boundary, for 4- and 8-byte elements alike. Cell arrays simply leave their
// last row/plane/column unused, so a kernel can address every array with one
// (px, pxy) pair. 1D coordinate arrays are indexed from min-2.
//
// Several chunks (the decks of an ensemble) can share one allocation per
// array: deck d then starts o3 elements into every 3D allocation and o1
// elements into every 1D allocation. A single chunk has o3 = o1 = 0.
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

namespace clover {

struct Geom {
  int x_min, x_max, y_min, y_max, z_min, z_max;
  int px;         // row pitch in elements
  int o1;         // offset of this chunk in the shared 1D allocations
  long long pxy;  // plane pitch in elements
  long long o3;   // offset of this chunk in the shared 3D allocations
  // Cell volume and face areas of the chunk's uniform mesh: every element of
  // the volume, xarea, yarea and zarea arrays holds these values
  // (initialise_chunk_kernel.f90:113-175: volume = dx*dy*dz, xarea =
  // celldy*celldz = dy*dz, yarea = dx*dz, zarea = dx*dy). The native step
  // kernels read them here instead of streaming four 3D arrays; the drop-in
  // kernels, whose callers own the arrays, read the arrays.
  double vol, xa, ya, za;
  // Per-chunk quotients of those constants, formed on the host in the
  // precision the kernels use them in (IEEE division either side): 1/volume
  // (PdV_kernel.f90:105) and calc_dt's ds = 1/min(dx,dy,dz)^2
  // (calc_dt_kernel.f90:112), in FP64 and FP32.
  double rvol, ds;
  float rvol_f, ds_f;
};

// Elements per 128 bytes for a storage type.
template <class T>
constexpr int kAlignElems = 128 / (int)sizeof(T);

// Front padding so that element j = x_min (2 after the first) is aligned.
template <class T>
constexpr int kFrontPad = kAlignElems<T> - 2;

inline Geom make_geom(int x_min, int x_max, int y_min, int y_max, int z_min, int z_max) {
  Geom g;
  g.x_min = x_min; g.x_max = x_max; g.y_min = y_min;
  g.y_max = y_max; g.z_min = z_min; g.z_max = z_max;
  const int align = 32;
  int nxv = x_max - x_min + 6;
  g.px = (nxv + align - 1) / align * align;
  g.pxy = (long long)g.px * (y_max - y_min + 6);
  g.o1 = 0;
  g.o3 = 0;
  g.vol = g.xa = g.ya = g.za = 0.0;
  g.rvol = g.ds = 0.0;
  g.rvol_f = g.ds_f = 0.0f;
  return g;
}

// Elements (after the front pad) one 3D array of the chunk occupies.
inline long long array_elems(const Geom& g) {
  return g.pxy * (long long)(g.z_max - g.z_min + 6);
}

__host__ __device__ __forceinline__ long long off3(const Geom& g, int j, int k, int l) {
  return g.o3 + (long long)(j - g.x_min + 2) + (long long)(k - g.y_min + 2) * g.px +
         (long long)(l - g.z_min + 2) * g.pxy;
}

// Elements of one 1D coordinate array (any axis) of a chunk, rounded so that
// the next chunk's arrays start on a 256-byte boundary.
inline int array1d_elems(const Geom& g) {
  int n = g.x_max - g.x_min;
  if (g.y_max - g.y_min > n) n = g.y_max - g.y_min;
  if (g.z_max - g.z_min > n) n = g.z_max - g.z_min;
  return (n + 6 + 31) / 32 * 32;
}

}  // namespace clover
