// field_summary without any device allocation (clover_field_summary_kernel_noalloc).
//
// For callers that cannot let the library call cudaMalloc: a host code whose
// device memory is all owned by its own pool allocator or reserved up front
// (a framework holding the GPU's memory in a caching pool), or one that runs
// under a fixed device-memory budget, where an allocation made behind its
// back could fail or fragment the pool. The regular entry point mirrors host
// arrays and keeps its reduction scratch in memory it allocates on first use;
// this one takes device arrays and keeps its scratch in a file-scope device
// array that exists as soon as the library is loaded on a GPU.
//
// Scratch: kNoAllocMaxPlanes x 5 partial sums + 5 totals (160 KiB), held by
// every GPU that loads the library until the process exits. The grid may
// have at most kNoAllocMaxPlanes cells along z; larger grids are rejected.
// Every call overwrites the partials it reads, so nothing must start at zero,
// but all calls share the one array: calls that overlap on the GPU (from two
// host threads, or queued on different streams) race.
#include <cstdio>

#include "../../include/clover_kernels.h"
#include "clover_layout.cuh"

namespace clover {
namespace {

constexpr int kNoAllocMaxPlanes = CLOVER_NOALLOC_MAX_Z_CELLS;
constexpr int kThreads = 256;
constexpr int kMaxDevices = 64;

// per-plane partials at [5*p, 5*p+5), totals at [5*kNoAllocMaxPlanes, +5)
__device__ __align__(256) double g_summary_scratch[5 * kNoAllocMaxPlanes + 8];

// Device address of g_summary_scratch per device, resolved once.
double* g_scratch_addr[kMaxDevices] = {nullptr};

// One block per z plane: the cells of the plane in (j fastest, k) order,
// strided over the block's threads, then a fixed tree over the threads.
__global__ void __launch_bounds__(kThreads) k_summary_planes(Geom g, const double* __restrict__ volume,
    const double* __restrict__ density0, const double* __restrict__ energy0,
    const double* __restrict__ pressure, const double* __restrict__ xvel0,
    const double* __restrict__ yvel0, const double* __restrict__ zvel0, double* scratch) {
  __shared__ double sh[5 * kThreads];
  const int l = g.z_min + blockIdx.x;
  const int nx = g.x_max - g.x_min + 1, ny = g.y_max - g.y_min + 1;
  const long long n = (long long)nx * ny;
  double acc[5] = {0.0, 0.0, 0.0, 0.0, 0.0};
  for (long long c = threadIdx.x; c < n; c += kThreads) {
    const int j = g.x_min + (int)(c % nx);
    const int k = g.y_min + (int)(c / nx);
    double vsqrd = 0.0;
    for (int lv = l; lv <= l + 1; lv++)
      for (int kv = k; kv <= k + 1; kv++)
        for (int jv = j; jv <= j + 1; jv++) {
          const long long o = off3(g, jv, kv, lv);
          const double u = xvel0[o], v = yvel0[o], w = zvel0[o];
          vsqrd = vsqrd + 0.125 * (u * u + v * v + w * w);
        }
    const long long o = off3(g, j, k, l);
    const double cell_vol = volume[o];
    const double cell_mass = cell_vol * density0[o];
    acc[0] = acc[0] + cell_vol;
    acc[1] = acc[1] + cell_mass;
    acc[2] = acc[2] + cell_mass * energy0[o];
    acc[3] = acc[3] + cell_mass * 0.5 * vsqrd;
    acc[4] = acc[4] + cell_vol * pressure[o];
  }
  const int t = threadIdx.x;
  for (int q = 0; q < 5; q++) sh[q * kThreads + t] = acc[q];
  __syncthreads();
  for (int s = kThreads / 2; s > 0; s >>= 1) {
    if (t < s)
      for (int q = 0; q < 5; q++) sh[q * kThreads + t] += sh[q * kThreads + t + s];
    __syncthreads();
  }
  if (t == 0)
    for (int q = 0; q < 5; q++) scratch[5 * blockIdx.x + q] = sh[q * kThreads];
}

// The plane partials added in plane order by one thread.
__global__ void k_summary_planes_total(int planes, double* scratch) {
  double t[5] = {0.0, 0.0, 0.0, 0.0, 0.0};
  for (int p = 0; p < planes; p++)
    for (int q = 0; q < 5; q++) t[q] = t[q] + scratch[5 * p + q];
  for (int q = 0; q < 5; q++) scratch[5 * kNoAllocMaxPlanes + q] = t[q];
}

bool on_device(const void* p) {
  cudaPointerAttributes a;
  if (cudaPointerGetAttributes(&a, p) != cudaSuccess) {
    cudaGetLastError();
    return false;
  }
  return a.type == cudaMemoryTypeDevice || a.type == cudaMemoryTypeManaged;
}

}  // namespace
}  // namespace clover

using namespace clover;

extern "C" int clover_field_summary_kernel_noalloc(
    const int* x_min, const int* x_max, const int* y_min, const int* y_max, const int* z_min,
    const int* z_max, const double* volume, const double* density0, const double* energy0,
    const double* pressure, const double* xvel0, const double* yvel0, const double* zvel0,
    double* vol, double* mass, double* ie, double* ke, double* press) {
  const int planes = *z_max - *z_min + 1;
  if (*x_max < *x_min || *y_max < *y_min || planes < 1) {
    fprintf(stderr, "clover_field_summary_kernel_noalloc: empty grid\n");
    return CLOVER_STATUS_BAD_ARG;
  }
  if (planes > kNoAllocMaxPlanes) {
    fprintf(stderr,
            "clover_field_summary_kernel_noalloc: %d cells along z exceed the maximum of %d "
            "that its fixed scratch holds; use clover_field_summary_kernel\n",
            planes, kNoAllocMaxPlanes);
    return CLOVER_STATUS_BAD_ARG;
  }
  const void* in[7] = {volume, density0, energy0, pressure, xvel0, yvel0, zvel0};
  for (const void* p : in)
    if (!p || !on_device(p)) {
      fprintf(stderr,
              "clover_field_summary_kernel_noalloc: every array must be device memory in the "
              "chunk layout (host arrays would need a device copy)\n");
      return CLOVER_STATUS_BAD_ARG;
    }
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= kMaxDevices) {
    cudaGetLastError();
    return CLOVER_STATUS_NO_DEVICE;
  }
  // Set-up, once per device with that device current: the host-side name of
  // a __device__ array is not a device address, so look the address up.
  if (!g_scratch_addr[dev]) {
    void* p = nullptr;
    const cudaError_t e = cudaGetSymbolAddress(&p, g_summary_scratch);
    if (e != cudaSuccess || !p) {
      fprintf(stderr, "clover_field_summary_kernel_noalloc: scratch address: %s\n",
              cudaGetErrorString(e));
      cudaGetLastError();
      return CLOVER_STATUS_CUDA_ERROR;
    }
    g_scratch_addr[dev] = (double*)p;
  }
  double* scratch = g_scratch_addr[dev];
  const Geom g = make_geom(*x_min, *x_max, *y_min, *y_max, *z_min, *z_max);
  k_summary_planes<<<planes, kThreads>>>(g, volume, density0, energy0, pressure, xvel0, yvel0,
                                         zvel0, scratch);
  k_summary_planes_total<<<1, 1>>>(planes, scratch);
  const cudaError_t le = cudaGetLastError();
  if (le != cudaSuccess) {
    fprintf(stderr, "clover_field_summary_kernel_noalloc: launch: %s\n", cudaGetErrorString(le));
    return CLOVER_STATUS_CUDA_ERROR;
  }
  double s[5];
  const cudaError_t e = cudaMemcpy(s, scratch + 5 * kNoAllocMaxPlanes, sizeof(s),
                                   cudaMemcpyDeviceToHost);
  if (e != cudaSuccess) {
    fprintf(stderr, "clover_field_summary_kernel_noalloc: %s\n", cudaGetErrorString(e));
    return CLOVER_STATUS_CUDA_ERROR;
  }
  *vol = s[0];
  *mass = s[1];
  *ie = s[2];
  *ke = s[3];
  *press = s[4];
  return 0;
}
