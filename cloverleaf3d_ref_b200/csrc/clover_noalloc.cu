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
// Scratch: kNoAllocMaxPlanes x 10 doubles (five compensated partial sums and
// their five compensation terms per z plane) + 10 for the totals, 320 KiB,
// held by every GPU that loads the library until the process exits. The grid
// may have at most kNoAllocMaxPlanes cells along z; larger grids are rejected.
// Every call overwrites the partials it reads, so nothing must start at zero,
// but all calls share the one array: calls that overlap on the GPU (from two
// host threads, or queued on different streams) race.
//
// Ordering: the drop-in entry points queue their kernels on the library's
// own stream and return without waiting. This call launches on that stream
// when the library's context lives on the current device, so it reads the
// arrays only after every library kernel queued before it; otherwise it uses
// the legacy default stream. Work the caller queued on its own streams must
// be finished (or ordered before this call) by the caller.
#include <cstdio>
#include <mutex>

#include "../../include/clover_kernels.h"
#include "clover_layout.cuh"
#include "clover_sum.cuh"

namespace clover {

cudaStream_t abi_stream_on(int dev);  // clover_abi.cu

namespace {

constexpr int kNoAllocMaxPlanes = CLOVER_NOALLOC_MAX_Z_CELLS;
constexpr int kThreads = 256;
constexpr int kMaxDevices = 64;
constexpr int kTotals = 2 * kSumQ * kNoAllocMaxPlanes;  // offset of the totals

// per-plane (s, c) at [10*p, 10*p+10), totals (s, c) at [kTotals, kTotals+10)
__device__ __align__(256) double g_summary_scratch[2 * kSumQ * kNoAllocMaxPlanes + 16];

// Device address of g_summary_scratch per device, looked up once per device
// (the module, and with it the array, lives until the process exits; a
// cudaDeviceReset after the first call on a device is not supported).
double* g_scratch_addr[kMaxDevices] = {nullptr};
std::mutex g_setup;

// One block per z plane: the cells of the plane in (j fastest, k) order,
// strided over the block's threads, then a fixed tree over the threads; every
// sum compensated (clover_sum.cuh).
__global__ void __launch_bounds__(kThreads) k_summary_planes(Geom g, const double* __restrict__ volume,
    const double* __restrict__ density0, const double* __restrict__ energy0,
    const double* __restrict__ pressure, const double* __restrict__ xvel0,
    const double* __restrict__ yvel0, const double* __restrict__ zvel0, double* scratch) {
  __shared__ double sh[2 * kSumQ * kThreads];
  const int l = g.z_min + blockIdx.x;
  const int nx = g.x_max - g.x_min + 1, ny = g.y_max - g.y_min + 1;
  const long long n = (long long)nx * ny;
  double s[kSumQ] = {0.0, 0.0, 0.0, 0.0, 0.0}, c[kSumQ] = {0.0, 0.0, 0.0, 0.0, 0.0};
  for (long long i = threadIdx.x; i < n; i += kThreads) {
    const int j = g.x_min + (int)(i % nx);
    const int k = g.y_min + (int)(i / nx);
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
    csum_add(s[0], c[0], cell_vol);
    csum_add(s[1], c[1], cell_mass);
    csum_add(s[2], c[2], cell_mass * energy0[o]);
    csum_add(s[3], c[3], cell_mass * 0.5 * vsqrd);
    csum_add(s[4], c[4], cell_vol * pressure[o]);
  }
  block_csum<kThreads>(s, c, sh);
  if (threadIdx.x == 0)
    for (int q = 0; q < kSumQ; q++) {
      scratch[2 * kSumQ * blockIdx.x + q] = s[q];
      scratch[2 * kSumQ * blockIdx.x + kSumQ + q] = c[q];
    }
}

// The plane partials merged in plane order by one thread; totals s + c.
__global__ void k_summary_planes_total(int planes, double* scratch) {
  double s[kSumQ] = {0.0, 0.0, 0.0, 0.0, 0.0}, c[kSumQ] = {0.0, 0.0, 0.0, 0.0, 0.0};
  for (int p = 0; p < planes; p++)
    for (int q = 0; q < kSumQ; q++)
      csum_merge(s[q], c[q], scratch[2 * kSumQ * p + q], scratch[2 * kSumQ * p + kSumQ + q]);
  for (int q = 0; q < kSumQ; q++) scratch[kTotals + q] = s[q] + c[q];
}

// Device memory of device dev (or managed memory): a pointer into another
// GPU's memory is refused, since reading it here needs peer access.
bool on_device(const void* p, int dev) {
  cudaPointerAttributes a;
  if (cudaPointerGetAttributes(&a, p) != cudaSuccess) {
    cudaGetLastError();
    return false;
  }
  if (a.type == cudaMemoryTypeManaged) return true;
  return a.type == cudaMemoryTypeDevice && a.device == dev;
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
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= kMaxDevices) {
    cudaGetLastError();
    return CLOVER_STATUS_NO_DEVICE;
  }
  const void* in[7] = {volume, density0, energy0, pressure, xvel0, yvel0, zvel0};
  for (const void* p : in)
    if (!p || !on_device(p, dev)) {
      fprintf(stderr,
              "clover_field_summary_kernel_noalloc: every array must be memory of the current "
              "device in the chunk layout (host arrays would need a device copy, another "
              "GPU's arrays peer access)\n");
      return CLOVER_STATUS_BAD_ARG;
    }
  // Set-up, once per device with that device current: the host-side name of
  // a __device__ array is not a device address, so look the address up.
  double* scratch = nullptr;
  {
    std::lock_guard<std::mutex> lock(g_setup);
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
    scratch = g_scratch_addr[dev];
  }
  // after any kernel the drop-in entry points queued on this device
  cudaStream_t st = abi_stream_on(dev);
  const Geom g = make_geom(*x_min, *x_max, *y_min, *y_max, *z_min, *z_max);
  k_summary_planes<<<planes, kThreads, 0, st>>>(g, volume, density0, energy0, pressure, xvel0,
                                                yvel0, zvel0, scratch);
  k_summary_planes_total<<<1, 1, 0, st>>>(planes, scratch);
  const cudaError_t le = cudaGetLastError();
  if (le != cudaSuccess) {
    fprintf(stderr, "clover_field_summary_kernel_noalloc: launch: %s\n", cudaGetErrorString(le));
    return CLOVER_STATUS_CUDA_ERROR;
  }
  double s[5];
  cudaError_t e = cudaMemcpyAsync(s, scratch + kTotals, sizeof(s), cudaMemcpyDeviceToHost, st);
  if (e == cudaSuccess) e = cudaStreamSynchronize(st);
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
