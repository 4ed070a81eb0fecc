// Drop-in C ABI (include/clover_kernels.h): host-pointer mirrors and the
// extern "C" entry points that replace the reference's *_kernel procedures.
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <map>
#include <mutex>
#include <string>
#include <tuple>
#include <unordered_map>
#include <vector>

#include "../../include/clover_kernels.h"
#include "clover_launch.h"
#include "clover_tma.cuh"

namespace clover {
namespace {

// Host-side extents of a reference array argument (Fortran declared shape).
struct HostShape {
  int hx, hy, hz;  // 1D arrays: hy = hz = 1
  bool one_d;
};

struct Mirror {
  void* raw = nullptr;      // cudaMalloc'd base
  double* dev = nullptr;    // element (min-2, min-2, min-2)
  HostShape shape{};        // largest declared shape seen
  int planes = 0;           // host planes copied up so far
  bool pinned = false;
  Geom g{};                 // the bounds of the chunk the array belongs to (3D arrays)
};

struct Context {
  bool ready = false;
  Geom g{};
  cudaStream_t stream = nullptr;
  int device = -1;  // the device current when the context was created
  std::unordered_map<const void*, Mirror> mirrors;
  std::vector<void*> scratch;  // arrays standing in for mirrors passed with another chunk's bounds
  unsigned long long* d_key = nullptr;
  double* d_partials = nullptr;
  double* d_sum = nullptr;
  double* stage = nullptr;  // contiguous copy of host planes on their way up or down
  size_t stage_bytes = 0;
  double* msg = nullptr;    // one halo message (pack_kernel.f90) on the device
  size_t msg_bytes = 0;
  // advec_mom's pre/post volumes (advec_mom_kernel.f90 recomputes them in each
  // of a sweep's three velocity calls): the call that formed them last, and
  // the number of library calls made up to it
  long long calls = 0;
  struct {
    long long at = -1;
    int variant = -1;
    const void* in[4] = {nullptr, nullptr, nullptr, nullptr};  // vol_flux_x/y/z, volume
    const void* out[2] = {nullptr, nullptr};                  // pre_vol, post_vol
    Geom g{};
  } mom_vol;
  int status = 0;
  std::string err;
  bool pin_host = true;
  // Bulk-tensor staging of the stencils that have a staged form: allowed
  // (clover_gpu_use_staging), and whether the staged kernels could be set up
  // (0 not tried yet, 1 ready, -1 unavailable). Tensor maps are made once per
  // (array, box rows, layout) and kept until release; a staged kernel whose
  // bounded wait gives up sets a bit in d_status, read back at the next sync.
  bool staging = true;
  int tma_state = 0;
  std::map<std::tuple<const void*, int, int, long long, int>, CUtensorMap> tmaps;
  int* d_status = nullptr;
};

Context& ctx() {
  static Context c;
  return c;
}

void set_error(int bit, const std::string& msg) {
  Context& c = ctx();
  c.status |= bit;
  if (c.err.empty()) c.err = msg;
}

bool check(cudaError_t e, const char* what) {
  if (e == cudaSuccess) return true;
  set_error(CLOVER_STATUS_CUDA_ERROR, std::string(what) + ": " + cudaGetErrorString(e));
  return false;
}

void check_launch(const char* what) { check(cudaGetLastError(), what); }

// Create the context on first use. Each call's bounds select the geometry of
// that call: several chunks may share the process (the reference runs one
// chunk per task; the brick driver runs the bricks of a deck in one process),
// and every array belongs to the chunk whose bounds it was first passed with.
bool enter(const int* x_min, const int* x_max, const int* y_min, const int* y_max,
           const int* z_min, const int* z_max) {
  Context& c = ctx();
  c.calls++;
  if (*x_max < *x_min || *y_max < *y_min || *z_max < *z_min) {
    set_error(CLOVER_STATUS_BAD_ARG, "empty chunk bounds");
    return false;
  }
  if (!c.ready) {
    int n = 0;
    if (cudaGetDeviceCount(&n) != cudaSuccess || n == 0) {
      set_error(CLOVER_STATUS_NO_DEVICE, "no CUDA device");
      return false;
    }
    c.g = make_geom(*x_min, *x_max, *y_min, *y_max, *z_min, *z_max);
    if (!check(cudaGetDevice(&c.device), "device")) return false;
    if (!check(cudaStreamCreateWithFlags(&c.stream, cudaStreamNonBlocking), "stream")) return false;
    if (!check(cudaMalloc(&c.d_key, sizeof(unsigned long long)), "malloc")) return false;
    if (!check(cudaMalloc(&c.d_partials, summary_partials_len() * sizeof(double)), "malloc"))
      return false;
    if (!check(cudaMalloc(&c.d_sum, 5 * sizeof(double)), "malloc")) return false;
    if (!check(cudaMalloc(&c.d_status, sizeof(int)), "malloc")) return false;
    if (!check(cudaMemsetAsync(c.d_status, 0, sizeof(int), c.stream), "status clear")) return false;
    const char* pin = getenv("CLOVER_GPU_PIN_HOST");
    c.pin_host = !(pin && pin[0] == '0');
    c.ready = true;
    return true;
  }
  const Geom& g = c.g;
  if (g.x_min != *x_min || g.x_max != *x_max || g.y_min != *y_min || g.y_max != *y_max ||
      g.z_min != *z_min || g.z_max != *z_max)
    c.g = make_geom(*x_min, *x_max, *y_min, *y_max, *z_min, *z_max);
  return true;
}

bool same_chunk(const Geom& a, const Geom& b) {
  return a.x_min == b.x_min && a.x_max == b.x_max && a.y_min == b.y_min && a.y_max == b.y_max &&
         a.z_min == b.z_min && a.z_max == b.z_max;
}

bool is_device_pointer(const void* p) {
  cudaPointerAttributes a;
  if (cudaPointerGetAttributes(&a, p) != cudaSuccess) {
    cudaGetLastError();
    return false;
  }
  return a.type == cudaMemoryTypeDevice || a.type == cudaMemoryTypeManaged;
}

// The tensor map of a chunk-layout FP64 array with boxes of `rows` rows, made
// on first use; null if the array cannot be staged (the driver refuses the
// map, e.g. a device array passed in place whose base is not 16-byte aligned).
const CUtensorMap* tmap(Context& c, const double* base, const Geom& g, int rows,
                        bool rows_along_z = false) {
  if (!base) return nullptr;
  // box rows along z are keyed as negative row counts
  const auto key = std::make_tuple((const void*)base, rows_along_z ? -rows : rows, g.px, g.pxy,
                                   g.z_max - g.z_min);
  auto it = c.tmaps.find(key);
  if (it != c.tmaps.end()) return &it->second;
  CUtensorMap m;
  if (!encode_plane_map(&m, base, 8, g, rows, rows_along_z)) return nullptr;
  return &(c.tmaps[key] = m);
}

// The maps of n arrays (base, box rows) into out[], in order; false if any
// array has none.
bool tmaps_of(Context& c, const Geom& g, int n, const double* const* base, const int* rows,
              CUtensorMap* out, bool rows_along_z = false) {
  for (int q = 0; q < n; q++) {
    const CUtensorMap* m = tmap(c, base[q], g, rows[q], rows_along_z);
    if (!m) return false;
    out[q] = *m;
  }
  return true;
}

// Whether the staged drop-in kernels may run: allowed, and set up once.
bool staged(Context& c) {
  if (!c.staging) return false;
  if (c.tma_state == 0)
    c.tma_state = pdv_dropin_tma_prepare() && stencils_dropin_tma_prepare() &&
                          mom_node_dropin_tma_prepare()
                      ? 1
                      : -1;
  if (c.tma_state < 0) cudaGetLastError();
  return c.tma_state > 0;
}

// After a synchronisation of the library stream: a staged kernel's bounded
// wait that gave up left a status bit on the device.
void poll_device_status(Context& c) {
  if (!c.d_status) return;
  int st = 0;
  if (cudaMemcpy(&st, c.d_status, sizeof(int), cudaMemcpyDeviceToHost) != cudaSuccess) {
    cudaGetLastError();
    return;
  }
  if (st) {
    set_error(st, "a staged kernel's wait for its bulk copies gave up");
    cudaMemset(c.d_status, 0, sizeof(int));
  }
}

}  // namespace

// The stream the drop-in entry points queue their kernels on, if the library
// context exists and was created on device dev; null otherwise. A call that
// reads arrays those kernels write in place orders itself after them by
// launching on this stream.
cudaStream_t abi_stream_on(int dev) {
  Context& c = ctx();
  return c.ready && c.device == dev ? c.stream : nullptr;
}

// Rows of hx elements between the host's contiguous planes (hy rows each) and
// the mirror's pitched layout (row pitch px, plane pitch pxy): one block per
// row, grid-strided.
__global__ void k_rows_to_pitched(const double* __restrict__ src, double* __restrict__ dst, int hx,
                                  int hy, long long rows, int px, long long pxy) {
  for (long long r = blockIdx.x; r < rows; r += gridDim.x) {
    const double* s = src + r * hx;
    double* d = dst + (r / hy) * pxy + (r % hy) * px;
    for (int i = threadIdx.x; i < hx; i += blockDim.x) d[i] = s[i];
  }
}
__global__ void k_pitched_to_rows(const double* __restrict__ src, double* __restrict__ dst, int hx,
                                  int hy, long long rows, int px, long long pxy) {
  for (long long r = blockIdx.x; r < rows; r += gridDim.x) {
    const double* s = src + (r / hy) * pxy + (r % hy) * px;
    double* d = dst + r * hx;
    for (int i = threadIdx.x; i < hx; i += blockDim.x) d[i] = s[i];
  }
}

// Host <-> device copy of planes [p0,p1) of a 3D mirror: one contiguous DMA
// of the host planes to or from a staging buffer, and a kernel that moves the
// rows between the staging buffer and the pitched mirror (a strided copy of
// ~4 KB rows runs at a fraction of the link's rate).
static void xfer3d(const void* host, Mirror& m, int p0, int p1, bool up) {
  Context& c = ctx();
  if (p1 <= p0) return;
  const HostShape& s = m.shape;
  const size_t host_plane = (size_t)s.hx * s.hy * 8;
  const size_t bytes = host_plane * (size_t)(p1 - p0);
  if (bytes > c.stage_bytes) {
    cudaStreamSynchronize(c.stream);
    cudaFree(c.stage);
    c.stage = nullptr;
    c.stage_bytes = 0;
    if (!check(cudaMalloc(&c.stage, bytes), "staging malloc")) return;
    c.stage_bytes = bytes;
  }
  char* hp = (char*)host + host_plane * p0;
  double* dp = m.dev + m.g.pxy * p0;
  const long long rows = (long long)s.hy * (p1 - p0);
  if (up) {
    check(cudaMemcpyAsync(c.stage, hp, bytes, cudaMemcpyHostToDevice, c.stream), "upload");
    k_rows_to_pitched<<<148 * 8, 256, 0, c.stream>>>(c.stage, dp, s.hx, s.hy, rows, m.g.px,
                                                     m.g.pxy);
    check_launch("upload rows");
  } else {
    k_pitched_to_rows<<<148 * 8, 256, 0, c.stream>>>(dp, c.stage, s.hx, s.hy, rows, m.g.px,
                                                     m.g.pxy);
    check_launch("download rows");
    check(cudaMemcpyAsync(hp, c.stage, bytes, cudaMemcpyDeviceToHost, c.stream), "download");
  }
}

// Resolve a 3D array argument to its device copy.
static double* dev3(double* host, int hx, int hy, int hz) {
  Context& c = ctx();
  if (!host) return nullptr;
  auto it = c.mirrors.find(host);
  if (it == c.mirrors.end()) {
    if (is_device_pointer(host)) return host;
    Mirror m;
    m.g = c.g;
    const long long elems = array_elems(c.g) + kFrontPad<double>;
    if (!check(cudaMalloc(&m.raw, (size_t)elems * 8), "mirror malloc")) return nullptr;
    m.dev = (double*)m.raw + kFrontPad<double>;
    check(cudaMemsetAsync(m.raw, 0, (size_t)elems * 8, c.stream), "mirror clear");
    m.shape = HostShape{hx, hy, hz, false};
    // Page-lock large host arrays for full-bandwidth copies. Only arrays of
    // 64 MiB and more: those are mapped on pages of their own, whereas small
    // heap arrays share pages with their neighbours, and a copy that
    // straddles the end of a locked range is rejected.
    const size_t bytes = (size_t)hx * hy * hz * 8;
    if (c.pin_host && bytes >= ((size_t)64 << 20)) {
      m.pinned = cudaHostRegister(host, bytes, cudaHostRegisterDefault) == cudaSuccess;
      if (!m.pinned) cudaGetLastError();
    }
    it = c.mirrors.emplace(host, m).first;
  }
  Mirror& m = it->second;
  if (!same_chunk(m.g, c.g)) {
    // an array of another chunk: the call runs on a zeroed array of this
    // call's bounds instead (so no access leaves an allocation) and fails
    set_error(CLOVER_STATUS_BOUNDS, "array passed with the bounds of another chunk");
    void* raw = nullptr;
    const long long elems = array_elems(c.g) + kFrontPad<double>;
    if (!check(cudaMalloc(&raw, (size_t)elems * 8), "scratch malloc")) return nullptr;
    check(cudaMemsetAsync(raw, 0, (size_t)elems * 8, c.stream), "scratch clear");
    c.scratch.push_back(raw);
    return (double*)raw + kFrontPad<double>;
  }
  if (hz > m.shape.hz) {
    // A later declaration covers more planes (e.g. post_ener is declared to
    // z_max+2, the same work array elsewhere to z_max+3): a copy may not
    // straddle the end of a page-locked range, so lock the larger range.
    if (m.pinned) {
      cudaHostUnregister(host);
      m.pinned = cudaHostRegister(host, (size_t)hx * hy * hz * 8, cudaHostRegisterDefault) ==
                 cudaSuccess;
      if (!m.pinned) cudaGetLastError();
    }
    m.shape.hz = hz;
  }
  if (hz > m.planes) {
    xfer3d(host, m, m.planes, hz, true);
    m.planes = hz;
  }
  return m.dev;
}

// Resolve a 1D coordinate array argument (n elements from min-2).
static double* dev1(double* host, int n) {
  Context& c = ctx();
  if (!host) return nullptr;
  auto it = c.mirrors.find(host);
  if (it == c.mirrors.end()) {
    if (is_device_pointer(host)) return host;
    Mirror m;
    if (!check(cudaMalloc(&m.raw, (size_t)(n + 32) * 8), "mirror malloc")) return nullptr;
    m.dev = (double*)m.raw;
    m.shape = HostShape{n, 1, 1, true};
    m.shape.hy = n + 32;  // capacity (1D mirrors)
    it = c.mirrors.emplace(host, m).first;
  }
  Mirror& m = it->second;
  if (n > m.shape.hy) {  // a 1D array of a smaller chunk passed with larger bounds
    set_error(CLOVER_STATUS_BOUNDS, "array passed with the bounds of another chunk");
    void* raw = nullptr;
    if (!check(cudaMalloc(&raw, (size_t)(n + 32) * 8), "scratch malloc")) return nullptr;
    check(cudaMemsetAsync(raw, 0, (size_t)(n + 32) * 8, c.stream), "scratch clear");
    c.scratch.push_back(raw);
    return (double*)raw;
  }
  if (m.planes == 0 || n > m.shape.hx) {
    m.shape.hx = n > m.shape.hx ? n : m.shape.hx;
    check(cudaMemcpyAsync(m.dev, host, (size_t)m.shape.hx * 8, cudaMemcpyHostToDevice, c.stream),
          "upload");
    m.planes = 1;
  }
  return m.dev;
}

}  // namespace clover


namespace clover {
// ---------------------------------------------------------------------------
// Halo messages between chunks (pack_kernel.f90). Side 0..5 = left, right,
// bottom, top, back, front. A message holds `depth` layers of the field next
// to that side, over the other two axes' full extents including their halos;
// element (j,k,l) of the loop space goes to the reference's 1-based buffer
// index of pack_kernel.f90 (:78 left/right, :310 bottom/top, :542 back/front).
// pack: field -> buf, unpack: buf -> field; buf[0] holds buffer index `lo`.
struct FaceMsg {
  int side, depth, xi, yi, zi;  // x_inc, y_inc, z_inc of the field type
  int off_a, off_b;             // left/right: y, z offsets; bottom/top: x, z; back/front: x, y
  int gx, gy, gz;               // g_x_max, g_y_max, g_z_max
  long long base, lo;           // buffer_offset; the first buffer index the message covers
  int n0, n1, n2;               // extents of the loop space (j, k, l)
  int j0, k0, l0;               // their first values
};

__host__ __device__ inline long long face_index(const FaceMsg& f, int j, int k, int l) {
  const int d = f.depth;
  if (f.side < 2)
    return f.base + (j + (long long)(k + f.off_a + d - 1) * d) +
           (long long)(l + f.off_b + d - 1) * (f.gy + f.yi + 2 * d) * d;
  const long long rx = f.gx + f.xi + 2 * d;
  if (f.side < 4)
    return f.base + (j + f.off_a + d) + (long long)(l + f.off_b - 1 + d) * rx +
           (long long)(k - 1) * (rx * (f.gz + f.zi + 2 * d));
  return f.base + (j + f.off_a + d) + (long long)(k + f.off_b - 1 + d) * rx +
         (long long)(l - 1) * (rx * (f.gy + f.yi + 2 * d));
}

// The field element a message element comes from (pack) or goes to (unpack).
__device__ inline void face_cell(const Geom& g, const FaceMsg& f, bool pack, int& j, int& k, int& l) {
  switch (f.side) {
    case 0: j = pack ? g.x_min + f.xi - 1 + j : g.x_min - j; break;
    case 1: j = pack ? g.x_max + 1 - j : g.x_max + f.xi + j; break;
    case 2: k = pack ? g.y_min + f.yi - 1 + k : g.y_min - k; break;
    case 3: k = pack ? g.y_max + 1 - k : g.y_max + f.yi + k; break;
    case 4: l = pack ? g.z_min + f.zi - 1 + l : g.z_min - l; break;
    default: l = pack ? g.z_max + 1 - l : g.z_max + f.zi + l; break;
  }
}

__global__ void k_face_msg(Geom g, FaceMsg f, double* __restrict__ field, double* __restrict__ buf,
                           int pack) {
  const long long n = (long long)f.n0 * f.n1 * f.n2;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n;
       i += (long long)gridDim.x * blockDim.x) {
    const int a = (int)(i % f.n0), b = (int)((i / f.n0) % f.n1), c = (int)(i / ((long long)f.n0 * f.n1));
    int j = f.j0 + a, k = f.k0 + b, l = f.l0 + c;
    const long long q = face_index(f, j, k, l) - f.lo;
    face_cell(g, f, pack != 0, j, k, l);
    double* e = field + off3(g, j, k, l);
    if (pack) buf[q] = *e;
    else *e = buf[q];
  }
}

// Several halo messages between chunks of this process in one launch, each
// copied straight from the sender's layers to the receiver's halo: element i
// of the loop space is message element i on both sides (the two chunks share
// the extents of the face), so no buffer is needed. blockIdx.y = message.
struct FaceCopy {
  Geom gs, gd;
  FaceMsg fs, fd;
  const double* src;
  double* dst;
};

__global__ void k_face_copy_batch(const FaceCopy* __restrict__ list) {
  const FaceCopy& c = list[blockIdx.y];
  const long long n = (long long)c.fs.n0 * c.fs.n1 * c.fs.n2;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n;
       i += (long long)gridDim.x * blockDim.x) {
    const int a = (int)(i % c.fs.n0), b = (int)((i / c.fs.n0) % c.fs.n1),
              e = (int)(i / ((long long)c.fs.n0 * c.fs.n1));
    int js = c.fs.j0 + a, ks = c.fs.k0 + b, ls = c.fs.l0 + e;
    int jd = c.fd.j0 + a, kd = c.fd.k0 + b, ld = c.fd.l0 + e;
    face_cell(c.gs, c.fs, true, js, ks, ls);
    face_cell(c.gd, c.fd, false, jd, kd, ld);
    c.dst[off3(c.gd, jd, kd, ld)] = c.src[off3(c.gs, js, ks, ls)];
  }
}

namespace {

// The loop space of pack_kernel.f90 for one side (j innermost), and the
// buffer index range it covers (the index grows with every loop variable).
FaceMsg face_msg(const Geom& g, int side, int depth, int xi, int yi, int zi, int off_a, int off_b,
                 int gx, int gy, int gz, long long base) {
  FaceMsg f;
  f.side = side; f.depth = depth; f.xi = xi; f.yi = yi; f.zi = zi;
  f.off_a = off_a; f.off_b = off_b; f.gx = gx; f.gy = gy; f.gz = gz; f.base = base;
  const int d = depth;
  f.j0 = side < 2 ? 1 : g.x_min - d;
  f.n0 = side < 2 ? d : (g.x_max + xi + d) - (g.x_min - d) + 1;
  f.k0 = (side == 2 || side == 3) ? 1 : g.y_min - d;
  f.n1 = (side == 2 || side == 3) ? d : (g.y_max + yi + d) - (g.y_min - d) + 1;
  f.l0 = side >= 4 ? 1 : g.z_min - d;
  f.n2 = side >= 4 ? d : (g.z_max + zi + d) - (g.z_min - d) + 1;
  f.lo = 0;
  f.lo = face_index(f, f.j0, f.k0, f.l0);
  return f;
}

long long face_len(const FaceMsg& f) {
  return face_index(f, f.j0 + f.n0 - 1, f.k0 + f.n1 - 1, f.l0 + f.n2 - 1) - f.lo + 1;
}

// x_inc, y_inc, z_inc of pack_kernel.f90's field types; false if unknown
bool field_incs(int type, int& xi, int& yi, int& zi) {
  switch (type) {
    case 1: xi = 0; yi = 0; zi = 0; return true;  // cell
    case 2: xi = 1; yi = 1; zi = 1; return true;  // vertex
    case 3: xi = 1; yi = 0; zi = 0; return true;  // x face
    case 4: xi = 0; yi = 1; zi = 0; return true;  // y face
    case 5: xi = 0; yi = 0; zi = 1; return true;  // z face
  }
  return false;
}

// The device copy of a 3D field argument of the given pack_kernel field type.
double* dev_of_type(double* host, int type) {
  const Geom& g = ctx().g;
  const int nx = g.x_max - g.x_min + 1, ny = g.y_max - g.y_min + 1, nz = g.z_max - g.z_min + 1;
  int xi, yi, zi;
  field_incs(type, xi, yi, zi);
  return dev3(host, nx + 4 + xi, ny + 4 + yi, nz + 4 + zi);
}

double* msg_buffer(long long n) {
  Context& c = ctx();
  const size_t bytes = (size_t)n * 8;
  if (bytes > c.msg_bytes) {
    cudaStreamSynchronize(c.stream);
    cudaFree(c.msg);
    c.msg = nullptr;
    c.msg_bytes = 0;
    if (!check(cudaMalloc(&c.msg, bytes), "message malloc")) return nullptr;
    c.msg_bytes = bytes;
  }
  return c.msg;
}

void launch_face(const Geom& g, const FaceMsg& f, double* field, double* buf, bool pack) {
  const long long n = (long long)f.n0 * f.n1 * f.n2;
  const int blocks = (int)((n + 255) / 256 < 148 * 8 ? (n + 255) / 256 : 148 * 8);
  k_face_msg<<<blocks > 0 ? blocks : 1, 256, 0, ctx().stream>>>(g, f, field, buf, pack ? 1 : 0);
  check_launch(pack ? "pack" : "unpack");
}

// clover_pack_message_* / clover_unpack_message_* with a host buffer: the
// message is formed on the device and copied to (or from) the caller's buffer
// at its 1-based buffer_offset indices.
void message(const int* x_min, const int* x_max, const int* y_min, const int* y_max,
             const int* z_min, const int* z_max, double* field, double* buffer,
             const int* cell_data, const int* vertex_data, const int* x_face_data,
             const int* y_face_data, const int* z_face_data, const int* depth,
             const int* field_type, const int* buffer_offset, const int* off_a, const int* off_b,
             const int* g_x_max, const int* g_y_max, const int* g_z_max, int side, bool pack) {
  if (!enter(x_min, x_max, y_min, y_max, z_min, z_max)) return;
  Context& c = ctx();
  int type = 0;
  if (*field_type == *cell_data) type = 1;
  else if (*field_type == *vertex_data) type = 2;
  else if (*field_type == *x_face_data) type = 3;
  else if (*field_type == *y_face_data) type = 4;
  else if (*field_type == *z_face_data) type = 5;
  if (type == 0 || *depth < 1 || *depth > 2) {
    set_error(CLOVER_STATUS_BAD_ARG, "pack/unpack: unknown field type or depth");
    return;
  }
  int xi, yi, zi;
  field_incs(type, xi, yi, zi);
  const FaceMsg f = face_msg(c.g, side, *depth, xi, yi, zi, *off_a, *off_b, *g_x_max, *g_y_max,
                             *g_z_max, *buffer_offset);
  if (f.lo < 1) {
    set_error(CLOVER_STATUS_BAD_ARG, "pack/unpack: buffer index below 1");
    return;
  }
  const long long n = face_len(f);
  double* d_field = dev_of_type(field, type);
  double* d_buf = msg_buffer(n);
  if (!d_field || !d_buf) return;
  double* h = buffer + (f.lo - 1);
  if (pack) {
    // the index range can have gaps (tile offsets, g_*_max beyond the tile)
    // that hold other messages: the range goes up first, so that copying it
    // back rewrites those entries with their own values
    check(cudaMemcpyAsync(d_buf, h, (size_t)n * 8, cudaMemcpyHostToDevice, c.stream), "message up");
    launch_face(c.g, f, d_field, d_buf, true);
    check(cudaMemcpyAsync(h, d_buf, (size_t)n * 8, cudaMemcpyDeviceToHost, c.stream), "message down");
    check(cudaStreamSynchronize(c.stream), "message sync");
  } else {
    check(cudaMemcpyAsync(d_buf, h, (size_t)n * 8, cudaMemcpyHostToDevice, c.stream), "message up");
    launch_face(c.g, f, d_field, d_buf, false);
  }
}

}  // namespace
}  // namespace clover

using namespace clover;

#define BOUNDS x_min, x_max, y_min, y_max, z_min, z_max
#define ENTER()                                   \
  if (!enter(BOUNDS)) return;                     \
  Context& c = ctx();                             \
  const Geom& g = c.g;                            \
  const int nx = *x_max - *x_min + 1, ny = *y_max - *y_min + 1, nz = *z_max - *z_min + 1; \
  (void)nx; (void)ny; (void)nz; (void)g
// declared shapes (build_field.f90:41-146)
#define CELL(p) dev3(p, nx + 4, ny + 4, nz + 4)
#define VERT(p) dev3(p, nx + 5, ny + 5, nz + 5)
#define VERTZ2(p) dev3(p, nx + 5, ny + 5, nz + 4) /* z declared to z_max+2 */
#define XF(p) dev3(p, nx + 5, ny + 4, nz + 4)
#define YF(p) dev3(p, nx + 4, ny + 5, nz + 4)
#define ZF(p) dev3(p, nx + 4, ny + 4, nz + 5)
#define CX(p) dev1(p, nx + 4)
#define CY(p) dev1(p, ny + 4)
#define CZ(p) dev1(p, nz + 4)
#define VX(p) dev1(p, nx + 5)
#define VY(p) dev1(p, ny + 5)
#define VZ(p) dev1(p, nz + 5)

static GeomArrays no_geom() {
  GeomArrays ga;
  memset(&ga, 0, sizeof(ga));
  return ga;
}

extern "C" {

void clover_ideal_gas_kernel(const int* x_min, const int* x_max, const int* y_min,
                             const int* y_max, const int* z_min, const int* z_max,
                             double* density, double* energy, double* pressure,
                             double* soundspeed) {
  ENTER();
  launch_ideal_gas<F64>(g, c.stream, CELL(density), CELL(energy), CELL(pressure), CELL(soundspeed));
  check_launch("ideal_gas");
}

void clover_viscosity_kernel(const int* x_min, const int* x_max, const int* y_min,
                             const int* y_max, const int* z_min, const int* z_max,
                             double* xarea, double* yarea, double* zarea, double* celldx,
                             double* celldy, double* celldz, double* density0,
                             double* pressure, double* viscosity, double* xvel0,
                             double* yvel0, double* zvel0) {
  ENTER();
  GeomArrays ga = no_geom();
  ga.xarea = XF(xarea); ga.yarea = YF(yarea); ga.zarea = ZF(zarea);
  ga.celldx = CX(celldx); ga.celldy = CY(celldy); ga.celldz = CZ(celldz);
  double *d0 = CELL(density0), *pr = CELL(pressure), *vi = CELL(viscosity);
  double *u0 = VERT(xvel0), *v0 = VERT(yvel0), *w0 = VERT(zvel0);
  if (staged(c)) {
    const double* base[8] = {u0, v0, w0, pr, ga.xarea, ga.yarea, ga.zarea, d0};
    const int rows[8] = {9, 9, 9, 10, 8, 8, 8, 8};
    CUtensorMap m[8];
    if (tmaps_of(c, g, 8, base, rows, m)) {
      ViscDropMaps maps;
      maps.u = m[0]; maps.v = m[1]; maps.w = m[2]; maps.p = m[3];
      maps.xa = m[4]; maps.ya = m[5]; maps.za = m[6]; maps.d = m[7];
      launch_viscosity_dropin_tma(g, c.stream, ga, maps, vi, c.d_status);
      check_launch("viscosity");
      return;
    }
  }
  launch_viscosity<F64>(g, c.stream, ga, d0, pr, vi, u0, v0, w0);
  check_launch("viscosity");
}

void clover_calc_dt_kernel(const int* x_min, const int* x_max, const int* y_min,
                           const int* y_max, const int* z_min, const int* z_max,
                           const double* g_small, const double* g_big, const double* dtmin,
                           const double* dtc_safe, const double* dtu_safe,
                           const double* dtv_safe, const double* dtw_safe,
                           const double* dtdiv_safe, double* xarea, double* yarea,
                           double* zarea, double* cellx, double* celly, double* cellz,
                           double* celldx, double* celldy, double* celldz, double* volume,
                           double* density0, double* energy0, double* pressure,
                           double* viscosity_a, double* soundspeed, double* xvel0,
                           double* yvel0, double* zvel0, double* dt_min, double* dt_min_val,
                           int* dtl_control, double* xl_pos, double* yl_pos, double* zl_pos,
                           int* jldt, int* kldt, int* lldt, int* small) {
  ENTER();
  (void)energy0;
  (void)pressure;
  GeomArrays ga = no_geom();
  ga.xarea = XF(xarea); ga.yarea = YF(yarea); ga.zarea = ZF(zarea);
  ga.celldx = CX(celldx); ga.celldy = CY(celldy); ga.celldz = CZ(celldz);
  ga.volume = CELL(volume);
  const unsigned long long init = min_key_of(*g_big);
  check(cudaMemcpyAsync(c.d_key, &init, sizeof(init), cudaMemcpyHostToDevice, c.stream), "key");
  double *d0 = CELL(density0), *qa = CELL(viscosity_a), *ss = CELL(soundspeed);
  double *u0 = VERT(xvel0), *v0 = VERT(yvel0), *w0 = VERT(zvel0), *dtm = VERT(dt_min);
  bool done = false;
  if (staged(c)) {
    const double* base[10] = {u0, v0, w0, ss, qa, d0, ga.volume, ga.xarea, ga.yarea, ga.zarea};
    const int rows[10] = {9, 9, 9, 8, 8, 8, 8, 8, 8, 8};
    CUtensorMap m[10];
    if (tmaps_of(c, g, 10, base, rows, m)) {
      DtDropMaps maps;
      maps.u = m[0]; maps.v = m[1]; maps.w = m[2]; maps.ss = m[3]; maps.q = m[4];
      maps.d = m[5]; maps.vol = m[6]; maps.xa = m[7]; maps.ya = m[8]; maps.za = m[9];
      launch_calc_dt_dropin_tma(g, c.stream, ga, *g_small, *dtc_safe, *dtu_safe, *dtv_safe,
                                *dtw_safe, *dtdiv_safe, maps, dtm, c.d_key, c.d_status);
      done = true;
    }
  }
  if (!done)
    launch_calc_dt<F64>(g, c.stream, ga, *g_small, *dtc_safe, *dtu_safe, *dtv_safe, *dtw_safe,
                        *dtdiv_safe, d0, qa, ss, u0, v0, w0, dtm, c.d_key);
  check_launch("calc_dt");
  unsigned long long key = init;
  check(cudaMemcpyAsync(&key, c.d_key, sizeof(key), cudaMemcpyDeviceToHost, c.stream), "key");
  check(cudaStreamSynchronize(c.stream), "calc_dt sync");
  poll_device_status(c);
  *dt_min_val = min_key_value(key);
  // calc_dt_kernel.f90:154-161: jkl_control is the constant 1.1 (a default
  // REAL), so these outputs never depend on the field.
  double jkl_control = (double)1.1f;
  *dtl_control = (int)((double)10.01f * (jkl_control - (double)(int)jkl_control));
  jkl_control = jkl_control - (jkl_control - (double)(int)jkl_control);
  *jldt = ((int)jkl_control) % (*x_max);
  *kldt = (int)(1.0 + (jkl_control / (double)(*x_max)));
  *lldt = (int)(1.0 + (jkl_control / (double)(*x_max)));
  const double* px = is_device_pointer(cellx) ? nullptr : cellx;
  const double* py = is_device_pointer(celly) ? nullptr : celly;
  const double* pz = is_device_pointer(cellz) ? nullptr : cellz;
  *xl_pos = px ? px[*jldt - *x_min + 2] : 0.0;
  *yl_pos = py ? py[*kldt - *y_min + 2] : 0.0;
  *zl_pos = pz ? pz[*lldt - *z_min + 2] : 0.0;
  *small = *dt_min_val < *dtmin ? 1 : 0;
  if (*small) {
    c.status |= CLOVER_STATUS_SMALL_DT;
    fprintf(stderr, "Timestep information:\n timestep : %.17g\n", *dt_min_val);
  }
}

void clover_pdv_kernel(const int32_t* predict, const int* x_min, const int* x_max,
                       const int* y_min, const int* y_max, const int* z_min, const int* z_max,
                       const double* dt, double* xarea, double* yarea, double* zarea,
                       double* volume, double* density0, double* density1, double* energy0,
                       double* energy1, double* pressure, double* viscosity, double* xvel0,
                       double* xvel1, double* yvel0, double* yvel1, double* zvel0,
                       double* zvel1) {
  ENTER();
  GeomArrays ga = no_geom();
  ga.xarea = XF(xarea); ga.yarea = YF(yarea); ga.zarea = ZF(zarea); ga.volume = CELL(volume);
  double *d0 = CELL(density0), *d1 = CELL(density1), *e0 = CELL(energy0), *e1 = CELL(energy1);
  double *pr = CELL(pressure), *vi = CELL(viscosity);
  double *u0 = VERT(xvel0), *u1 = VERT(xvel1), *v0 = VERT(yvel0), *v1 = VERT(yvel1);
  double *w0 = VERT(zvel0), *w1 = VERT(zvel1);
  const bool pred = *predict != 0;
  // the planes staged by bulk-tensor copies when every staged array has a map
  // (the corrector's time level 1 velocities too)
  if (staged(c)) {
    const CUtensorMap* m[9] = {tmap(c, u0, g, 9), tmap(c, v0, g, 9), tmap(c, w0, g, 9),
                               pred ? nullptr : tmap(c, u1, g, 9),
                               pred ? nullptr : tmap(c, v1, g, 9),
                               pred ? nullptr : tmap(c, w1, g, 9),
                               tmap(c, ga.xarea, g, 8), tmap(c, ga.yarea, g, 9),
                               tmap(c, ga.zarea, g, 8)};
    bool ok = true;
    for (int q = 0; q < 9; q++) ok = ok && (m[q] || (pred && q >= 3 && q <= 5));
    if (ok) {
      PdvDropMaps maps;
      maps.u0 = *m[0]; maps.v0 = *m[1]; maps.w0 = *m[2];
      if (!pred) { maps.u1 = *m[3]; maps.v1 = *m[4]; maps.w1 = *m[5]; }
      else { maps.u1 = *m[0]; maps.v1 = *m[1]; maps.w1 = *m[2]; }
      maps.xa = *m[6]; maps.ya = *m[7]; maps.za = *m[8];
      launch_pdv_dropin_tma(g, c.stream, pred, *dt, maps, ga.volume, d0, d1, e0, e1, pr, vi,
                            c.d_status);
      check_launch("PdV");
      return;
    }
  }
  launch_pdv<F64>(g, c.stream, pred, *dt, nullptr, ga, d0, d1, e0, e1, pr, vi, u0, u1, v0, v1, w0,
                  w1);
  check_launch("PdV");
}

void clover_revert_kernel(const int* x_min, const int* x_max, const int* y_min,
                          const int* y_max, const int* z_min, const int* z_max,
                          double* density0, double* density1, double* energy0,
                          double* energy1) {
  ENTER();
  launch_revert<F64>(g, c.stream, CELL(density0), CELL(density1), CELL(energy0), CELL(energy1));
  check_launch("revert");
}

void clover_accelerate_kernel(const int* x_min, const int* x_max, const int* y_min,
                              const int* y_max, const int* z_min, const int* z_max,
                              const double* dt, double* xarea, double* yarea, double* zarea,
                              double* volume, double* density0, double* pressure,
                              double* viscosity, double* xvel0, double* yvel0, double* zvel0,
                              double* xvel1, double* yvel1, double* zvel1) {
  ENTER();
  GeomArrays ga = no_geom();
  ga.xarea = XF(xarea); ga.yarea = YF(yarea); ga.zarea = ZF(zarea); ga.volume = CELL(volume);
  double *d0 = CELL(density0), *pr = CELL(pressure), *vi = CELL(viscosity);
  double *u0 = VERT(xvel0), *v0 = VERT(yvel0), *w0 = VERT(zvel0);
  double *u1 = VERT(xvel1), *v1 = VERT(yvel1), *w1 = VERT(zvel1);
  if (staged(c)) {
    const double* base[10] = {d0, ga.volume, pr, vi, ga.xarea, ga.zarea, ga.yarea, u0, v0, w0};
    const int rows[10] = {9, 9, 9, 9, 9, 9, 8, 8, 8, 8};
    CUtensorMap m[10];
    if (tmaps_of(c, g, 10, base, rows, m)) {
      AccDropMaps maps;
      maps.d = m[0]; maps.vol = m[1]; maps.p = m[2]; maps.q = m[3]; maps.xa = m[4];
      maps.za = m[5]; maps.ya = m[6]; maps.u = m[7]; maps.v = m[8]; maps.w = m[9];
      launch_accelerate_dropin_tma(g, c.stream, *dt, maps, u1, v1, w1, c.d_status);
      check_launch("accelerate");
      return;
    }
  }
  launch_accelerate<F64>(g, c.stream, *dt, nullptr, ga, d0, pr, vi, u0, v0, w0, u1, v1, w1);
  check_launch("accelerate");
}

void clover_flux_calc_kernel(const int* x_min, const int* x_max, const int* y_min,
                             const int* y_max, const int* z_min, const int* z_max,
                             const double* dt, double* xarea, double* yarea, double* zarea,
                             double* xvel0, double* yvel0, double* zvel0, double* xvel1,
                             double* yvel1, double* zvel1, double* vol_flux_x,
                             double* vol_flux_y, double* vol_flux_z) {
  ENTER();
  GeomArrays ga = no_geom();
  ga.xarea = XF(xarea); ga.yarea = YF(yarea); ga.zarea = ZF(zarea);
  launch_flux_calc<F64>(g, c.stream, *dt, nullptr, ga, VERT(xvel0), VERT(yvel0), VERT(zvel0),
                        VERT(xvel1), VERT(yvel1), VERT(zvel1), XF(vol_flux_x), YF(vol_flux_y),
                        ZF(vol_flux_z));
  check_launch("flux_calc");
}

void clover_advec_cell_kernel(const int* x_min, const int* x_max, const int* y_min,
                              const int* y_max, const int* z_min, const int* z_max,
                              const int32_t* advect_x, const int* dir, const int* sweep_number,
                              double* vertexdx, double* vertexdy, double* vertexdz,
                              double* volume, double* density1, double* energy1,
                              double* mass_flux_x, double* vol_flux_x, double* mass_flux_y,
                              double* vol_flux_y, double* mass_flux_z, double* vol_flux_z,
                              double* pre_vol, double* post_vol, double* pre_mass,
                              double* post_mass, double* advec_vol, double* post_ener,
                              double* ener_flux) {
  ENTER();
  GeomArrays ga = no_geom();
  ga.vertexdx = VX(vertexdx); ga.vertexdy = VY(vertexdy); ga.vertexdz = VZ(vertexdz);
  ga.volume = CELL(volume);
  double* work[7] = {VERT(pre_vol), VERT(post_vol), VERT(pre_mass), VERT(post_mass),
                     VERT(advec_vol), VERTZ2(post_ener), VERTZ2(ener_flux)};
  launch_advec_cell<F64>(g, c.stream, *advect_x != 0, *dir, *sweep_number, ga, CELL(density1),
                         CELL(energy1), XF(mass_flux_x), XF(vol_flux_x), YF(mass_flux_y),
                         YF(vol_flux_y), ZF(mass_flux_z), ZF(vol_flux_z), work);
  check_launch("advec_cell");
}

void clover_advec_mom_kernel(const int* x_min, const int* x_max, const int* y_min,
                             const int* y_max, const int* z_min, const int* z_max,
                             double* vel1, double* mass_flux_x, double* vol_flux_x,
                             double* mass_flux_y, double* vol_flux_y, double* mass_flux_z,
                             double* vol_flux_z, double* volume, double* density1,
                             double* node_flux, double* node_mass_post, double* node_mass_pre,
                             double* advec_vel, double* mom_flux, double* pre_vol,
                             double* post_vol, double* celldx, double* celldy, double* celldz,
                             const int32_t* advect_x, const int* which_vel,
                             const int* sweep_number, const int* direction) {
  ENTER();
  GeomArrays ga = no_geom();
  ga.volume = CELL(volume);
  ga.celldx = CX(celldx); ga.celldy = CY(celldy); ga.celldz = CZ(celldz);
  double* work[7] = {VERT(node_flux), VERT(node_mass_post), VERT(node_mass_pre),
                     VERT(advec_vel), VERT(mom_flux), VERT(pre_vol), VERT(post_vol)};
  // The pre/post volumes depend only on the sweep's variant, the volume
  // fluxes and the volume. They are formed again only if another library call
  // (or a host change: clover_gpu_invalidate*) came since the advec_mom call
  // that last formed them, or that call had another variant or other arrays.
  // A call whose other outputs alias them forms them again too.
  const int variant = mom_vol_variant(*advect_x != 0, *sweep_number, *direction);
  const void* in[4] = {vol_flux_x, vol_flux_y, vol_flux_z, volume};
  const void* out[2] = {pre_vol, post_vol};
  const void* others[6] = {vel1, node_flux, node_mass_post, node_mass_pre, advec_vel, mom_flux};
  bool skip = variant >= 0 && c.mom_vol.at == c.calls - 1 && c.mom_vol.variant == variant &&
              same_chunk(c.mom_vol.g, g);
  for (int q = 0; q < 4 && skip; q++) skip = c.mom_vol.in[q] == in[q];
  for (int q = 0; q < 2 && skip; q++) skip = c.mom_vol.out[q] == out[q];
  bool aliased = pre_vol == post_vol;
  for (int q = 0; q < 6; q++) aliased = aliased || others[q] == pre_vol || others[q] == post_vol;
  for (int q = 0; q < 4; q++) aliased = aliased || in[q] == pre_vol || in[q] == post_vol;
  skip = skip && !aliased;
  double *v1 = VERT(vel1), *mfx = XF(mass_flux_x), *vfx = XF(vol_flux_x);
  double *mfy = YF(mass_flux_y), *vfy = YF(vol_flux_y), *mfz = ZF(mass_flux_z);
  double *vfz = ZF(vol_flux_z), *d1 = CELL(density1);
  // the node pass staged by bulk-tensor copies, between the volumes it reads
  // and the flux + update
  bool staged_node = false;
  NodeDropMaps nmaps;
  const int dir = *direction;
  if (*which_vel == 1 && staged(c)) {
    const double* base[3] = {dir == 1 ? mfx : dir == 2 ? mfy : mfz, d1, work[6]};
    const int rows[3] = {9, 9, 9};
    CUtensorMap m[3];
    if (tmaps_of(c, g, 3, base, rows, m, dir == 2)) {
      nmaps.mf = m[0]; nmaps.d = m[1]; nmaps.pv = m[2];
      staged_node = true;
    }
  }
  if (staged_node) {
    launch_advec_mom<F64>(g, c.stream, v1, mfx, vfx, mfy, vfy, mfz, vfz, ga, d1, work,
                          *advect_x != 0, *which_vel, *sweep_number, dir, skip, kMomVolumes);
    launch_mom_node_dropin_tma(g, c.stream, dir, nmaps, work[0], work[1], work[2], c.d_status);
    launch_advec_mom<F64>(g, c.stream, v1, mfx, vfx, mfy, vfy, mfz, vfz, ga, d1, work,
                          *advect_x != 0, *which_vel, *sweep_number, dir, true, kMomFluxUpdate);
  } else {
    launch_advec_mom<F64>(g, c.stream, v1, mfx, vfx, mfy, vfy, mfz, vfz, ga, d1, work,
                          *advect_x != 0, *which_vel, *sweep_number, dir, skip);
  }
  check_launch("advec_mom");
  c.mom_vol.at = (variant >= 0 && !aliased && c.status == 0) ? c.calls : -1;
  c.mom_vol.variant = variant;
  c.mom_vol.g = g;
  for (int q = 0; q < 4; q++) c.mom_vol.in[q] = in[q];
  for (int q = 0; q < 2; q++) c.mom_vol.out[q] = out[q];
}

void clover_reset_field_kernel(const int* x_min, const int* x_max, const int* y_min,
                               const int* y_max, const int* z_min, const int* z_max,
                               double* density0, double* density1, double* energy0,
                               double* energy1, double* xvel0, double* xvel1, double* yvel0,
                               double* yvel1, double* zvel0, double* zvel1) {
  ENTER();
  launch_reset_field<F64>(g, c.stream, CELL(density0), CELL(density1), CELL(energy0),
                          CELL(energy1), VERT(xvel0), VERT(xvel1), VERT(yvel0), VERT(yvel1),
                          VERT(zvel0), VERT(zvel1));
  check_launch("reset_field");
}

void clover_field_summary_kernel(const int* x_min, const int* x_max, const int* y_min,
                                 const int* y_max, const int* z_min, const int* z_max,
                                 double* volume, double* density0, double* energy0,
                                 double* pressure, double* xvel0, double* yvel0, double* zvel0,
                                 double* vol, double* mass, double* ie, double* ke,
                                 double* press) {
  ENTER();
  launch_field_summary<F64>(g, c.stream, CELL(volume), CELL(density0), CELL(energy0),
                            CELL(pressure), VERTZ2(xvel0), VERTZ2(yvel0), VERTZ2(zvel0),
                            c.d_partials, c.d_sum);
  check_launch("field_summary");
  double s[5] = {0, 0, 0, 0, 0};
  check(cudaMemcpyAsync(s, c.d_sum, sizeof(s), cudaMemcpyDeviceToHost, c.stream), "summary");
  check(cudaStreamSynchronize(c.stream), "summary sync");
  poll_device_status(c);
  *vol = s[0]; *mass = s[1]; *ie = s[2]; *ke = s[3]; *press = s[4];
}

void clover_update_halo_kernel(const int* x_min, const int* x_max, const int* y_min,
                               const int* y_max, const int* z_min, const int* z_max,
                               const int* chunk_neighbours, const int* tile_neighbours,
                               double* density0, double* energy0, double* pressure,
                               double* viscosity, double* soundspeed, double* density1,
                               double* energy1, double* xvel0, double* yvel0, double* zvel0,
                               double* xvel1, double* yvel1, double* zvel1,
                               double* vol_flux_x, double* vol_flux_y, double* vol_flux_z,
                               double* mass_flux_x, double* mass_flux_y, double* mass_flux_z,
                               const int* fields, const int* depth) {
  ENTER();
  if (*depth < 1 || *depth > 2) {  // the halo is two cells deep
    set_error(CLOVER_STATUS_BAD_ARG, "update_halo depth must be 1 or 2");
    return;
  }
  int ext[6];
  for (int f = 0; f < 6; f++) ext[f] = chunk_neighbours[f] == -1 && tile_neighbours[f] == -1;
  HaloFields hf;
  double* host[19] = {density0, density1, energy0, energy1, pressure, viscosity, soundspeed,
                      xvel0, xvel1, yvel0, yvel1, zvel0, zvel1, vol_flux_x, vol_flux_y,
                      vol_flux_z, mass_flux_x, mass_flux_y, mass_flux_z};
  for (int i = 0; i < 19; i++) {
    hf.f[i] = nullptr;
    if (fields[i] != 1) continue;
    if (i < 7) hf.f[i] = CELL(host[i]);
    else if (i < 13) hf.f[i] = VERT(host[i]);
    else if (i == 13 || i == 16) hf.f[i] = XF(host[i]);
    else if (i == 14 || i == 17) hf.f[i] = YF(host[i]);
    else hf.f[i] = ZF(host[i]);
  }
  launch_update_halo<F64>(g, c.stream, hf, fields, *depth, ext);
  check_launch("update_halo");
}

void clover_initialise_chunk_kernel(const int* x_min, const int* x_max, const int* y_min,
                                    const int* y_max, const int* z_min, const int* z_max,
                                    const double* xmin, const double* ymin, const double* zmin,
                                    const double* dx, const double* dy, const double* dz,
                                    double* vertexx, double* vertexdx, double* vertexy,
                                    double* vertexdy, double* vertexz, double* vertexdz,
                                    double* cellx, double* celldx, double* celly,
                                    double* celldy, double* cellz, double* celldz,
                                    double* volume, double* xarea, double* yarea,
                                    double* zarea) {
  ENTER();
  launch_initialise_chunk(g, c.stream, *xmin, *ymin, *zmin, *dx, *dy, *dz, VX(vertexx),
                          VX(vertexdx), VY(vertexy), VY(vertexdy), VZ(vertexz), VZ(vertexdz),
                          CX(cellx), CX(celldx), CY(celly), CY(celldy), CZ(cellz), CZ(celldz),
                          CELL(volume), XF(xarea), YF(yarea), ZF(zarea));
  check_launch("initialise_chunk");
}

void clover_generate_chunk_kernel(const int* x_min, const int* x_max, const int* y_min,
                                  const int* y_max, const int* z_min, const int* z_max,
                                  double* vertexx, double* vertexy, double* vertexz,
                                  double* cellx, double* celly, double* cellz,
                                  double* density0, double* energy0, double* xvel0,
                                  double* yvel0, double* zvel0, const int* number_of_states,
                                  const double* state_density, const double* state_energy,
                                  const double* state_xvel, const double* state_yvel,
                                  const double* state_zvel, const double* state_xmin,
                                  const double* state_xmax, const double* state_ymin,
                                  const double* state_ymax, const double* state_zmin,
                                  const double* state_zmax, const double* state_radius,
                                  const int* state_geometry, const int* g_rect,
                                  const int* g_circ, const int* g_point) {
  ENTER();
  if (*number_of_states < 1 || *number_of_states > 16) {
    set_error(CLOVER_STATUS_BAD_ARG, "generate_chunk supports 1..16 states");
    return;
  }
  StateTable st;
  st.n = *number_of_states;
  for (int i = 0; i < st.n; i++) {
    st.density[i] = state_density[i]; st.energy[i] = state_energy[i];
    st.xvel[i] = state_xvel[i]; st.yvel[i] = state_yvel[i]; st.zvel[i] = state_zvel[i];
    st.xmin[i] = state_xmin[i]; st.xmax[i] = state_xmax[i];
    st.ymin[i] = state_ymin[i]; st.ymax[i] = state_ymax[i];
    st.zmin[i] = state_zmin[i]; st.zmax[i] = state_zmax[i];
    st.radius[i] = state_radius[i];
    // map the caller's geometry codes onto 1 cuboid, 2 sphere, 3 point
    const int gc = state_geometry[i];
    st.geometry[i] = gc == *g_rect ? 1 : gc == *g_circ ? 2 : gc == *g_point ? 3 : 0;
  }
  GeomArrays ga = no_geom();
  ga.vertexx = VX(vertexx); ga.vertexy = VY(vertexy); ga.vertexz = VZ(vertexz);
  ga.cellx = CX(cellx); ga.celly = CY(celly); ga.cellz = CZ(cellz);
  launch_generate_chunk<F64>(g, c.stream, ga, CELL(density0), CELL(energy0), VERT(xvel0),
                             VERT(yvel0), VERT(zvel0), st);
  check_launch("generate_chunk");
}


#define MSG_ARGS                                                                                  \
  const int *x_min, const int *x_max, const int *y_min, const int *y_max, const int *z_min,      \
      const int *z_max, double *field, double *buffer, const int *cell_data,                     \
      const int *vertex_data, const int *x_face_data, const int *y_face_data,                    \
      const int *z_face_data, const int *depth, const int *field_type, const int *buffer_offset, \
      const int *off_a, const int *off_b, const int *g_x_max, const int *g_y_max,                \
      const int *g_z_max
#define MSG_PASS                                                                                  \
  x_min, x_max, y_min, y_max, z_min, z_max, field, buffer, cell_data, vertex_data, x_face_data,  \
      y_face_data, z_face_data, depth, field_type, buffer_offset, off_a, off_b, g_x_max,         \
      g_y_max, g_z_max
void clover_pack_message_left(MSG_ARGS) { message(MSG_PASS, 0, true); }
void clover_unpack_message_left(MSG_ARGS) { message(MSG_PASS, 0, false); }
void clover_pack_message_right(MSG_ARGS) { message(MSG_PASS, 1, true); }
void clover_unpack_message_right(MSG_ARGS) { message(MSG_PASS, 1, false); }
void clover_pack_message_bottom(MSG_ARGS) { message(MSG_PASS, 2, true); }
void clover_unpack_message_bottom(MSG_ARGS) { message(MSG_PASS, 2, false); }
void clover_pack_message_top(MSG_ARGS) { message(MSG_PASS, 3, true); }
void clover_unpack_message_top(MSG_ARGS) { message(MSG_PASS, 3, false); }
void clover_pack_message_back(MSG_ARGS) { message(MSG_PASS, 4, true); }
void clover_unpack_message_back(MSG_ARGS) { message(MSG_PASS, 4, false); }
void clover_pack_message_front(MSG_ARGS) { message(MSG_PASS, 5, true); }
void clover_unpack_message_front(MSG_ARGS) { message(MSG_PASS, 5, false); }
#undef MSG_PASS
#undef MSG_ARGS

int clover_gpu_face_copy_many(int n, const int* src_bounds, double* const* src,
                              const int* dst_bounds, double* const* dst, const int* sides,
                              const int* field_types, int depth) {
  if (n <= 0) return 0;
  if (depth < 1 || depth > 2) {
    set_error(CLOVER_STATUS_BAD_ARG, "face_copy_many: depth must be 1 or 2");
    return -1;
  }
  std::vector<FaceCopy> list((size_t)n);
  long long longest = 0;
  for (int m = 0; m < n; m++) {
    int xi, yi, zi;
    const int side = sides[m];
    if (side < 0 || side > 5 || !field_incs(field_types[m], xi, yi, zi)) {
      set_error(CLOVER_STATUS_BAD_ARG, "face_copy_many: bad side or field type");
      return -1;
    }
    const int* a = src_bounds + 6 * m;
    const int* b = dst_bounds + 6 * m;
    FaceCopy& c = list[m];
    if (!enter(a, a + 1, a + 2, a + 3, a + 4, a + 5)) return -1;
    c.gs = ctx().g;
    c.fs = face_msg(c.gs, side, depth, xi, yi, zi, 0, 0, c.gs.x_max, c.gs.y_max, c.gs.z_max, 1);
    c.src = dev_of_type(src[m], field_types[m]);
    if (!enter(b, b + 1, b + 2, b + 3, b + 4, b + 5)) return -1;
    c.gd = ctx().g;
    c.fd = face_msg(c.gd, side ^ 1, depth, xi, yi, zi, 0, 0, c.gd.x_max, c.gd.y_max, c.gd.z_max, 1);
    c.dst = dev_of_type(dst[m], field_types[m]);
    if (c.fs.n0 != c.fd.n0 || c.fs.n1 != c.fd.n1 || c.fs.n2 != c.fd.n2) {
      set_error(CLOVER_STATUS_BAD_ARG, "face_copy_many: the two chunks' faces differ in extent");
      return -1;
    }
    if (!c.src || !c.dst) return -1;
    const long long len = (long long)c.fs.n0 * c.fs.n1 * c.fs.n2;
    if (len > longest) longest = len;
  }
  Context& c = ctx();
  const size_t bytes = list.size() * sizeof(FaceCopy);
  double* d_list = msg_buffer((long long)((bytes + 7) / 8));
  if (!d_list) return -1;
  check(cudaMemcpyAsync(d_list, list.data(), bytes, cudaMemcpyHostToDevice, c.stream), "face list");
  // the list is read by the kernel before the next call can change the host copy:
  // the copy above is from pageable memory, which the runtime stages before returning
  long long bx = (longest + 255) / 256;
  if (bx > 64) bx = 64;
  k_face_copy_batch<<<dim3((unsigned)bx, (unsigned)n), 256, 0, c.stream>>>((const FaceCopy*)d_list);
  check_launch("face_copy_many");
  return c.status == 0 ? 0 : -1;
}

long long clover_gpu_message_len(const int* bounds, int side, int field_type, int depth) {
  int xi, yi, zi;
  if (side < 0 || side > 5 || depth < 1 || depth > 2 || !field_incs(field_type, xi, yi, zi))
    return -1;
  const Geom g = make_geom(bounds[0], bounds[1], bounds[2], bounds[3], bounds[4], bounds[5]);
  return face_len(face_msg(g, side, depth, xi, yi, zi, 0, 0, g.x_max, g.y_max, g.z_max, 1));
}

int clover_gpu_pack_device(const int* bounds, double* field, int side, int field_type, int depth,
                           double* dev_msg, int unpack) {
  int xi, yi, zi;
  if (side < 0 || side > 5 || depth < 1 || depth > 2 || !field_incs(field_type, xi, yi, zi)) {
    set_error(CLOVER_STATUS_BAD_ARG, "pack_device: bad side, depth or field type");
    return -1;
  }
  if (!enter(bounds, bounds + 1, bounds + 2, bounds + 3, bounds + 4, bounds + 5)) return -1;
  Context& c = ctx();
  const Geom g = c.g;
  const FaceMsg f = face_msg(g, side, depth, xi, yi, zi, 0, 0, g.x_max, g.y_max, g.z_max, 1);
  double* d_field = dev_of_type(field, field_type);
  if (!d_field || !dev_msg) return -1;
  launch_face(g, f, d_field, dev_msg, unpack == 0);
  return c.status == 0 ? 0 : -1;
}

void clover_gpu_face_copy(const int* src_bounds, double* src, const int* dst_bounds, double* dst,
                          int side, int field_type, int depth) {
  const int* a = src_bounds;
  const int* b = dst_bounds;
  int xi, yi, zi;
  if (side < 0 || side > 5 || depth < 1 || depth > 2 || !field_incs(field_type, xi, yi, zi)) {
    set_error(CLOVER_STATUS_BAD_ARG, "face_copy: bad side, depth or field type");
    return;
  }
  if (!enter(a, a + 1, a + 2, a + 3, a + 4, a + 5)) return;
  Context& c = ctx();
  const Geom gs = c.g;
  const FaceMsg fs = face_msg(gs, side, depth, xi, yi, zi, 0, 0, gs.x_max, gs.y_max, gs.z_max, 1);
  double* d_src = dev_of_type(src, field_type);
  if (!enter(b, b + 1, b + 2, b + 3, b + 4, b + 5)) return;
  const Geom gd = c.g;
  const int other = side ^ 1;  // the receiver unpacks on the opposite side
  const FaceMsg fd = face_msg(gd, other, depth, xi, yi, zi, 0, 0, gd.x_max, gd.y_max, gd.z_max, 1);
  if (face_len(fs) != face_len(fd)) {
    set_error(CLOVER_STATUS_BAD_ARG, "face_copy: the two chunks' faces differ in extent");
    return;
  }
  double* d_dst = dev_of_type(dst, field_type);
  double* d_buf = msg_buffer(face_len(fs));
  if (!d_src || !d_dst || !d_buf) return;
  launch_face(gs, fs, d_src, d_buf, true);
  launch_face(gd, fd, d_dst, d_buf, false);
}

int clover_gpu_status(void) { return ctx().status; }

void clover_gpu_use_staging(int on) { ctx().staging = on != 0; }

int clover_gpu_wait_selftest_queued(long long cycles) {
  Context& c = ctx();
  if (!c.ready) return CLOVER_STATUS_NO_DEVICE;
  launch_wait_selftest(c.stream, cycles, c.d_status);
  return check(cudaGetLastError(), "wait selftest") ? 0 : CLOVER_STATUS_CUDA_ERROR;
}

const char* clover_gpu_error_string(void) { return ctx().err.c_str(); }

void clover_gpu_clear_status(void) {
  ctx().status = 0;
  ctx().err.clear();
}

void clover_gpu_sync_to_host(void) {
  Context& c = ctx();
  if (!c.ready) return;
  for (auto& kv : c.mirrors) {
    Mirror& m = kv.second;
    if (m.shape.one_d)
      check(cudaMemcpyAsync((void*)kv.first, m.dev, (size_t)m.shape.hx * 8,
                            cudaMemcpyDeviceToHost, c.stream), "download");
    else
      xfer3d(kv.first, m, 0, m.planes, false);
  }
  check(cudaStreamSynchronize(c.stream), "sync_to_host");
  poll_device_status(c);
}

void clover_gpu_invalidate(const void* host_array) {
  Context& c = ctx();
  c.mom_vol.at = -1;
  auto it = c.mirrors.find(host_array);
  if (it != c.mirrors.end()) it->second.planes = 0;
}

void clover_gpu_invalidate_all(void) {
  Context& c = ctx();
  c.mom_vol.at = -1;
  for (auto& kv : c.mirrors) kv.second.planes = 0;
}

void clover_gpu_synchronize(void) {
  Context& c = ctx();
  if (!c.ready) return;
  check(cudaStreamSynchronize(c.stream), "synchronize");
  poll_device_status(c);
}

void clover_gpu_release(void) {
  Context& c = ctx();
  if (!c.ready) return;
  cudaStreamSynchronize(c.stream);
  for (auto& kv : c.mirrors) {
    if (kv.second.pinned) cudaHostUnregister((void*)kv.first);
    cudaFree(kv.second.raw);
  }
  c.mirrors.clear();
  c.mom_vol.at = -1;
  for (void* p : c.scratch) cudaFree(p);
  c.scratch.clear();
  cudaFree(c.d_key);
  cudaFree(c.d_partials);
  cudaFree(c.d_sum);
  cudaFree(c.d_status);
  c.d_status = nullptr;
  c.tmaps.clear();
  c.tma_state = 0;
  cudaFree(c.stage);
  c.stage = nullptr;
  c.stage_bytes = 0;
  cudaFree(c.msg);
  c.msg = nullptr;
  c.msg_bytes = 0;
  cudaStreamDestroy(c.stream);
  c.stream = nullptr;
  c.device = -1;
  c.ready = false;
}

void clover_gpu_layout(const int* x_min, const int* x_max, const int* y_min, const int* y_max,
                       const int* z_min, const int* z_max, int* px, long long* pxy,
                       long long* elems) {
  const Geom g = make_geom(*x_min, *x_max, *y_min, *y_max, *z_min, *z_max);
  *px = g.px;
  *pxy = g.pxy;
  *elems = array_elems(g);
}

void clover_gpu_mirror_stats(int* arrays, long long* bytes) {
  Context& c = ctx();
  long long b = 0;
  for (auto& kv : c.mirrors)
    b += kv.second.shape.one_d ? (long long)(kv.second.shape.hx + 32) * 8
                               : (array_elems(kv.second.g) + kFrontPad<double>) * 8;
  *arrays = (int)c.mirrors.size();
  *bytes = b;
}

}  // extern "C"
