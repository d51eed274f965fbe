// sph_noalloc.cu — SPH density by direct summation for callers that cannot
// allocate device memory.
//
// Some callers of this library must not call cudaMalloc: a code that runs
// inside another application's fixed device-memory budget (an in-situ
// analysis hook handed particle arrays by a host simulation, or a process
// whose allocator is owned by a framework), or a caller that must not risk
// the implicit device synchronisation of cudaMalloc/cudaFree in a
// latency-critical loop.  sph_density_noalloc serves them: the caller passes
// device pointers to the inputs and the output, and every intermediate array
// (cell keys, sorted order, cell starts, sorted positions, radix-sort
// workspace) lives in one file-scope __device__ array of fixed size.
//
// The array is SPH_NOALLOC_SCRATCH_BYTES per GPU and exists on every GPU that
// loads the library until the process exits.  Its device address is looked
// up once per device, with that device current, on the first call made on
// it (cudaGetSymbolAddress).  Every call uses the same array, so calls that
// overlap on the GPU (concurrent streams, several host threads) race and
// give wrong results; the function synchronises its stream before
// returning.  What must start at zero or at a sentinel is cleared by the
// call itself.
//
// The density is circuit1's direct summation (circuit1.f90:253-296):
//   rho_i = sum_{j != i, r_ij <= krad h_i} m_j W(r_ij, h_i) + m_i W(0, h_i)
// over the particles as given (no periodic images), with the neighbour
// test of the kd-tree search (kdtree2.f90:1673-1678) in FP64.
#include <cub/device/device_radix_sort.cuh>

#include <cmath>
#include <mutex>
#include <string>

#include "sph_internal.h"

namespace sph {
namespace {

constexpr size_t kScratchBytes = SPH_NOALLOC_SCRATCH_BYTES;
static __device__ __align__(256) unsigned char g_noalloc_scratch[kScratchBytes];

constexpr int kMaxDevices = 64;
void* g_scratch_ptr[kMaxDevices] = {nullptr};
std::mutex g_scratch_mu;

// Device address of the scratch array on the current device (looked up once).
int scratch_address(void** out) {
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return sph_fail(SPH_ERR_CUDA, std::string("cudaGetDevice: ") + cudaGetErrorString(e));
  if (dev < 0 || dev >= kMaxDevices) return sph_fail(SPH_ERR_CUDA, "device index out of range");
  std::lock_guard<std::mutex> lk(g_scratch_mu);
  if (!g_scratch_ptr[dev]) {
    void* p = nullptr;
    e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
    if (e != cudaSuccess || !p)
      return sph_fail(SPH_ERR_CUDA, std::string("cudaGetSymbolAddress: ") + cudaGetErrorString(e));
    g_scratch_ptr[dev] = p;
  }
  *out = g_scratch_ptr[dev];
  return SPH_OK;
}

constexpr int TPB = 256;
inline int nblocks(int64_t n) { return int((n + TPB - 1) / TPB > 0 ? (n + TPB - 1) / TPB : 1); }

__device__ __forceinline__ double pos_of(const double* a, int64_t i) { return a ? a[i] : 0.0; }

// bbox (min/max per axis) and smallest h, order-preserving keys in red[0..6]
__global__ void k_na_init(unsigned long long* red) {
  int t = threadIdx.x;
  if (t < 3) red[t] = dkey(1e308);
  else if (t < 6) red[t] = dkey(-1e308);
  else if (t == 6) red[t] = dkey(1e308);
}

__global__ void k_na_reduce(const double* x, const double* y, const double* z, const double* h,
                            int64_t n, unsigned long long* red) {
  int64_t i = blockIdx.x * int64_t(blockDim.x) + threadIdx.x;
  if (i >= n) return;
  const double p[3] = {pos_of(x, i), pos_of(y, i), pos_of(z, i)};
  for (int k = 0; k < 3; ++k) {
    atomicMin(&red[k], dkey(p[k]));
    atomicMax(&red[3 + k], dkey(p[k]));
  }
  atomicMin(&red[6], dkey(h[i]));
}

__device__ __forceinline__ int na_cell(double v, double o, double invL, int nc) {
  double f = floor((v - o) * invL);
  if (!(f >= 0.0)) return 0;
  if (f >= double(nc - 1)) return nc - 1;
  return int(f);
}

__global__ void k_na_keys(const double* x, const double* y, const double* z, int64_t n, Grid g,
                          uint32_t* keys, int32_t* vals) {
  int64_t i = blockIdx.x * int64_t(blockDim.x) + threadIdx.x;
  if (i >= n) return;
  uint32_t cx = na_cell(pos_of(x, i), g.ox, g.invL, g.nx);
  uint32_t cy = na_cell(pos_of(y, i), g.oy, g.invL, g.ny);
  uint32_t cz = na_cell(pos_of(z, i), g.oz, g.invL, g.nz);
  keys[i] = cx + uint32_t(g.nx) * (cy + uint32_t(g.ny) * cz);
  vals[i] = int32_t(i);
}

__global__ void k_na_starts(const uint32_t* keys, int64_t n, int64_t ncell, int32_t* cstart) {
  int64_t k = blockIdx.x * int64_t(blockDim.x) + threadIdx.x;
  if (k > n) return;
  int64_t lo, hi;
  if (k == 0) { lo = -1; hi = n > 0 ? int64_t(keys[0]) : ncell; }
  else if (k == n) { lo = int64_t(keys[n - 1]); hi = ncell; }
  else { lo = int64_t(keys[k - 1]); hi = int64_t(keys[k]); }
  for (int64_t c = lo + 1; c <= hi; ++c) cstart[c] = int32_t(k);
}

__global__ void k_na_gather(const double* x, const double* y, const double* z, const double* m,
                            const int32_t* order, int64_t n, double4* sorted) {
  int64_t k = blockIdx.x * int64_t(blockDim.x) + threadIdx.x;
  if (k >= n) return;
  int64_t i = order[k];
  sorted[k] = make_double4(pos_of(x, i), pos_of(y, i), pos_of(z, i), m[i]);
}

template <int K, int DIM>
__global__ void k_na_density(const double* x, const double* y, const double* z, const double* m,
                             const double* h, int64_t n, Grid g, double krad, double wcv,
                             const int32_t* cstart, const int32_t* order, const double4* sorted,
                             double* rho, int* status) {
  int64_t i = blockIdx.x * int64_t(blockDim.x) + threadIdx.x;
  if (i >= n) return;
  const double xi = pos_of(x, i), yi = pos_of(y, i), zi = pos_of(z, i);
  const double hi = h[i];
  const double kh = __dmul_rn(krad, hi);
  const double R2 = __dmul_rn(kh, kh);
  const double R = sqrt(R2) * (1.0 + 1e-9) + 1e-300;
  const double ih = 1.0 / hi;
  const double xs[3] = {xi, yi, zi}, os[3] = {g.ox, g.oy, g.oz};
  const int ns[3] = {g.nx, g.ny, g.nz};
  int c0[3], c1[3];
  for (int a = 0; a < 3; ++a) {
    const double sl = fabs(xs[a]) * 1e-15;
    c0[a] = na_cell(xs[a] - R - sl, os[a], g.invL, ns[a]);
    c1[a] = na_cell(xs[a] + R + sl, os[a], g.invL, ns[a]);
  }
  double sum = 0.0;
  bool bad = false;
  for (int cz = c0[2]; cz <= c1[2]; ++cz)
    for (int cy = c0[1]; cy <= c1[1]; ++cy) {
      const int64_t row = int64_t(g.nx) * (cy + int64_t(g.ny) * cz);
      const int32_t s = cstart[row + c0[0]], e = cstart[row + c1[0] + 1];
      for (int32_t q = s; q < e; ++q) {
        if (order[q] == i) continue;  // neighboursearch.f90:190
        const double4 pj = sorted[q];
        const double d0 = __dadd_rn(pj.x, -xi), d1 = __dadd_rn(pj.y, -yi), d2 = __dadd_rn(pj.z, -zi);
        const double sd = __dadd_rn(__dadd_rn(__dmul_rn(d0, d0), __dmul_rn(d1, d1)), __dmul_rn(d2, d2));
        if (sd > R2) continue;
        const double q_ = sqrt(sd) * ih;
        bad |= !(q_ >= 0.0);
        sum += pj.w * kshape_f<K, double>(q_);
      }
    }
  const double self = m[i] * kshape_f<K, double>(0.0);
  rho[i] = wcv * (sum + self) / ipow<DIM>(hi);
  if (bad) atomicCAS(status, 0, SPH_ERR_Q_NAN);
}

template <int K>
void launch_density(int dim, const double* x, const double* y, const double* z, const double* m,
                    const double* h, int64_t n, Grid g, double krad, double wcv,
                    const int32_t* cstart, const int32_t* order, const double4* sorted,
                    double* rho, int* status, cudaStream_t s) {
  if (dim == 3)
    k_na_density<K, 3><<<nblocks(n), TPB, 0, s>>>(x, y, z, m, h, n, g, krad, wcv, cstart, order, sorted, rho, status);
  else if (dim == 2)
    k_na_density<K, 2><<<nblocks(n), TPB, 0, s>>>(x, y, z, m, h, n, g, krad, wcv, cstart, order, sorted, rho, status);
  else
    k_na_density<K, 1><<<nblocks(n), TPB, 0, s>>>(x, y, z, m, h, n, g, krad, wcv, cstart, order, sorted, rho, status);
}

// carve `bytes` (256-aligned) out of the scratch array
struct Carver {
  unsigned char* base;
  size_t used = 0;
  void* take(size_t bytes) {
    void* p = base + used;
    used += (bytes + 255) & ~size_t(255);
    return p;
  }
};

}  // namespace
}  // namespace sph

using namespace sph;

extern "C" int sph_density_noalloc(const double* x, const double* y, const double* z,
                                   const double* m, const double* h, int64_t n, int dim,
                                   int kernel_id, double* rho, void* stream) {
  if (n < 1 || n > SPH_NOALLOC_MAX_PARTICLES)
    return sph_fail(SPH_ERR_ARG, "sph_density_noalloc: n must be in 1.." +
                                     std::to_string(SPH_NOALLOC_MAX_PARTICLES) + ", got " +
                                     std::to_string(n));
  if (dim < 1 || dim > 3) return sph_fail(SPH_ERR_ARG, "sph_density_noalloc: dim must be 1, 2 or 3");
  if (kernel_id < 0 || kernel_id > 2) return sph_fail(SPH_ERR_ARG, "sph_density_noalloc: bad kernel id");
  if (!x || !m || !h || !rho || (dim >= 2 && !y) || (dim == 3 && !z))
    return sph_fail(SPH_ERR_ARG, "sph_density_noalloc: null device pointer");
  if (dim < 2) y = nullptr;
  if (dim < 3) z = nullptr;
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  // The scratch address is the current device's; a stream of another device
  // would run the kernels there with this device's address.
  if (s) {
    int cur = -1, sdev = -1;
    cudaError_t ge = cudaGetDevice(&cur);
    if (ge == cudaSuccess) ge = cudaStreamGetDevice(s, &sdev);
    if (ge != cudaSuccess)
      return sph_fail(SPH_ERR_CUDA, std::string("sph_density_noalloc: ") + cudaGetErrorString(ge));
    if (sdev != cur)
      return sph_fail(SPH_ERR_ARG, "sph_density_noalloc: the stream belongs to device " +
                                       std::to_string(sdev) + ", the current device is " +
                                       std::to_string(cur));
  }
  void* base = nullptr;
  int rc = scratch_address(&base);
  if (rc) return rc;
  // knorm / krad of the kernel bases (base_m4.f90:12,18; base_m6.f90:13,17; base_gauss.f90:15,19)
  const double pi = 4.0 * std::atan(1.0);
  const double norms[3][3] = {{2. / 3., 10. / (7. * pi), 1. / pi},
                              {1. / 120., 7. / (478. * pi), 1. / (120. * pi)},
                              {1. / std::sqrt(pi), 1. / pi, 1. / std::pow(pi, 1.5)}};
  const double krads[3] = {2.0, 3.0, 10.0};
  const double wcv = norms[kernel_id][dim - 1], krad = krads[kernel_id];

  Carver cv{static_cast<unsigned char*>(base)};
  auto* red = static_cast<unsigned long long*>(cv.take(8 * sizeof(unsigned long long)));
  auto* status = static_cast<int*>(cv.take(sizeof(int)));
  auto* keys = static_cast<uint32_t*>(cv.take(sizeof(uint32_t) * n));
  auto* keys2 = static_cast<uint32_t*>(cv.take(sizeof(uint32_t) * n));
  auto* vals = static_cast<int32_t*>(cv.take(sizeof(int32_t) * n));
  auto* vals2 = static_cast<int32_t*>(cv.take(sizeof(int32_t) * n));
  auto* sorted = static_cast<double4*>(cv.take(sizeof(double4) * n));
  const int64_t max_cells = 4 * n + 4096;
  auto* cstart = static_cast<int32_t*>(cv.take(sizeof(int32_t) * (max_cells + 1)));
  size_t sort_bytes = 0;
  cub::DeviceRadixSort::SortPairs(nullptr, sort_bytes, keys, keys2, vals, vals2, int(n), 0, 32, s);
  void* sort_tmp = cv.take(sort_bytes);
  if (cv.used > kScratchBytes) return sph_fail(SPH_ERR_ARG, "sph_density_noalloc: scratch too small for n");

  cudaError_t e = cudaMemsetAsync(status, 0, sizeof(int), s);
  if (e != cudaSuccess) return sph_fail(SPH_ERR_CUDA, cudaGetErrorString(e));
  k_na_init<<<1, 32, 0, s>>>(red);
  k_na_reduce<<<nblocks(n), TPB, 0, s>>>(x, y, z, h, n, red);
  unsigned long long hred[7];
  e = cudaMemcpyAsync(hred, red, sizeof(hred), cudaMemcpyDeviceToHost, s);
  if (e == cudaSuccess) e = cudaStreamSynchronize(s);
  if (e != cudaSuccess) return sph_fail(SPH_ERR_CUDA, std::string("sph_density_noalloc: ") + cudaGetErrorString(e));
  double lo[3], hi[3];
  for (int k = 0; k < 3; ++k) { lo[k] = dkey_inv(hred[k]); hi[k] = dkey_inv(hred[3 + k]); }
  const double hmin = dkey_inv(hred[6]);
  if (!(hmin > 0) || !std::isfinite(hmin)) return sph_fail(SPH_ERR_IC_H, "smoothing length <= 0");
  for (int k = 0; k < 3; ++k)
    if (!std::isfinite(lo[k]) || !std::isfinite(hi[k])) return sph_fail(SPH_ERR_Q_NAN, "q is nan");
  // cell edge krad*h_min, widened until the grid fits the scratch
  double L = krad * hmin;
  int64_t ncell = 0;
  int n3[3] = {1, 1, 1};
  for (int guard = 0;; ++guard) {
    double ex[3];
    for (int k = 0; k < 3; ++k) ex[k] = (hi[k] - lo[k]) / L;
    if (grid_dims(ex, max_cells, n3, &ncell)) break;
    L *= 1.25;
    if (guard > 400) return sph_fail(SPH_ERR_GRID, "cell grid would not fit");
  }
  Grid g;
  g.ox = lo[0]; g.oy = lo[1]; g.oz = lo[2];
  g.L = L; g.invL = 1.0 / L;
  g.nx = n3[0]; g.ny = n3[1]; g.nz = n3[2];
  int end_bit = 1;
  while ((int64_t(1) << end_bit) < ncell) ++end_bit;
  k_na_keys<<<nblocks(n), TPB, 0, s>>>(x, y, z, n, g, keys, vals);
  cub::DeviceRadixSort::SortPairs(sort_tmp, sort_bytes, keys, keys2, vals, vals2, int(n), 0, end_bit, s);
  k_na_starts<<<nblocks(n + 1), TPB, 0, s>>>(keys2, n, ncell, cstart);
  k_na_gather<<<nblocks(n), TPB, 0, s>>>(x, y, z, m, vals2, n, sorted);
  if (kernel_id == SPH_KERNEL_M6)
    launch_density<KM6>(dim, x, y, z, m, h, n, g, krad, wcv, cstart, vals2, sorted, rho, status, s);
  else if (kernel_id == SPH_KERNEL_M4)
    launch_density<KM4>(dim, x, y, z, m, h, n, g, krad, wcv, cstart, vals2, sorted, rho, status, s);
  else
    launch_density<KGAUSS>(dim, x, y, z, m, h, n, g, krad, wcv, cstart, vals2, sorted, rho, status, s);
  // this library's own kernels (init, reduce, keys, starts, gather,
  // density); the radix sort's kernels are CUB's and are not counted, as
  // in the engine's launch counter
  note_launch(6);
  int hstatus = 0;
  e = cudaMemcpyAsync(&hstatus, status, sizeof(int), cudaMemcpyDeviceToHost, s);
  if (e == cudaSuccess) e = cudaStreamSynchronize(s);
  if (e == cudaSuccess) e = cudaGetLastError();
  if (e != cudaSuccess) return sph_fail(SPH_ERR_CUDA, std::string("sph_density_noalloc: ") + cudaGetErrorString(e));
  if (hstatus) return sph_fail(hstatus, "q is nan");
  return SPH_OK;
}
