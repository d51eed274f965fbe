// sph_grid.cu — the non-pair kernels of one SPH step on the device:
// store upload/download and re-ordering, periodic wrap and periodic images
// (BC.f90:102-475), Morton cell keys + radix sort + cell ranges (replacing the
// kd-tree of neighboursearch.f90:74-180), the FP64 fixed-ball neighbour
// predicate (kdtree2.f90:1673-1678), packing of pair data, the leapfrog
// predictor/corrector (main.f90:323-362), timestep reductions
// (timestep.f90:40-166), EOS (eos.f90:21-45) and the STS stage update
// (sts_integrator.f90:87-124).
#include <cub/device/device_radix_sort.cuh>
#include <cub/device/device_scan.cuh>

#include "sph_internal.h"

namespace sph {

namespace {

constexpr int TPB = 256;

inline int nblocks(int64_t n, int tpb = TPB) {
  int64_t b = (n + tpb - 1) / tpb;
  return int(b < 1 ? 1 : b);
}

__device__ __forceinline__ void red_min(unsigned long long* slot, double v) {
  atomicMin(slot, dkey(v));
}
__device__ __forceinline__ void red_max(unsigned long long* slot, double v) {
  atomicMax(slot, dkey(v));
}

// warp-level min/max of doubles, then one atomic per warp
__device__ __forceinline__ double warp_min(double v) {
  for (int o = 16; o > 0; o >>= 1) v = fmin(v, __shfl_xor_sync(0xffffffffu, v, o));
  return v;
}
__device__ __forceinline__ double warp_max(double v) {
  for (int o = 16; o > 0; o >>= 1) v = fmax(v, __shfl_xor_sync(0xffffffffu, v, o));
  return v;
}

// ---- store transposes -----------------------------------------------------------
// Row-major (n x NCOL) table <-> column store, through 32 x 32 tiles in
// shared memory so that both the row reads / writes and the column writes /
// reads are contiguous runs of 256 bytes.  Block (32, 8): tile of 32 rows.
static_assert(NCOL == 32, "the tile transposes assume 32 fields");
__global__ void __launch_bounds__(256)
k_upload(const double* __restrict__ rm, double* __restrict__ cols, int32_t* __restrict__ orig,
         int64_t n, int64_t a, int64_t b) {
  // rows a .. b - 1 of the n (a a multiple of 32)
  __shared__ double tile[32][33];
  const int64_t r0 = a + int64_t(blockIdx.x) * 32;
  for (int k = threadIdx.y; k < 32; k += 8) {  // row r0 + k, field threadIdx.x
    const int64_t i = r0 + k;
    if (i < b) tile[k][threadIdx.x] = rm[i * NCOL + threadIdx.x];
  }
  __syncthreads();
  for (int f = threadIdx.y; f < NCOL; f += 8) {  // field f, row r0 + threadIdx.x
    const int64_t i = r0 + threadIdx.x;
    if (i < b) cols[f * n + i] = tile[threadIdx.x][f];
  }
  if (threadIdx.y == 0 && r0 + threadIdx.x < b) orig[r0 + threadIdx.x] = int32_t(r0 + threadIdx.x);
}
// caller rows a .. b - 1 of the row-major table from the column store:
// caller row j is physical row inv[j] (inv the inverse of orig)
__global__ void __launch_bounds__(256)
k_download_gather(const double* __restrict__ cols, const int32_t* __restrict__ inv,
                  double* __restrict__ rm, int64_t n, int64_t a, int64_t b) {
  __shared__ double tile[32][33];
  const int64_t r0 = a + int64_t(blockIdx.x) * 32;
  const int64_t j = r0 + threadIdx.x;
  const int64_t p = j < b ? int64_t(inv[j]) : 0;
  for (int f = threadIdx.y; f < NCOL; f += 8)  // field f of caller row j
    if (j < b) tile[threadIdx.x][f] = cols[f * n + p];
  __syncthreads();
  for (int k = threadIdx.y; k < 32; k += 8) {
    const int64_t i = r0 + k;
    if (i < b) rm[i * NCOL + threadIdx.x] = tile[k][threadIdx.x];
  }
}

__global__ void __launch_bounds__(256)
k_download(const double* __restrict__ cols, const int32_t* __restrict__ orig,
           double* __restrict__ rm, int64_t n) {
  __shared__ double tile[32][33];
  const int64_t r0 = int64_t(blockIdx.x) * 32;
  for (int f = threadIdx.y; f < NCOL; f += 8) {  // field f of physical row r0 + threadIdx.x
    const int64_t i = r0 + threadIdx.x;
    if (i < n) tile[threadIdx.x][f] = cols[f * n + i];
  }
  __syncthreads();
  for (int k = threadIdx.y; k < 32; k += 8) {  // physical row r0 + k to its original row
    const int64_t i = r0 + k;
    if (i < n) rm[int64_t(orig[i]) * NCOL + threadIdx.x] = tile[k][threadIdx.x];
  }
}

__global__ void k_reorder(const double* __restrict__ cin, double* __restrict__ cout,
                          const int32_t* __restrict__ oin, int32_t* __restrict__ oout,
                          const int32_t* __restrict__ perm, int64_t n, int64_t ldi,
                          int64_t ldo) {
  int64_t i = blockIdx.x * int64_t(blockDim.x) + threadIdx.x;
  if (i >= n) return;
  int64_t src = perm[i];
  for (int f = 0; f < NCOL; ++f) cout[f * ldo + i] = cin[f * ldi + src];
  oout[i] = oin[src];
}

// ---- periodic wrap of real particles (BC.f90:102-194) ----------------------------
__global__ void k_reflect(double* __restrict__ cols, int64_t ld, int64_t nreal, BoxGeom g) {
  int64_t i = blockIdx.x * int64_t(blockDim.x) + threadIdx.x;
  if (i >= nreal) return;
  double r[3], dxmin[3], dxmax[3];
  for (int k = 0; k < 3; ++k) {
    r[k] = cols[(es_rx + k) * ld + i];
    dxmin[k] = __dadd_rn(g.emin[k], -r[k]);
    dxmax[k] = __dadd_rn(r[k], -g.emax[k]);
  }
  for (int k = 0; k < 3; ++k) {
    if (!g.reflect[k]) continue;
    double v = r[k];
    if (dxmax[k] > 0) v = __dadd_rn(g.emin[k], dxmax[k]);
    if (dxmin[k] > 0) v = __dadd_rn(g.emax[k], -dxmin[k]);
    cols[(es_rx + k) * ld + i] = v;
  }
}

// ---- periodic images --------------------------------------------------------------
// Image rule equivalent to createPeriodicBorder's list walk (BC.f90:311-475):
// an image shifts a subset S of the periodic axes; the first axis of S (in x,
// y, z order) is tested on the real particle with the padding bound of
// findInsideBorderParticles (BC.f90:277-303), every later axis of S is tested
// on the intermediate image without it (BC.f90:342-354, 402-407).  On each
// axis at most one of the two sides can hold, so S fixes the image.
struct AxisSigns {
  int pad[3];   // +1 low strip, -1 high strip, 0 none (padded test)
  int npad[3];  // same without the padding bound
};

__device__ __forceinline__ int type_of(double t) { return int(t); }

__device__ __forceinline__ bool ghost_source(double t) {
  int ty = type_of(t);
  return ty == ept_real || ty == ept_fixed || ty == ept_fixedreal;
}

__device__ __forceinline__ AxisSigns axis_signs(const double* r, const BoxGeom& g, int dim) {
  AxisSigns s;
  for (int k = 0; k < 3; ++k) {
    s.pad[k] = 0;
    s.npad[k] = 0;
    if (k >= dim || !g.periodic[k]) continue;
    double ra = r[k];
    if (ra < g.boxmin[k]) {
      if (ra > g.pmin[k]) s.pad[k] = +1;
      s.npad[k] = +1;
    } else if (ra > g.boxmax[k]) {
      if (ra < g.pmax[k]) s.pad[k] = -1;
      s.npad[k] = -1;
    }
  }
  return s;
}

// Image `mask` (bits of S) -> shift signs; returns false if the image does not exist.
__device__ __forceinline__ bool image_of(const AxisSigns& s, int mask, int sg[3]) {
  bool first = true;
  for (int k = 0; k < 3; ++k) {
    sg[k] = 0;
    if (!(mask & (1 << k))) continue;
    int v = first ? s.pad[k] : s.npad[k];
    if (v == 0) return false;
    sg[k] = v;
    first = false;
  }
  return true;
}

__device__ __forceinline__ double image_coord(double x, int sign, double emin, double emax) {
  if (sign > 0) return __dadd_rn(emax, __dadd_rn(x, -emin));  // xmax + (x - xmin)
  if (sign < 0) return __dadd_rn(emin, __dadd_rn(x, -emax));  // xmin + (x - xmax)
  return x;
}

// Reduction of per-thread partial minima / maxima over the block: one value
// per slot leaves the block (then one atomic per block and slot, so that the
// slots see a few thousand atomics per launch rather than one per warp).
template <int K>
__device__ __forceinline__ void block_minmax(double (&v)[K], const bool (&is_max)[K]) {
  __shared__ double part[TPB / 32][K];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
  for (int j = 0; j < K; ++j) v[j] = is_max[j] ? warp_max(v[j]) : warp_min(v[j]);
  if (lane == 0) {
#pragma unroll
    for (int j = 0; j < K; ++j) part[warp][j] = v[j];
  }
  __syncthreads();
  if (warp == 0) {
#pragma unroll
    for (int j = 0; j < K; ++j) {
      double x = lane < int(blockDim.x >> 5) ? part[lane][j] : (is_max[j] ? -1e308 : 1e308);
      v[j] = is_max[j] ? warp_max(x) : warp_min(x);
    }
  }
}
// grid of the reduction kernels: a few blocks per SM, each thread striding
// over the rows
inline int reduce_blocks(int64_t n) {
  const int64_t b = (n + TPB - 1) / TPB;
  return int(b < 148 * 8 ? (b > 0 ? b : 1) : 148 * 8);
}

__global__ void __launch_bounds__(TPB)
k_ghost_count(const double* __restrict__ cols, int64_t ld, int64_t nrows, int64_t nreal,
              BoxGeom g, int dim, int32_t* __restrict__ count,
              unsigned long long* __restrict__ red) {
  // slots: lo x, y, z (min), hi x, y, z (max), hmin (min)
  double v[7] = {1e300, 1e300, 1e300, -1e300, -1e300, -1e300, 1e300};
  const bool is_max[7] = {false, false, false, true, true, true, false};
  for (int64_t i = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; i < nrows;
       i += int64_t(gridDim.x) * blockDim.x) {
    int c = 0;
    double r[3] = {cols[es_rx * ld + i], cols[es_ry * ld + i], cols[es_rz * ld + i]};
    for (int k = 0; k < 3; ++k) { v[k] = fmin(v[k], r[k]); v[3 + k] = fmax(v[3 + k], r[k]); }
    if (i < nreal) v[6] = fmin(v[6], cols[es_h * ld + i]);
    if (ghost_source(cols[es_type * ld + i])) {
      AxisSigns sg_ = axis_signs(r, g, dim);
      for (int mask = 1; mask < 8; ++mask) {
        int sg[3];
        if (!image_of(sg_, mask, sg)) continue;
        ++c;
        for (int k = 0; k < 3; ++k) {
          double x = image_coord(r[k], sg[k], g.emin[k], g.emax[k]);
          v[k] = fmin(v[k], x);
          v[3 + k] = fmax(v[3 + k], x);
        }
      }
    }
    count[i] = c;
  }
  block_minmax<7>(v, is_max);
  if (threadIdx.x == 0) {
    for (int k = 0; k < 3; ++k) {
      if (v[k] < 1e300) red_min(&red[RED_LO_X + k], v[k]);
      if (v[3 + k] > -1e300) red_max(&red[RED_HI_X + k], v[3 + k]);
    }
    if (v[6] < 1e300) red_min(&red[RED_HMIN], v[6]);
  }
}

__global__ void k_ghost_write(const double* __restrict__ cols, int64_t ld, int64_t nrows,
                              BoxGeom g, int dim, const int32_t* __restrict__ offset, int64_t cap,
                              double* __restrict__ gx, double* __restrict__ gy,
                              double* __restrict__ gz, int32_t* __restrict__ gsrc,
                              int8_t* __restrict__ gcode) {
  int64_t i = blockIdx.x * int64_t(blockDim.x) + threadIdx.x;
  if (i >= nrows) return;
  if (!ghost_source(cols[es_type * ld + i])) return;
  double r[3] = {cols[es_rx * ld + i], cols[es_ry * ld + i], cols[es_rz * ld + i]};
  AxisSigns s = axis_signs(r, g, dim);
  int64_t o = offset[i];
  for (int mask = 1; mask < 8; ++mask) {
    int sg[3];
    if (!image_of(s, mask, sg)) continue;
    if (o >= cap) return;  // a device-resident step found more images than room
    gx[o] = image_coord(r[0], sg[0], g.emin[0], g.emax[0]);
    gy[o] = image_coord(r[1], sg[1], g.emin[1], g.emax[1]);
    gz[o] = image_coord(r[2], sg[2], g.emin[2], g.emax[2]);
    gsrc[o] = int32_t(i);
    gcode[o] = int8_t((sg[0] + 1) + 3 * (sg[1] + 1) + 9 * (sg[2] + 1));
    ++o;
  }
}

// ---- cell keys ----------------------------------------------------------------------
// Cells are numbered row-major (x fastest), so the cells of one (y, z) row are
// contiguous in the sorted particle order and a search visits one index range
// per row instead of one per cell.
__device__ __forceinline__ int cell_coord(double x, double o, double invL, int n) {
  // clamped to [0, n-1]; NaN and -inf map to 0 and +inf to n-1 before any
  // float-to-int conversion happens
  double f = floor((x - o) * invL);
  if (!(f >= 0.0)) return 0;
  if (f >= double(n - 1)) return n - 1;
  return int(f);
}

// With a device plan the particle count and grid come from it, and the
// slots up to the capacity ncap get the padding key (sorted behind every
// cell) so that the sort can run over a size fixed on the host.
__global__ void k_keys(const double* __restrict__ cols, int64_t ld, int64_t nrows,
                       const double* __restrict__ gx, const double* __restrict__ gy,
                       const double* __restrict__ gz, int64_t nghost, Grid g,
                       uint32_t* __restrict__ keys, int32_t* __restrict__ vals,
                       const DevPlan* __restrict__ plan, int64_t ncap) {
  int64_t u = blockIdx.x * int64_t(blockDim.x) + threadIdx.x;
  int64_t n = nrows + nghost;
  if (plan) {
    n = plan->nall;
    g = plan->grid;
    if (u >= n && u < ncap) {
      keys[u] = plan->pad_key;
      vals[u] = int32_t(u);
      return;
    }
  }
  if (u >= n) return;
  double x, y, z;
  if (u < nrows) {
    x = cols[es_rx * ld + u]; y = cols[es_ry * ld + u]; z = cols[es_rz * ld + u];
  } else {
    int64_t q = u - nrows;
    x = gx[q]; y = gy[q]; z = gz[q];
  }
  uint32_t cx = cell_coord(x, g.ox, g.invL, g.nx);
  uint32_t cy = cell_coord(y, g.oy, g.invL, g.ny);
  uint32_t cz = cell_coord(z, g.oz, g.invL, g.nz);
  keys[u] = cx + uint32_t(g.nx) * (cy + uint32_t(g.ny) * cz);
  vals[u] = int32_t(u);
}

// ---- counting sort of the records by cell ------------------------------------------------
// The keys are cell indices, so one pass of counting sort orders them: the
// records of each cell are counted, the counts scanned into the cells'
// starts, and every record placed at its cell's start plus a slot taken
// with an atomic.  The slots within a cell come out in arbitrary order;
// each cell's records are then sorted by index (a thread per cell for up to
// kCellSmall records, a block per cell for up to kCellBig), which gives the
// order of a stable sort by key.
constexpr int kCellSmall = 32;
constexpr int kCellBig = 4096;

__global__ void k_cell_count(const uint32_t* __restrict__ keys, int64_t n,
                             int32_t* __restrict__ count, int32_t* __restrict__ maxc) {
  const int64_t u = blockIdx.x * int64_t(blockDim.x) + threadIdx.x;
  int m = 0;
  if (u < n) m = atomicAdd(&count[keys[u]], 1) + 1;
  unsigned long long v[1] = {(unsigned long long)m};
  const bool is_max[1] = {true};
  block_counters<1>(v, is_max);
  if (threadIdx.x == 0 && v[0]) atomicMax(maxc, int(v[0]));
}
__global__ void k_cell_scatter(const uint32_t* __restrict__ keys, int64_t n,
                               const int32_t* __restrict__ cstart, int32_t* __restrict__ fill,
                               int32_t* __restrict__ vout, uint32_t* __restrict__ kout) {
  const int64_t u = blockIdx.x * int64_t(blockDim.x) + threadIdx.x;
  if (u >= n) return;
  const uint32_t key = keys[u];
  const int32_t pos = cstart[key] + atomicAdd(&fill[key], 1);
  vout[pos] = int32_t(u);
  kout[pos] = key;
}
// cells of up to kCellSmall records: insertion sort by a thread; larger
// ones go to `big`
__global__ void k_cell_sort_small(const int32_t* __restrict__ cstart, int64_t ncell,
                                  int32_t* __restrict__ v, int32_t* __restrict__ big,
                                  int32_t* __restrict__ nbig) {
  const int64_t c = blockIdx.x * int64_t(blockDim.x) + threadIdx.x;
  if (c >= ncell) return;
  const int32_t a = cstart[c], b = cstart[c + 1];
  const int k = b - a;
  if (k <= 1) return;
  if (k > kCellSmall) {
    big[atomicAdd(nbig, 1)] = int32_t(c);
    return;
  }
  int32_t r[kCellSmall];
  for (int i = 0; i < k; ++i) r[i] = v[a + i];
  for (int i = 1; i < k; ++i) {
    const int32_t x = r[i];
    int j = i - 1;
    while (j >= 0 && r[j] > x) { r[j + 1] = r[j]; --j; }
    r[j + 1] = x;
  }
  for (int i = 0; i < k; ++i) v[a + i] = r[i];
}
// cells of up to kCellBig records: a block per cell (the blocks stride over
// the list), bitonic sort in shared memory padded to a power of two
__global__ void __launch_bounds__(256)
k_cell_sort_big(const int32_t* __restrict__ cstart, int32_t* __restrict__ v,
                const int32_t* __restrict__ big, const int32_t* __restrict__ nbig) {
  __shared__ int32_t sh[kCellBig];
  const int nb = *nbig;
  for (int i = blockIdx.x; i < nb; i += gridDim.x) {
    const int32_t c = big[i];
    const int32_t a = cstart[c];
    const int k = cstart[c + 1] - a;  // kCellSmall < k <= kCellBig (checked on the host)
    int m = 1;
    while (m < k) m <<= 1;
    for (int t = threadIdx.x; t < m; t += blockDim.x) sh[t] = t < k ? v[a + t] : INT32_MAX;
    __syncthreads();
    for (int size = 2; size <= m; size <<= 1)
      for (int stride = size >> 1; stride > 0; stride >>= 1) {
        for (int t = threadIdx.x; t < m; t += blockDim.x) {
          const int o = t ^ stride;
          if (o > t) {
            const bool up = (t & size) == 0;
            const int32_t x = sh[t], y = sh[o];
            if ((x > y) == up) { sh[t] = y; sh[o] = x; }
          }
        }
        __syncthreads();
      }
    for (int t = threadIdx.x; t < k; t += blockDim.x) v[a + t] = sh[t];
    __syncthreads();
  }
}

// cstart[c] = number of particles in cells before c (ncell + 1 entries), from
// the sorted keys: each key change fills the empty cells it skips.
__global__ void k_cell_starts(const uint32_t* __restrict__ keys, int64_t n, int64_t ncell,
                              int32_t* __restrict__ cstart, const DevPlan* __restrict__ plan) {
  int64_t k = blockIdx.x * int64_t(blockDim.x) + threadIdx.x;
  if (plan) {
    n = plan->nall;
    ncell = plan->ncell;
  }
  if (k > n) return;
  int64_t lo, hi;  // cells (lo, hi] start at k
  if (k == 0) { lo = -1; hi = n > 0 ? int64_t(keys[0]) : ncell; }
  else if (k == n) { lo = int64_t(keys[n - 1]); hi = ncell; }
  else { lo = int64_t(keys[k - 1]); hi = int64_t(keys[k]); }
  for (int64_t c = lo + 1; c <= hi; ++c) cstart[c] = int32_t(k);
}

// Sorted-order gather of positions and source rows; compaction of centres
// (the real rows, which the reference iterates as alllistlv1 = 1..realpn).
__global__ void k_sorted_gather(const int32_t* __restrict__ sidx, int64_t n, int64_t nrows,
                                int64_t nreal, const double* __restrict__ cols, int64_t ld,
                                const double* __restrict__ gx, const double* __restrict__ gy,
                                const double* __restrict__ gz, const int32_t* __restrict__ gsrc,
                                double* __restrict__ sx, double* __restrict__ sy,
                                double* __restrict__ sz, int32_t* __restrict__ ssrc,
                                int32_t* __restrict__ centre_slot, float4* __restrict__ s32,
                                PackGeom pg, const DevPlan* __restrict__ plan, int64_t ncap) {
  int64_t k = blockIdx.x * int64_t(blockDim.x) + threadIdx.x;
  if (plan) {
    n = plan->nall;
    pg = plan->pg;
    if (k >= n && k <= ncap) {  // no centres past the particles (the scan covers ncap + 1)
      centre_slot[k] = 0;
      return;
    }
  }
  if (k >= n) return;
  int64_t u = sidx[k];
  double x, y, z;
  if (u < nrows) {
    x = cols[es_rx * ld + u]; y = cols[es_ry * ld + u]; z = cols[es_rz * ld + u];
    ssrc[k] = int32_t(u);
    centre_slot[k] = (u < nreal) ? 1 : 0;
  } else {
    int64_t q = u - nrows;
    x = gx[q]; y = gy[q]; z = gz[q];
    ssrc[k] = gsrc[q];
    centre_slot[k] = 0;
  }
  sx[k] = x; sy[k] = y; sz[k] = z;
  // FP32 image of the position, one binade for the whole extent (see PackGeom)
  // (w carries the record's own sorted index, so that a copy of a run of
  // records still knows where each came from)
  s32[k] = make_float4(__double2float_rn((x - pg.ox) + pg.shift),
                       __double2float_rn((y - pg.oy) + pg.shift),
                       __double2float_rn((z - pg.oz) + pg.shift), __int_as_float(int32_t(k)));
}

__global__ void k_centres(const int32_t* __restrict__ sidx, const int32_t* __restrict__ flag,
                          const int32_t* __restrict__ pos, int64_t n,
                          int32_t* __restrict__ centre_k, int32_t* __restrict__ centre_p) {
  int64_t k = blockIdx.x * int64_t(blockDim.x) + threadIdx.x;
  if (k >= n) return;
  if (!flag[k]) return;
  int64_t c = pos[k];
  centre_k[c] = int32_t(k);
  centre_p[c] = sidx[k];
}

// ---- bulk copies into shared memory (the TMA engine's 1-D form) --------------------
// cp.async.bulk moves a contiguous run of bytes from global to shared memory
// and reports its bytes to an mbarrier; both addresses 16-byte aligned, the
// size a multiple of 16.  No cluster multicast.
__device__ __forceinline__ uint32_t smem_u32(const void* p) {
  return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}
__device__ __forceinline__ void mbar_init(unsigned long long* m, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(m)), "r"(count) : "memory");
}
__device__ __forceinline__ void mbar_init_fence() {
  asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}
__device__ __forceinline__ void mbar_arrive_expect_tx(unsigned long long* m, uint32_t bytes) {
  asm volatile("{\n .reg .b64 st;\n mbarrier.arrive.expect_tx.shared::cta.b64 st, [%0], %1;\n}\n"
               ::"r"(smem_u32(m)), "r"(bytes) : "memory");
}
__device__ __forceinline__ bool mbar_test_wait(unsigned long long* m, uint32_t parity) {
  uint32_t ok;
  asm volatile("{\n .reg .pred p;\n mbarrier.test_wait.parity.shared::cta.b64 p, [%1], %2;\n"
               " selp.u32 %0, 1, 0, p;\n}\n"
               : "=r"(ok) : "r"(smem_u32(m)), "r"(parity) : "memory");
  return ok != 0u;
}
__device__ __forceinline__ void fence_proxy_async_smem() {
  asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}
__device__ __forceinline__ void bulk_g2s(void* dst, const void* src, uint32_t bytes,
                                         unsigned long long* m) {
  asm volatile(
      "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];"
      ::"r"(smem_u32(dst)), "l"(__cvta_generic_to_global(src)), "r"(bytes), "r"(smem_u32(m))
      : "memory");
}
// waits for the phase with the given parity, at most `limit` polls; false
// when it did not complete
__device__ __forceinline__ bool mbar_wait_bounded(unsigned long long* m, uint32_t parity,
                                                  int limit) {
  for (int i = 0; i < limit; ++i)
    if (mbar_test_wait(m, parity)) return true;
  return false;
}

// ---- neighbour-set digest ----------------------------------------------------------------
// Per centre, in original row order: the neighbour count and the sum (mod
// 2^64) of a 64-bit mix of each neighbour's (row << 5) | image code, the
// encoding of sph_get_neighbours.  The sum does not depend on the order of a
// row, so two engines with the same sets give the same digests; a differing
// set changes the sum unless 64-bit mixes cancel.  One warp per centre.
__device__ __forceinline__ unsigned long long mix64(unsigned long long z) {
  z += 0x9e3779b97f4a7c15ull;
  z = (z ^ (z >> 30)) * 0xbf58476d1ce4e5b9ull;
  z = (z ^ (z >> 27)) * 0x94d049bb133111ebull;
  return z ^ (z >> 31);
}
__global__ void k_neib_digest(int64_t nc, const int32_t* __restrict__ centre_p,
                              const int32_t* __restrict__ orig, const int64_t* __restrict__ rowoff,
                              const int32_t* __restrict__ ncnt, const int32_t* __restrict__ nl,
                              const int32_t* __restrict__ sidx, const int32_t* __restrict__ ssrc,
                              const int8_t* __restrict__ gcode, int64_t nrows,
                              unsigned long long* __restrict__ out) {
  const int64_t c = (blockIdx.x * int64_t(blockDim.x) + threadIdx.x) >> 5;
  const int lane = threadIdx.x & 31;
  if (c >= nc) return;
  const int n = ncnt[c];
  const int32_t* row = nl + rowoff[c];
  unsigned long long s = 0;
  for (int l = lane; l < n; l += 32) {
    const int64_t q = row[l];
    const int64_t u = sidx[q];
    const long long rj = orig[ssrc[q]];
    const long long code = u < nrows ? 13 : gcode[u - nrows];
    s += mix64((unsigned long long)((rj << 5) | code));
  }
  for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
  if (lane == 0) {
    const int64_t o = orig[centre_p[c]];
    out[2 * o] = (unsigned long long)n;
    out[2 * o + 1] = s;
  }
}

// ---- neighbour search -------------------------------------------------------------------
// One lane per centre; a group of G consecutive centres (in cell order, so
// neighbours in space) shares one stream of candidates.  The centres of a
// group whose home cell lies in the same (y, z) row of cells form a segment
// (almost always the whole group); for every row of cells that the segment's
// spheres reach, the x-extent of the union of the spheres selects a run of
// cells, which is one contiguous range of the sorted particles.  The group
// stages the ranges of RPL G rows at a time (a chunk) in shared memory with a
// prefix of their lengths and walks their concatenation G candidates at a time: every lane loads one
// candidate (coalesced) into shared memory, then every lane tests all G of
// them against its own centre and appends the hits to its centre's list.  A
// candidate is fetched once for the G centres, and no lane computes a range
// of cells for itself alone.
//
// Inclusion is the kd-tree's FP64 test, summed x, y, z in order without
// fused multiply-adds: ((dx*dx + dy*dy) + dz*dz) <= (krad*h)^2
// (kdtree2.f90:1673-1678, neighboursearch.f90:126), self excluded
// (neighboursearch.f90:190).  Most candidates are far from the sphere's
// surface, so a FP32 test on the one-binade position images decides them
// first: with per-axis image error e = 2^-23 * shift, the FP32 distance differs
// from the exact one by less than 2 sqrt(3) e R + 3 e^2 (plus FP32 rounding)
// near the surface, so delta = 8 e / R + 4 (e / R)^2 + 1e-6 bounds it.  Only
// the candidates with |sd32 - R^2| <= delta R^2 are tested in FP64; the FP64
// test alone decides membership, so the sets equal the FP64 predicate's.
constexpr int kNeibRowsPerLane = 2;  // RPL: rows of cells per lane and chunk (measured
                                     // best of 1-8 on the 128^3 Sedov step)

// minimum / maximum over the G lanes of a group (all lanes of the warp call)
template <int G>
__device__ __forceinline__ float group_min(float v) {
#pragma unroll
  for (int d = 1; d < G; d <<= 1) v = fminf(v, __shfl_xor_sync(0xffffffffu, v, d, G));
  return v;
}
template <int G>
__device__ __forceinline__ float group_max(float v) {
#pragma unroll
  for (int d = 1; d < G; d <<= 1) v = fmaxf(v, __shfl_xor_sync(0xffffffffu, v, d, G));
  return v;
}

// squared distance of two FP32 images, rounded the same way wherever it is
// computed (the guard-band pass recomputes it bit for bit)
__device__ __forceinline__ float dist2_f32(const float4& b, const float4& a) {
  const float fx = __fsub_rn(b.x, a.x), fy = __fsub_rn(b.y, a.y), fz = __fsub_rn(b.z, a.z);
  return __fmaf_rn(fz, fz, __fmaf_rn(fy, fy, __fmul_rn(fx, fx)));
}

// STAGED: each chunk's candidate runs (contiguous ranges of sorted records)
// are copied into shared memory by bulk copies, one per run, and tested
// from there, instead of being fetched a batch at a time by the lanes; a
// chunk that does not fit the stage falls back to the fetch.
constexpr int kStageRecords = 96;  // records staged per group and chunk
template <int DIM, int G, bool STAGED>
__global__ void __launch_bounds__(128, STAGED ? 4 : 7)
k_neighbours(NeibArgs a) {
  constexpr int RPL = STAGED ? 1 : kNeibRowsPerLane;
  constexpr int STG = kStageRecords;
  constexpr int NG = 128 / G;
  constexpr unsigned FULL = 0xffffffffu;
  // Staged ranges per group, stored [entry of the lane][lane] so that the
  // lanes' stores hit distinct banks.  Entry = (first sorted index of the
  // range - its offset in the concatenation, end of the range in the
  // concatenation).
  __shared__ int2 ranges[NG][RPL * G];
  // The batch of candidates: FP32 image and sorted index; one float4 of
  // padding per group puts the groups of a warp on different banks.
  __shared__ float4 batch[NG][G + 1];
  // Each lane's hits wait in its own slice of `held` and go to its list in
  // runs, written by the whole warp at once (coalesced), whenever a lane
  // holds FLUSH_AT or more.  At most G hits arrive between two checks, so
  // a slice of 33 words (a stride that spreads the slices over the banks)
  // never overflows and a run never exceeds the warp's 32 lanes.
  constexpr int FLUSH_AT = 33 - G;
  __shared__ int32_t held[128][33];
  // the staged runs of a chunk, then sentinels up to the warp's longest
  // concatenation + G; one mbarrier per group counts the copies' bytes
  __shared__ __align__(16) float4 stage[STAGED ? NG : 1][STAGED ? STG + G : 1];
  __shared__ __align__(8) unsigned long long mbar[STAGED ? NG : 1];
  const int64_t c = blockIdx.x * int64_t(blockDim.x) + threadIdx.x;
  const int lane = threadIdx.x & (G - 1);
  const int wl = threadIdx.x & 31;
  const unsigned gmask = (G == 32) ? FULL : (((1u << G) - 1u) << (wl & ~(G - 1)));
  int2* rs = ranges[threadIdx.x / G];
  float4* bt = batch[threadIdx.x / G];
  float4* const sg = stage[STAGED ? threadIdx.x / G : 0];
  unsigned long long* const mb = &mbar[STAGED ? threadIdx.x / G : 0];
  uint32_t mphase = 0;  // parity of the group's mbarrier phase in use
  if constexpr (STAGED) {
    if (lane == 0) mbar_init(mb, 1);
    mbar_init_fence();
    __syncwarp();
  }
  unsigned int ncand = 0, nexact = 0, nfound = 0;
  Grid g = a.g;
  double shift = a.shift;
  if (a.plan) {
    g = a.plan->grid;
    shift = a.plan->pg.shift;
  }
  // Every loop below runs the same number of passes on all lanes of the warp
  // (the maximum over its groups), so votes and shuffles take the full mask.
  const bool active = c < a.nc;
  int32_t k = -1, p = 0;
  double xi = 0.0, yi = 0.0, zi = 0.0, R2 = 0.0;
  float4 pi = make_float4(0.f, 0.f, 0.f, 0.f);
  float lo_thr = -1.f, hi_thr = -1.f, ux = 0.f, uy = 0.f, uz = 0.f, rc = 0.f, mrg = 0.f;
  int rcap = 0, home = -1;
  int64_t off = 0;
  int64_t cg = c;  // the centre's index in centre_k / centre_p / rowoff / rowcap / ncnt
  auto clampc = [](float v, int n) {
    float f = floorf(v);
    if (!(f >= 0.f)) return 0;
    if (f >= float(n - 1)) return n - 1;
    return int(f);
  };
  if (active) {
    if (a.cmap) cg = a.cmap[c];
    k = a.centre_k[cg];
    p = a.centre_p[cg];
    xi = a.sx[k]; yi = a.sy[k]; zi = a.sz[k];
    pi = a.s32[k];
    double kh = __dmul_rn(a.krad, a.hcol[p]);
    const double kf = a.kfac_dev ? *a.kfac_dev : a.kfac;
    if (kf > 0.0 && kf != 1.0) kh = __dmul_rn(kh, kf);  // a skin search
    R2 = __dmul_rn(kh, kh);
    const double R = sqrt(R2) * (1.0 + 1e-9) + 1e-300;
    const double er = (shift * 1.1920928955078125e-7) / R;  // per-axis image error / R
    const double delta = 8.0 * er + 4.0 * er * er + 1e-6;
    lo_thr = float(R2 * (1.0 - delta));
    hi_thr = float(R2 * (1.0 + delta));
    // Row selection in cell units and FP32: every quantity is widened by a
    // margin far above its rounding, so the selected cells are a superset of
    // the ones the spheres touch; membership is decided per candidate below.
    ux = float((xi - g.ox) * g.invL); uy = float((yi - g.oy) * g.invL);
    uz = float((zi - g.oz) * g.invL);
    mrg = 1e-3f + 1e-6f * (fabsf(ux) + fabsf(uy) + fabsf(uz));
    rc = float((R + a.reach) * g.invL) * (1.f + 1e-5f) + mrg;
    home = (DIM >= 2 ? clampc(uy, g.ny) : 0) + (DIM == 3 ? clampc(uz, g.nz) : 0) * g.ny;
    off = a.rowoff[cg];
    // slots usable without leaving the table; a shorter row is an overflow
    const int rcap0 = a.rowcap[cg];
    const int64_t room = a.nl_size - off;
    rcap = room <= 0 ? 0 : (room < int64_t(rcap0) ? int(room) : rcap0);
  }
  int cnt = 0;   // hits found so far (written to the list while they fit)
  int nheld = 0;  // hits waiting in held[threadIdx.x]
  int32_t* dst = a.nl + off;  // the list slot of hit number cnt
  int32_t* const mine_held = held[threadIdx.x];
  int32_t* const warp_held = held[threadIdx.x & ~31];
  // writes the held hits of the lanes in `who` to their lists, all 32
  // lanes of the warp carrying one lane's run at a time; a lane's run is
  // cut at its row's capacity (the hits past it are only counted)
  auto flush = [&](unsigned who) {
    const int nw = max(0, min(nheld, rcap - cnt));
    __syncwarp();
    while (who) {
      const int L = __ffs(who) - 1;
      who &= who - 1u;
      const int nL = __shfl_sync(FULL, nw, L);
      int32_t* const dL = reinterpret_cast<int32_t*>(
          __shfl_sync(FULL, reinterpret_cast<unsigned long long>(dst), L));
      if (wl < nL) __stcg(dL + wl, warp_held[L * 33 + wl]);
    }
    __syncwarp();
  };
  unsigned todo = __ballot_sync(FULL, active) & gmask;
  while (__any_sync(FULL, todo != 0u)) {
    // this pass: the centres that share the home row of the first one left
    const int lead = todo ? __ffs(todo) - 1 : wl;
    const int lead_home = __shfl_sync(FULL, home, lead);
    const bool mine = ((todo >> wl) & 1u) && home == lead_home;
    const unsigned seg = __ballot_sync(FULL, mine) & gmask;
    todo &= ~seg;
    // bounding box of the segment's centres and its largest radius (cells)
    const float BIG = 3.0e38f;
    const float bx0 = group_min<G>(mine ? ux : BIG), bx1 = group_max<G>(mine ? ux : -BIG);
    const float by0 = group_min<G>(mine ? uy : BIG), by1 = group_max<G>(mine ? uy : -BIG);
    const float bz0 = group_min<G>(mine ? uz : BIG), bz1 = group_max<G>(mine ? uz : -BIG);
    const float rmax = group_max<G>(mine ? rc : 0.f);
    const float bm = group_max<G>(mine ? mrg : 0.f);
    int cy0 = 0, cy1 = -1, cz0 = 0, cz1 = 0;
    if (seg) {
      cy0 = DIM >= 2 ? clampc(by0 - rmax, g.ny) : 0;
      cy1 = DIM >= 2 ? clampc(by1 + rmax, g.ny) : 0;
      cz0 = DIM == 3 ? clampc(bz0 - rmax, g.nz) : 0;
      cz1 = DIM == 3 ? clampc(bz1 + rmax, g.nz) : 0;
    }
    const int ny_r = cy1 - cy0 + 1;
    const int nrows_r = seg ? ny_r * (cz1 - cz0 + 1) : 0;
    const float r2 = rmax * rmax;
    // tests a batch of G candidates (cand[0 .. G-1], broadcast from shared
    // memory) against each lane's centre, then flushes the lanes whose held
    // hits reached FLUSH_AT
    auto test_batch = [&](const float4* cand) {
      if (mine) {
        // FP32 decisions for the batch: 0 < sd32 < lo is inside for sure.
        // The guard band and sd32 = 0 (the centre itself, or a particle
        // closer than the FP32 images resolve) are decided in FP64 after
        // the batch, which recomputes sd32 bit for bit to find them (rare:
        // about once per centre)
        // The candidate is written to the next free slot whether or not it
        // is a hit and kept only by counting it (no branch per test): a
        // lane starts a batch with at most FLUSH_AT - 1 = 32 - G held
        // hits, so test t writes slot <= 32 - G + t <= 31 of its 33.
        bool anyband = false;
#pragma unroll
        for (int t = 0; t < G; ++t) {
          const float4 pj = cand[t];
          const float sd32 = dist2_f32(pj, pi);
          const bool in32 = sd32 < lo_thr && sd32 > 0.f;
          anyband |= !in32 && !(sd32 > hi_thr);
          mine_held[nheld] = __float_as_int(pj.w);
          nheld += in32 ? 1 : 0;
        }
        if (anyband) {
#pragma unroll 1
        for (int t = 0; t < G; ++t) {
          const float4 pj = cand[t];
          const float sd32 = dist2_f32(pj, pi);
          if ((sd32 < lo_thr && sd32 > 0.f) || sd32 > hi_thr) continue;
          const int32_t q = __float_as_int(pj.w);
          if (q == k) continue;
          ++nexact;
          double d0 = __dadd_rn(a.sx[q], -xi);
          double d1 = __dadd_rn(a.sy[q], -yi);
          double d2 = __dadd_rn(a.sz[q], -zi);
          double sd = __dadd_rn(__dadd_rn(__dmul_rn(d0, d0), __dmul_rn(d1, d1)),
                                __dmul_rn(d2, d2));
          const bool take = !(sd > R2);
          if (take) mine_held[nheld] = q;
          nheld += take ? 1 : 0;
        }
        }
      }
      __syncwarp();  // the next batch overwrites this one
      const unsigned full = __ballot_sync(FULL, nheld >= FLUSH_AT);
      if (full) {
        flush(full);
        if ((full >> wl) & 1u) {
          cnt += nheld;
          dst += nheld;
          nheld = 0;
        }
      }
    };
    const int nch = __reduce_max_sync(FULL, (nrows_r + RPL * G - 1) / (RPL * G));
    for (int ch = 0; ch < nch; ++ch) {
      // Each lane takes RPL consecutive rows of the chunk (row rbase + i is
      // its i-th), so the lanes' runs concatenated in lane order follow the
      // rows in cell order: the candidates, and each centre's hits, come in
      // increasing record order.  First each lane finds its rows' runs of
      // cells, then issues all their cell-start loads at once.
      const int rbase = ch * RPL * G + lane * RPL;
      unsigned ia[RPL], ib[RPL];  // cstart indices of each run's ends
#pragma unroll
      for (int i = 0; i < RPL; ++i) ia[i] = ib[i] = 0u;
      if (nrows_r > 0) {  // then ny_r >= 1
        int cy = cy0 + rbase % ny_r, cz = cz0 + rbase / ny_r;
#pragma unroll
        for (int i = 0; i < RPL; ++i) {
          if (rbase + i < nrows_r) {
            float dzc = 0.f, dyc = 0.f;
            if (DIM == 3) dzc = fmaxf(0.f, fmaxf(float(cz) - bz1, bz0 - float(cz + 1)));
            if (DIM >= 2) dyc = fmaxf(0.f, fmaxf(float(cy) - by1, by0 - float(cy + 1)));
            const float rem = r2 - dyc * dyc - dzc * dzc;
            if (rem >= 0.f) {
              const float w = sqrtf(rem) + bm;
              const int cx0 = clampc(bx0 - w, g.nx);
              const int cx1 = clampc(bx1 + w, g.nx);
              const int64_t rowc = int64_t(g.nx) * (cy + int64_t(g.ny) * cz);
              ia[i] = unsigned(rowc + cx0);
              ib[i] = unsigned(rowc + cx1 + 1);
            }
          }
          if (++cy > cy1) { cy = cy0; ++cz; }
        }
      }
      int mysum = 0;
      {
        int32_t sa[RPL], sb[RPL];
#pragma unroll
        for (int i = 0; i < RPL; ++i) {
          sa[i] = __ldg(a.cstart + ia[i]);
          sb[i] = __ldg(a.cstart + ib[i]);
        }
#pragma unroll
        for (int i = 0; i < RPL; ++i) {
          rs[i * G + lane] = make_int2(sa[i], sb[i] - sa[i]);
          mysum += sb[i] - sa[i];
        }
      }
      // exclusive prefix of the lanes' sums over the group
      int incl = mysum;
#pragma unroll
      for (int d = 1; d < G; d <<= 1) {
        const int t = __shfl_up_sync(FULL, incl, d, G);
        if (lane >= d) incl += t;
      }
      const int total = __shfl_sync(FULL, incl, G - 1, G);
      int run = incl - mysum;
      int soff[RPL], ssa[RPL], slen[RPL];  // each run: offset in the concatenation, start, length
#pragma unroll
      for (int i = 0; i < RPL; ++i) {
        const int2 v = rs[i * G + lane];
        soff[i] = run;
        ssa[i] = v.x;
        slen[i] = v.y;
        rs[i * G + lane] = make_int2(v.x - run, run + v.y);
        run += v.y;
      }
      __syncwarp();
      if (mine) ncand += unsigned(total);
      const int tmax = __reduce_max_sync(FULL, total);
      const float4 far = make_float4(3.0e38f, 3.0e38f, 3.0e38f, __int_as_float(-1));
      if constexpr (STAGED) {
        if (__all_sync(FULL, total <= STG)) {
          // earlier generic reads and writes of the stage before the async
          // copies overwrite it
          __syncwarp();
          fence_proxy_async_smem();
          __syncwarp();
          if (total > 0) {  // the same on all lanes of the group
            if (lane == 0) mbar_arrive_expect_tx(mb, uint32_t(total) * 16u);
            __syncwarp(gmask);  // the expected bytes are set before any copy lands
#pragma unroll
            for (int i = 0; i < RPL; ++i)
              if (slen[i] > 0)
                bulk_g2s(sg + soff[i], a.s32 + ssa[i], uint32_t(slen[i]) * 16u, mb);
          }
          for (int pos = total + lane; pos < tmax + G; pos += G) sg[pos] = far;
          if (total > 0) {
            if (!mbar_wait_bounded(mb, mphase, 1 << 20)) {
              atomicOr(a.overflow, 2);  // reported as a timeout by the host
              mbar_wait_bounded(mb, mphase, 1 << 20);
            }
            mphase ^= 1u;
          }
          __syncwarp();
          for (int p0 = 0; p0 < tmax; p0 += G) test_batch(sg + p0);
          __syncwarp();  // the next chunk overwrites the ranges and the stage
          continue;
        }
      }
      // The walk: lane j of the group fetches candidate p0 + j of every
      // batch, one batch ahead of the tests (software pipelining), past the
      // end a far-away sentinel that no test accepts.
      int r = 0;
      int2 rw = rs[0];
      float4 nxt = far;
      int32_t nxt_q = -1;
      if (lane < total) {
        while (lane >= rw.y) {
          ++r;
          rw = rs[(r % RPL) * G + r / RPL];
        }
        nxt_q = lane + rw.x;
        nxt = __ldg(a.s32 + nxt_q);
      }
      for (int p0 = 0; p0 < tmax; p0 += G) {
        const float4 cur = make_float4(nxt.x, nxt.y, nxt.z, __int_as_float(nxt_q));
        const int pos = p0 + G + lane;
        nxt = far;
        nxt_q = -1;
        if (pos < total) {
          // the range holding pos: ends are increasing and the last one is
          // total, so the walk stays inside the chunk
          while (pos >= rw.y) {
            ++r;
            rw = rs[(r % RPL) * G + r / RPL];
          }
          nxt_q = pos + rw.x;
          nxt = __ldg(a.s32 + nxt_q);
        }
        bt[lane] = cur;
        __syncwarp();
        test_batch(bt);
      }
      __syncwarp();  // the next chunk overwrites the ranges
    }
  }
  {
    const unsigned left = __ballot_sync(FULL, nheld > 0);
    if (left) flush(left);
    cnt += nheld;
    nheld = 0;
  }
  if (active) {
    a.ncnt[cg] = cnt;
    a.count_prev[a.orig[p]] = cnt;
    a.h_prev[a.orig[p]] = float(a.hcol[p]);
    nfound = unsigned(cnt);
  }
  // the longest row, any overflow and the counters leave the block as one
  // atomic each (one per centre or warp on a single address would
  // serialise in its L2 slice)
  unsigned long long v[5] = {active ? (unsigned long long)cnt : 0ull,
                             (active && cnt > rcap) ? 1ull : 0ull, ncand, nfound, nexact};
  const bool is_max[5] = {true, true, false, false, false};
  block_counters<5>(v, is_max);
  if (threadIdx.x == 0) {
    if (v[0]) atomicMax(a.maxcnt, int(v[0]));
    if (v[1]) atomicOr(a.overflow, 1);
    if (v[2]) atomicAdd(&a.dcnt[DC_CANDIDATES], v[2]);
    if (v[3] && !a.skin_search) atomicAdd(&a.dcnt[DC_NEIB_PAIRS], v[3]);
    if (v[4]) atomicAdd(&a.dcnt[DC_EXACT_TESTS], v[4]);
  }
}

// ---- skin lists (SPH_P_SKIN) -------------------------------------------------------------
// A search of radius kfac krad h (kfac = 1 + s) at step b leaves each centre
// its skin list: every record within that radius at b.  At a later step t
// every record has moved by at most d (the running maximum of its FP64
// distance from its position at b), so a record j outside centre i's skin
// list lies at least kfac krad h_b - d_i - d_j from it (triangle
// inequality): it cannot pass i's predicate at t while
// krad h_t + d_i + d_j < kfac krad h_b.  Each centre takes one of three
// ways at t:
//  * fresh search (the search over the cells of step b, its cell range
//    widened by the largest displacement D): a record that moved more than
//    tau ("fast") is within reach, the centre moved more than tau itself, or
//    its h grew too far for the inequality above;
//  * keep: no record of its skin list moved more than eps, nor did the
//    centre, and 2 eps + krad |h_t - h_b| (running maximum) stays below the
//    gap of step b (the smallest distance of a skin-list record from the
//    sphere krad h_b): no record crossed the sphere, so the row written at
//    b is the set at t (the row is not touched; the ways are monotone, so a
//    kept row was never rewritten since b);
//  * filter: its skin list through the FP64 predicate.
// Either way each centre's set is the FP64 predicate's over all records,
// i.e. that of a fresh search.  The image records of step b are reused when
// no row's image signature changed (the image set is then the one the image
// builder would make at t) and are placed by the same arithmetic
// (image_coord).

// which periodic sides hold the row: per axis the unpadded side (-1, 0, +1)
// and whether the padded test agrees, 6 states per axis
__device__ __forceinline__ uint8_t image_sig(const double* r, const BoxGeom& g, int dim) {
  const AxisSigns sg = axis_signs(r, g, dim);
  int v = 0, m = 1;
  for (int k = 0; k < 3; ++k) {
    v += m * ((sg.npad[k] + 1) + 3 * (sg.pad[k] != 0 ? 1 : 0));
    m *= 6;
  }
  return uint8_t(v);
}

__global__ void k_skin_sig(const double* __restrict__ cols, int64_t ld, int64_t nrows,
                           BoxGeom g, int dim, uint8_t* __restrict__ sig) {
  const int64_t i = blockIdx.x * int64_t(blockDim.x) + threadIdx.x;
  if (i >= nrows) return;
  const double r[3] = {cols[es_rx * ld + i], cols[es_ry * ld + i], cols[es_rz * ld + i]};
  sig[i] = ghost_source(cols[es_type * ld + i]) ? image_sig(r, g, dim) : uint8_t(0);
}

__global__ void __launch_bounds__(TPB)
k_skin_refresh(const int32_t* __restrict__ sidx, int64_t n, int64_t nrows, int64_t nreal,
               const double* __restrict__ cols, int64_t ld, const int32_t* __restrict__ gsrc,
               const int8_t* __restrict__ gcode, BoxGeom g, int dim,
               const uint8_t* __restrict__ sig_b, const double* __restrict__ bx,
               const double* __restrict__ by, const double* __restrict__ bz,
               double* __restrict__ sx, double* __restrict__ sy, double* __restrict__ sz,
               float4* __restrict__ s32, PackGeom pg, float* __restrict__ dsp, float tau,
               float eps, double* __restrict__ hrec, unsigned long long* __restrict__ red,
               const DevPlan* __restrict__ plan, const DevSkin* __restrict__ gate) {
  if (gate && !gate->live) return;
  if (plan) {
    n = plan->nall;
    pg = plan->pg;
  }
  // slots: lo x, y, z (min), hi x, y, z (max), D (max), h of the real rows (max)
  double v[8] = {1e300, 1e300, 1e300, -1e300, -1e300, -1e300, 0.0, 0.0};
  const bool is_max[8] = {false, false, false, true, true, true, true, true};
  unsigned nfast = 0, nmove = 0;
  bool sigchg = false;
  for (int64_t k = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; k < n;
       k += int64_t(gridDim.x) * blockDim.x) {
    const int64_t u = sidx[k];
    double x, y, z;
    if (u < nrows) {
      x = cols[es_rx * ld + u]; y = cols[es_ry * ld + u]; z = cols[es_rz * ld + u];
      const double h = cols[es_h * ld + u];
      hrec[k] = h;  // (for the centres' ways, read in record order)
      if (u < nreal) v[7] = fmax(v[7], h);
      if (ghost_source(cols[es_type * ld + u])) {
        const double r[3] = {x, y, z};
        sigchg |= image_sig(r, g, dim) != sig_b[u];
      }
    } else {
      const int64_t q = u - nrows;
      const int64_t src = gsrc[q];
      const int code = gcode[q];
      x = image_coord(cols[es_rx * ld + src], code % 3 - 1, g.emin[0], g.emax[0]);
      y = image_coord(cols[es_ry * ld + src], (code / 3) % 3 - 1, g.emin[1], g.emax[1]);
      z = image_coord(cols[es_rz * ld + src], code / 9 - 1, g.emin[2], g.emax[2]);
    }
    sx[k] = x; sy[k] = y; sz[k] = z;
    s32[k] = make_float4(__double2float_rn((x - pg.ox) + pg.shift),
                         __double2float_rn((y - pg.oy) + pg.shift),
                         __double2float_rn((z - pg.oz) + pg.shift), __int_as_float(int32_t(k)));
    const double ex = x - bx[k], ey = y - by[k], ez = z - bz[k];
    // a few ulp of rounding in the differences, squares, sum and root: the
    // factor and the floor make the stored value an upper bound
    const double d = sqrt(ex * ex + ey * ey + ez * ez) * (1.0 + 1e-12) + 1e-300;
    const float df = fmaxf(dsp[k], __double2float_ru(d));  // running maximum since b
    dsp[k] = df;
    nfast += df > tau ? 1u : 0u;
    nmove += df > eps ? 1u : 0u;
    v[6] = fmax(v[6], double(df));
    v[0] = fmin(v[0], x); v[1] = fmin(v[1], y); v[2] = fmin(v[2], z);
    v[3] = fmax(v[3], x); v[4] = fmax(v[4], y); v[5] = fmax(v[5], z);
  }
  const unsigned wf = __reduce_add_sync(0xffffffffu, nfast);
  const unsigned wm = __reduce_add_sync(0xffffffffu, nmove);
  const unsigned ws = __ballot_sync(0xffffffffu, sigchg);
  if ((threadIdx.x & 31) == 0) {
    if (wf) atomicAdd(&red[RED_SKIN_NFAST], (unsigned long long)wf);
    if (wm) atomicAdd(&red[RED_SKIN_NMOVE], (unsigned long long)wm);
    if (ws) atomicMax(&red[RED_SKIN_SIG], 1ull);
  }
  block_minmax<8>(v, is_max);
  if (threadIdx.x == 0) {
    for (int k = 0; k < 3; ++k) {
      if (v[k] < 1e300) red_min(&red[RED_LO_X + k], v[k]);
      if (v[3 + k] > -1e300) red_max(&red[RED_HI_X + k], v[3 + k]);
    }
    red_max(&red[RED_SKIN_D], v[6]);
    red_max(&red[RED_SKIN_HMAX], v[7]);
  }
}

// clamped cell coordinate of an FP64 cell-unit value (NaN -> 0)
__device__ __forceinline__ int clamp_cell(double f, int n) {
  f = floor(f);
  if (!(f >= 0.0)) return 0;
  if (f >= double(n - 1)) return n - 1;
  return int(f);
}

// Marks at the level of cells: a record that moved more than eps flags the
// cell it was sorted into (its position at b), one that moved more than tau
// the cell of its position now (clamped to the grid); each flag field is
// then dilated by a box of w cells per side (k_dilate, one axis per pass),
// w = ceil(reach / L) + 1, which holds every cell within `reach` of any
// point of the flagged cell.  A centre is near a fast (moving) record when
// the cell it was sorted into carries the dilated flag.
__global__ void k_skin_cells(int64_t n, const float* __restrict__ dsp, float tau, float eps,
                             const uint32_t* __restrict__ keys, const double* __restrict__ sx,
                             const double* __restrict__ sy, const double* __restrict__ sz,
                             Grid g, uint8_t* __restrict__ fast_cell,
                             uint8_t* __restrict__ move_cell) {
  const int64_t k = blockIdx.x * int64_t(blockDim.x) + threadIdx.x;
  if (k >= n) return;
  const float d = dsp[k];
  if (move_cell && d > eps) move_cell[keys[k]] = 1;
  if (d > tau) {
    const int cx = clamp_cell((sx[k] - g.ox) * g.invL, g.nx);
    const int cy = clamp_cell((sy[k] - g.oy) * g.invL, g.ny);
    const int cz = clamp_cell((sz[k] - g.oz) * g.invL, g.nz);
    fast_cell[cx + int64_t(g.nx) * (cy + int64_t(g.ny) * cz)] = 1;
  }
}
// out[c] = OR of in over the cells within w of c along `axis` (out zeroed
// before): every marked cell writes its window, so the work follows the
// marks (a few per cent of the cells while the lists serve), not the grid
__global__ void k_dilate(const uint8_t* __restrict__ in, uint8_t* __restrict__ out, Grid g,
                         int axis, const int* __restrict__ wp) {
  const int64_t c = blockIdx.x * int64_t(blockDim.x) + threadIdx.x;
  const int64_t ncell = int64_t(g.nx) * g.ny * g.nz;
  if (c >= ncell || !in[c]) return;
  const int w = *wp;
  int n, i;
  int64_t stride;
  if (axis == 0) { n = g.nx; i = int(c % g.nx); stride = 1; }
  else if (axis == 1) { n = g.ny; i = int((c / g.nx) % g.ny); stride = g.nx; }
  else { n = g.nz; i = int(c / (int64_t(g.nx) * g.ny)); stride = int64_t(g.nx) * g.ny; }
  const int a = max(0, i - w), b = min(n - 1, i + w);
  for (int j = a; j <= b; ++j) out[c + int64_t(j - i) * stride] = 1;
}

// The way of each centre (mode: 0 filter, 1 fresh search, 2 keep; dflag =
// 1 for the fresh search).  The margins of 1e-12 (relative) lie far above
// the FP64 rounding of the predicate and of the displacements, so that no
// record outside a list can pass the FP64 predicate at t; near_f / near_m
// are the dilated cell flags (near_m == NULL: no centre keeps its row).
__global__ void k_skin_classify(int64_t nc, const int32_t* __restrict__ centre_k,
                                const double* __restrict__ hrec, const double* __restrict__ hb,
                                double* __restrict__ hdev, const float* __restrict__ gap,
                                double krad, double kfac, float tau, float eps,
                                const float* __restrict__ dsp,
                                const uint32_t* __restrict__ keys,
                                const uint8_t* __restrict__ near_f,
                                const uint8_t* __restrict__ near_m,
                                uint8_t* __restrict__ mode, int64_t* __restrict__ ways,
                                const int32_t* __restrict__ ncnt,
                                unsigned long long* __restrict__ nkept) {
  const int64_t c = blockIdx.x * int64_t(blockDim.x) + threadIdx.x;
  uint8_t w = 1;
  if (c < nc) {
    const bool was_searched = mode[c] == 1;  // (a centre once searched afresh stays so)
    const int32_t k = centre_k[c];
    const double h = hrec[k], h0 = hb[c];
    const double hd = fmax(hdev[c], fabs(h - h0));
    hdev[c] = hd;
    const double di = double(dsp[k]);
    const double lhs = krad * h * (1.0 + 1e-12) + di + double(tau);
    const double rhs = krad * h0 * kfac * (1.0 - 1e-12);
    const uint32_t cell = keys[k];  // the cell the centre was sorted into
    const bool clean = !was_searched && !near_f[cell] && dsp[k] <= tau && lhs < rhs;
    if (clean) {
      const bool keep = near_m && !near_m[cell] && dsp[k] <= eps &&
                        2.0 * double(eps) + krad * hd * (1.0 + 1e-12) + 1e-12 * krad * h0 <
                            double(gap[c]);
      w = keep ? 2 : 0;
    }
    mode[c] = w;
    // one scan counts both lists: fresh searches in the low word, filters
    // in the high one
    ways[c] = (w == 1 ? 1ll : 0ll) | (w == 0 ? (1ll << 32) : 0ll);
  }
  // rows kept and their neighbours: nkept[0], nkept[1]
  const bool kp = c < nc && w == 2;
  unsigned long long v[2] = {kp ? 1ull : 0ull, kp ? (unsigned long long)ncnt[c] : 0ull};
  const bool is_max[2] = {false, false};
  block_counters<2>(v, is_max);
  if (threadIdx.x == 0 && v[0]) {
    atomicAdd(nkept, v[0]);
    atomicAdd(nkept + 1, v[1]);
  }
}

// the lists of the centres searched afresh and of those that filter, in
// centre order, from the scan of k_skin_classify's ways
__global__ void k_skin_lists(int64_t nc, const int64_t* __restrict__ ways,
                             const int64_t* __restrict__ pos, int32_t* __restrict__ dlist,
                             int32_t* __restrict__ flist) {
  const int64_t c = blockIdx.x * int64_t(blockDim.x) + threadIdx.x;
  if (c >= nc) return;
  const int64_t w = ways[c], p = pos[c];
  if (w & 1) dlist[p & 0xffffffffll] = int32_t(c);
  if (w >> 32) flist[p >> 32] = int32_t(c);
}

__global__ void k_skin_compact(int64_t nc, const int32_t* __restrict__ dflag,
                               const int32_t* __restrict__ dpos, int32_t* __restrict__ dlist) {
  const int64_t c = blockIdx.x * int64_t(blockDim.x) + threadIdx.x;
  if (c < nc && dflag[c]) dlist[dpos[c]] = int32_t(c);
}

// hb[c] = h of centre c, and the largest of them into red[slot] (dkey max)
__global__ void __launch_bounds__(TPB)
k_gather_h(int64_t nc, const int32_t* __restrict__ centre_p, const double* __restrict__ hcol,
           double* __restrict__ hb, unsigned long long* __restrict__ red, int slot) {
  const int64_t c = blockIdx.x * int64_t(blockDim.x) + threadIdx.x;
  double v[1] = {0.0};
  const bool is_max[1] = {true};
  if (c < nc) {
    v[0] = hcol[centre_p[c]];
    hb[c] = v[0];
  }
  block_minmax<1>(v, is_max);
  if (threadIdx.x == 0) red_max(&red[slot], v[0]);
}

// G lanes per centre walk its skin list 4 G records at a time: every lane
// loads 4 consecutive entries at once (rows start on 16-byte boundaries:
// row capacities are multiples of 4) and gathers their 4 FP32 images
// together; FP32 test with the search's guard band, FP64 predicate in the
// band (the same arithmetic as the search, so the same decisions); the
// round's hits go to the row in list order (prefix of the lanes' counts).
// With gap != NULL each centre also records the smallest distance of a
// list record from its sphere, less the FP32 images' error bound.
// Counters and the longest row are summed over the block's whole share of
// centres (a grid of a few blocks per SM strides over them) and leave it as
// one atomic each: one atomic per centre on a single address would
// serialise in its L2 slice.
template <int G>
__global__ void __launch_bounds__(128) k_skin_filter(SkinFilterArgs a) {
  constexpr unsigned FULL = 0xffffffffu;
  if (a.plan) a.shift = a.plan->pg.shift;
  constexpr int V = 4;
  constexpr int PER = G * V;
  constexpr int CPB = 128 / G;  // centres per block and pass
  const int lane = threadIdx.x & (G - 1);
  unsigned long long ncand = 0, nfound = 0, nexact = 0;
  int maxc = 0;
  bool ovf = false;
  for (int64_t cb = blockIdx.x; cb * CPB < a.nc; cb += gridDim.x) {
    const int64_t i = cb * CPB + threadIdx.x / G;
    int64_t c = i;
    bool active = i < a.nc;
    if (a.list) {
      c = active ? a.list[i] : 0;  // (the list holds the centres that filter)
    } else if (active && a.mode) {
      const uint8_t w = a.mode[c];
      active = w == 0 || (w == 2 && !a.keep);
    }
    int32_t k = -1, n = 0, rcap = 0;
    int64_t off = 0;
    const int4* src = reinterpret_cast<const int4*>(a.skin_nl);
    double xi = 0.0, yi = 0.0, zi = 0.0, R2 = 0.0, hi_ = 0.0, Rx = 0.0;
    float4 pi = make_float4(0.f, 0.f, 0.f, 0.f);
    float lo_thr = -1.f, hi_thr = -1.f, Rf = 0.f;
    if (active) {
      k = a.centre_k[c];
      const int32_t p = a.centre_p[c];
      xi = a.sx[k]; yi = a.sy[k]; zi = a.sz[k];
      pi = a.s32[k];
      hi_ = a.hcol[p];
      const double kh = __dmul_rn(a.krad, hi_);
      R2 = __dmul_rn(kh, kh);
      Rx = sqrt(R2);
      Rf = float(Rx);
      const double R = Rx * (1.0 + 1e-9) + 1e-300;
      const double er = (a.shift * 1.1920928955078125e-7) / R;
      const double delta = 8.0 * er + 4.0 * er * er + 1e-6;
      lo_thr = float(R2 * (1.0 - delta));
      hi_thr = float(R2 * (1.0 + delta));
      n = a.skin_cnt[c];
      if (a.skin_cap) {
        const int64_t sroom = a.skin_size - a.skin_off[c];
        const int scap = sroom <= 0 ? 0 : int(min(int64_t(a.skin_cap[c]), sroom));
        n = min(n, scap);
      }
      src = reinterpret_cast<const int4*>(a.skin_nl + a.skin_off[c]);
      off = a.rowoff[c];
      const int rcap0 = a.rowcap[c];
      const int64_t room = a.nl_size - off;
      rcap = room <= 0 ? 0 : (room < int64_t(rcap0) ? int(room) : rcap0);
    }
    const int rounds = __reduce_max_sync(FULL, active ? (n + PER - 1) / PER : 0);
    int cnt = 0;
    float gmin = 3.0e38f;
    int32_t* const dst = a.nl + off;
    for (int r = 0; r < rounds; ++r) {
      const int base = r * PER + lane * V;
      int32_t q[V] = {-1, -1, -1, -1};
      unsigned m = 0;
      if (active && base < n) {
        // the int4 holding entry base lies inside the row's capacity
        const int4 v = __ldcs(src + (r * G + lane));
        q[0] = v.x; q[1] = v.y; q[2] = v.z; q[3] = v.w;
        float4 pj[V];
#pragma unroll
        for (int j = 0; j < V; ++j)
          if (base + j < n) pj[j] = __ldg(a.s32 + q[j]);
#pragma unroll
        for (int j = 0; j < V; ++j) {
          if (base + j >= n) continue;
          const float sd32 = dist2_f32(pj[j], pi);
          if ((sd32 < lo_thr && sd32 > 0.f) || sd32 > hi_thr) {
            if (sd32 <= hi_thr) m |= 1u << j;
            if (a.gap) {
              // |r - R| from the images: their error (eimg) and the FP32
              // rounding of the distance, the root and the difference
              const float r32 = sqrtf(sd32);
              gmin = fminf(gmin, fabsf(r32 - Rf) - (a.eimg + 4e-7f * (Rf + r32)));
            }
          } else if (q[j] != k) {
            ++nexact;
            const double d0 = __dadd_rn(a.sx[q[j]], -xi);
            const double d1 = __dadd_rn(a.sy[q[j]], -yi);
            const double d2 = __dadd_rn(a.sz[q[j]], -zi);
            const double sd = __dadd_rn(__dadd_rn(__dmul_rn(d0, d0), __dmul_rn(d1, d1)),
                                        __dmul_rn(d2, d2));
            if (!(sd > R2)) m |= 1u << j;
            if (a.gap) gmin = fminf(gmin, __double2float_rd(fabs(sqrt(sd) - Rx) - 1e-9 * Rx));
          }
        }
      }
      // exclusive prefix of the hit counts over the group's lanes
      const int nh = __popc(m);
      int incl = nh;
#pragma unroll
      for (int d = 1; d < G; d <<= 1) {
        const int t = __shfl_up_sync(FULL, incl, d, G);
        if (lane >= d) incl += t;
      }
      const int total = __shfl_sync(FULL, incl, G - 1, G);
      int pos = cnt + incl - nh;
#pragma unroll
      for (int j = 0; j < V; ++j)
        if ((m >> j) & 1u) {
          if (pos < rcap) __stcg(dst + pos, q[j]);
          ++pos;
        }
      cnt += total;
    }
    if (a.gap) {
#pragma unroll
      for (int d = 1; d < G; d <<= 1) gmin = fminf(gmin, __shfl_xor_sync(FULL, gmin, d, G));
    }
    if (active && lane == 0) {
      const int32_t p = a.centre_p[c];
      a.ncnt[c] = cnt;
      a.count_prev[a.orig[p]] = cnt;
      a.h_prev[a.orig[p]] = float(hi_);
      if (a.gap) a.gap[c] = gmin;
      maxc = max(maxc, cnt);
      ovf |= cnt > rcap;
      nfound += unsigned(cnt);
      ncand += unsigned(n);
    }
  }
  // block totals: warp reductions, then the 4 warps through shared memory
  __shared__ unsigned long long part[4][3];
  __shared__ int pmax[4], povf[4];
  const int w = threadIdx.x >> 5, wl = threadIdx.x & 31;
  for (int o = 16; o > 0; o >>= 1) {
    ncand += __shfl_xor_sync(FULL, ncand, o);
    nfound += __shfl_xor_sync(FULL, nfound, o);
    nexact += __shfl_xor_sync(FULL, nexact, o);
  }
  const int wmax = __reduce_max_sync(FULL, maxc);
  const bool wovf = __any_sync(FULL, ovf);
  if (wl == 0) {
    part[w][0] = ncand; part[w][1] = nfound; part[w][2] = nexact;
    pmax[w] = wmax;
    povf[w] = wovf ? 1 : 0;
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    unsigned long long t[3] = {0, 0, 0};
    int mx = 0, ov = 0;
    for (int i = 0; i < int(blockDim.x >> 5); ++i) {
      for (int j = 0; j < 3; ++j) t[j] += part[i][j];
      mx = max(mx, pmax[i]);
      ov |= povf[i];
    }
    if (t[0]) atomicAdd(&a.dcnt[DC_CANDIDATES], t[0]);
    if (t[1]) atomicAdd(&a.dcnt[DC_NEIB_PAIRS], t[1]);
    if (t[2]) atomicAdd(&a.dcnt[DC_EXACT_TESTS], t[2]);
    if (mx) atomicMax(a.maxcnt, mx);
    if (ov) atomicOr(a.overflow, 1);
  }
}

// ---- rows renamed under skin lists (a re-sort, a table upload) -----------------------------
// Old row perm[i] becomes row i; the sorted records, the images and the
// centres name rows, so they follow through inv[old] = new; the rows' image
// signatures move with their rows.
__global__ void k_inv_perm(const int32_t* __restrict__ perm, int64_t n, int32_t* __restrict__ inv) {
  const int64_t i = blockIdx.x * int64_t(blockDim.x) + threadIdx.x;
  if (i < n) inv[perm[i]] = int32_t(i);
}
// *changed = 1 if a row's particle type differs from the one its row had
// (old types by old row, perm[new] = old)
__global__ void k_type_changed(const double* __restrict__ cols, int64_t ld, int64_t n,
                               const double* __restrict__ old_type,
                               const int32_t* __restrict__ perm, int32_t* __restrict__ changed) {
  const int64_t i = blockIdx.x * int64_t(blockDim.x) + threadIdx.x;
  if (i < n && !(cols[es_type * ld + i] == old_type[perm[i]])) *changed = 1;
}
__global__ void k_rows_renamed(const int32_t* __restrict__ inv, const int32_t* __restrict__ perm,
                               int64_t nall, int64_t nrows, int64_t nghost, int64_t nreal,
                               int32_t* __restrict__ sidx, int32_t* __restrict__ ssrc,
                               int32_t* __restrict__ gsrc, int32_t* __restrict__ centre_p,
                               const uint8_t* __restrict__ sig_in, uint8_t* __restrict__ sig_out) {
  const int64_t k = blockIdx.x * int64_t(blockDim.x) + threadIdx.x;
  if (k < nall) {
    const int32_t u = sidx[k];
    if (u < nrows) sidx[k] = inv[u];
    ssrc[k] = inv[ssrc[k]];
  }
  if (k < nghost) gsrc[k] = inv[gsrc[k]];
  if (k < nreal) centre_p[k] = inv[centre_p[k]];
  if (k < nrows) sig_out[k] = sig_in[perm[k]];
}

// ---- rows of the centres searched afresh (skin-list iterates) -----------------------------
// They are laid out anew every iterate after the table's fixed part (whose
// rows the other centres keep): cap[i] for centre list[i] from its last
// count as k_rowcap sizes rows, then (after the scan) rowoff / rowcap.
__global__ void k_dyn_caps(int64_t nd, const int32_t* __restrict__ list,
                           const int32_t* __restrict__ centre_p, const int32_t* __restrict__ orig,
                           const int32_t* __restrict__ count_prev,
                           const float* __restrict__ h_prev, const double* __restrict__ hcol,
                           int dim, float slack, int64_t* __restrict__ cap) {
  const int64_t i = blockIdx.x * int64_t(blockDim.x) + threadIdx.x;
  if (i > nd) return;
  if (i == nd) { cap[i] = 0; return; }
  const int32_t p = centre_p[list[i]];
  const int32_t o = orig[p];
  float est = float(count_prev[o]);
  const float hp = h_prev[o];
  if (hp > 0.f) {
    float g = float(hcol[p]) / hp;
    g = fminf(fmaxf(g, 0.5f), 4.f);
    est *= dim == 3 ? g * g * g : (dim == 2 ? g * g : g);
  }
  cap[i] = (int64_t(fminf(est * slack, 1.0e9f)) + 8 + 3) & ~int64_t(3);
}
__global__ void k_dyn_assign(int64_t nd, const int32_t* __restrict__ list,
                             const int64_t* __restrict__ off, const int64_t* __restrict__ cap,
                             const int64_t* __restrict__ base, int64_t* __restrict__ rowoff,
                             int32_t* __restrict__ rowcap) {
  const int64_t i = blockIdx.x * int64_t(blockDim.x) + threadIdx.x;
  if (i >= nd) return;
  const int32_t c = list[i];
  rowoff[c] = *base + off[i];
  rowcap[c] = int32_t(cap[i]);
}
// end[0] = rowoff[n - 1] + rowcap[n - 1] (the end of a freshly laid-out table)
__global__ void k_table_end(const int64_t* __restrict__ rowoff, const int32_t* __restrict__ rowcap,
                            int64_t n, int64_t* __restrict__ end) {
  end[0] = n > 0 ? rowoff[n - 1] + rowcap[n - 1] : 0;
}
// filter rows that overflowed their place join the centres searched afresh:
// mode[c] = 1, and dflag[c] = 1 for every centre of mode 1
__global__ void k_overflow_to_search(int64_t nc, const int32_t* __restrict__ ncnt,
                                     const int64_t* __restrict__ rowoff,
                                     const int32_t* __restrict__ rowcap, int64_t nl_size,
                                     uint8_t* __restrict__ mode, int32_t* __restrict__ dflag) {
  const int64_t c = blockIdx.x * int64_t(blockDim.x) + threadIdx.x;
  if (c >= nc) return;
  uint8_t w = mode[c];
  if (w == 0) {
    const int64_t room = nl_size - rowoff[c];
    const int64_t rc = room < int64_t(rowcap[c]) ? (room > 0 ? room : 0) : int64_t(rowcap[c]);
    if (int64_t(ncnt[c]) > rc) w = 1;
  }
  mode[c] = w;
  dflag[c] = w == 1 ? 1 : 0;
}

// Search of a few centres (a list): G lanes per centre walk the rows of
// cells its sphere reaches (radius krad h + reach, the records having moved
// up to `reach` from the positions they were sorted by), each row's x-run of
// cells one contiguous run of records, G records at a time: the search's FP32
// test with its guard band, the FP64 predicate in the band, the hits in walk
// order (ballot + prefix within the group).  Row by row in increasing cell
// index, so each row of the list is in increasing record order.
template <int DIM, int G>
__global__ void __launch_bounds__(128) k_search_few(FewArgs a) {
  constexpr int CPB = 128 / G;
  const int lane = threadIdx.x & (G - 1);
  const unsigned gmask = (G == 32) ? 0xffffffffu
                                   : (((1u << G) - 1u) << ((threadIdx.x & 31) & ~(G - 1)));
  const unsigned below = (1u << lane) - 1u;
  unsigned long long ncand = 0, nfound = 0, nexact = 0;
  int maxc = 0;
  bool ovf = false;
  for (int64_t cb = blockIdx.x; cb * CPB < a.n; cb += gridDim.x) {
    const int64_t i = cb * CPB + threadIdx.x / G;
    if (i >= a.n) continue;  // (the whole group)
    const int32_t c = a.list[i];
    const int32_t k = a.centre_k[c], p = a.centre_p[c];
    const double xi = a.sx[k], yi = a.sy[k], zi = a.sz[k];
    const float4 pi = a.s32[k];
    const double hi_ = a.hcol[p];
    const double kh = __dmul_rn(a.krad, hi_);
    const double R2 = __dmul_rn(kh, kh);
    const double R = sqrt(R2) * (1.0 + 1e-9) + 1e-300;
    const double er = (a.shift * 1.1920928955078125e-7) / R;
    const double delta = 8.0 * er + 4.0 * er * er + 1e-6;
    const float lo_thr = float(R2 * (1.0 - delta)), hi_thr = float(R2 * (1.0 + delta));
    const Grid& g = a.g;
    const double ux = (xi - g.ox) * g.invL, uy = (yi - g.oy) * g.invL, uz = (zi - g.oz) * g.invL;
    // radius in cells, widened far above its rounding
    const double rr = (R + a.reach) * g.invL * (1.0 + 1e-9) +
                      1e-9 * (fabs(ux) + fabs(uy) + fabs(uz)) + 1e-6;
    const int cy0 = DIM >= 2 ? clamp_cell(uy - rr, g.ny) : 0;
    const int cy1 = DIM >= 2 ? clamp_cell(uy + rr, g.ny) : 0;
    const int cz0 = DIM == 3 ? clamp_cell(uz - rr, g.nz) : 0;
    const int cz1 = DIM == 3 ? clamp_cell(uz + rr, g.nz) : 0;
    const int64_t off = a.rowoff[c];
    const int rcap0 = a.rowcap[c];
    const int64_t room = a.nl_size - off;
    const int rcap = room <= 0 ? 0 : (room < int64_t(rcap0) ? int(room) : rcap0);
    int32_t* const dst = a.nl + off;
    int cnt = 0;
    // the rows of cells in (z, y) order, G at a time: each lane finds one
    // row's run of records (its two cell-start loads issued side by side
    // with the other lanes'), then the group walks the G runs in order
    const int ny_r = cy1 - cy0 + 1;
    const int nrows_r = ny_r * (cz1 - cz0 + 1);
    for (int r0 = 0; r0 < nrows_r; r0 += G) {
      int32_t mq0 = 0, mq1 = 0;
      const int r = r0 + lane;
      if (r < nrows_r) {
        const int cy = cy0 + r % ny_r, cz = cz0 + r / ny_r;
        const double dzc = DIM == 3 ? fmax(0.0, fmax(double(cz) - uz, uz - double(cz + 1))) : 0.0;
        const double dyc = DIM >= 2 ? fmax(0.0, fmax(double(cy) - uy, uy - double(cy + 1))) : 0.0;
        const double rem = rr * rr - dyc * dyc - dzc * dzc;
        if (rem >= 0.0) {
          const double w = sqrt(rem);
          const int cx0 = clamp_cell(ux - w, g.nx), cx1 = clamp_cell(ux + w, g.nx);
          const int64_t rowc = int64_t(g.nx) * (cy + int64_t(g.ny) * cz);
          mq0 = __ldg(a.cstart + rowc + cx0);
          mq1 = __ldg(a.cstart + rowc + cx1 + 1);
        }
      }
      for (int jr = 0; jr < G; ++jr) {
        const int32_t q0 = __shfl_sync(gmask, mq0, jr, G), q1 = __shfl_sync(gmask, mq1, jr, G);
        ncand += (lane == 0) ? unsigned(q1 - q0) : 0u;
        for (int32_t b = q0; b < q1; b += G) {
          const int32_t q = b + lane;
          bool hit = false;
          if (q < q1) {
            const float sd32 = dist2_f32(__ldg(a.s32 + q), pi);
            if (sd32 < lo_thr && sd32 > 0.f) {
              hit = true;
            } else if (!(sd32 > hi_thr) && q != k) {
              ++nexact;
              const double d0 = __dadd_rn(a.sx[q], -xi);
              const double d1 = __dadd_rn(a.sy[q], -yi);
              const double d2 = __dadd_rn(a.sz[q], -zi);
              const double sd = __dadd_rn(__dadd_rn(__dmul_rn(d0, d0), __dmul_rn(d1, d1)),
                                          __dmul_rn(d2, d2));
              hit = !(sd > R2);
            }
          }
          const unsigned hb = __ballot_sync(gmask, hit) >> ((threadIdx.x & 31) & ~(G - 1));
          if (hit) {
            const int pos = cnt + __popc(hb & below);
            if (pos < rcap) __stcg(dst + pos, q);
          }
          cnt += __popc(hb);
        }
      }
    }
    if (lane == 0) {
      a.ncnt[c] = cnt;
      a.count_prev[a.orig[p]] = cnt;
      a.h_prev[a.orig[p]] = float(hi_);
      maxc = max(maxc, cnt);
      ovf |= cnt > rcap;
      nfound += unsigned(cnt);
    }
  }
  // block totals (as k_skin_filter)
  constexpr unsigned FULL = 0xffffffffu;
  __shared__ unsigned long long part[4][3];
  __shared__ int pmax[4], povf[4];
  const int w = threadIdx.x >> 5, wl = threadIdx.x & 31;
  __syncwarp();
  for (int o = 16; o > 0; o >>= 1) {
    ncand += __shfl_xor_sync(FULL, ncand, o);
    nfound += __shfl_xor_sync(FULL, nfound, o);
    nexact += __shfl_xor_sync(FULL, nexact, o);
  }
  const int wmax = __reduce_max_sync(FULL, maxc);
  const bool wovf = __any_sync(FULL, ovf);
  if (wl == 0) {
    part[w][0] = ncand; part[w][1] = nfound; part[w][2] = nexact;
    pmax[w] = wmax;
    povf[w] = wovf ? 1 : 0;
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    unsigned long long t[3] = {0, 0, 0};
    int mx = 0, ov = 0;
    for (int j = 0; j < int(blockDim.x >> 5); ++j) {
      for (int q = 0; q < 3; ++q) t[q] += part[j][q];
      mx = max(mx, pmax[j]);
      ov |= povf[j];
    }
    if (t[0]) atomicAdd(&a.dcnt[DC_CANDIDATES], t[0]);
    if (t[1]) atomicAdd(&a.dcnt[DC_NEIB_PAIRS], t[1]);
    if (t[2]) atomicAdd(&a.dcnt[DC_EXACT_TESTS], t[2]);
    if (mx) atomicMax(a.maxcnt, mx);
    if (ov) atomicOr(a.overflow, 1);
  }
}

// Row capacity of each centre's neighbour list: the particle's count from
// the previous search, scaled by (h / h_then)^dim for the change of its
// search radius since, plus 20% and 8 slots of slack (or the initial
// estimate, which comes with h_then = 0).
__global__ void k_rowcap(int64_t nc, const int32_t* __restrict__ centre_p,
                         const int32_t* __restrict__ orig, const int32_t* __restrict__ count_prev,
                         const float* __restrict__ h_prev, const double* __restrict__ hcol,
                         int dim, float slack, int64_t* __restrict__ rowcap64,
                         int32_t* __restrict__ rowcap) {
  int64_t c = blockIdx.x * int64_t(blockDim.x) + threadIdx.x;
  if (c >= nc) return;
  const int32_t p = centre_p[c];
  const int32_t o = orig[p];
  float est = float(count_prev[o]);
  const float hp = h_prev[o];
  if (hp > 0.f) {
    float g = float(hcol[p]) / hp;
    g = fminf(fmaxf(g, 0.5f), 4.f);
    est *= dim == 3 ? g * g * g : (dim == 2 ? g * g : g);
  }
  // a multiple of 4, so that every row starts on a 16-byte boundary
  const int cap = (int(fminf(est * slack, 1.0e9f)) + 8 + 3) & ~3;
  rowcap[c] = cap;
  rowcap64[c] = cap;
}

// ---- pair-data packing (sorted order) --------------------------------------------------------
// a position in fixed-point units of the packing frame, in [0, 2^31)
__device__ __forceinline__ int32_t fixpos(double t) {
  t = rint(t);
  if (!(t >= 0.0)) return 0;
  if (t > 2147483647.0) return 2147483647;
  return int32_t(t);
}
__global__ void k_pack(int prec, int groups, int64_t n, const int32_t* __restrict__ ssrc,
                       const double* __restrict__ sx, const double* __restrict__ sy,
                       const double* __restrict__ sz, const double* __restrict__ cols, int64_t ld,
                       PackGeom pg, PackBufs pb, const DevPlan* __restrict__ plan) {
  int64_t k = blockIdx.x * int64_t(blockDim.x) + threadIdx.x;
  if (plan) {
    n = plan->nall;
    pg = plan->pg;
  }
  if (k >= n) return;
  const int64_t p = ssrc[k];
  auto C = [&](int f) { return cols[f * ld + p]; };
  const double m = C(es_m) / pg.mref;
  if (prec == SPH_PREC_FP64) {
    if (groups & PACK_POS) {
      pb.p[0][k] = make_double2(sx[k], sy[k]);
      pb.p[1][k] = make_double2(sz[k], m);
      if (groups & PACK_TEMP) pb.p[6][k] = make_double2(C(es_vz), C(es_t));
    }
    if (groups & PACK_HYDRO) {
      double h = C(es_h), rho = C(es_den), om = C(es_om), P = C(es_p);
      pb.p[2][k] = make_double2(1.0 / h, rho);
      pb.p[3][k] = make_double2(1.0 / (rho * rho * om), P);
      pb.p[4][k] = make_double2(C(es_c), C(es_u));
      pb.p[5][k] = make_double2(C(es_vx), C(es_vy));
      pb.p[6][k] = make_double2(C(es_vz), C(es_t));
    }
    if (groups & PACK_EXTRA) {
      pb.p[7][k] = make_double2(C(es_kappa), C(es_dtdx));
      pb.p[8][k] = make_double2(C(es_dtdy), C(es_dtdz));
      pb.p[9][k] = make_double2(C(es_bx), C(es_by));
      pb.p[10][k] = make_double2(C(es_bz), 0.0);
    }
  } else {
    if (groups & PACK_POS) {
      // the density pass: 31-bit fixed point over the frame (every record
      // has 0 <= x - origin < shift), one 16-byte record per neighbour
      const double sc = 2147483648.0 / pg.shift;  // (a power of two)
      const int32_t xi = fixpos((sx[k] - pg.ox) * sc);
      const int32_t yi = fixpos((sy[k] - pg.oy) * sc);
      const int32_t zi = fixpos((sz[k] - pg.oz) * sc);
      pb.q[6][k] = make_float4(__int_as_float(xi), __int_as_float(yi), __int_as_float(zi), float(m));
      if (k == 0) *pb.unit = float(pg.shift / 2147483648.0);
      if (groups & PACK_TEMP)
        pb.q[4][k] = make_float4(float(C(es_t)), float(C(es_kappa)), float(C(es_dtdx)),
                               float(C(es_dtdy)));
    }
    if (groups & PACK_HYDRO) {
      // the force pass: high and low FP32 parts in one binade (the highs'
      // differences are exact)
      const double xs = (sx[k] - pg.ox) + pg.shift;
      const double ys = (sy[k] - pg.oy) + pg.shift;
      const double zs = (sz[k] - pg.oz) + pg.shift;
      const float xh = __double2float_rn(xs), yh = __double2float_rn(ys), zh = __double2float_rn(zs);
      const float xl = __double2float_rn(xs - double(xh));
      const float yl = __double2float_rn(ys - double(yh));
      const float zl = __double2float_rn(zs - double(zh));
      double h = C(es_h), rho = C(es_den), om = C(es_om), P = C(es_p);
      pb.q[0][k] = make_float4(xh, yh, zh, float(m));
      pb.q[1][k] = make_float4(xl, yl, zl, float(1.0 / h));
      // wCv / (h^(d+1) rho^2 Omega): the neighbour's kernel factor and
      // 1/(rho^2 Omega) always meet as this product in the force pass
      const double ih = 1.0 / h;
      double kp = pb.kp_wcv;
      for (int d = 0; d <= pb.kp_dim; ++d) kp *= ih;
      pb.q[2][k] = make_float4(float(0.5 * rho), float(kp / (rho * rho * om)), float(P),
                               float(pb.kp_alpha * C(es_c)));
      pb.q[3][k] = make_float4(float(pb.kp_au * C(es_u)), float(C(es_vx)), float(C(es_vy)),
                               float(C(es_vz)));
    }
    if (groups & PACK_EXTRA) {
      pb.q[4][k] = make_float4(float(C(es_t)), float(C(es_kappa)), float(C(es_dtdx)),
                               float(C(es_dtdy)));
      pb.q[5][k] = make_float4(float(C(es_dtdz)), float(C(es_bx)), float(C(es_by)),
                               float(C(es_bz)));
    }
  }
}

// ---- leapfrog (main.f90:323-362) ----------------------------------------------------------
// Integrated rows: the reals and the fixedreal rows that follow them
// (main.f90:181-184), selected by original row index.  Arithmetic in the
// reference's evaluation order without contraction, so the update is bitwise
// reproducible by the CPU oracle.  B (T) is left as it is when no equation
// gives it a derivative (dB/dt = 0, dT/dt = 0 every step): x + dt 0 = x,
// except that a stored -0 would become +0.
enum SaveSlot : int { SV_AX = 0, SV_AY, SV_AZ, SV_DU, SV_DH, SV_DDT, SV_DBX, SV_DBY, SV_DBZ, SV_N };

__global__ void k_predict(double* __restrict__ cols, int64_t ld, const int32_t* __restrict__ orig,
                          int64_t nrows, int64_t n_int, double* __restrict__ save,
                          const double* __restrict__ ctrl, int mode) {
  int64_t i = blockIdx.x * int64_t(blockDim.x) + threadIdx.x;
  if (i >= nrows || orig[i] >= n_int) return;
  const bool do_b = !(mode & LF_NO_B), do_t = !(mode & (LF_STS | LF_NO_T));
  const double dt = ctrl[0];
  const double hdt2 = __dmul_rn(__dmul_rn(0.5, dt), dt);
  auto C = [&](int f) -> double& { return cols[f * ld + i]; };
  double ta[3], tv[3];
  for (int k = 0; k < 3; ++k) {
    ta[k] = C(es_ax + k);
    tv[k] = C(es_vx + k);
    save[(SV_AX + k) * ld + i] = ta[k];
    if (do_b) save[(SV_DBX + k) * ld + i] = C(es_dbx + k);
  }
  double tdu = C(es_du), tdh = C(es_dh);
  save[SV_DU * ld + i] = tdu;
  save[SV_DH * ld + i] = tdh;
  const double tddt = do_t ? C(es_ddt) : 0.0;
  if (do_t) save[SV_DDT * ld + i] = tddt;
  for (int k = 0; k < 3; ++k) {
    C(es_rx + k) = __dadd_rn(__dadd_rn(C(es_rx + k), __dmul_rn(dt, tv[k])), __dmul_rn(hdt2, ta[k]));
    C(es_vx + k) = __dadd_rn(tv[k], __dmul_rn(dt, ta[k]));
  }
  C(es_u) = __dadd_rn(C(es_u), __dmul_rn(dt, tdu));
  C(es_h) = __dadd_rn(C(es_h), __dmul_rn(dt, tdh));
  if (do_t) C(es_t) = __dadd_rn(C(es_t), __dmul_rn(dt, tddt));
  if (do_b)
    for (int k = 0; k < 3; ++k)
      C(es_bx + k) = __dadd_rn(C(es_bx + k), __dmul_rn(dt, save[(SV_DBX + k) * ld + i]));
}

__global__ void k_correct(double* __restrict__ cols, int64_t ld, const int32_t* __restrict__ orig,
                          int64_t nrows, int64_t n_int, const double* __restrict__ save,
                          const double* __restrict__ ctrl, int mode) {
  int64_t i = blockIdx.x * int64_t(blockDim.x) + threadIdx.x;
  if (i >= nrows || orig[i] >= n_int) return;
  const bool do_b = !(mode & LF_NO_B), do_t = !(mode & (LF_STS | LF_NO_T));
  const double hdt = __dmul_rn(0.5, ctrl[0]);
  auto C = [&](int f) -> double& { return cols[f * ld + i]; };
  for (int k = 0; k < 3; ++k)
    C(es_vx + k) = __dadd_rn(C(es_vx + k), __dmul_rn(hdt, __dadd_rn(C(es_ax + k), -save[(SV_AX + k) * ld + i])));
  C(es_u) = __dadd_rn(C(es_u), __dmul_rn(hdt, __dadd_rn(C(es_du), -save[SV_DU * ld + i])));
  C(es_h) = __dadd_rn(C(es_h), __dmul_rn(hdt, __dadd_rn(C(es_dh), -save[SV_DH * ld + i])));
  if (do_b)
    for (int k = 0; k < 3; ++k)
      C(es_bx + k) = __dadd_rn(C(es_bx + k), __dmul_rn(hdt, __dadd_rn(C(es_dbx + k), -save[(SV_DBX + k) * ld + i])));
  if (do_t) C(es_t) = __dadd_rn(C(es_t), __dmul_rn(hdt, __dadd_rn(C(es_ddt), -save[SV_DDT * ld + i])));
}

// ---- timestep reductions (timestep.f90:40-166) -----------------------------------------------
// Over the first realpn rows in original order.
__global__ void __launch_bounds__(TPB)
k_timestep_reduce(const double* __restrict__ cols, int64_t ld, const int32_t* __restrict__ orig,
                  int64_t nrows, int64_t n_ts, Params P, unsigned long long* __restrict__ red) {
  // slots: hmin, cmax, denmin, cmin, kapmax, bmax, kapmin, lammax
  // kappa (slots 4, 6) enters only the diffusion / FLD timesteps and B
  // (slot 5) only the MHD one: their columns are read only when those
  // equations are on (a slot left at its start value is not used)
  double v[8] = {1e308, -1e308, 1e308, 1e308, -1e308, -1e308, 1e308, -1e308};
  const bool is_max[8] = {false, true, false, false, true, true, false, true};
  const bool need_ka = P.eq_diff || P.eq_fld, need_b = P.eq_magneto;
  for (int64_t i = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; i < nrows;
       i += int64_t(gridDim.x) * blockDim.x) {
    if (orig[i] >= n_ts) continue;
    double h = cols[es_h * ld + i], c = cols[es_c * ld + i], d = cols[es_den * ld + i];
    v[0] = fmin(v[0], h);
    v[1] = fmax(v[1], c);
    v[2] = fmin(v[2], d);
    v[3] = fmin(v[3], c);
    double ka = 0.0;
    if (need_ka) {
      ka = cols[es_kappa * ld + i];
      v[4] = fmax(v[4], ka);
      v[6] = fmin(v[6], ka);
    }
    if (need_b)
      v[5] = fmax(v[5], fmax(fmax(cols[es_bx * ld + i], cols[es_by * ld + i]), cols[es_bz * ld + i]));
    if (P.eq_fld) {
      double n0 = cols[es_dtdx * ld + i], n1 = cols[es_dtdy * ld + i], n2 = cols[es_dtdz * ld + i];
      double ta = cols[es_t * ld + i];
      double gr = sqrt(((0.0 + n0 * n0) + n1 * n1) + n2 * n2);
      double fr = gr / (ka * d * d * ta);
      v[7] = fmax(v[7], (2. + fr) / (6. + 3 * fr + fr * fr));
    }
  }
  block_minmax<8>(v, is_max);
  if (threadIdx.x == 0) {
    red_min(&red[RED_TS_HMIN], v[0]);
    red_max(&red[RED_TS_CMAX], v[1]);
    red_min(&red[RED_TS_DENMIN], v[2]);
    red_min(&red[RED_TS_CMIN], v[3]);
    red_max(&red[RED_TS_KAPMAX], v[4]);
    red_max(&red[RED_TS_BMAX], v[5]);
    red_min(&red[RED_TS_KAPMIN], v[6]);
    red_max(&red[RED_TS_LAMMAX], v[7]);
  }
}

// ---- radiation - gas energy exchange (rad_exchange.f90:9-118) ---------------------------------
// Per integrated row: the gas energy u and the radiation energy xi = T
// exchange at fixed total e = u + xi; the new u solves, by at most 10 Newton
// steps from u0 until two iterates agree to 1e-16,
//   u/dt - u0/dt - du - 4 sigma kappa (rho (e - u) / a - (u cv1)^4) = 0,
// a = 4 sigma / c, cv1 = (gamma - 1) mu / Rg (rad_exchange.f90:111-126).
// Integer powers as repeated products, no fused multiply-adds.
__global__ void k_radexch(double* __restrict__ cols, int64_t ld, const int32_t* __restrict__ orig,
                          int64_t nrows, int64_t n_int, double dt, double gamma, double gmw,
                          int* __restrict__ status) {
  const int64_t i = blockIdx.x * int64_t(blockDim.x) + threadIdx.x;
  if (i >= nrows || orig[i] >= n_int) return;
  auto C = [&](int f) -> double& { return cols[f * ld + i]; };
  const double a = __ddiv_rn(__dmul_rn(4., kSigmaB), kLightspeed);
  const double cv1 = __ddiv_rn(__dmul_rn(gamma - 1., gmw), kRg);
  const double ack = __dmul_rn(__dmul_rn(4., kSigmaB), C(es_kappa));
  const double rho = C(es_den), u0 = C(es_u), dudt = C(es_du), xi = C(es_t);
  const double etot = __dadd_rn(u0, xi);
  double unew = u0, uold = __dmul_rn(2., u0);
  for (int iter = 0; fabs(__dadd_rn(unew, -uold)) > 1e-16 && iter < 10; ++iter) {
    uold = unew;
    const double uc = __dmul_rn(unew, cv1);
    const double uc2 = __dmul_rn(uc, uc);
    const double u3 = __dmul_rn(__dmul_rn(unew, unew), unew);
    const double cv2 = __dmul_rn(cv1, cv1);
    const double fu = __dadd_rn(
        __dadd_rn(__dadd_rn(__ddiv_rn(unew, dt), -__ddiv_rn(u0, dt)), -dudt),
        -__dmul_rn(ack, __dadd_rn(__ddiv_rn(__dmul_rn(rho, __dadd_rn(etot, -unew)), a),
                                  -__dmul_rn(uc2, uc2))));
    const double dfu = __dadd_rn(
        __ddiv_rn(1., dt),
        __dmul_rn(ack, __dadd_rn(__ddiv_rn(rho, a), __dmul_rn(4., __dmul_rn(u3, __dmul_rn(cv2, cv2))))));
    unew = __dadd_rn(unew, -__ddiv_rn(fu, dfu));
  }
  C(es_u) = unew;
  C(es_t) = __dadd_rn(etot, -unew);
  if (!(C(es_t) > 0.) || !(C(es_u) > 0.)) atomicCAS(status, 0, SPH_ERR_RAD_NEGATIVE);
}

// ---- device-resident step: the host's per-step arithmetic on the device ------------------
// k_plan repeats the host code between the image count and the sort (grid
// edge krad h_min f widened by 1.25 until the cell count fits, the FP32
// binade of the extent), with the same FP64 operations in the same order
// and no contraction, so a step planned here equals the host-planned one.
__global__ void k_plan(const unsigned long long* __restrict__ red,
                       const int32_t* __restrict__ nghost_dev, PlanIn in,
                       DevPlan* __restrict__ plan, int* __restrict__ err_out) {
  if (blockIdx.x != 0 || threadIdx.x != 0) return;
  DevPlan P{};
  P.err = 0;
  int64_t ng = nghost_dev[0];
  if (ng > in.nghost_cap || in.nrows + ng > in.nall_cap) {
    P.err = SPH_ERR_STATE;  // more images than room: redo on the host path
    ng = min(ng, in.nghost_cap);
    if (in.nrows + ng > in.nall_cap) ng = in.nall_cap - in.nrows;
  }
  P.nghost = ng;
  P.nall = in.nrows + ng;
  P.pad_key = in.end_bit_cap >= 32 ? 0xffffffffu : ((1u << in.end_bit_cap) - 1u);
  double lo[3], hi[3];
  for (int k = 0; k < 3; ++k) {
    lo[k] = dkey_inv(red[RED_LO_X + k]);
    hi[k] = dkey_inv(red[RED_HI_X + k]);
  }
  const double hmin = dkey_inv(red[RED_HMIN]);
  bool ok_in = true;
  if (!(hmin > 0) || !isfinite(hmin)) { P.err = P.err ? P.err : SPH_ERR_IC_H; ok_in = false; }
  for (int k = 0; k < 3; ++k)
    if (!isfinite(lo[k]) || !isfinite(hi[k])) { P.err = P.err ? P.err : SPH_ERR_Q_NAN; ok_in = false; }
  double L = __dmul_rn(__dmul_rn(in.krad, hmin), in.cf);
  const int64_t ncap = min(max(int64_t(8) * P.nall, int64_t(1) << 20), int64_t(1) << 31);
  int n3[3] = {1, 1, 1};
  int64_t ncell = 1;
  bool fits = ok_in;
  for (int guard = 0; fits; ++guard) {
    double e[3];
    for (int k = 0; k < 3; ++k) e[k] = __ddiv_rn(__dadd_rn(hi[k], -lo[k]), L);
    if (grid_dims(e, ncap, n3, &ncell)) break;
    L = __dmul_rn(L, 1.25);
    if (guard > 400) { fits = false; P.err = P.err ? P.err : SPH_ERR_GRID; }
  }
  if (!fits) {  // an error: a one-cell grid keeps every later launch in bounds
    n3[0] = n3[1] = n3[2] = 1;
    ncell = 1;
    L = 1.0;
    for (int k = 0; k < 3; ++k) lo[k] = hi[k] = 0.0;
  }
  P.ncell = ncell;
  P.grid.ox = lo[0]; P.grid.oy = lo[1]; P.grid.oz = lo[2];
  P.grid.L = L;
  P.grid.invL = __ddiv_rn(1.0, L);
  P.grid.nx = n3[0]; P.grid.ny = n3[1]; P.grid.nz = n3[2];
  const double e0 = __dadd_rn(hi[0], -lo[0]), e1 = __dadd_rn(hi[1], -lo[1]),
               e2 = __dadd_rn(hi[2], -lo[2]);
  const double ext = e0 < (e2 > e1 ? e2 : e1) ? (e2 > e1 ? e2 : e1) : e0;
  double sh = 1.0;
  if (ext > 0) {
    const double lim = __dmul_rn(ext, 1.0001);
    while (sh < lim) sh = __dmul_rn(sh, 2.0);
    while (__dmul_rn(sh, 0.5) >= lim) sh = __dmul_rn(sh, 0.5);
  }
  P.pg.ox = lo[0]; P.pg.oy = lo[1]; P.pg.oz = lo[2];
  P.pg.shift = sh;
  P.pg.mref = in.mref;
  *plan = P;
  if (P.err) atomicCAS(err_out, 0, P.err);
}
__global__ void k_flag_if_nonzero(const unsigned long long* __restrict__ v, int* __restrict__ err,
                                  int code) {
  if (blockIdx.x == 0 && threadIdx.x == 0 && *v != 0ull) atomicCAS(err, 0, code);
}

// dt of timestep.f90:40-166 and the clipping to tfinish / the next output
// time of main.f90:241-320, as the host does them (same operations, no
// contraction); writes dt to ctrl[0] for the predictor and corrector.
__device__ __forceinline__ double dmin_host(double a, double b) { return b < a ? b : a; }
__global__ void k_dt(const unsigned long long* __restrict__ red, DtIn in,
                     DevClock* __restrict__ clk, double* __restrict__ ctrl) {
  if (blockIdx.x != 0 || threadIdx.x != 0) return;
  const double hmin = dkey_inv(red[RED_TS_HMIN]), cmax = dkey_inv(red[RED_TS_CMAX]);
  const double denmin = dkey_inv(red[RED_TS_DENMIN]), cmin = dkey_inv(red[RED_TS_CMIN]);
  const double kapmax = dkey_inv(red[RED_TS_KAPMAX]), bmax = dkey_inv(red[RED_TS_BMAX]);
  const double kapmin = dkey_inv(red[RED_TS_KAPMIN]), lammax = dkey_inv(red[RED_TS_LAMMAX]);
  double dt = 1.7976931348623157e308;
  double dtdiff = __longlong_as_double(0x7ff0000000000000LL), dtfld = dtdiff;
  if (in.eq_hydro) dt = dmin_host(dt, __ddiv_rn(__dmul_rn(in.cn_hydro, hmin), cmax));
  if (in.eq_magneto)
    dt = dmin_host(dt, __ddiv_rn(__ddiv_rn(__dmul_rn(.1, hmin), cmax), bmax));
  if (in.eq_diff) {
    dtdiff = __ddiv_rn(__dmul_rn(__dmul_rn(__dmul_rn(in.cnd2, denmin), cmin), __dmul_rn(hmin, hmin)),
                       kapmax);
    dt = dmin_host(dt, dtdiff);
  }
  if (in.eq_fld) {
    dtfld = __ddiv_rn(__ddiv_rn(__dmul_rn(__dmul_rn(__dmul_rn(__dmul_rn(in.cnd2, hmin), hmin),
                                                    denmin), kapmin), kLightspeed), lammax);
    dt = dmin_host(dt, dtfld);
  }
  if (in.sts_fixed) {
    const double sts_dt_min = dmin_host(dtdiff, dtfld);
    dt = __dmul_rn(__dmul_rn(double(in.sts_s * in.sts_s + in.sts_s) - 2., 0.25), sts_dt_min);
  }
  DevClock c = *clk;
  const double t = c.t;
  if (__dadd_rn(t, dt) > c.tfinish) { dt = __dadd_rn(c.tfinish, -t); c.stopped = 1; }
  if (c.dtout > 0) {
    if (t >= c.ltout) { while (c.ltout <= t) c.ltout = __dadd_rn(c.ltout, c.dtout); }
    if (__dadd_rn(t, dt) > c.ltout) {
      if (c.dtout < dt) c.ltout = __dadd_rn(__dadd_rn(c.ltout, -c.dtout), dt);
      else dt = __dadd_rn(c.ltout, -t);
    }
  }
  c.dt = dt;
  *clk = c;
  ctrl[0] = dt;
}
__global__ void k_clock_advance(DevClock* __restrict__ clk) {
  if (blockIdx.x == 0 && threadIdx.x == 0) clk->t = __dadd_rn(clk->t, clk->dt);
}

// ---- selected columns in caller row order (the split step's exchanges) -------------
// out[k * nrows + orig[p]] = column fs.f[k] of physical row p, and back
__global__ void k_get_columns(const double* __restrict__ cols, int64_t ld,
                              const int32_t* __restrict__ orig, int64_t nrows, ColumnSet fs,
                              double* __restrict__ out) {
  const int64_t p = blockIdx.x * int64_t(blockDim.x) + threadIdx.x;
  if (p >= nrows) return;
  const int64_t o = orig[p];
  for (int k = 0; k < fs.n; ++k) out[k * nrows + o] = cols[fs.f[k] * ld + p];
}
__global__ void k_set_columns(double* __restrict__ cols, int64_t ld,
                              const int32_t* __restrict__ orig, int64_t nrows, ColumnSet fs,
                              const double* __restrict__ in) {
  const int64_t p = blockIdx.x * int64_t(blockDim.x) + threadIdx.x;
  if (p >= nrows) return;
  const int64_t o = orig[p];
  for (int k = 0; k < fs.n; ++k) cols[fs.f[k] * ld + p] = in[k * nrows + o];
}

// ---- the device loop of a batch ----------------------------------------------------
// the time loop's condition of main.f90:241 as the host evaluates it
// (t < tfinish + epsilon(1d0) and not stopped)
__device__ __forceinline__ bool inst_runs(const BatchInst& b) {
  const DevClock& c = *b.clk;
  return !b.failed && b.steps < b.limit &&
         c.t < __dadd_rn(c.tfinish, 2.220446049250313080847e-16) && !c.stopped;
}
__global__ void k_batch_gate(BatchInst* __restrict__ bi, int n,
                             const cudaGraphConditionalHandle* __restrict__ ifh) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const int r = inst_runs(bi[i]) ? 1 : 0;
  bi[i].running = r;
  cudaGraphSetConditional(ifh[i], r);
}
__global__ void k_batch_ctl(const BatchInst* __restrict__ bi, int n, cudaGraphConditionalHandle wh,
                            int* __restrict__ iter, int cap) {
  if (blockIdx.x != 0 || threadIdx.x != 0) return;
  bool any = false, failed = false;
  for (int i = 0; i < n; ++i) {
    failed |= bi[i].failed != 0;
    any |= inst_runs(bi[i]);
  }
  const int it = *iter + 1;
  *iter = it;
  // the cap bounds every launch of the loop, whatever the clocks say
  cudaGraphSetConditional(wh, (any && !failed && it < cap) ? 1u : 0u);
}
__global__ void k_inst_begin(BatchInst* __restrict__ b, const DevClock* __restrict__ clk,
                             DevClock* __restrict__ clk_save) {
  if (blockIdx.x != 0 || threadIdx.x != 0) return;
  *clk_save = *clk;
  b->since_before = b->since;
  b->reorder = (b->every > 0 && b->since >= b->every) ? 1 : 0;
  if (b->reorder) b->since = 0;
}
__global__ void k_inst_end(BatchInst* __restrict__ b, const int* __restrict__ err,
                           const int32_t* __restrict__ overflow, const int* __restrict__ status) {
  if (blockIdx.x != 0 || threadIdx.x != 0) return;
  if (*err || *overflow || *status) {
    b->failed = 1;
  } else {
    b->steps += 1;
    b->since += 1;
  }
}
__global__ void k_reorder_gather_gated(const BatchInst* __restrict__ b,
                                       const double* __restrict__ cin, double* __restrict__ cout,
                                       const int32_t* __restrict__ oin, int32_t* __restrict__ oout,
                                       const int32_t* __restrict__ centre_p, int64_t nreal,
                                       int64_t n) {
  if (!b->reorder) return;
  const int64_t i = blockIdx.x * int64_t(blockDim.x) + threadIdx.x;
  if (i >= n) return;
  const int64_t src = i < nreal ? int64_t(centre_p[i]) : i;
  for (int f = 0; f < NCOL; ++f) cout[f * n + i] = cin[f * n + src];
  oout[i] = oin[src];
}
__global__ void k_reorder_back_gated(const BatchInst* __restrict__ b, const double* __restrict__ cin,
                                     double* __restrict__ cout, const int32_t* __restrict__ oin,
                                     int32_t* __restrict__ oout, int64_t n, DevSkin* ds) {
  if (!b->reorder) return;
  const int64_t i = blockIdx.x * int64_t(blockDim.x) + threadIdx.x;
  if (ds && i == 0) ds->live = 0;  // the lists name records by the old rows
  if (i >= n) return;
  for (int f = 0; f < NCOL; ++f) cout[f * n + i] = cin[f * n + i];
  oout[i] = oin[i];
}

__global__ void k_fill_i32(int32_t* p, int64_t n, int32_t v) {
  int64_t i = blockIdx.x * int64_t(blockDim.x) + threadIdx.x;
  if (i < n) p[i] = v;
}

__global__ void k_fill_u64(unsigned long long* p, int n, unsigned long long v) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) p[i] = v;
}

// ---- STS stage updates (sts_integrator.f90:100-123) ------------------------------------------
// Y holds six columns of length ld: Y0, Yjm1, Yjm2, Yj, DY0, DYjm1.
enum { Y0 = 0, YJM1, YJM2, YJ, DY0, DYJM1 };
__global__ void k_sts(int kind, double* __restrict__ cols, int64_t ld, int64_t n,
                      double* __restrict__ Y, double a0, double a1, double a2, double a3,
                      double a4, const double* __restrict__ ctrl,
                      const double* __restrict__ coef = nullptr, const int* __restrict__ jdev = nullptr) {
  int64_t i = blockIdx.x * int64_t(blockDim.x) + threadIdx.x;
  if (i >= n) return;
  if (coef) {  // stage j of the device-resident loop
    const double* c = coef + 4 * (*jdev - 2);
    a0 = c[0]; a1 = c[1]; a2 = c[2]; a3 = c[3];
  }
  auto y = [&](int s) -> double& { return Y[s * ld + i]; };
  double* T = cols + es_t * ld;
  const double* ddt = cols + es_ddt * ld;
  const double dt = ctrl[0];
  switch (kind) {
    case 0:  // Y0 = T
      y(Y0) = T[i];
      break;
    case 1:  // after the first iterate: DY0, Yjm2 = Y0, Yjm1 = Y0 + muhat1*dt*DY0
      y(DY0) = ddt[i];
      y(YJM2) = y(Y0);
      y(YJM1) = __dadd_rn(y(Y0), __dmul_rn(__dmul_rn(a0, dt), y(DY0)));
      y(YJ) = y(YJM1);
      T[i] = y(YJM1);
      break;
    case 2: {  // stage j: a0 = mu, a1 = nu, a2 = muhat, a3 = gmhat
      y(DYJM1) = ddt[i];
      double v = __dadd_rn(__dmul_rn(a0, y(YJM1)), __dmul_rn(a1, y(YJM2)));
      v = __dadd_rn(v, __dmul_rn(__dadd_rn(__dadd_rn(1.0, -a0), -a1), y(Y0)));
      v = __dadd_rn(v, __dmul_rn(__dmul_rn(a2, dt), y(DYJM1)));
      v = __dadd_rn(v, __dmul_rn(__dmul_rn(a3, dt), y(DY0)));
      y(YJ) = v;
      y(YJM2) = y(YJM1);
      y(YJM1) = v;
      T[i] = v;
      break;
    }
    case 3:  // final: T = Yj
      T[i] = y(YJ);
      break;
    default:
      break;
  }
}

// ---- EOS (eos.f90:21-45), only for a separate call; circuit1 fuses it ------------------------
__global__ void k_eos(double* __restrict__ cols, int64_t ld, int64_t nreal, Params P) {
  int64_t i = blockIdx.x * int64_t(blockDim.x) + threadIdx.x;
  if (i >= nreal) return;
  double rho = cols[es_den * ld + i];
  if (P.eos_kind == 1) {
    double p = (P.gamma - 1.) * rho * cols[es_u * ld + i];
    cols[es_p * ld + i] = p;
    cols[es_c * ld + i] = sqrt(P.gamma * p / rho);
  } else if (P.eos_kind == 2) {
    cols[es_p * ld + i] = rho * P.c_iso * P.c_iso;
  }
}

// iterator.f90:143, :153-163 — the MTI set-ups add a gravity term after c2
__global__ void k_mti(double* __restrict__ cols, int64_t ld, const int32_t* __restrict__ orig,
                      int64_t nrows, int64_t nreal, int lowres) {
  int64_t i = blockIdx.x * int64_t(blockDim.x) + threadIdx.x;
  if (i >= nrows || orig[i] >= nreal) return;
  double ay = cols[es_ay * ld + i];
  if (lowres) ay = ay - erf(cols[es_ry * ld + i] * 8.);
  else ay = ay - 1.;
  cols[es_ay * ld + i] = ay;
}

__global__ void k_set(double* col, int64_t n, double v) {
  int64_t i = blockIdx.x * int64_t(blockDim.x) + threadIdx.x;
  if (i < n) col[i] = v;
}

}  // namespace

// ---- launchers ------------------------------------------------------------------------------
void launch_upload_store(const double* rm, double* cols, int32_t* orig, int64_t n, cudaStream_t s) {
  if (n <= 0) return;
  k_upload<<<unsigned((n + 31) / 32), dim3(32, 8), 0, s>>>(rm, cols, orig, n, 0, n);
  note_launch();
}
void launch_upload_rows(const double* rm, double* cols, int32_t* orig, int64_t n, int64_t a,
                        int64_t b, cudaStream_t s) {
  if (b <= a) return;
  k_upload<<<unsigned((b - a + 31) / 32), dim3(32, 8), 0, s>>>(rm, cols, orig, n, a, b);
  note_launch();
}
void launch_download_rows(const double* cols, const int32_t* inv, double* rm, int64_t n, int64_t a,
                          int64_t b, cudaStream_t s) {
  if (b <= a) return;
  k_download_gather<<<unsigned((b - a + 31) / 32), dim3(32, 8), 0, s>>>(cols, inv, rm, n, a, b);
  note_launch();
}
void launch_download_store(const double* cols, const int32_t* orig, double* rm, int64_t n,
                           cudaStream_t s) {
  if (n <= 0) return;
  k_download<<<unsigned((n + 31) / 32), dim3(32, 8), 0, s>>>(cols, orig, rm, n);
  note_launch();
}
void launch_reorder(const double* cin, double* cout, const int32_t* oin, int32_t* oout,
                    const int32_t* perm, int64_t n, int64_t ldi, int64_t ldo, cudaStream_t s) {
  k_reorder<<<nblocks(n), TPB, 0, s>>>(cin, cout, oin, oout, perm, n, ldi, ldo);
  note_launch();
}
void launch_reflect(double* cols, int64_t ld, int64_t nreal, BoxGeom g, cudaStream_t s) {
  if (nreal > 0) {
    k_reflect<<<nblocks(nreal), TPB, 0, s>>>(cols, ld, nreal, g);
    note_launch();
  }
}
void launch_ghost_count(const double* cols, int64_t nrows, int64_t nreal, BoxGeom g, int dim,
                        int32_t* count, unsigned long long* red, cudaStream_t s) {
  k_ghost_count<<<reduce_blocks(nrows), TPB, 0, s>>>(cols, nrows, nrows, nreal, g, dim, count,
                                                     red);
  note_launch();
}
void launch_ghost_write(const double* cols, int64_t nrows, BoxGeom g, int dim,
                        const int32_t* offset, double* gx, double* gy, double* gz,
                        int32_t* gsrc, int8_t* gcode, unsigned long long*, cudaStream_t s) {
  k_ghost_write<<<nblocks(nrows), TPB, 0, s>>>(cols, nrows, nrows, g, dim, offset, INT64_MAX, gx,
                                               gy, gz, gsrc, gcode);
  note_launch();
}
void launch_ghost_write_cap(const double* cols, int64_t nrows, BoxGeom g, int dim,
                            const int32_t* offset, int64_t cap, double* gx, double* gy,
                            double* gz, int32_t* gsrc, int8_t* gcode, cudaStream_t s) {
  k_ghost_write<<<nblocks(nrows), TPB, 0, s>>>(cols, nrows, nrows, g, dim, offset, cap, gx, gy, gz,
                                               gsrc, gcode);
  note_launch();
}
void launch_keys(const double* cols, int64_t nrows, const double* gx, const double* gy,
                 const double* gz, int64_t nghost, Grid g, uint32_t* keys, int32_t* vals,
                 cudaStream_t s) {
  k_keys<<<nblocks(nrows + nghost), TPB, 0, s>>>(cols, nrows, nrows, gx, gy, gz, nghost, g,
                                                 keys, vals, nullptr, 0);
  note_launch();
}
void launch_keys_dev(const double* cols, int64_t nrows, const double* gx, const double* gy,
                     const double* gz, const DevPlan* plan, int64_t ncap, uint32_t* keys,
                     int32_t* vals, cudaStream_t s) {
  k_keys<<<nblocks(ncap), TPB, 0, s>>>(cols, nrows, nrows, gx, gy, gz, 0, Grid{}, keys, vals, plan,
                                       ncap);
  note_launch();
}
void launch_cell_starts(const uint32_t* keys, int64_t n, int64_t ncell, int32_t* cstart,
                        cudaStream_t s) {
  k_cell_starts<<<nblocks(n + 1), TPB, 0, s>>>(keys, n, ncell, cstart, nullptr);
  note_launch();
}
void launch_cell_starts_dev(const uint32_t* keys, int64_t ncap, const DevPlan* plan,
                            int32_t* cstart, cudaStream_t s) {
  k_cell_starts<<<nblocks(ncap + 1), TPB, 0, s>>>(keys, ncap, 0, cstart, plan);
  note_launch();
}
void launch_sorted_gather(const int32_t* sidx, int64_t n, int64_t nrows, int64_t nreal,
                          const double* cols, const double* gx, const double* gy,
                          const double* gz, const int32_t* gsrc, double* sx, double* sy,
                          double* sz, int32_t* ssrc, int32_t* centre_slot, float4* s32,
                          PackGeom pg, cudaStream_t s) {
  k_sorted_gather<<<nblocks(n), TPB, 0, s>>>(sidx, n, nrows, nreal, cols, nrows, gx, gy, gz,
                                             gsrc, sx, sy, sz, ssrc, centre_slot, s32, pg,
                                             nullptr, 0);
  note_launch();
}
void launch_sorted_gather_dev(const int32_t* sidx, int64_t ncap, int64_t nrows, int64_t nreal,
                              const double* cols, const double* gx, const double* gy,
                              const double* gz, const int32_t* gsrc, double* sx, double* sy,
                              double* sz, int32_t* ssrc, int32_t* centre_slot, float4* s32,
                              const DevPlan* plan, cudaStream_t s) {
  k_sorted_gather<<<nblocks(ncap + 1), TPB, 0, s>>>(sidx, ncap, nrows, nreal, cols, nrows, gx, gy,
                                                    gz, gsrc, sx, sy, sz, ssrc, centre_slot, s32,
                                                    PackGeom{}, plan, ncap);
  note_launch();
}
void launch_centres(const int32_t* sidx, const int32_t* flag, const int32_t* pos, int64_t n,
                    int32_t* centre_k, int32_t* centre_p, cudaStream_t s) {
  k_centres<<<nblocks(n), TPB, 0, s>>>(sidx, flag, pos, n, centre_k, centre_p);
  note_launch();
}
void launch_neib_digest(int64_t nc, const int32_t* centre_p, const int32_t* orig,
                        const int64_t* rowoff, const int32_t* ncnt, const int32_t* nl,
                        const int32_t* sidx, const int32_t* ssrc, const int8_t* gcode,
                        int64_t nrows, unsigned long long* out, cudaStream_t s) {
  if (nc <= 0) return;
  k_neib_digest<<<nblocks(nc * 32), TPB, 0, s>>>(nc, centre_p, orig, rowoff, ncnt, nl, sidx,
                                                  ssrc, gcode, nrows, out);
  note_launch();
}
template <int DIM, int G>
static void neighbours_g(bool staged, const NeibArgs& a, cudaStream_t s) {
  const int tpb = 128;
  // (4-lane groups keep the fetch: 32 stages would not fit 48 KB)
  if (staged && G >= 8) k_neighbours<DIM, G, (G >= 8)><<<nblocks(a.nc, tpb), tpb, 0, s>>>(a);
  else k_neighbours<DIM, G, false><<<nblocks(a.nc, tpb), tpb, 0, s>>>(a);
}
template <int DIM>
static void neighbours_dim(int G, bool staged, const NeibArgs& a, cudaStream_t s) {
  switch (G) {
    case 4: neighbours_g<DIM, 4>(staged, a, s); break;
    case 8: neighbours_g<DIM, 8>(staged, a, s); break;
    case 16: neighbours_g<DIM, 16>(staged, a, s); break;
    default: neighbours_g<DIM, 32>(staged, a, s); break;
  }
}
void launch_neighbours(int dim, int G, bool staged, const NeibArgs& a, cudaStream_t s) {
  if (dim == 3) neighbours_dim<3>(G, staged, a, s);
  else if (dim == 2) neighbours_dim<2>(G, staged, a, s);
  else neighbours_dim<1>(G, staged, a, s);
  note_launch();
}
void launch_rowcap(int64_t nc, const int32_t* centre_p, const int32_t* orig,
                   const int32_t* count_prev, const float* h_prev, const double* hcol,
                   int dim, float slack, int64_t* rowcap64, int32_t* rowcap,
                   cudaStream_t s) {
  k_rowcap<<<nblocks(nc), TPB, 0, s>>>(nc, centre_p, orig, count_prev, h_prev, hcol, dim, slack,
                                       rowcap64, rowcap);
  note_launch();
}
void launch_skin_sig(const double* cols, int64_t nrows, BoxGeom g, int dim, uint8_t* sig,
                     cudaStream_t s) {
  if (nrows <= 0) return;
  k_skin_sig<<<nblocks(nrows), TPB, 0, s>>>(cols, nrows, nrows, g, dim, sig);
  note_launch();
}
void launch_skin_refresh(const int32_t* sidx, int64_t n, int64_t nrows, int64_t nreal,
                         const double* cols, const int32_t* gsrc, const int8_t* gcode,
                         BoxGeom g, int dim, const uint8_t* sig_b, const double* bx,
                         const double* by, const double* bz, double* sx, double* sy, double* sz,
                         float4* s32, PackGeom pg, float* dsp, float tau, float eps,
                         double* hrec, unsigned long long* red, cudaStream_t s,
                         const DevPlan* plan, const DevSkin* gate) {
  if (n <= 0) return;
  k_skin_refresh<<<reduce_blocks(n), TPB, 0, s>>>(sidx, n, nrows, nreal, cols, nrows, gsrc, gcode,
                                                  g, dim, sig_b, bx, by, bz, sx, sy, sz, s32, pg,
                                                  dsp, tau, eps, hrec, red, plan, gate);
  note_launch();
}

// ---- skin lists of the device-resident step ---------------------------------------------
__global__ void k_dskin_check(int64_t nc, const int32_t* __restrict__ centre_p,
                              const double* __restrict__ hcol, const double* __restrict__ hb,
                              double krad, const DevSkin* __restrict__ ds,
                              unsigned long long* __restrict__ red) {
  if (!ds->live) return;
  const double D = dkey_inv(red[RED_SKIN_D]);
  const double kfb = ds->kfac_b;
  bool bad = false;
  for (int64_t c = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; c < nc;
       c += int64_t(gridDim.x) * blockDim.x) {
    // relative margins far above the rounding of both sides and of the
    // search's own radius kfac (krad h)
    const double need = (krad * hcol[centre_p[c]] + 2.0 * D) * (1.0 + 1e-12);
    const double have = kfb * (krad * hb[c]) * (1.0 - 1e-12);
    bad |= !(need <= have);
  }
  if (__any_sync(0xffffffffu, bad) && (threadIdx.x & 31) == 0) atomicMax(&red[RED_DSKIN_FAIL], 1ull);
}
__global__ void k_dskin_decide(DevSkin* __restrict__ ds, const unsigned long long* __restrict__ red,
                               const DevPlan* __restrict__ plan, double krad, double skin,
                               int short_age, int pause0, int pause_max,
                               cudaGraphConditionalHandle hsearch,
                               unsigned long long* __restrict__ dcnt) {
  if (blockIdx.x != 0 || threadIdx.x != 0) return;
  DevSkin d = *ds;
  bool ok = d.live != 0;
  if (ok) {
    const double D = dkey_inv(red[RED_SKIN_D]), hmax = dkey_inv(red[RED_SKIN_HMAX]);
    ok = red[RED_SKIN_SIG] == 0ull && red[RED_DSKIN_FAIL] == 0ull && D <= krad * d.hmin_b &&
         hmax > 0.0 && isfinite(hmax);
    // every record inside the FP32 packing's binade: 0 <= x - origin < shift
    const double o[3] = {plan->pg.ox, plan->pg.oy, plan->pg.oz};
    for (int k = 0; k < 3; ++k) {
      const double lo = dkey_inv(red[RED_LO_X + k]), hi = dkey_inv(red[RED_HI_X + k]);
      ok = ok && lo >= o[k] && hi - o[k] < plan->pg.shift * (1.0 - 1e-9);
    }
  }
  if (ok) {
    ++d.age;
    ++dcnt[DC_SKIN_REUSES];
  } else {
    if (d.live) {  // the lists ended: short-lived ones start a pause of plain searches
      if (d.age < short_age) {
        d.pause_len = d.pause_len ? min(2 * d.pause_len, pause_max) : pause0;
        d.pause = d.pause_len;
      } else {
        d.pause_len = 0;
      }
    }
    if (d.pause > 0) {
      --d.pause;
      d.kfac = 1.0;
    } else {
      d.kfac = 1.0 + skin;
      ++dcnt[DC_SKIN_BUILDS];
    }
    d.live = 0;
    ++dcnt[DC_SEARCHES];
  }
  *ds = d;
  cudaGraphSetConditional(hsearch, ok ? 0u : 1u);
}
__global__ void k_dskin_built(DevSkin* __restrict__ ds, const unsigned long long* __restrict__ red) {
  if (blockIdx.x != 0 || threadIdx.x != 0) return;
  ds->live = ds->kfac > 1.0 ? 1 : 0;
  ds->age = 0;
  ds->kfac_b = ds->kfac;
  ds->hmin_b = dkey_inv(red[RED_HMIN]);
}
void launch_dskin_check(int64_t nc, const int32_t* centre_p, const double* hcol, const double* hb,
                        double krad, const DevSkin* ds, unsigned long long* red, cudaStream_t s) {
  if (nc <= 0) return;
  k_dskin_check<<<reduce_blocks(nc), TPB, 0, s>>>(nc, centre_p, hcol, hb, krad, ds, red);
  note_launch();
}
void launch_dskin_decide(DevSkin* ds, const unsigned long long* red, const DevPlan* plan,
                         double krad, double skin, int short_age, int pause0, int pause_max,
                         cudaGraphConditionalHandle hsearch, unsigned long long* dcnt,
                         cudaStream_t s) {
  k_dskin_decide<<<1, 32, 0, s>>>(ds, red, plan, krad, skin, short_age, pause0, pause_max, hsearch,
                                  dcnt);
  note_launch();
}
void launch_dskin_built(DevSkin* ds, const unsigned long long* red, cudaStream_t s) {
  k_dskin_built<<<1, 32, 0, s>>>(ds, red);
  note_launch();
}
void launch_skin_marks(int64_t n, const float* dsp, float tau, float eps, const uint32_t* keys,
                       const double* sx, const double* sy, const double* sz, Grid g, int dim,
                       const int* w, uint8_t* fast_cell, uint8_t* move_cell, uint8_t* tmp,
                       cudaStream_t s) {
  const int64_t ncell = int64_t(g.nx) * g.ny * g.nz;
  if (n <= 0 || ncell <= 0) return;
  cudaMemsetAsync(fast_cell, 0, size_t(ncell), s);
  if (move_cell) cudaMemsetAsync(move_cell, 0, size_t(ncell), s);
  k_skin_cells<<<nblocks(n), TPB, 0, s>>>(n, dsp, tau, eps, keys, sx, sy, sz, g, fast_cell,
                                          move_cell);
  note_launch();
  // dilate in place through tmp: axis 0 into tmp, 1 back, 2 into tmp, copy back
  auto dilate = [&](uint8_t* f, const int* wp) {
    uint8_t* a = f;
    uint8_t* b = tmp;
    for (int axis = 0; axis < dim; ++axis) {
      cudaMemsetAsync(b, 0, size_t(ncell), s);
      k_dilate<<<nblocks(ncell), TPB, 0, s>>>(a, b, g, axis, wp);
      note_launch();
      std::swap(a, b);
    }
    if (a != f) cudaMemcpyAsync(f, a, size_t(ncell), cudaMemcpyDeviceToDevice, s);
  };
  dilate(fast_cell, w);
  if (move_cell) dilate(move_cell, w + 1);
}
__global__ void k_skin_gate(const unsigned long long* __restrict__ red, SkinGateIn in,
                            int* __restrict__ gate) {
  if (blockIdx.x != 0 || threadIdx.x != 0) return;
  const double D = dkey_inv(red[RED_SKIN_D]);
  const double hmax = dkey_inv(red[RED_SKIN_HMAX]);
  const double hmaxb = dkey_inv(red[RED_SKIN_HMAXB]);
  int why = 0;
  if (red[RED_SKIN_SIG]) why = 1;
  else if (!(D <= in.dcap)) why = 2;
  else if (!(hmax > 0) || !isfinite(hmax) || !(hmaxb > 0)) why = 3;
  if (!why) {
    // every record inside the FP32 packing's binade: 0 <= x - origin < shift
    const double o[3] = {in.pg.ox, in.pg.oy, in.pg.oz};
    for (int k = 0; k < 3; ++k) {
      const double lo = dkey_inv(red[RED_LO_X + k]), hi = dkey_inv(red[RED_HI_X + k]);
      if (!(lo >= o[k]) || !(hi - o[k] < in.pg.shift * (1.0 - 1e-9))) why = 4;
    }
  }
  int wf = 0, wm = 0;
  if (!why) {
    // around fast records every centre that may see them now (reach_f),
    // around moving ones every skin list holding them (reach_m)
    const double reach_f = (in.krad * hmax + in.tau) * (1.0 + 1e-9);
    const double reach_m = in.kfac * in.krad * hmaxb * (1.0 + 1e-9);
    const double ef = ceil(reach_f * in.invL) + 1.0, em = ceil(reach_m * in.invL) + 1.0;
    if (!(ef <= 256.0) || !(em <= 256.0)) why = 5;
    else { wf = int(ef); wm = int(em); }
  }
  gate[0] = why;
  gate[1] = wf;
  gate[2] = wm;
}
void launch_skin_gate(const unsigned long long* red, SkinGateIn in, int* gate, cudaStream_t s) {
  k_skin_gate<<<1, 32, 0, s>>>(red, in, gate);
  note_launch();
}
void launch_skin_classify(int64_t nc, const int32_t* centre_k, const double* hrec,
                          const double* hb, double* hdev, const float* gap, double krad,
                          double kfac, float tau, float eps, const float* dsp,
                          const uint32_t* keys, const uint8_t* near_f, const uint8_t* near_m,
                          uint8_t* mode, int64_t* ways, int64_t* pos, int32_t* dlist,
                          int32_t* flist, void* scan_tmp, size_t scan_bytes,
                          const int32_t* ncnt, unsigned long long* nkept, cudaStream_t s) {
  if (nc <= 0) return;
  k_skin_classify<<<nblocks(nc), TPB, 0, s>>>(nc, centre_k, hrec, hb, hdev, gap, krad, kfac, tau,
                                              eps, dsp, keys, near_f, near_m, mode, ways, ncnt,
                                              nkept);
  cudaMemsetAsync(ways + nc, 0, sizeof(int64_t), s);
  exclusive_scan64(scan_tmp, scan_bytes, ways, pos, nc + 1, s);
  k_skin_lists<<<nblocks(nc), TPB, 0, s>>>(nc, ways, pos, dlist, flist);
  note_launch(2);
}
void launch_inverse(const int32_t* p, int64_t n, int32_t* q, cudaStream_t s) {
  if (n <= 0) return;
  k_inv_perm<<<nblocks(n), TPB, 0, s>>>(p, n, q);
  note_launch();
}
void launch_type_changed(const double* cols, int64_t n, const double* old_type,
                         const int32_t* perm, int32_t* changed, cudaStream_t s) {
  if (n <= 0) return;
  k_type_changed<<<nblocks(n), TPB, 0, s>>>(cols, n, n, old_type, perm, changed);
  note_launch();
}
void launch_rows_renamed(const int32_t* perm, const int32_t* inv, int64_t nall, int64_t nrows,
                         int64_t nghost, int64_t nreal, int32_t* sidx, int32_t* ssrc,
                         int32_t* gsrc, int32_t* centre_p, const uint8_t* sig_in,
                         uint8_t* sig_out, cudaStream_t s) {
  if (nrows <= 0) return;
  k_rows_renamed<<<nblocks(nall), TPB, 0, s>>>(inv, perm, nall, nrows, nghost, nreal, sidx, ssrc,
                                               gsrc, centre_p, sig_in, sig_out);
  note_launch();
}
void launch_dyn_rows(int64_t nd, const int32_t* list, const int32_t* centre_p,
                     const int32_t* orig, const int32_t* count_prev, const float* h_prev,
                     const double* hcol, int dim, int64_t* cap, int64_t* off, void* scan_tmp,
                     size_t scan_bytes, const int64_t* base, int64_t* rowoff, int32_t* rowcap,
                     cudaStream_t s) {
  if (nd <= 0) return;
  k_dyn_caps<<<nblocks(nd + 1), TPB, 0, s>>>(nd, list, centre_p, orig, count_prev, h_prev, hcol,
                                             dim, 1.2f, cap);
  exclusive_scan64(scan_tmp, scan_bytes, cap, off, nd + 1, s);
  k_dyn_assign<<<nblocks(nd), TPB, 0, s>>>(nd, list, off, cap, base, rowoff, rowcap);
  note_launch(2);
}
void launch_table_end(const int64_t* rowoff, const int32_t* rowcap, int64_t n, int64_t* end,
                      cudaStream_t s) {
  k_table_end<<<1, 1, 0, s>>>(rowoff, rowcap, n, end);
  note_launch();
}
void launch_overflow_to_search(int64_t nc, const int32_t* ncnt, const int64_t* rowoff,
                               const int32_t* rowcap, int64_t nl_size, uint8_t* mode,
                               int32_t* dflag, cudaStream_t s) {
  if (nc <= 0) return;
  k_overflow_to_search<<<nblocks(nc), TPB, 0, s>>>(nc, ncnt, rowoff, rowcap, nl_size, mode, dflag);
  note_launch();
}
template <int DIM>
static void search_few_dim(const FewArgs& a, cudaStream_t s) {
  constexpr int G = 8;
  const int64_t need = (a.n * G + 127) / 128;
  const int grid = int(need < 148 * 8 ? need : 148 * 8);
  k_search_few<DIM, G><<<grid, 128, 0, s>>>(a);
}
void launch_search_few(int dim, const FewArgs& a, cudaStream_t s) {
  if (a.n <= 0) return;
  if (dim == 3) search_few_dim<3>(a, s);
  else if (dim == 2) search_few_dim<2>(a, s);
  else search_few_dim<1>(a, s);
  note_launch();
}
void launch_skin_compact(int64_t nc, const int32_t* dflag, const int32_t* dpos, int32_t* dlist,
                         cudaStream_t s) {
  if (nc <= 0) return;
  k_skin_compact<<<nblocks(nc), TPB, 0, s>>>(nc, dflag, dpos, dlist);
  note_launch();
}
void launch_gather_h(int64_t nc, const int32_t* centre_p, const double* hcol, double* hb,
                     unsigned long long* red, int slot, cudaStream_t s) {
  if (nc <= 0) return;
  k_gather_h<<<nblocks(nc), TPB, 0, s>>>(nc, centre_p, hcol, hb, red, slot);
  note_launch();
}
void launch_skin_filter(const SkinFilterArgs& a, cudaStream_t s) {
  constexpr int G = 8;
  if (a.nc <= 0) return;
  // 6 blocks of 128 threads fit an SM (76 registers a thread)
  const int64_t need = (a.nc * G + 127) / 128;
  const int grid = int(need < 148 * 6 ? need : 148 * 6);
  k_skin_filter<G><<<grid, 128, 0, s>>>(a);
  note_launch();
}
size_t scan64_temp_bytes(int64_t n) {
  size_t b = 0;
  cub::DeviceScan::ExclusiveSum(nullptr, b, (const int64_t*)nullptr, (int64_t*)nullptr, int(n));
  return b;
}
void exclusive_scan64(void* tmp, size_t tmp_bytes, const int64_t* in, int64_t* out, int64_t n,
                      cudaStream_t s) {
  cub::DeviceScan::ExclusiveSum(tmp, tmp_bytes, in, out, int(n), s);
}
void launch_pack(int prec, int groups, int64_t n, const int32_t* ssrc, const double* sx,
                 const double* sy, const double* sz, const double* cols, int64_t ld, PackGeom pg,
                 PackBufs pb, cudaStream_t s) {
  k_pack<<<nblocks(n), TPB, 0, s>>>(prec, groups, n, ssrc, sx, sy, sz, cols, ld, pg, pb, nullptr);
  note_launch();
}
void launch_pack_dev(int prec, int groups, int64_t ncap, const int32_t* ssrc, const double* sx,
                     const double* sy, const double* sz, const double* cols, int64_t ld,
                     const DevPlan* plan, PackBufs pb, cudaStream_t s) {
  k_pack<<<nblocks(ncap), TPB, 0, s>>>(prec, groups, ncap, ssrc, sx, sy, sz, cols, ld, PackGeom{},
                                       pb, plan);
  note_launch();
}
void launch_predict(double* cols, int64_t ld, const int32_t* orig, int64_t nrows, int64_t n_int,
                    double* save, const double* ctrl, int mode, cudaStream_t s) {
  k_predict<<<nblocks(nrows), TPB, 0, s>>>(cols, ld, orig, nrows, n_int, save, ctrl, mode);
  note_launch();
}
void launch_correct(double* cols, int64_t ld, const int32_t* orig, int64_t nrows, int64_t n_int,
                    const double* save, const double* ctrl, int mode, cudaStream_t s) {
  k_correct<<<nblocks(nrows), TPB, 0, s>>>(cols, ld, orig, nrows, n_int, save, ctrl, mode);
  note_launch();
}
void launch_timestep_reduce(const double* cols, int64_t ld, const int32_t* orig, int64_t nrows,
                            int64_t n_ts, Params P, unsigned long long* red, cudaStream_t s) {
  k_timestep_reduce<<<reduce_blocks(nrows), TPB, 0, s>>>(cols, ld, orig, nrows, n_ts, P, red);
  note_launch();
}
void launch_radexch(double* cols, int64_t ld, const int32_t* orig, int64_t nrows, int64_t n_int,
                    double dt, double gamma, double gmw, int* status, cudaStream_t s) {
  k_radexch<<<nblocks(nrows), TPB, 0, s>>>(cols, ld, orig, nrows, n_int, dt, gamma, gmw, status);
  note_launch();
}
void launch_plan(const unsigned long long* red, const int32_t* nghost_dev, PlanIn in,
                 DevPlan* plan, int* err_out, cudaStream_t s) {
  k_plan<<<1, 32, 0, s>>>(red, nghost_dev, in, plan, err_out);
  note_launch();
}
__global__ void k_sweeps_init(int* __restrict__ iter, cudaGraphConditionalHandle h) {
  if (blockIdx.x != 0 || threadIdx.x != 0) return;
  *iter = 0;
  cudaGraphSetConditional(h, 1u);
}
__global__ void k_sweeps_ctl(int* __restrict__ iter, const unsigned long long* __restrict__ active,
                             int sweeps, int maxiter, int* __restrict__ err,
                             cudaGraphConditionalHandle h) {
  if (blockIdx.x != 0 || threadIdx.x != 0) return;
  const int it = *iter + 1;
  *iter = it;
  const bool act = *active != 0ull;
  if (act && it >= sweeps && sweeps < maxiter) atomicCAS(err, 0, SPH_ERR_STATE);
  cudaGraphSetConditional(h, (act && it < sweeps) ? 1u : 0u);
}
void launch_sweeps_init(int* iter, cudaGraphConditionalHandle h, cudaStream_t s) {
  k_sweeps_init<<<1, 32, 0, s>>>(iter, h);
  note_launch();
}
void launch_sweeps_ctl(int* iter, const unsigned long long* active, int sweeps, int maxiter,
                       int* err, cudaGraphConditionalHandle h, cudaStream_t s) {
  k_sweeps_ctl<<<1, 32, 0, s>>>(iter, active, sweeps, maxiter, err, h);
  note_launch();
}
void launch_flag_if_nonzero(const unsigned long long* v, int* err, int code, cudaStream_t s) {
  k_flag_if_nonzero<<<1, 32, 0, s>>>(v, err, code);
  note_launch();
}
void launch_dt(const unsigned long long* red, DtIn in, DevClock* clk, double* ctrl, cudaStream_t s) {
  k_dt<<<1, 32, 0, s>>>(red, in, clk, ctrl);
  note_launch();
}
void launch_clock_advance(DevClock* clk, cudaStream_t s) {
  k_clock_advance<<<1, 32, 0, s>>>(clk);
  note_launch();
}
void launch_get_columns(const double* cols, int64_t ld, const int32_t* orig, int64_t nrows,
                        ColumnSet fs, double* out, cudaStream_t s) {
  k_get_columns<<<nblocks(nrows), TPB, 0, s>>>(cols, ld, orig, nrows, fs, out);
  note_launch();
}
void launch_set_columns(double* cols, int64_t ld, const int32_t* orig, int64_t nrows,
                        ColumnSet fs, const double* in, cudaStream_t s) {
  k_set_columns<<<nblocks(nrows), TPB, 0, s>>>(cols, ld, orig, nrows, fs, in);
  note_launch();
}
void launch_batch_gate(BatchInst* bi, int n, const cudaGraphConditionalHandle* ifh,
                       cudaStream_t s) {
  k_batch_gate<<<(n + 127) / 128, 128, 0, s>>>(bi, n, ifh);
  note_launch();
}
void launch_batch_ctl(const BatchInst* bi, int n, cudaGraphConditionalHandle wh, int* iter,
                      int cap, cudaStream_t s) {
  k_batch_ctl<<<1, 32, 0, s>>>(bi, n, wh, iter, cap);
  note_launch();
}
void launch_inst_begin(BatchInst* b, const DevClock* clk, DevClock* clk_save, cudaStream_t s) {
  k_inst_begin<<<1, 32, 0, s>>>(b, clk, clk_save);
  note_launch();
}
void launch_inst_end(BatchInst* b, const int* err, const int32_t* overflow, const int* status,
                     cudaStream_t s) {
  k_inst_end<<<1, 32, 0, s>>>(b, err, overflow, status);
  note_launch();
}
void launch_reorder_gated(const BatchInst* b, double* cols, double* cols_alt, int32_t* orig,
                          int32_t* orig_alt, const int32_t* centre_p, int64_t nreal,
                          int64_t nrows, DevSkin* ds, cudaStream_t s) {
  k_reorder_gather_gated<<<nblocks(nrows), TPB, 0, s>>>(b, cols, cols_alt, orig, orig_alt,
                                                        centre_p, nreal, nrows);
  k_reorder_back_gated<<<nblocks(nrows), TPB, 0, s>>>(b, cols_alt, cols, orig_alt, orig, nrows, ds);
  note_launch(2);
}
void launch_fill_i32(int32_t* p, int64_t n, int32_t v, cudaStream_t s) {
  k_fill_i32<<<nblocks(n), TPB, 0, s>>>(p, n, v);
  note_launch();
}
void launch_fill_u64(unsigned long long* p, int n, unsigned long long v, cudaStream_t s) {
  k_fill_u64<<<nblocks(n), TPB, 0, s>>>(p, n, v);
  note_launch();
}
__global__ void k_init_slots(unsigned long long* p, SlotInit in) {
  const int i = threadIdx.x;
  if (i < in.n) p[in.off[i]] = in.val[i];
}
void launch_init_slots(unsigned long long* p, const SlotInit& in, cudaStream_t s) {
  k_init_slots<<<1, 32, 0, s>>>(p, in);
  note_launch();
}
void launch_sts_stage(int kind, double* cols, int64_t ld, int64_t n, double* Y, double a0,
                      double a1, double a2, double a3, double a4, const double* ctrl,
                      cudaStream_t s) {
  k_sts<<<nblocks(n), TPB, 0, s>>>(kind, cols, ld, n, Y, a0, a1, a2, a3, a4, ctrl);
  note_launch();
}
void launch_sts_stage_dev(double* cols, int64_t ld, int64_t n, double* Y, const double* coef,
                          const int* jdev, const double* ctrl, cudaStream_t s) {
  k_sts<<<nblocks(n), TPB, 0, s>>>(2, cols, ld, n, Y, 0., 0., 0., 0., 0., ctrl, coef, jdev);
  note_launch();
}
__global__ void k_sts_loop(int* __restrict__ jdev, int sts_s, cudaGraphConditionalHandle h,
                           int init) {
  if (blockIdx.x != 0 || threadIdx.x != 0) return;
  const int j = init ? 2 : *jdev + 1;
  *jdev = j;
  cudaGraphSetConditional(h, j <= sts_s ? 1u : 0u);
}
void launch_sts_loop_init(int* jdev, int sts_s, cudaGraphConditionalHandle h, cudaStream_t s) {
  k_sts_loop<<<1, 32, 0, s>>>(jdev, sts_s, h, 1);
  note_launch();
}
void launch_sts_loop_ctl(int* jdev, int sts_s, cudaGraphConditionalHandle h, cudaStream_t s) {
  k_sts_loop<<<1, 32, 0, s>>>(jdev, sts_s, h, 0);
  note_launch();
}
void launch_eos(double* cols, int64_t ld, int64_t nreal, Params P, cudaStream_t s) {
  k_eos<<<nblocks(nreal), TPB, 0, s>>>(cols, ld, nreal, P);
  note_launch();
}
void launch_apply_mti(double* cols, int64_t ld, const int32_t* orig, int64_t nrows, int64_t nreal,
                      int lowres, cudaStream_t s) {
  k_mti<<<nblocks(nrows), TPB, 0, s>>>(cols, ld, orig, nrows, nreal, lowres);
  note_launch();
}
void launch_set_col(double* col, int64_t n, double v, cudaStream_t s) {
  k_set<<<nblocks(n), TPB, 0, s>>>(col, n, v);
  note_launch();
}

bool cell_sort(const uint32_t* keys, int64_t n, int64_t ncell, int32_t* count, int32_t* cstart,
               int32_t* vout, uint32_t* kout, int32_t* big, int32_t* ctr, void* scan_tmp,
               size_t scan_bytes, int32_t* h_ctr, cudaStream_t s) {
  // ctr[0]: the largest cell, ctr[1]: cells for the block sort
  cudaMemsetAsync(count, 0, sizeof(int32_t) * size_t(ncell + 1), s);
  cudaMemsetAsync(ctr, 0, 2 * sizeof(int32_t), s);
  if (n > 0) k_cell_count<<<nblocks(n), TPB, 0, s>>>(keys, n, count, ctr);
  cudaMemcpyAsync(h_ctr, ctr, sizeof(int32_t), cudaMemcpyDeviceToHost, s);
  cudaStreamSynchronize(s);
  note_launch();
  if (h_ctr[0] > kCellBig) return false;  // (nothing written)
  exclusive_scan(scan_tmp, scan_bytes, count, cstart, ncell + 1, s);
  cudaMemsetAsync(count, 0, sizeof(int32_t) * size_t(ncell), s);
  if (n > 0) k_cell_scatter<<<nblocks(n), TPB, 0, s>>>(keys, n, cstart, count, vout, kout);
  if (h_ctr[0] > 1) {
    k_cell_sort_small<<<nblocks(ncell), TPB, 0, s>>>(cstart, ncell, vout, big, ctr + 1);
    if (h_ctr[0] > kCellSmall) k_cell_sort_big<<<148 * 4, 256, 0, s>>>(cstart, vout, big, ctr + 1);
  }
  note_launch(3);
  return true;
}
size_t sort_temp_bytes(int64_t n) {
  size_t b = 0;
  cub::DeviceRadixSort::SortPairs(nullptr, b, (const uint32_t*)nullptr, (uint32_t*)nullptr,
                                  (const int32_t*)nullptr, (int32_t*)nullptr, int(n), 0, 30);
  return b;
}
void sort_pairs(void* tmp, size_t tmp_bytes, const uint32_t* kin, uint32_t* kout, const int32_t* vin,
                int32_t* vout, int64_t n, int end_bit, cudaStream_t s) {
  cub::DeviceRadixSort::SortPairs(tmp, tmp_bytes, kin, kout, vin, vout, int(n), 0, end_bit, s);
}
size_t scan_temp_bytes(int64_t n) {
  size_t b = 0;
  cub::DeviceScan::ExclusiveSum(nullptr, b, (const int32_t*)nullptr, (int32_t*)nullptr, int(n));
  return b;
}
void exclusive_scan(void* tmp, size_t tmp_bytes, const int32_t* in, int32_t* out, int64_t n,
                    cudaStream_t s) {
  cub::DeviceScan::ExclusiveSum(tmp, tmp_bytes, in, out, int(n), s);
}

}  // namespace sph
