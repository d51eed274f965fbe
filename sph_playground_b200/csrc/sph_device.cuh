// sph_device.cuh — device-side building blocks of the SPH step engine:
// kernel shapes (M4/M6/Gauss), two-sum accumulators, packed pair-data
// layouts and the launch-parameter block shared by all kernels.
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

#include "sph_abi.h"

namespace sph {

// ---- enums mirrored from playground/src/const.f90 --------------------------
enum : int { esd_fab = 400, esd_n2w = 401, esd_fw = 402, esd_2nw_ds = 403,
             esd_2nw_sd = 404 };
enum : int { ept_empty = 0, ept_real = 1, ept_fixed = 2, ept_fixedreal = 21,
             ept_fixedmirror = 22, ept_periodic = 3 };
// 0-based store columns (const.f90:69-103 minus one)
enum : int {
  es_rx = 0, es_ry, es_rz, es_vx, es_vy, es_vz, es_ax, es_ay, es_az, es_m,
  es_den, es_h, es_dh, es_p, es_u, es_du, es_t, es_kappa, es_dtdx, es_dtdy,
  es_dtdz, es_ddt, es_bx, es_by, es_bz, es_dbx, es_dby, es_dbz, es_c, es_om,
  es_type, es_vfld
};
constexpr int NCOL = SPH_ES_TOTAL;
constexpr double kLightspeed = 2.997924e10;  // const.f90:6
constexpr double kRg = 8.314e7;              // const.f90:7
constexpr double kSigmaB = 5.67051e-5;       // const.f90:8

// ---- kernel shapes ------------------------------------------------------------
// The reference evaluates f(q), f'(q), f''(q) piecewise (kernel/base_m6.f90:36-97,
// base_m4.f90:35-90, base_gauss.f90:39-82).  On the device the pieces are
// written branch-free with clamped terms t_k = max(k - q, 0): for q beyond a
// break point the clamped term is exactly zero, so the sum equals the
// reference's piece without divergent branches inside a warp.
enum KernelId : int { KM4 = SPH_KERNEL_M4, KM6 = SPH_KERNEL_M6, KGAUSS = SPH_KERNEL_GAUSS };

template <int K> struct KRad;
template <> struct KRad<KM4> { static constexpr double v = 2.0; };
template <> struct KRad<KM6> { static constexpr double v = 3.0; };
template <> struct KRad<KGAUSS> { static constexpr double v = 10.0; };

template <class R> __device__ __forceinline__ R rmax0(R x) { return x > R(0) ? x : R(0); }

template <int K, class R>
__device__ __forceinline__ void kshape_f_df(R q, R& f, R& df) {
  if constexpr (K == KM6) {
    R t3 = rmax0(R(3) - q), t2 = rmax0(R(2) - q), t1 = rmax0(R(1) - q);
    R s3 = t3 * t3, s2 = t2 * t2, s1 = t1 * t1;
    R q3 = s3 * s3, q2 = s2 * s2, q1 = s1 * s1;
    f = q3 * t3 - R(6) * (q2 * t2) + R(15) * (q1 * t1);
    df = R(-5) * q3 + R(30) * q2 - R(75) * q1;
  } else if constexpr (K == KM4) {
    R t2 = rmax0(R(2) - q), t1 = rmax0(R(1) - q);
    R s2 = t2 * t2, s1 = t1 * t1;
    f = R(0.25) * (s2 * t2) - s1 * t1;
    df = R(-0.75) * s2 + R(3) * s1;
  } else {
    R e = exp(-q * q);
    f = e;
    df = R(-2) * e * q;
  }
}

template <int K, class R>
__device__ __forceinline__ R kshape_df(R q) {
  if constexpr (K == KM6) {
    R t3 = rmax0(R(3) - q), t2 = rmax0(R(2) - q), t1 = rmax0(R(1) - q);
    R s3 = t3 * t3, s2 = t2 * t2, s1 = t1 * t1;
    return R(-5) * (s3 * s3) + R(30) * (s2 * s2) - R(75) * (s1 * s1);
  } else if constexpr (K == KM4) {
    R t2 = rmax0(R(2) - q), t1 = rmax0(R(1) - q);
    return R(-0.75) * (t2 * t2) + R(3) * (t1 * t1);
  } else {
    return R(-2) * exp(-q * q) * q;
  }
}

template <int K, class R>
__device__ __forceinline__ void kshape_all(R q, R& f, R& df, R& ddf) {
  if constexpr (K == KM6) {
    R t3 = rmax0(R(3) - q), t2 = rmax0(R(2) - q), t1 = rmax0(R(1) - q);
    R s3 = t3 * t3, s2 = t2 * t2, s1 = t1 * t1;
    R c3 = s3 * t3, c2 = s2 * t2, c1 = s1 * t1;
    R q3 = s3 * s3, q2 = s2 * s2, q1 = s1 * s1;
    f = q3 * t3 - R(6) * (q2 * t2) + R(15) * (q1 * t1);
    df = R(-5) * q3 + R(30) * q2 - R(75) * q1;
    ddf = R(20) * c3 - R(120) * c2 + R(300) * c1;
  } else if constexpr (K == KM4) {
    R t2 = rmax0(R(2) - q), t1 = rmax0(R(1) - q);
    R s2 = t2 * t2, s1 = t1 * t1;
    f = R(0.25) * (s2 * t2) - s1 * t1;
    df = R(-0.75) * s2 + R(3) * s1;
    ddf = R(1.5) * t2 - R(6) * t1;
  } else {
    R e = exp(-q * q);
    f = e;
    df = R(-2) * e * q;
    ddf = R(-2) * e + R(4) * e * q * q;
  }
}

// FP32 f(q) that follows q below FP32 resolution, for the Newton iteration on
// h.  q_lo is the rounding residual of q = r/h.  q is split as qh + dq with
// qh on the 2^-21 grid (for q < 4, q + 4 carries an ulp of 2^-21, so the add
// rounds q to it and the subtraction back is exact), which makes every piece
// t_k = c_k - qh exact; dq = (q - qh) + q_lo (the first difference exact)
// enters f to first order, f(q) = f(qh) + f'(qh) dq, the second-order term
// being below 1e-12 of f.  The density sum then changes smoothly with h
// instead of in steps of one FP32 ulp of q, so the Newton iterates settle.
template <int K>
__device__ __forceinline__ void kshape_f_df_res(float q, float q_lo, float& f, float& df) {
  if constexpr (K == KM6 || K == KM4) {
    const float qh = __fsub_rn(__fadd_rn(q, 4.0f), 4.0f);
    const float dq = __fadd_rn(__fsub_rn(q, qh), q_lo);
    constexpr int NP = (K == KM6) ? 3 : 2;
    const float cs[3] = {K == KM6 ? 3.f : 2.f, K == KM6 ? 2.f : 1.f, 1.f};
    const float as[3] = {K == KM6 ? 1.f : 0.25f, K == KM6 ? -6.f : -1.f, 15.f};
    f = 0.f;
    df = 0.f;
#pragma unroll
    for (int k = 0; k < NP; ++k) {
      const float th = fmaxf(cs[k] - qh, 0.f);  // exact: both on the 2^-21 grid
      const float s = th * th;
      if constexpr (K == KM6) {
        const float q4 = s * s;
        f = fmaf(as[k], q4 * th, f);
        df = fmaf(-5.f * as[k], q4, df);
      } else {
        f = fmaf(as[k], s * th, f);
        df = fmaf(-3.f * as[k], s, df);
      }
    }
    f = fmaf(df, dq, f);
  } else {
    float e = expf(-q * q);
    f = e;
    df = -2.f * e * q;
    f = fmaf(df, q_lo, f);
  }
}

template <int K, class R>
__device__ __forceinline__ R kshape_f(R q) {
  R f, df;
  kshape_f_df<K, R>(q, f, df);
  return f;
}

// Reciprocal square root, square root and division of the pair arithmetic.
// FP64 keeps IEEE operations (the parity path); FP32 uses the MUFU
// approximations (about 2 ulp), inside the FP32 path's error budget.
template <class R> __device__ __forceinline__ R frsqrt(R x);
template <> __device__ __forceinline__ double frsqrt<double>(double x) { return 1.0 / sqrt(x); }
template <> __device__ __forceinline__ float frsqrt<float>(float x) { return rsqrtf(x); }
template <class R> __device__ __forceinline__ R fsqrt(R x);
template <> __device__ __forceinline__ double fsqrt<double>(double x) { return sqrt(x); }
template <> __device__ __forceinline__ float fsqrt<float>(float x) {
  return x > 0.f ? x * rsqrtf(x) : 0.f;
}
template <class R> __device__ __forceinline__ R fdiv(R a, R b);
template <> __device__ __forceinline__ double fdiv<double>(double a, double b) { return a / b; }
template <> __device__ __forceinline__ float fdiv<float>(float a, float b) { return __fdividef(a, b); }

// h^n for small non-negative n (the reference's h**dim, h**(dim+2)).
template <int N, class R>
__device__ __forceinline__ R ipow(R x) {
  if constexpr (N == 0) return R(1);
  else if constexpr (N == 1) return x;
  else if constexpr (N == 2) return x * x;
  else if constexpr (N == 3) return x * (x * x);
  else if constexpr (N == 4) { R s = x * x; return s * s; }
  else { R s = x * x; return (s * s) * x; }
}

// ---- compensated accumulation ---------------------------------------------------
// Two-sum (Knuth): s + e == a + b exactly.  The FP32 path keeps every
// per-particle sum as (s, c) so that summing ~200 pair terms loses no more
// than one rounding of the final value.
template <class R> struct Acc {
  R s, c;
  __device__ __forceinline__ void init() { s = R(0); c = R(0); }
  __device__ __forceinline__ void add(R x) {
    R t = s + x;
    R bp = t - s;
    R e = (s - (t - bp)) + (x - bp);
    s = t;
    c += e;
  }
  __device__ __forceinline__ R val() const { return s + c; }
  __device__ __forceinline__ double dval() const { return double(s) + double(c); }
};
// Plain running sum in R with the same interface: a lane's share of a pair
// loop (n terms) carries at most gamma_n * sum|t| of rounding, about 2e-6
// sum|t| in FP32 for the n ~ 30 terms of a force lane; the lanes are then
// added in FP64.
template <class R> struct SumAcc {
  R s;
  __device__ __forceinline__ void init() { s = R(0); }
  __device__ __forceinline__ void add(R x) { s += x; }
  __device__ __forceinline__ R val() const { return s; }
  __device__ __forceinline__ double dval() const { return double(s); }
};
// Plain FP64 accumulator with the same interface.
template <> struct Acc<double> {
  double s;
  __device__ __forceinline__ void init() { s = 0.0; }
  __device__ __forceinline__ void add(double x) { s += x; }
  __device__ __forceinline__ double val() const { return s; }
  __device__ __forceinline__ double dval() const { return s; }
};

// ---- packed pair data (sorted order; the streams are listed at PackBufs) ----------
// FP64 positions are the sorted records' own; the FP32 force pass takes a
// hi/lo float pair of (x - origin + 2^E), all in one binade, so hi_i - hi_j
// is exact and dx = (hi_i - hi_j) + (lo_i - lo_j) carries one FP32 rounding;
// the FP32 density pass takes 31-bit fixed point (FixPos).
template <class R> struct PairPos;  // position handle for dx computation
template <> struct PairPos<double> {
  double x, y, z;
};
template <> struct PairPos<float> {
  float xh, yh, zh, xl, yl, zl;
};

__device__ __forceinline__ void pos_delta(const PairPos<double>& a, const PairPos<double>& b,
                                          double& dx, double& dy, double& dz) {
  dx = a.x - b.x; dy = a.y - b.y; dz = a.z - b.z;
}
// the density pass's FP32 positions: 31-bit fixed point over the packing
// frame; a separation is an exact integer difference rounded once to FP32
// (the scaling by the power-of-two unit is exact)
struct FixPos {
  int32_t x, y, z;
};
__device__ __forceinline__ void pos_delta(const FixPos& a, const FixPos& b, float& dx, float& dy,
                                          float& dz, float unit) {
  dx = __int2float_rn(a.x - b.x) * unit;
  dy = __int2float_rn(a.y - b.y) * unit;
  dz = __int2float_rn(a.z - b.z) * unit;
}
__device__ __forceinline__ void pos_delta(const PairPos<double>& a, const PairPos<double>& b,
                                          double& dx, double& dy, double& dz, double) {
  pos_delta(a, b, dx, dy, dz);
}
__device__ __forceinline__ void pos_delta(const PairPos<float>& a, const PairPos<float>& b,
                                          float& dx, float& dy, float& dz) {
  dx = (a.xh - b.xh) + (a.xl - b.xl);
  dy = (a.yh - b.yh) + (a.yl - b.yl);
  dz = (a.zh - b.zh) + (a.zl - b.zl);
}

// ---- launch parameters -------------------------------------------------------------
struct Params {
  int dim;
  int kernel;
  double krad;
  double wCv;      // knorm(dim)
  double fwc;      // fwcl(dim)
  double hfac;
  double alpha, beta, au;
  double gamma;
  double muzero;
  double difcond;
  int difiso;
  int ddw;
  int full_tensor;
  int eq_hydro, eq_magneto, eq_diff, eq_fld;
  int adden, artts;
  double tol;
  int maxiter;
  int eos_kind;  // 0 none, 1 adiabatic, 2 isothermal
  double c_iso;  // c of row 1 for eos_isothermal
};

// Counters of a block: each v[k] summed (or, with is_max[k], maximised) over
// the block's threads into thread 0's v[k], through shared memory, so that
// a kernel issues its counter atomics once per block, not once per warp
// (hundreds of thousands of same-address atomics per launch otherwise).
// Every thread of the block must call it; blocks of at most 1024 threads.
template <int N>
__device__ __forceinline__ void block_counters(unsigned long long (&v)[N], const bool (&is_max)[N]) {
  __shared__ unsigned long long part[32][N];
#pragma unroll
  for (int k = 0; k < N; ++k)
    for (int o = 16; o > 0; o >>= 1) {
      const unsigned long long t = __shfl_xor_sync(0xffffffffu, v[k], o);
      v[k] = is_max[k] ? (t > v[k] ? t : v[k]) : v[k] + t;
    }
  const int w = threadIdx.x >> 5;
  if ((threadIdx.x & 31) == 0)
    for (int k = 0; k < N; ++k) part[w][k] = v[k];
  __syncthreads();
  if (threadIdx.x == 0)
    for (int i = 1; i < int((blockDim.x + 31) >> 5); ++i)
      for (int k = 0; k < N; ++k)
        v[k] = is_max[k] ? (part[i][k] > v[k] ? part[i][k] : v[k]) : v[k] + part[i][k];
}

// status word helper: first error wins
__device__ __forceinline__ void raise_status(int* status, int code) {
  atomicCAS(status, 0, code);
}

}  // namespace sph
