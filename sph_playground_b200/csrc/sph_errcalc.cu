// sph_errcalc.cu — the engine's closing error evaluation on the device
// (main.f90:374-402 with the calculators of errcalc.f90): one thread per
// table row computes err of a real particle from its own fields, stored at
// the particle's original row; the L1 sum runs over the original order in
// fixed blocks and a fixed tree, so it does not depend on how the table's
// rows are currently ordered.
//
// Each formula keeps the reference's evaluation order; the transcendental
// functions are CUDA's double-precision ones (erf, exp, sin, atan2), so the
// results agree with a libm evaluation to a few ulp.
#include <cmath>

#include "sph_internal.h"

namespace sph {
namespace {

constexpr int TPB = 256;
constexpr double kPi = 3.141592653589793;  // 4 atan(1) in double (const.f90:4)

inline int nblocks(int64_t n, int tpb = TPB) {
  int64_t b = (n + tpb - 1) / tpb;
  return int(b < 1 ? 1 : b);
}

// density of the exact Riemann solution at x, time t (the wave pattern
// sampled along x / t; Toro, Riemann Solvers and Numerical Methods, ch. 4)
__device__ double riemann_density(const RiemannFan& f, double x, double t) {
  if (!(t > 0.0)) return x < f.x0 ? f.rl : f.rr;
  const double s = (x - f.x0) / t;
  const double g = f.gamma;
  if (s <= f.us) {  // left of the contact
    if (f.shock_l) return s <= f.sl ? f.rl : f.rsl;
    if (s <= f.hl) return f.rl;
    if (s <= f.tl) {  // inside the left fan
      const double w = 2.0 / (g + 1.0) + (g - 1.0) / ((g + 1.0) * f.cl) * (f.ul - s);
      return f.rl * pow(w, 2.0 / (g - 1.0));
    }
    return f.rsl;
  }
  if (f.shock_r) return s >= f.sr ? f.rr : f.rsr;
  if (s >= f.hr) return f.rr;
  if (s >= f.tr) {  // inside the right fan
    const double w = 2.0 / (g + 1.0) - (g - 1.0) / ((g + 1.0) * f.cr) * (f.ur - s);
    return f.rr * pow(w, 2.0 / (g - 1.0));
  }
  return f.rsr;
}

__global__ void k_errcalc(const double* __restrict__ cols, int64_t ld,
                          const int32_t* __restrict__ orig, int64_t nrows, int64_t nreal,
                          ErrCalcIn in, double* __restrict__ err) {
  const int64_t i = blockIdx.x * int64_t(blockDim.x) + threadIdx.x;
  if (i >= nrows) return;
  const int64_t o = orig[i];
  if (o >= nreal) return;
  auto C = [&](int f) { return cols[f * ld + i]; };
  const double x = C(es_rx), y = C(es_ry), z = C(es_rz), t = in.t;
  double e = 0.0;
  switch (in.kind) {
    case EK_SHOCK12: {  // errcalc.f90:140-170
      double tt = t;
      if (in.diso != 1 && !(C(es_bx) == 1.0)) tt = 1e-15;
      const double exact = (2.0 + 1.0) / 2.0 + (2.0 - 1.0) / 2.0 * erf(x / sqrt(4.0 * tt));
      e = fabs(exact - C(es_t));
      break;
    }
    case EK_RING: {  // errcalc.f90:99-138
      const double rho = sqrt(x * x + y * y);
      const double phi = atan2(y, x);
      const double d = rho - 0.3;
      const double exact =
          exp(-0.5 * (d * d / (0.05 * 0.05) + phi * phi / (0.5 * 0.5 + 2.0 * 1.0 * t / rho / rho)));
      e = fabs(exact - C(es_t));
      break;
    }
    case EK_PULSE: {  // errcalc.f90:46-97
      double exact;
      if (in.diso == 1)
        exact = in.pifac / in.ektd2 * exp(-0.5 * ((x * x + y * y + z * z) / in.ekt));
      else
        exact = in.pifac / in.epsdm1 / in.ektsq *
                exp(-0.5 * (x * x / in.ekt + (y * y + z * z) / 0.1 / 0.1));
      e = fabs(exact - C(es_t));
      break;
    }
    case EK_SOUNDWAVE:  // errcalc.f90:220-236
      e = fabs(1.0 + 0.005 * sin(kPi * (x - t)) - C(es_den));
      break;
    case EK_HYDROSHOCK:  // errcalc.f90:26-44
      e = fabs(C(es_den) - riemann_density(in.fan, x, t));
      break;
    case EK_ALFVEN: {  // errcalc.f90:198-218
      const double x1 = (x + 2.0 * y + 2.0 * z) / 3.0;
      const double b2 = (C(es_by) - 2.0 * C(es_bx)) / sqrt(5.0);
      e = fabs(0.1 * sin(2.0 * kPi * (x1 - t)) - b2);
      break;
    }
    default:
      break;
  }
  err[o] = e;
}

// part[b] = sum of err[b TPB .. (b+1) TPB) by a fixed tree
__global__ void __launch_bounds__(TPB) k_sum_blocks(const double* __restrict__ v, int64_t n,
                                                    double* __restrict__ part) {
  __shared__ double sh[TPB];
  const int64_t i = blockIdx.x * int64_t(TPB) + threadIdx.x;
  sh[threadIdx.x] = i < n ? v[i] : 0.0;
  __syncthreads();
  for (int w = TPB / 2; w > 0; w >>= 1) {
    if (threadIdx.x < w) sh[threadIdx.x] += sh[threadIdx.x + w];
    __syncthreads();
  }
  if (threadIdx.x == 0) part[blockIdx.x] = sh[0];
}

}  // namespace

RiemannFan riemann_fan(double gamma, double rl, double ul, double pl, double rr, double ur,
                       double pr, double x0) {
  RiemannFan f{};
  f.gamma = gamma;
  f.x0 = x0;
  f.rl = rl; f.ul = ul; f.pl = pl;
  f.rr = rr; f.ur = ur; f.pr = pr;
  f.cl = std::sqrt(gamma * pl / rl);
  f.cr = std::sqrt(gamma * pr / rr);
  const double g = gamma;
  // pressure function of one side and its derivative (Toro 4.6-4.7)
  auto side = [&](double p, double rk, double pk, double ck, double& d) {
    if (p > pk) {
      const double A = 2.0 / ((g + 1.0) * rk), B = (g - 1.0) / (g + 1.0) * pk;
      const double q = std::sqrt(A / (p + B));
      d = q * (1.0 - (p - pk) / (2.0 * (B + p)));
      return (p - pk) * q;
    }
    d = 1.0 / (rk * ck) * std::pow(p / pk, -(g + 1.0) / (2.0 * g));
    return 2.0 * ck / (g - 1.0) * (std::pow(p / pk, (g - 1.0) / (2.0 * g)) - 1.0);
  };
  // Newton from the two-rarefaction estimate (Toro 4.46), kept positive
  const double z = (g - 1.0) / (2.0 * g);
  double p = std::pow((f.cl + f.cr - 0.5 * (g - 1.0) * (ur - ul)) /
                          (f.cl / std::pow(pl, z) + f.cr / std::pow(pr, z)),
                      1.0 / z);
  if (!(p > 1e-12)) p = 1e-12;
  for (int it = 0; it < 100; ++it) {
    double dl, dr;
    const double fl = side(p, rl, pl, f.cl, dl), fr = side(p, rr, pr, f.cr, dr);
    double pn = p - (fl + fr + (ur - ul)) / (dl + dr);
    if (!(pn > 0.0)) pn = 0.5 * p;
    const double ch = std::fabs(pn - p) / (0.5 * (pn + p));
    p = pn;
    if (ch < 1e-15) break;
  }
  double dl, dr;
  const double fl = side(p, rl, pl, f.cl, dl), fr = side(p, rr, pr, f.cr, dr);
  f.ps = p;
  f.us = 0.5 * (ul + ur) + 0.5 * (fr - fl);
  const double gg = (g - 1.0) / (g + 1.0);
  f.shock_l = p > pl;
  f.shock_r = p > pr;
  if (f.shock_l) {
    f.rsl = rl * ((p / pl + gg) / (gg * p / pl + 1.0));
    f.sl = ul - f.cl * std::sqrt((g + 1.0) / (2.0 * g) * p / pl + z);
  } else {
    f.rsl = rl * std::pow(p / pl, 1.0 / g);
    f.hl = ul - f.cl;
    f.tl = f.us - f.cl * std::pow(p / pl, z);
  }
  if (f.shock_r) {
    f.rsr = rr * ((p / pr + gg) / (gg * p / pr + 1.0));
    f.sr = ur + f.cr * std::sqrt((g + 1.0) / (2.0 * g) * p / pr + z);
  } else {
    f.rsr = rr * std::pow(p / pr, 1.0 / g);
    f.hr = ur + f.cr;
    f.tr = f.us + f.cr * std::pow(p / pr, z);
  }
  return f;
}

// scratch of the fixed-order sum: one partial per block at every level
int64_t errcalc_parts(int64_t nreal) {
  int64_t total = 1, n = nreal;
  while (n > 1) {
    n = (n + TPB - 1) / TPB;
    total += n;
  }
  return total;
}

void launch_errcalc(const double* cols, int64_t ld, const int32_t* orig, int64_t nrows,
                    int64_t nreal, const ErrCalcIn& in, double* err, double* part, double* sum,
                    cudaStream_t s) {
  k_errcalc<<<nblocks(nrows), TPB, 0, s>>>(cols, ld, orig, nrows, nreal, in, err);
  note_launch();
  // block sums of block sums until one value is left
  const double* v = err;
  int64_t n = nreal;
  double* out = part;
  while (n > 1) {
    const int64_t nb = (n + TPB - 1) / TPB;
    k_sum_blocks<<<int(nb), TPB, 0, s>>>(v, n, out);
    note_launch();
    v = out;
    out += nb;
    n = nb;
  }
  cudaMemcpyAsync(sum, v, sizeof(double), cudaMemcpyDeviceToDevice, s);
}

}  // namespace sph
