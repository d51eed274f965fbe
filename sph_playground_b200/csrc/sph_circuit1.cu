// sph_circuit1.cu — circuit1 on the device: density summation, the Newton
// iteration on h with the grad-h term Omega (circuit1.f90:76-224), the
// direct-summation variant (circuit1.f90:227-305) and the temperature
// gradient used by the diffusion methods, with the adiabatic / isothermal EOS
// (eos.f90:21-45) fused into the epilogue.
//
// Two schedules give the reference's Jacobi iteration:
//  * k_c1_newton — without diffusion no particle reads another particle's
//    h, rho or Omega inside the loop (only positions and masses), so each
//    particle's sequence of iterates is independent of the others: one
//    thread runs its own Newton loop until |h_new - h|/h_0 <= tol or the
//    sweep cap, exactly the iterates the global loop gives it.
//  * k_c1_sweep — with a temperature gradient the sum reads the neighbours'
//    previous-sweep h, rho, Omega (circuit1.f90:163-179); one launch per
//    sweep over snapshot arrays, the host loops while any eps > tol.
#include "sph_internal.h"

namespace sph {
namespace {

constexpr int TPB = 128;

inline int nblocks(int64_t n, int tpb = TPB) {
  int64_t b = (n + tpb - 1) / tpb;
  return int(b < 1 ? 1 : b);
}

template <class R> struct PosAccess;
template <> struct PosAccess<double> {
  using Pos = PairPos<double>;
  static __device__ __forceinline__ double unit(const PackBufs&) { return 1.0; }
  static __device__ __forceinline__ PairPos<double> load(const PackBufs& pb, int64_t j, double& m) {
    double2 a = __ldg(&pb.p[0][j]);
    double2 b = __ldg(&pb.p[1][j]);
    m = b.y;
    PairPos<double> r;
    r.x = a.x; r.y = a.y; r.z = b.x;
    return r;
  }
  static __device__ __forceinline__ double temp(const PackBufs& pb, int64_t j) {
    return __ldg(&pb.p[6][j]).y;
  }
};
template <> struct PosAccess<float> {
  using Pos = FixPos;
  static __device__ __forceinline__ float unit(const PackBufs& pb) { return *pb.unit; }
  static __device__ __forceinline__ FixPos load(const PackBufs& pb, int64_t j, float& m) {
    const float4 a = __ldg(&pb.q[6][j]);
    m = a.w;
    FixPos r;
    r.x = __float_as_int(a.x); r.y = __float_as_int(a.y); r.z = __float_as_int(a.z);
    return r;
  }
  static __device__ __forceinline__ float temp(const PackBufs& pb, int64_t j) {
    return __ldg(&pb.q[4][j]).x;
  }
};

template <class R> __device__ __forceinline__ R rsq(R x) { return fsqrt<R>(x); }

// One Newton update from the summed density and dW/dh terms
// (circuit1.f90:191-206).  Returns eps; writes rho, Omega, h_new.
template <int DIM>
__device__ __forceinline__ double newton_update(double ha, double ha0, double ma, double hfac,
                                                double wsum, double osum, double& rho,
                                                double& om, double& hn) {
  rho = wsum;
  om = 1. - osum * (-ha / (DIM * rho));
  double dfdh = -DIM * rho * om / ha;
  double fh = ma * ipow<DIM>(hfac / ha) - rho;
  hn = ha - fh / dfdh;
  return fabs(hn - ha) / ha0;
}

__device__ __forceinline__ void eos_epilogue(double* cols, int64_t ld, int64_t p, double rho,
                                             const Params& P) {
  if (P.eos_kind == 1) {
    double pr = (P.gamma - 1.) * rho * cols[es_u * ld + p];
    cols[es_p * ld + p] = pr;
    cols[es_c * ld + p] = sqrt(P.gamma * pr / rho);
  } else if (P.eos_kind == 2) {
    cols[es_p * ld + p] = rho * P.c_iso * P.c_iso;
  }
}

// Sum a per-lane double over the G lanes of a group (all lanes get the sum).
template <int G>
__device__ __forceinline__ double group_sum(double v, unsigned gmask) {
#pragma unroll
  for (int o = G / 2; o > 0; o >>= 1) v += __shfl_xor_sync(gmask, v, o);
  return v;
}

template <int G>
__device__ __forceinline__ unsigned group_mask() {
  const int wl = threadIdx.x & 31;
  return (G == 32) ? 0xffffffffu : (((1u << G) - 1u) << (wl & ~(G - 1)));
}

// ---- fused Newton loop (no temperature gradient) ------------------------------------------
// G lanes per centre: each lane sums every G-th neighbour of the centre's
// row of the neighbour list (coalesced), the group adds its lanes' two-sum
// partials in FP64, and every lane takes the same FP64 Newton step.
template <int K, int DIM, class R, int G>
__global__ void __launch_bounds__(TPB, 8)
k_c1_newton(C1Args a, PackBufs pb, Params P) {
  const int64_t c = (blockIdx.x * int64_t(blockDim.x) + threadIdx.x) / G;
  const int lane = threadIdx.x & (G - 1);
  const unsigned gmask = group_mask<G>();
  unsigned long long pairs = 0, sweeps = 0;
  int maxit = 0;
  if (c < a.nc) {
    const int64_t k = a.centre_k[c];
    const int64_t p = a.centre_p[c];
    double* cols = a.cols;
    const int64_t ld = a.ld;
    R mi;
    const typename PosAccess<R>::Pos pi = PosAccess<R>::load(pb, k, mi);
    const R punit = PosAccess<R>::unit(pb);
    const double ma = cols[es_m * ld + p];
    const double ha0 = cols[es_h * ld + p];
    const int n = a.ncnt[c];
    const int32_t* __restrict__ row = a.nl + a.rowoff[c];
    const double wcv = P.wCv;
    // kernel shape at q = 0 for the self term (circuit1.f90:191-194)
    R f0, df0;
    kshape_f_df<K, R>(R(0), f0, df0);
    double ha = ha0, rho = 0., om = 1., hn = ha0, eps_prev = 1e300;
    int it = 0;
    bool bad = false;
    for (;;) {
      ++it;
      // (the separations stay in fixed-point units: 1/h carries the unit, a
      // power of two, so q is the same as from physical separations)
      const double ihd_full = 1.0 / ha;
      const R ih0 = R(ihd_full);
      const R ih = ih0 * punit;
      const R ih_lo = R(ihd_full - double(ih0)) * punit;
      // the density sum keeps its two-sum partials (its smoothness in h is
      // what the Newton iteration needs); the d rho / dh sum only scales the
      // Newton step and Omega, so a plain per-lane sum suffices
      Acc<R> sw;
      SumAcc<R> so;
      sw.init();
      so.init();
      // U neighbours per lane per round: their pair data are all requested
      // before the first is used, so the gathers overlap; the list entries
      // of the next round are read one round ahead
      constexpr int U = sizeof(R) == 4 ? 4 : 2;
      int32_t jn[U];
#pragma unroll
      for (int u = 0; u < U; ++u) jn[u] = (lane + u * G < n) ? row[lane + u * G] : -1;
      for (int l0 = lane; l0 < n; l0 += G * U) {
        int64_t jj[U];
#pragma unroll
        for (int u = 0; u < U; ++u) jj[u] = jn[u];
        typename PosAccess<R>::Pos pj[U];
        R mj[U];
#pragma unroll
        for (int u = 0; u < U; ++u) pj[u] = PosAccess<R>::load(pb, jj[u] >= 0 ? jj[u] : 0, mj[u]);
#pragma unroll
        for (int u = 0; u < U; ++u) {
          const int l = l0 + (U + u) * G;
          jn[u] = l < n ? row[l] : -1;
        }
#pragma unroll
        for (int u = 0; u < U; ++u) {
          if (jj[u] < 0) continue;
          R dx, dy, dz;
          pos_delta(pi, pj[u], dx, dy, dz, R(1));
          R r2 = dx * dx;
          if (DIM >= 2) r2 += dy * dy;
          if (DIM == 3) r2 += dz * dz;
          const R r = rsq<R>(r2);
          const R q = r * ih;
          bad |= !(q >= R(0));
          R f, df;
          if constexpr (sizeof(R) == 4) {
            // q carries the FP32 rounding of r/h; its residual (exact via FMA)
            // and the residuals of the kernel pieces enter f to first order,
            // so the density sum varies smoothly with h below FP32 resolution
            // and the Newton iterates converge instead of cycling between
            // neighbouring FP32 values (kshape_f_df_res).
            const R q_lo = fmaf(r, ih, -q) + r * ih_lo;
            kshape_f_df_res<K>(q, q_lo, f, df);
          } else {
            kshape_f_df<K, R>(q, f, df);
          }
          sw.add(mj[u] * f);
          so.add(mj[u] * (R(DIM) * f + q * df));
        }
      }
      const double swt = group_sum<G>(sw.dval(), gmask);
      const double sot = group_sum<G>(so.dval(), gmask);
      // W = wCv f / h^d; dW/dh = -wCv / h^(d+1) (d f + q f')  (kernel.f90:178-187, 239-249)
      const double ihd = 1.0 / ipow<DIM>(ha);
      const double wsum = wcv * ihd * (a.mref * swt + ma * double(f0));
      const double osum = -wcv * ihd / ha * (a.mref * sot + ma * (DIM * double(f0)));
      const double eps = newton_update<DIM>(ha, ha0, ma, P.hfac, wsum, osum, rho, om, hn);
      if (hn <= 0.) {
        if (lane == 0) raise_status(a.status, SPH_ERR_H_NEG);
        break;
      }
      if (!(eps > P.tol) || it >= P.maxiter) break;
      if constexpr (sizeof(R) == 4) {
        // FP32 sums carry a noise floor of a few 1e-9 in rho, i.e. ~1e-8 in
        // the Newton step, and the FP32 force pass moves a lattice at rest
        // by its rounding, so h drifts by ~1e-8 per step.  An eps below 1e-7
        // puts the stored rho within 3e-7 of the converged one, inside the
        // FP32 path's budget: stop there on the first sweep, and later once
        // eps no longer at least halves (further sweeps move h only within
        // that noise).  At 160^3 Sedov this keeps the sweeps per particle at
        // 1.00 instead of 1.4 (whole steps where every particle would take
        // a second sweep for an eps just above 1e-8).
        if (eps < 1e-7 && (it == 1 || eps >= 0.5 * eps_prev)) break;
      }
      eps_prev = eps;
      ha = hn;
    }
    if (bad) raise_status(a.status, (ha > 0.0) ? SPH_ERR_Q_NAN : SPH_ERR_Q_NEG);
    if (lane == 0) {
      pairs = (unsigned long long)n * it;
      sweeps = it;
      maxit = it;
      cols[es_h * ld + p] = hn;
      cols[es_den * ld + p] = rho;
      cols[es_om * ld + p] = om;
      cols[es_dtdx * ld + p] = 0.;
      cols[es_dtdy * ld + p] = 0.;
      cols[es_dtdz * ld + p] = 0.;
      eos_epilogue(cols, ld, p, rho, P);
    }
  }
  unsigned long long wp = pairs, ws = sweeps;
  for (int o = 16; o > 0; o >>= 1) {
    wp += __shfl_xor_sync(0xffffffffu, wp, o);
    ws += __shfl_xor_sync(0xffffffffu, ws, o);
    maxit = max(maxit, __shfl_xor_sync(0xffffffffu, maxit, o));
  }
  if ((threadIdx.x & 31) == 0) {
    if (wp) atomicAdd(&a.dcnt[DC_C1_PAIRS], wp);
    if (ws) atomicAdd(&a.dcnt[DC_C1_CENTRE_SWEEPS], ws);
    if (maxit) atomicMax(&a.dcnt[DC_C1_MAXSWEEPS], (unsigned long long)maxit);
  }
}

// ---- one Jacobi sweep (diffusion / FLD, and the direct summation) ------------------------
template <int K, int DIM, class R, int G>
__global__ void __launch_bounds__(TPB)
k_c1_sweep(C1Args a, PackBufs pb, Params P) {
  if (a.gate && *a.gate == 0ull) return;  // the previous sweep left no particle active
  const int64_t c = (blockIdx.x * int64_t(blockDim.x) + threadIdx.x) / G;
  const int lane = threadIdx.x & (G - 1);
  const unsigned gmask = group_mask<G>();
  unsigned long long pairs = 0, sweeps = 0;
  int active_left = 0;
  if (c < a.nc) {
    const int64_t k = a.centre_k[c];
    const int64_t p = a.centre_p[c];
    double* cols = a.cols;
    const int64_t ld = a.ld;
    if (a.simple || a.eps[p] > P.tol) {
      R mi;
      const typename PosAccess<R>::Pos pi = PosAccess<R>::load(pb, k, mi);
      const R punit = PosAccess<R>::unit(pb);
      const double ma = cols[es_m * ld + p];
      const double ha0 = cols[es_h * ld + p];
      const double ha = a.hk_s[k], rhoa = a.dk_s[k], oma = a.ok_s[k];
      const double ta = cols[es_t * ld + p];
      const int n = a.ncnt[c];
      const int32_t* __restrict__ row = a.nl + a.rowoff[c];
      const bool dT = a.simple ? (P.eq_diff && (P.ddw == esd_2nw_ds || P.ddw == esd_2nw_sd))
                               : (P.eq_diff || P.eq_fld);
      const R ih = R(1.0 / ha);
      const R ih_lo = R(1.0 / ha - double(ih));
      const double Ka = P.wCv / ipow<DIM + 1>(ha);  // wCv / h^(d+1)
      Acc<R> sw, so;
      sw.init();
      so.init();
      Acc<R> g[3];
      g[0].init(); g[1].init(); g[2].init();
      bool bad = false;
      const R rta = R(ta), rrhoa = R(rhoa), roma = R(oma);
      int32_t jnext = lane < n ? row[lane] : 0;  // list entry read one round ahead
      for (int l = lane; l < n; l += G) {
        const int64_t j = jnext;
        R mj;
        const typename PosAccess<R>::Pos pj = PosAccess<R>::load(pb, j, mj);
        if (l + G < n) jnext = row[l + G];
        R dx, dy, dz;
        pos_delta(pi, pj, dx, dy, dz, punit);
        R r2 = dx * dx;
        if (DIM >= 2) r2 += dy * dy;
        if (DIM == 3) r2 += dz * dz;
        const R r = rsq<R>(r2);
        const R q = r * ih;
        bad |= !(q >= R(0));
        R f, df;
        if constexpr (sizeof(R) == 4) kshape_f_df_res<K>(q, fmaf(r, ih, -q) + r * ih_lo, f, df);
        else kshape_f_df<K, R>(q, f, df);
        sw.add(mj * f);
        if (!a.simple) so.add(mj * (R(DIM) * f + q * df));
        if (dT) {
          const R tb = PosAccess<R>::temp(pb, j);
          // nabla W_a = wCv f'(q_a) r_ab / (h_a^(d+1) r)   (kernel.f90:189-197)
          const R ga = fdiv<R>(R(Ka) * df, r);
          R coef;
          if (P.ddw == esd_2nw_sd) {
            const double hb = a.hk_s[j], rhob = a.dk_s[j], omb = a.ok_s[j];
            const R qb = r * R(1.0 / hb);
            const R dfb = kshape_df<K, R>(qb);
            const R gb = fdiv<R>(R(P.wCv / ipow<DIM + 1>(hb)) * dfb, r);
            R ca, cb;
            if (a.simple) {  // circuit1.f90:289
              ca = rta / rrhoa / rrhoa;
              cb = tb / R(rhob) / R(rhob);
            } else {  // circuit1.f90:176
              ca = rta * rrhoa / roma / rrhoa / rrhoa;
              cb = tb * rrhoa / R(omb) / R(rhob) / R(rhob);
            }
            coef = mj * (ca * ga + cb * gb);
          } else if (a.simple) {  // 2nw_ds, circuit1.f90:284
            coef = mj / rrhoa * (tb - rta) * ga;
          } else {  // circuit1.f90:179
            const R rhob = R(a.dk_s[j]);
            coef = mj / rrhoa / roma * (tb * rhob - rta * rrhoa) * ga;
          }
          g[0].add(coef * dx);
          if (DIM >= 2) g[1].add(coef * dy);
          if (DIM == 3) g[2].add(coef * dz);
        }
      }
      pairs = (lane == 0) ? n : 0;
      sweeps = (lane == 0) ? 1 : 0;
      if (bad) raise_status(a.status, (ha > 0.0) ? SPH_ERR_Q_NAN : SPH_ERR_Q_NEG);
      const double swt = group_sum<G>(sw.dval(), gmask);
      const double sot = group_sum<G>(so.dval(), gmask);
      const double g0 = group_sum<G>(g[0].dval(), gmask);
      const double g1 = group_sum<G>(g[1].dval(), gmask);
      const double g2 = group_sum<G>(g[2].dval(), gmask);
      R f0, df0;
      kshape_f_df<K, R>(R(0), f0, df0);
      const double ihd = 1.0 / ipow<DIM>(ha);
      const double wsum = P.wCv * ihd * (a.mref * swt + ma * double(f0));
      if (lane == 0) {
        cols[es_dtdx * ld + p] = a.mref * g0;
        cols[es_dtdy * ld + p] = a.mref * g1;
        cols[es_dtdz * ld + p] = a.mref * g2;
        if (a.simple) {
          // circuit1.f90:293-301
          const double hnew = P.hfac * pow(ma / wsum, 1. / DIM);
          a.dkp1[p] = wsum;
          a.hkp1[p] = hnew;
          a.okp1[p] = 1.;
        } else {
          const double osum = -P.wCv * ihd / ha * (a.mref * sot + ma * (DIM * double(f0)));
          double rho, om, hn;
          double eps = newton_update<DIM>(ha, ha0, ma, P.hfac, wsum, osum, rho, om, hn);
          if (hn <= 0.) raise_status(a.status, SPH_ERR_H_NEG);
          if constexpr (sizeof(R) == 4) {
            // FP32 noise floor, as in k_c1_newton: an eps below 1e-7 on the
            // first sweep, or a stagnating one later, counts as converged
            // (a table at rest otherwise takes 2-3 sweeps per iterate that
            // move h only within the FP32 sums' noise)
            const double eps_prev = a.eps[p];
            const bool first = a.iter_dev ? *a.iter_dev == 0 : a.first != 0;
            if (eps > P.tol && eps < 1e-7 && (first || eps >= 0.5 * eps_prev)) eps = 0.0;
          }
          a.eps[p] = eps;
          a.dkp1[p] = rho;
          a.okp1[p] = om;
          a.hkp1[p] = hn;
          active_left = eps > P.tol ? 1 : 0;
        }
      }
    }
  }
  unsigned long long wp = pairs, ws = sweeps;
  for (int o = 16; o > 0; o >>= 1) {
    wp += __shfl_xor_sync(0xffffffffu, wp, o);
    ws += __shfl_xor_sync(0xffffffffu, ws, o);
    active_left |= __shfl_xor_sync(0xffffffffu, active_left, o);
  }
  if ((threadIdx.x & 31) == 0) {
    if (wp) atomicAdd(&a.dcnt[DC_C1_PAIRS], wp);
    if (ws) atomicAdd(&a.dcnt[DC_C1_CENTRE_SWEEPS], ws);
    if (active_left) atomicOr(&a.red[a.active_slot], 1ull);
  }
}

__global__ void k_c1_snapshot(int64_t n, const int32_t* __restrict__ ssrc,
                              const double* __restrict__ hkp1, const double* __restrict__ dkp1,
                              const double* __restrict__ okp1, double* __restrict__ hk_s,
                              double* __restrict__ dk_s, double* __restrict__ ok_s,
                              const DevPlan* __restrict__ plan,
                              const unsigned long long* __restrict__ gate) {
  if (gate && *gate == 0ull) return;
  int64_t k = blockIdx.x * int64_t(blockDim.x) + threadIdx.x;
  if (plan) n = plan->nall;  // launched over the capacity
  if (k >= n) return;
  int64_t p = ssrc[k];
  hk_s[k] = hkp1[p];
  dk_s[k] = dkp1[p];
  ok_s[k] = okp1[p];
}

// Store the converged iterates (circuit1.f90:213-215 / 299-301) and run the EOS.
__global__ void k_c1_finalize(int64_t nrows, int64_t nreal, double* __restrict__ cols, int64_t ld,
                              const double* __restrict__ hkp1, const double* __restrict__ dkp1,
                              const double* __restrict__ okp1, int simple, Params P) {
  int64_t p = blockIdx.x * int64_t(blockDim.x) + threadIdx.x;
  if (p >= nrows) return;
  if (p < nreal) {
    cols[es_h * ld + p] = hkp1[p];
    cols[es_den * ld + p] = dkp1[p];
    cols[es_om * ld + p] = okp1[p];
    eos_epilogue(cols, ld, p, dkp1[p], P);
  } else if (simple) {
    cols[es_om * ld + p] = 1.;  // circuit1.f90:62 sets every row
  }
}

template <int K, int DIM, class R>
void dispatch_newton(int G, const C1Args& a, const PackBufs& pb, const Params& P, cudaStream_t s) {
  switch (G) {
    case 4: k_c1_newton<K, DIM, R, 4><<<nblocks(a.nc * 4), TPB, 0, s>>>(a, pb, P); break;
    case 8: k_c1_newton<K, DIM, R, 8><<<nblocks(a.nc * 8), TPB, 0, s>>>(a, pb, P); break;
    case 16: k_c1_newton<K, DIM, R, 16><<<nblocks(a.nc * 16), TPB, 0, s>>>(a, pb, P); break;
    default: k_c1_newton<K, DIM, R, 32><<<nblocks(a.nc * 32), TPB, 0, s>>>(a, pb, P); break;
  }
  note_launch();
}
template <int K, int DIM, class R>
void dispatch_sweep(int G, const C1Args& a, const PackBufs& pb, const Params& P, cudaStream_t s) {
  switch (G) {
    case 4: k_c1_sweep<K, DIM, R, 4><<<nblocks(a.nc * 4), TPB, 0, s>>>(a, pb, P); break;
    case 8: k_c1_sweep<K, DIM, R, 8><<<nblocks(a.nc * 8), TPB, 0, s>>>(a, pb, P); break;
    case 16: k_c1_sweep<K, DIM, R, 16><<<nblocks(a.nc * 16), TPB, 0, s>>>(a, pb, P); break;
    default: k_c1_sweep<K, DIM, R, 32><<<nblocks(a.nc * 32), TPB, 0, s>>>(a, pb, P); break;
  }
  note_launch();
}

#define SPH_DISPATCH(FN)                                                             \
  template <int K, int DIM>                                                          \
  void FN##_prec(int prec, const C1Args& a, const PackBufs& pb, const Params& P,    \
                 cudaStream_t s) {                                                   \
    if (prec == SPH_PREC_FP64) FN<K, DIM, double>(a.G, a, pb, P, s);                 \
    else FN<K, DIM, float>(a.G, a, pb, P, s);                                        \
  }                                                                                  \
  template <int K>                                                                   \
  void FN##_dim(int prec, int dim, const C1Args& a, const PackBufs& pb,             \
                const Params& P, cudaStream_t s) {                                   \
    if (dim == 3) FN##_prec<K, 3>(prec, a, pb, P, s);                                \
    else if (dim == 2) FN##_prec<K, 2>(prec, a, pb, P, s);                           \
    else FN##_prec<K, 1>(prec, a, pb, P, s);                                         \
  }                                                                                  \
  void FN##_all(int prec, int kernel, int dim, const C1Args& a, const PackBufs& pb, \
                const Params& P, cudaStream_t s) {                                   \
    if (kernel == KM6) FN##_dim<KM6>(prec, dim, a, pb, P, s);                        \
    else if (kernel == KM4) FN##_dim<KM4>(prec, dim, a, pb, P, s);                   \
    else FN##_dim<KGAUSS>(prec, dim, a, pb, P, s);                                   \
  }

SPH_DISPATCH(dispatch_newton)
SPH_DISPATCH(dispatch_sweep)

}  // namespace

void launch_c1_newton(int prec, int kernel, int dim, const C1Args& a, PackBufs pb, Params P,
                      cudaStream_t s) {
  dispatch_newton_all(prec, kernel, dim, a, pb, P, s);
}
void launch_c1_sweep(int prec, int kernel, int dim, const C1Args& a, PackBufs pb, Params P,
                     cudaStream_t s) {
  dispatch_sweep_all(prec, kernel, dim, a, pb, P, s);
}
void launch_c1_finalize(int64_t nrows, int64_t nreal, double* cols, int64_t ld, const double* hkp1,
                        const double* dkp1, const double* okp1, int simple, Params P,
                        cudaStream_t s) {
  k_c1_finalize<<<nblocks(nrows, 256), 256, 0, s>>>(nrows, nreal, cols, ld, hkp1, dkp1, okp1,
                                                    simple, P);
  note_launch();
}
void launch_c1_snapshot(int64_t n, const int32_t* ssrc, const double* hkp1, const double* dkp1,
                        const double* okp1, double* hk_s, double* dk_s, double* ok_s,
                        cudaStream_t s, const DevPlan* plan, const unsigned long long* gate) {
  k_c1_snapshot<<<nblocks(n, 256), 256, 0, s>>>(n, ssrc, hkp1, dkp1, okp1, hk_s, dk_s, ok_s,
                                                plan, gate);
  note_launch();
}

}  // namespace sph
