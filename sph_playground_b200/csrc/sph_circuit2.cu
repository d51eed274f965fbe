// sph_circuit2.cu — circuit2 on the device: the per-pair forces of
// circuit2.f90:58-505 (hydro pressure force and energy, Monaghan artificial
// viscosity :558-575, artificial conductivity :520-529, dh/dt from the
// continuity term, anisotropic / isotropic / flux-limited diffusion with the
// run-time second-derivative method, ideal-MHD stress and induction).
//
// G lanes per centre walk its neighbour list (lane l takes entries l, l + G,
// ...); neighbour data come from the packed sorted-order streams.  All
// nabla W terms are written as g * r_ab with
//   g_a = wCv f'(q_a) / (h_a^(d+1) r)      (nw_cart, kernel.f90:189-197)
// and the reference's per-pair divisions by rho^2 Omega are the per-particle
// factor Pi = 1/(rho^2 Omega) computed once when the streams are packed.
// The "ddw device function table" of kernel.f90:19-23 (procedure pointers
// nw, fab, n2w, hessian) is the run-time switch on P.ddw below; the branch
// is uniform across a launch, so it does not diverge.
#include "sph_internal.h"

namespace sph {
namespace {

constexpr int TPB = 128;

inline int nblocks(int64_t n, int tpb = TPB) {
  int64_t b = (n + tpb - 1) / tpb;
  return int(b < 1 ? 1 : b);
}

template <class R> struct Part {
  PairPos<R> pos;
  R m, invh, rho, Pi, P, c, u, vx, vy, vz;
  R hrho, ac;  // rho / 2 and alpha c (the FP32 record's own fields)
};
template <class R> struct PartX {
  R T, kappa, gx, gy, gz, bx, by, bz;
};

template <class R> struct Loader;
template <> struct Loader<double> {
  static __device__ __forceinline__ void hydro(const PackBufs& pb, int64_t j, Part<double>& o) {
    double2 a = __ldg(&pb.p[0][j]), b = __ldg(&pb.p[1][j]), c = __ldg(&pb.p[2][j]),
            d = __ldg(&pb.p[3][j]), e = __ldg(&pb.p[4][j]), f = __ldg(&pb.p[5][j]),
            g = __ldg(&pb.p[6][j]);
    o.pos.x = a.x; o.pos.y = a.y; o.pos.z = b.x; o.m = b.y;
    o.invh = c.x; o.rho = c.y; o.Pi = d.x; o.P = d.y; o.c = e.x; o.u = e.y;
    o.vx = f.x; o.vy = f.y; o.vz = g.x;
  }
  static __device__ __forceinline__ void extra(const PackBufs& pb, int64_t j, PartX<double>& o) {
    double2 g = __ldg(&pb.p[6][j]), h = __ldg(&pb.p[7][j]), i = __ldg(&pb.p[8][j]),
            k = __ldg(&pb.p[9][j]), l = __ldg(&pb.p[10][j]);
    o.T = g.y; o.kappa = h.x; o.gx = h.y; o.gy = i.x; o.gz = i.y;
    o.bx = k.x; o.by = k.y; o.bz = l.x;
  }
};
template <> struct Loader<float> {
  static __device__ __forceinline__ void hydro(const PackBufs& pb, int64_t j, Part<float>& o) {
    float4 a = __ldg(&pb.q[0][j]), b = __ldg(&pb.q[1][j]), c = __ldg(&pb.q[2][j]),
           d = __ldg(&pb.q[3][j]);
    o.pos.xh = a.x; o.pos.yh = a.y; o.pos.zh = a.z; o.m = a.w;
    o.pos.xl = b.x; o.pos.yl = b.y; o.pos.zl = b.z; o.invh = b.w;
    o.hrho = c.x; o.rho = 2.f * c.x; o.Pi = c.y; o.P = c.z; o.ac = c.w;
    o.u = d.x; o.vx = d.y; o.vy = d.z; o.vz = d.w;
  }
  static __device__ __forceinline__ void extra(const PackBufs& pb, int64_t j, PartX<float>& o) {
    float4 e = __ldg(&pb.q[4][j]), f = __ldg(&pb.q[5][j]);
    o.T = e.x; o.kappa = e.y; o.gx = e.z; o.gy = e.w;
    o.gz = f.x; o.bx = f.y; o.by = f.z; o.bz = f.w;
  }
};

template <class R> __device__ __forceinline__ R my_sqrt(R x);
template <> __device__ __forceinline__ double my_sqrt<double>(double x) { return sqrt(x); }
template <> __device__ __forceinline__ float my_sqrt<float>(float x) { return sqrtf(x); }

// diffusion tensor (3x3, symmetric) built from a unit vector (circuit2.f90:203-205,
// 371-373: diagonal form; the full k_par b b^T when full_tensor is set)
template <class R>
__device__ __forceinline__ void aniso_tensor(R difcond, const R* ub, int full, R K[3][3]) {
  for (int a = 0; a < 3; ++a)
    for (int b = 0; b < 3; ++b) K[a][b] = (a == b || full) ? difcond * ub[a] * ub[b] : R(0);
}

// flux-limited diffusion coefficient (circuit2.f90:180-183, 358-361)
template <class R>
__device__ __forceinline__ R fld_coef(R gnorm, R kappa, R rho, R T, R& lambda) {
  R fr = gnorm / (kappa * rho * rho * T);
  lambda = (R(2) + fr) / (R(6) + R(3) * fr + fr * fr);
  return R(kLightspeed) * lambda / kappa / rho;
}

template <int G>
__device__ __forceinline__ double group_sum(double v, unsigned gmask) {
#pragma unroll
  for (int o = G / 2; o > 0; o >>= 1) v += __shfl_xor_sync(gmask, v, o);
  return v;
}

// G lanes per centre: lane l takes neighbours l, l+G, ... of the centre's
// list row; per-lane partial sums are added over the group in FP64 and
// lane 0 stores the result.
// (FP32: 9 blocks of 128 threads per SM, 56 registers with a 4-byte spill,
// measured 2.01 -> 1.95 ms on the 128^3 Sedov step against 8 blocks at 64
// registers; 10 blocks spill 44 bytes and take 2.5 ms)
template <int K, int DIM, class R, bool GENERAL, int G>
__global__ void __launch_bounds__(TPB, sizeof(R) == 8 ? 5 : 9)
k_c2(C2Args a, PackBufs pb, Params P) {
  const int64_t c = (blockIdx.x * int64_t(blockDim.x) + threadIdx.x) / G;
  const int lane = threadIdx.x & (G - 1);
  const int wl = threadIdx.x & 31;
  const unsigned gmask = (G == 32) ? 0xffffffffu : (((1u << G) - 1u) << (wl & ~(G - 1)));
  unsigned long long pairs = 0;
  if (c < a.nc) {
    const int64_t k = a.centre_k[c];
    const int64_t p = a.centre_p[c];
    double* cols = a.cols;
    const int64_t ld = a.ld;
    Part<R> A;
    Loader<R>::hydro(pb, k, A);
    if constexpr (sizeof(R) == 4) {
      // the FP32 record's second rho field is wCv Pi / h^(d+1), the
      // neighbour-side product; the centre takes Pi itself
      const double rr = cols[es_den * ld + p], oo = cols[es_om * ld + p];
      A.Pi = float(1.0 / (rr * rr * oo));
    }
    const R wcv = R(P.wCv);
    R Ka = A.invh;
    for (int d = 0; d < DIM; ++d) Ka *= A.invh;
    Ka *= wcv;  // wCv / h_a^(d+1)
    const R alpha = R(P.alpha), beta = R(P.beta), au = R(P.au);
    const bool artts = P.artts == 1, adden = P.adden == 1, hydro = P.eq_hydro != 0;
    // the artificial conductivity term (circuit2.f90:316-331) is scaled by
    // au: au = -1 switches it off in the reference, and au = 0 makes it
    // vanish, so it is skipped for both
    const bool use_au = P.au != -1.0 && P.au != 0.0;
    const R rPiA = A.rho * A.Pi;  // 1 / (rho_a Omega_a)
    R alpha_ca;
    if constexpr (sizeof(R) == 4) alpha_ca = A.ac;
    else alpha_ca = alpha * A.c;
    const R hrhoa = R(-0.5) * A.rho, hrho_a = R(0.5) * A.rho, rPiA_h = R(0.5) * rPiA;
    const R PiPa = hydro ? A.Pi * A.P : R(0);  // Pi_a P_a (the FP32 path's F and du)
    // force-type sums: plain per lane (a few tens of terms), FP64 over lanes
    SumAcc<R> dv[3], du, drho, ddt, db[3];
    for (int d = 0; d < 3; ++d) { dv[d].init(); db[d].init(); }
    du.init(); drho.init(); ddt.init();

    // ---- per-centre set-up of the general path ----
    PartX<R> AX;
    R kta[3][3], ktb[3][3], uba[3] = {R(0), R(0), R(0)}, ubb[3] = {R(0), R(0), R(0)};
    R halfB2a = R(0);
    const R mu0inv = R(1.0 / P.muzero);
    if constexpr (GENERAL) {
      Loader<R>::extra(pb, k, AX);
      for (int x = 0; x < 3; ++x)
        for (int y = 0; y < 3; ++y) { kta[x][y] = R(0); ktb[x][y] = R(0); }
      R b2 = AX.bx * AX.bx + AX.by * AX.by + AX.bz * AX.bz;
      halfB2a = R(0.5) * b2;
      if (b2 != R(0)) {
        R ib = frsqrt<R>(b2);
        uba[0] = AX.bx * ib; uba[1] = AX.by * ib; uba[2] = AX.bz * ib;
      }
      if (P.eq_diff) {
        if (P.eq_fld) {
          R lam;
          R gn = my_sqrt<R>(AX.gx * AX.gx + AX.gy * AX.gy + AX.gz * AX.gz);
          R fd = fld_coef<R>(gn, AX.kappa, A.rho, AX.T, lam);
          kta[0][0] = kta[1][1] = kta[2][2] = fd;
          if (lane == 0)
            cols[es_vfld * ld + p] = double(fd) / ((double(AX.T) * double(A.rho)) / double(gn));
        } else if (P.difiso == 1) {
          R dc = R(P.difcond);
          kta[0][0] = kta[1][1] = kta[2][2] = dc;
          ktb[0][0] = ktb[1][1] = ktb[2][2] = dc;
        } else {
          aniso_tensor<R>(R(P.difcond), uba, P.full_tensor, kta);
        }
      }
    }
    R kga[3] = {R(0), R(0), R(0)};  // K_a grad T_a
    if constexpr (GENERAL) {
      if (P.eq_diff) {
        const R ga3[3] = {AX.gx, AX.gy, AX.gz};
        for (int x = 0; x < 3; ++x) kga[x] = kta[x][0] * ga3[0] + kta[x][1] * ga3[1] + kta[x][2] * ga3[2];
      }
    }

    bool bad = false;
    const int n = a.ncnt[c];
    const int32_t* __restrict__ row = a.nl + a.rowoff[c];
    // the next neighbour's index is read one round ahead, so that a round
    // waits on one dependent load (the neighbour's streams), not two
    int32_t jnext = lane < n ? row[lane] : 0;
    for (int l0 = lane; l0 < n; l0 += G) {
    {
      const int64_t j = jnext;
      Part<R> B;
      Loader<R>::hydro(pb, j, B);
      if (l0 + G < n) jnext = row[l0 + G];
      R rab[3];
      pos_delta(A.pos, B.pos, rab[0], rab[1], rab[2]);
      R r2 = rab[0] * rab[0];
      if (DIM >= 2) r2 += rab[1] * rab[1];
      if (DIM == 3) r2 += rab[2] * rab[2];
      const R invr = frsqrt<R>(r2);
      const R r = r2 * invr;
      const R vab[3] = {A.vx - B.vx, A.vy - B.vy, A.vz - B.vz};
      R vr = vab[0] * rab[0];
      if (DIM >= 2) vr += vab[1] * rab[1];
      if (DIM == 3) vr += vab[2] * rab[2];
      const R qa = r * A.invh, qb = r * B.invh;
      bad |= !(qa >= R(0)) || !(qb >= R(0));
      R fa = R(0), dfa, ddfa = R(0);
      if constexpr (GENERAL) {
        if (P.eq_diff && (P.ddw == esd_n2w || P.ddw == esd_fw)) kshape_all<K, R>(qa, fa, dfa, ddfa);
        else dfa = kshape_df<K, R>(qa);
      } else {
        dfa = kshape_df<K, R>(qa);
      }
      const R dfb = kshape_df<K, R>(qb);
      const R ga = (Ka * invr) * dfa;  // nabla W_a = ga * r_ab
      // nabla W_b = gb r_ab, which always meets Pi_b: gbPi = gb Pi_b, and
      // cbr = wCv f'_b rho_b Pi_b / h_b^(d+1) for the conductivity.  The FP32
      // record carries wCv Pi_b / h_b^(d+1) (a product formed in FP64 when
      // packed, five products per pair fewer); FP64 forms them per pair.
      R gb = R(0), gbPi, cbr;
      if constexpr (sizeof(R) == 4) {
        gbPi = (B.Pi * invr) * dfb;
        cbr = (B.Pi * dfb) * B.hrho;  // half of it: the conductivity's 1/2 is folded in
      } else {
        R Kb = B.invh;
        for (int d = 0; d < DIM; ++d) Kb *= B.invh;
        Kb *= wcv;
        gb = (Kb * invr) * dfb;
        gbPi = gb * B.Pi;
        cbr = Kb * dfb * B.rho * B.Pi;
      }
      // the neighbour's term gb x Pi_b of the general path
      auto gbx = [&](R x) {
        if constexpr (sizeof(R) == 4) return gbPi * x;
        else return gb * x * B.Pi;
      };
      const R mb = B.m;
      const R mgv = mb * ga * vr;      // m_b nabla W_a . v_ab
      if (adden) drho.add(mgv);        // circuit2.f90:265-267
      // F = ga Pi_a Fa + gb Pi_b Fb (dv -= mb F r_ab); du += mgv Pi_a Da.
      // With faba = Ka f'_a = ga r the viscous heating
      // mb dvr qav faba / (rho_a Omega_a) of circuit2.f90:329-334 is
      // mgv Pi_a (qav rho_a), and the pressure work of :343-344 is
      // mgv Pi_a P_a.
      R Fa = R(0), Fb = R(0), Da = R(0);
      R FaPi = PiPa, DaPi = PiPa;  // FP32: Pi_a Fa and Pi_a Da, Pi_a folded in
      if (artts) {
        // circuit2.f90:294-336; the Monaghan switch dvr < 0 as a clamp
        const R dvr = vr * invr;
        const R dneg = dvr < R(0) ? dvr : R(0);
        const R qav = hrhoa * (alpha_ca - beta * dneg) * dneg;
        // (FP32: the record carries rho_b / 2 and alpha c_b; the halvings
        // are exact, so only alpha c_b is rounded differently)
        R hrhob, acb;
        if constexpr (sizeof(R) == 4) {
          hrhob = B.hrho;
          acb = B.ac;
        } else {
          hrhob = R(0.5) * B.rho;
          acb = alpha * B.c;
        }
        const R qbv = (-hrhob) * (acb - beta * dneg) * dneg;
        Fa = qav;
        Fb = qbv;
        Da = qav * A.rho;
        FaPi = A.Pi * qav + PiPa;
        DaPi = qav * rPiA + PiPa;
        if (use_au) {
          const R faba = Ka * dfa;
          const R vsigu = fsqrt<R>(fdiv<R>(fabs(A.P - B.P), hrho_a + hrhob));
          if constexpr (sizeof(R) == 4)
            du.add(mb * (vsigu * (A.u - B.u) * (faba * rPiA_h + cbr)));  // (FP32 u is au u)
          else
            du.add(mb * (au * (vsigu * (A.u - B.u) * R(0.5) * (faba * rPiA + cbr))));
        }
      }
      if (hydro) {
        // circuit2.f90:338-345
        Fa += A.P;
        Fb += B.P;
        Da += A.P;
      }
      R F;
      if constexpr (sizeof(R) == 4) {
        F = ga * FaPi + gbPi * Fb;
        du.add(mgv * DaPi);
      } else {
        F = ga * A.Pi * Fa + gbPi * Fb;
        du.add(mgv * A.Pi * Da);
      }
      if constexpr (GENERAL) {
        PartX<R> BX;
        Loader<R>::extra(pb, j, BX);
        if (P.eq_diff) {
          // circuit2.f90:347-425
          if (P.eq_fld) {
            R lam;
            R gn = my_sqrt<R>(BX.gx * BX.gx + BX.gy * BX.gy + BX.gz * BX.gz);
            R fd = fld_coef<R>(gn, BX.kappa, B.rho, BX.T, lam);
            for (int x = 0; x < 3; ++x)
              for (int y = 0; y < 3; ++y) ktb[x][y] = (x == y) ? fd : R(0);
          } else if (P.difiso == 0) {
            R b2 = BX.bx * BX.bx + BX.by * BX.by + BX.bz * BX.bz;
            if (b2 != R(0)) {  // a zero B_b keeps the previous unit vector (:220-224)
              R ib = frsqrt<R>(b2);
              ubb[0] = BX.bx * ib; ubb[1] = BX.by * ib; ubb[2] = BX.bz * ib;
            }
            aniso_tensor<R>(R(P.difcond), ubb, P.full_tensor, ktb);
          }
          const int ddw = P.ddw;
          if (ddw == esd_fab || ddw == esd_fw || ddw == esd_n2w) {
            // K_bar : Hessian_a  (kernel.f90:377-539, circuit2.f90:390-397)
            R rr = R(0), tr = R(0);
            for (int x = 0; x < DIM; ++x) {
              tr += R(0.5) * (kta[x][x] + ktb[x][x]);
              for (int y = 0; y < DIM; ++y) rr += R(0.5) * (kta[x][y] + ktb[x][y]) * rab[x] * rab[y];
            }
            rr = rr * (invr * invr);
            R contr;
            if (ddw == esd_n2w) {
              contr = Ka * A.invh * ddfa * rr + ga * (tr - rr);
            } else {
              const R f2 = (ddw == esd_fab) ? -ga : R(0.5) * R(P.fwc) * Ka * A.invh * fa;
              contr = f2 * (R(DIM + 2) * rr - tr);
            }
            ddt.add(fdiv<R>(mb, B.rho * A.rho) * (BX.T * B.rho - AX.T * A.rho) * contr);
          } else {
            R kgb[3];
            const R gb3[3] = {BX.gx, BX.gy, BX.gz};
            for (int x = 0; x < 3; ++x) kgb[x] = ktb[x][0] * gb3[0] + ktb[x][1] * gb3[1] + ktb[x][2] * gb3[2];
            R ka_r = R(0), kb_r = R(0);
            for (int x = 0; x < DIM; ++x) { ka_r += kga[x] * rab[x]; kb_r += kgb[x] * rab[x]; }
            if (ddw == esd_2nw_ds) ddt.add(mb * (ga * ka_r * A.Pi + gbx(kb_r)));
            else ddt.add(mb * A.Pi * ga * (kb_r - ka_r));  // esd_2nw_sd
          }
        }
        if (P.eq_magneto) {
          // circuit2.f90:427-462
          const R Ba[3] = {AX.bx, AX.by, AX.bz}, Bb[3] = {BX.bx, BX.by, BX.bz};
          R Bar = R(0), Bbr = R(0);
          for (int x = 0; x < DIM; ++x) { Bar += Ba[x] * rab[x]; Bbr += Bb[x] * rab[x]; }
          const R halfB2b = R(0.5) * (Bb[0] * Bb[0] + Bb[1] * Bb[1] + Bb[2] * Bb[2]);
          for (int x = 0; x < 3; ++x) {
            const R rx = x < DIM ? rab[x] : R(0);
            const R ma_x = (halfB2a * rx - Ba[x] * Bar) * mu0inv;  // MPa . r_ab
            const R mb_x = (halfB2b * rx - Bb[x] * Bbr) * mu0inv;
            dv[x].add(-mb * (ga * ma_x * A.Pi + gbx(mb_x)));
            db[x].add(-mb * rPiA * ga * (vab[x] * Bar - Bb[x] * vr));
          }
        }
      }
      for (int d = 0; d < DIM; ++d) dv[d].add(-mb * F * rab[d]);
    }
    }
    if (bad) raise_status(a.status, SPH_ERR_Q_NAN);
    const double mref = a.mref;
    const double ax = group_sum<G>(dv[0].dval(), gmask);
    const double ay = DIM >= 2 || GENERAL ? group_sum<G>(dv[1].dval(), gmask) : 0.0;
    const double az = DIM == 3 || GENERAL ? group_sum<G>(dv[2].dval(), gmask) : 0.0;
    const double dus = group_sum<G>(du.dval(), gmask);
    const double drs = group_sum<G>(drho.dval(), gmask);
    double dts = 0.0, b0 = 0.0, b1 = 0.0, b2 = 0.0;
    if constexpr (GENERAL) {
      dts = group_sum<G>(ddt.dval(), gmask);
      b0 = group_sum<G>(db[0].dval(), gmask);
      b1 = group_sum<G>(db[1].dval(), gmask);
      b2 = group_sum<G>(db[2].dval(), gmask);
    }
    if (lane == 0) {
      pairs = n;
      cols[es_ax * ld + p] = mref * ax;
      cols[es_ay * ld + p] = mref * ay;
      cols[es_az * ld + p] = mref * az;
      cols[es_du * ld + p] = mref * dus;
      double dh = 0.;
      if (adden) {  // circuit2.f90:468-470
        const double ha = cols[es_h * ld + p];
        dh = -double(DIM) * ha * double(A.rho) * double(A.Pi) * (mref * drs);
      }
      cols[es_dh * ld + p] = dh;
      cols[es_ddt * ld + p] = mref * dts;
      cols[es_dbx * ld + p] = mref * b0;
      cols[es_dby * ld + p] = mref * b1;
      cols[es_dbz * ld + p] = mref * b2;
    }
  }
  unsigned long long wp = pairs;
  for (int o = 16; o > 0; o >>= 1) wp += __shfl_xor_sync(0xffffffffu, wp, o);
  if (wl == 0 && wp) atomicAdd(&a.dcnt[DC_C2_PAIRS], wp);
}

template <int K, int DIM, class R, bool GEN>
void run_g(const C2Args& a, const PackBufs& pb, const Params& P, cudaStream_t s) {
  switch (a.G) {
    case 4: k_c2<K, DIM, R, GEN, 4><<<nblocks(a.nc * 4), TPB, 0, s>>>(a, pb, P); break;
    case 8: k_c2<K, DIM, R, GEN, 8><<<nblocks(a.nc * 8), TPB, 0, s>>>(a, pb, P); break;
    case 16: k_c2<K, DIM, R, GEN, 16><<<nblocks(a.nc * 16), TPB, 0, s>>>(a, pb, P); break;
    default: k_c2<K, DIM, R, GEN, 32><<<nblocks(a.nc * 32), TPB, 0, s>>>(a, pb, P); break;
  }
}
template <int K, int DIM, class R>
void run(const C2Args& a, const PackBufs& pb, const Params& P, cudaStream_t s) {
  const bool general = P.eq_diff || P.eq_magneto;
  if (general) run_g<K, DIM, R, true>(a, pb, P, s);
  else run_g<K, DIM, R, false>(a, pb, P, s);
  note_launch();
}
template <int K, int DIM>
void run_prec(int prec, const C2Args& a, const PackBufs& pb, const Params& P, cudaStream_t s) {
  if (prec == SPH_PREC_FP64) run<K, DIM, double>(a, pb, P, s);
  else run<K, DIM, float>(a, pb, P, s);
}
template <int K>
void run_dim(int prec, int dim, const C2Args& a, const PackBufs& pb, const Params& P,
             cudaStream_t s) {
  if (dim == 3) run_prec<K, 3>(prec, a, pb, P, s);
  else if (dim == 2) run_prec<K, 2>(prec, a, pb, P, s);
  else run_prec<K, 1>(prec, a, pb, P, s);
}

}  // namespace

void launch_c2(int prec, int kernel, int dim, const C2Args& a, PackBufs pb, Params P,
               cudaStream_t s) {
  if (kernel == KM6) run_dim<KM6>(prec, dim, a, pb, P, s);
  else if (kernel == KM4) run_dim<KM4>(prec, dim, a, pb, P, s);
  else run_dim<KGAUSS>(prec, dim, a, pb, P, s);
}

}  // namespace sph
