// Adjoint (vector-Jacobian products) of one leapfrog step of the hydro path,
// for the gradient of a final-state misfit with respect to the initial
// velocities, energies, positions and the artificial-viscosity parameters;
// and of the diffusion path (fixed positions), with respect to the initial
// temperatures and the conductivity.
// No counterpart in the reference (its Fortran has no derivatives); the
// forward map differentiated here is exactly the engine's FP64 step for
// equations = hydro with the artificial viscosity of circuit2.f90:294-336
// (alpha, beta), the pressure force and energy terms of :338-345, the
// grad-h density of circuit1.f90:76-224 solved by Newton iteration, the
// adiabatic EOS of eos.f90:21-33 and the predictor / corrector of
// main.f90:323-362, taken with a fixed dt.
//
// The state of a step is (r, v, u, a, du); h follows r through the Newton
// solve, so it is not part of the state: at convergence h_a solves
//   g_a(h_a; r) = rho^(h_a; r) - m_a (hfac / h_a)^d = 0,
//   rho^(h; r) = sum_b m_b W(r_ab, h)   (self term included),
// rho_a = m_a (hfac / h_a)^d and Omega_a = 1 + h_a S_a / (d rho_a) with
// S_a = d rho^ / dh.  The adjoint of h follows from the implicit function
// theorem: dg/dh = d rho_a Omega_a / h_a.
//
// Pair terms of the force pass, with x = r_a - r_b, r = |x|, v = v_a - v_b,
// w = v.x, s = w / r, g_a = K_a f'(r/h_a) / r, K_a = wCv / h_a^(d+1),
// Pi_a = 1 / (rho_a^2 Omega_a), dn = min(s, 0),
// q_a = -rho_a (alpha c_a - beta dn) dn / 2:
//   a_a  += -m_b F x,  F = (q_a + P_a) g_a Pi_a + (q_b + P_b) g_b Pi_b
//   du_a +=  m_b g_a w Pi_a (q_a rho_a + P_a)
// Every partial derivative below is taken of these expressions.
#include <cuda_runtime.h>

#include "sph_abi.h"
#include "sph_device.cuh"
#include "sph_internal.h"

namespace sph {
namespace {

constexpr int TPB = 128;

inline int nblocks(int64_t n, int tpb = TPB) { return int((n + tpb - 1) / tpb); }

// sum over the G lanes of a group; only that group's lanes take part
template <int G>
__device__ __forceinline__ double gsum(double v) {
  const int wl = threadIdx.x & 31;
  const unsigned m = (G == 32) ? 0xffffffffu : (((1u << G) - 1u) << (wl & ~(G - 1)));
#pragma unroll
  for (int o = G / 2; o > 0; o >>= 1) v += __shfl_xor_sync(m, v, o);
  return v;
}

// W and its derivatives in r and h for the Newton-h adjoint:
//   dW/dr = wCv f' / h^(d+1)
//   d2W/dh dr = -wCv ((d+1) f' + q f'') / h^(d+2)
//   d2W/dh2 = wCv ((d+1) d f + 2 (d+1) q f' + q^2 f'') / h^(d+2)
template <int K, int DIM>
__device__ __forceinline__ void w_derivs(double r, double h, double wcv, double& dwdr,
                                         double& dwdhdr, double& dwdh2) {
  const double q = r / h;
  double f, df, ddf;
  kshape_all<K, double>(q, f, df, ddf);
  const double ih = 1.0 / h;
  const double k1 = wcv * ipow<DIM + 1>(ih);
  const double k2 = k1 * ih;
  dwdr = k1 * df;
  dwdhdr = -k2 * ((DIM + 1) * df + q * ddf);
  dwdh2 = k2 * ((DIM + 1) * DIM * f + 2.0 * (DIM + 1) * q * df + q * q * ddf);
}

// per-row column of the adjoint buffer
__device__ __forceinline__ double& AJ(const AdjArgs& a, int col, int64_t p) {
  return a.adj[int64_t(col) * a.ld + p];
}

// ---- VJP of the force pass (circuit2 hydro + AV) ------------------------------------------
template <int K, int DIM, int G>
__global__ void __launch_bounds__(TPB)
k_adj_c2(AdjArgs a) {
  const int64_t c = (blockIdx.x * int64_t(blockDim.x) + threadIdx.x) / G;
  const int lane = threadIdx.x & (G - 1);
  double gpar0 = 0.0, gpar1 = 0.0;
  if (c < a.nc) {
    const int64_t k = a.centre_k[c];
    const int64_t pa = a.centre_p[c];
    const double* cols = a.cols;
    const int64_t ld = a.ld;
    auto CA = [&](int f) { return cols[f * ld + pa]; };
    const double xa[3] = {a.sx[k], a.sy[k], a.sz[k]};
    const double va[3] = {CA(es_vx), CA(es_vy), CA(es_vz)};
    const double ha = CA(es_h), rhoa = CA(es_den), oma = CA(es_om), Pa = CA(es_p), ca = CA(es_c);
    const double Pia = 1.0 / (rhoa * rhoa * oma);
    const double Ka = a.wcv * ipow<DIM + 1>(1.0 / ha);
    const double Lam[3] = {AJ(a, AJ_LA, pa), AJ(a, AJ_LA + 1, pa), AJ(a, AJ_LA + 2, pa)};
    const double L = AJ(a, AJ_LDU, pa);
    const double al = a.alpha, be = a.beta;
    // a-side sums of this lane
    double gr[3] = {0, 0, 0}, gv[3] = {0, 0, 0};
    double gh = 0, grho = 0, gom = 0, gP = 0, gc = 0;
    const int n = a.ncnt[c];
    const int32_t* __restrict__ row = a.nl + a.rowoff[c];
    for (int l = lane; l < n; l += G) {
      const int64_t j = row[l];
      const int64_t pb = a.ssrc[j];
      auto CB = [&](int f) { return cols[f * ld + pb]; };
      double x[3] = {xa[0] - a.sx[j], xa[1] - a.sy[j], xa[2] - a.sz[j]};
      double v[3] = {va[0] - CB(es_vx), va[1] - CB(es_vy), va[2] - CB(es_vz)};
      double r2 = 0.0, w = 0.0, E = 0.0;
      for (int d = 0; d < DIM; ++d) { r2 += x[d] * x[d]; w += v[d] * x[d]; E += Lam[d] * x[d]; }
      const double r = sqrt(r2);
      const double invr = 1.0 / r;
      const double s = w * invr;
      const double mb = CB(es_m);
      const double hb = CB(es_h), rhob = CB(es_den), omb = CB(es_om), Pb = CB(es_p), cb = CB(es_c);
      const double Pib = 1.0 / (rhob * rhob * omb);
      const double Kb = a.wcv * ipow<DIM + 1>(1.0 / hb);
      double fa, dfa, ddfa, fb, dfb, ddfb;
      kshape_all<K, double>(r / ha, fa, dfa, ddfa);
      kshape_all<K, double>(r / hb, fb, dfb, ddfb);
      const double ga = Ka * dfa * invr, gb = Kb * dfb * invr;
      const bool neg = s < 0.0;
      const double dn = neg ? s : 0.0;
      double qa = 0, qb = 0;
      if (a.artts) {
        qa = -0.5 * rhoa * (al * ca - be * dn) * dn;
        qb = -0.5 * rhob * (al * cb - be * dn) * dn;
      }
      const double Aa = qa + (a.hydro ? Pa : 0.0), Ab = qb + (a.hydro ? Pb : 0.0);
      const double F = Aa * ga * Pia + Ab * gb * Pib;
      const double D = (a.artts ? qa * rhoa : 0.0) + (a.hydro ? Pa : 0.0);
      // J = mb (-F E + ga w Pia D L)
      const double dJ_dE = -mb * F;
      const double dJ_dF = -mb * E;
      const double JD = mb * ga * w * Pia * L;
      const double dJ_dga = dJ_dF * Aa * Pia + mb * w * Pia * D * L;
      const double dJ_dgb = dJ_dF * Ab * Pib;
      const double dJ_dqa = dJ_dF * ga * Pia + JD * rhoa;
      const double dJ_dqb = dJ_dF * gb * Pib;
      const double dJ_dPa = a.hydro ? dJ_dF * ga * Pia + JD : 0.0;
      const double dJ_dPb = a.hydro ? dJ_dF * gb * Pib : 0.0;
      const double dJ_dPia = dJ_dF * Aa * ga + mb * ga * w * D * L;
      const double dJ_dPib = dJ_dF * Ab * gb;
      double dJ_dw = mb * ga * Pia * D * L;
      double dJ_ds = 0.0;
      if (a.artts) {
        const double dqa_ddn = -0.5 * rhoa * (al * ca - 2.0 * be * dn);
        const double dqb_ddn = -0.5 * rhob * (al * cb - 2.0 * be * dn);
        if (neg) dJ_ds = dJ_dqa * dqa_ddn + dJ_dqb * dqb_ddn;
        grho += JD * qa + dJ_dqa * (-0.5 * (al * ca - be * dn) * dn);
        gc += dJ_dqa * (-0.5 * rhoa * al * dn);
        gpar0 += dJ_dqa * (-0.5 * rhoa * ca * dn) + dJ_dqb * (-0.5 * rhob * cb * dn);
        gpar1 += (dJ_dqa * rhoa + dJ_dqb * rhob) * (0.5 * dn * dn);
      }
      // ga(r, h_a) = K_a f'(r/h_a) / r
      const double dga_dr = Ka * invr * (ddfa / ha - dfa * invr);
      const double dgb_dr = Kb * invr * (ddfb / hb - dfb * invr);
      const double dga_dh = -(DIM + 1) * ga / ha - Ka * ddfa / (ha * ha);
      const double dgb_dh = -(DIM + 1) * gb / hb - Kb * ddfb / (hb * hb);
      const double dJ_dr = dJ_dga * dga_dr + dJ_dgb * dgb_dr - dJ_ds * w * invr * invr;
      dJ_dw += dJ_ds * invr;
      double lx[3], lv[3];
      for (int d = 0; d < 3; ++d) {
        lx[d] = d < DIM ? dJ_dE * Lam[d] + dJ_dr * x[d] * invr + dJ_dw * v[d] : 0.0;
        lv[d] = d < DIM ? dJ_dw * x[d] : 0.0;
        gr[d] += lx[d];
        gv[d] += lv[d];
      }
      gh += dJ_dga * dga_dh;
      grho += dJ_dPia * (-2.0 * Pia / rhoa);
      gom += dJ_dPia * (-Pia / oma);
      gP += dJ_dPa;
      // b side
      double* adj = a.adj;
      for (int d = 0; d < DIM; ++d) {
        atomicAdd(&adj[int64_t(AJ_GR + d) * ld + pb], -lx[d]);
        atomicAdd(&adj[int64_t(AJ_GV + d) * ld + pb], -lv[d]);
      }
      atomicAdd(&adj[int64_t(AJ_GH) * ld + pb], dJ_dgb * dgb_dh);
      double grb = dJ_dPib * (-2.0 * Pib / rhob);
      if (a.artts) grb += dJ_dqb * (-0.5 * (al * cb - be * dn) * dn);
      atomicAdd(&adj[int64_t(AJ_GRHO) * ld + pb], grb);
      atomicAdd(&adj[int64_t(AJ_GOM) * ld + pb], dJ_dPib * (-Pib / omb));
      if (a.hydro) atomicAdd(&adj[int64_t(AJ_GP) * ld + pb], dJ_dPb);
      if (a.artts) atomicAdd(&adj[int64_t(AJ_GC) * ld + pb], dJ_dqb * (-0.5 * rhob * al * dn));
    }
    // a side: the group's sums, written by lane 0
    for (int d = 0; d < DIM; ++d) { gr[d] = gsum<G>(gr[d]); gv[d] = gsum<G>(gv[d]); }
    gh = gsum<G>(gh); grho = gsum<G>(grho); gom = gsum<G>(gom); gP = gsum<G>(gP); gc = gsum<G>(gc);
    if (lane == 0) {
      double* adj = a.adj;
      for (int d = 0; d < DIM; ++d) {
        atomicAdd(&adj[int64_t(AJ_GR + d) * ld + pa], gr[d]);
        atomicAdd(&adj[int64_t(AJ_GV + d) * ld + pa], gv[d]);
      }
      atomicAdd(&adj[int64_t(AJ_GH) * ld + pa], gh);
      atomicAdd(&adj[int64_t(AJ_GRHO) * ld + pa], grho);
      atomicAdd(&adj[int64_t(AJ_GOM) * ld + pa], gom);
      atomicAdd(&adj[int64_t(AJ_GP) * ld + pa], gP);
      atomicAdd(&adj[int64_t(AJ_GC) * ld + pa], gc);
    }
  } else {
    (void)lane;
  }
  // viscosity parameters: one atomic per warp
  for (int o = 16; o > 0; o >>= 1) {
    gpar0 += __shfl_xor_sync(0xffffffffu, gpar0, o);
    gpar1 += __shfl_xor_sync(0xffffffffu, gpar1, o);
  }
  if ((threadIdx.x & 31) == 0 && (gpar0 != 0.0 || gpar1 != 0.0)) {
    atomicAdd(&a.gpar[0], gpar0);
    atomicAdd(&a.gpar[1], gpar1);
  }
}

// ---- S'_a = d2 rho^ / dh2 at h_a (self term included) -------------------------------------
template <int K, int DIM, int G>
__global__ void __launch_bounds__(TPB)
k_adj_c1_sum(AdjArgs a) {
  const int64_t c = (blockIdx.x * int64_t(blockDim.x) + threadIdx.x) / G;
  const int lane = threadIdx.x & (G - 1);
  if (c >= a.nc) return;  // whole groups leave together
  const int64_t k = a.centre_k[c];
  const int64_t pa = a.centre_p[c];
  const double ha = a.cols[es_h * a.ld + pa];
  const double xa[3] = {a.sx[k], a.sy[k], a.sz[k]};
  double sp = 0.0;
  const int n = a.ncnt[c];
  const int32_t* __restrict__ row = a.nl + a.rowoff[c];
  for (int l = lane; l < n; l += G) {
    const int64_t j = row[l];
    double x[3] = {xa[0] - a.sx[j], xa[1] - a.sy[j], xa[2] - a.sz[j]};
    double r2 = 0.0;
    for (int d = 0; d < DIM; ++d) r2 += x[d] * x[d];
    double dwdr, dwdhdr, dwdh2;
    w_derivs<K, DIM>(sqrt(r2), ha, a.wcv, dwdr, dwdhdr, dwdh2);
    sp += a.cols[es_m * a.ld + a.ssrc[j]] * dwdh2;
  }
  sp = gsum<G>(sp);
  if (lane == 0) {
    double dwdr, dwdhdr, dwdh2;
    w_derivs<K, DIM>(0.0, ha, a.wcv, dwdr, dwdhdr, dwdh2);
    AJ(a, AJ_SP, pa) = sp + a.cols[es_m * a.ld + pa] * dwdh2;
  }
}

// ---- per particle: EOS adjoint and the adjoint of h ---------------------------------------
__global__ void k_adj_particle(AdjArgs a, int dim) {
  const int64_t p = blockIdx.x * int64_t(blockDim.x) + threadIdx.x;
  if (p >= a.nreal) return;
  const double* cols = a.cols;
  const int64_t ld = a.ld;
  const double h = cols[es_h * ld + p], rho = cols[es_den * ld + p], om = cols[es_om * ld + p];
  const double u = cols[es_u * ld + p], cs = cols[es_c * ld + p];
  const double g1 = a.gamma - 1.0;
  // P = (gamma - 1) rho u; c = sqrt(gamma (gamma - 1) u)
  double grho = AJ(a, AJ_GRHO, p) + g1 * u * AJ(a, AJ_GP, p);
  double gu = g1 * rho * AJ(a, AJ_GP, p);
  if (cs > 0.0) gu += AJ(a, AJ_GC, p) * a.gamma * g1 / (2.0 * cs);
  AJ(a, AJ_GU, p) = gu;
  // Omega = 1 + h S / (d rho), S = (Omega - 1) d rho / h, rho = m (hfac / h)^d
  const double S = (om - 1.0) * dim * rho / h;
  const double Sp = AJ(a, AJ_SP, p);
  const double gom = AJ(a, AJ_GOM, p);
  const double dom_dh = S / (dim * rho) + h * Sp / (dim * rho) + S / rho;
  const double gh = AJ(a, AJ_GH, p) + gom * dom_dh + grho * (-dim * rho / h);
  AJ(a, AJ_MU, p) = gh / (dim * rho * om / h);
  AJ(a, AJ_WC, p) = gom * h / (dim * rho);
}

// ---- r-adjoint of h and Omega through the density sums ------------------------------------
template <int K, int DIM, int G>
__global__ void __launch_bounds__(TPB)
k_adj_c1_scatter(AdjArgs a) {
  const int64_t c = (blockIdx.x * int64_t(blockDim.x) + threadIdx.x) / G;
  const int lane = threadIdx.x & (G - 1);
  if (c >= a.nc) return;
  const int64_t k = a.centre_k[c];
  const int64_t pa = a.centre_p[c];
  const int64_t ld = a.ld;
  const double ha = a.cols[es_h * ld + pa];
  const double mu = AJ(a, AJ_MU, pa), wc = AJ(a, AJ_WC, pa);
  const double xa[3] = {a.sx[k], a.sy[k], a.sz[k]};
  double gr[3] = {0, 0, 0};
  const int n = a.ncnt[c];
  const int32_t* __restrict__ row = a.nl + a.rowoff[c];
  for (int l = lane; l < n; l += G) {
    const int64_t j = row[l];
    const int64_t pb = a.ssrc[j];
    double x[3] = {xa[0] - a.sx[j], xa[1] - a.sy[j], xa[2] - a.sz[j]};
    double r2 = 0.0;
    for (int d = 0; d < DIM; ++d) r2 += x[d] * x[d];
    const double r = sqrt(r2);
    double dwdr, dwdhdr, dwdh2;
    w_derivs<K, DIM>(r, ha, a.wcv, dwdr, dwdhdr, dwdh2);
    const double coef = a.cols[es_m * ld + pb] * (wc * dwdhdr - mu * dwdr) / r;
    for (int d = 0; d < DIM; ++d) {
      const double lx = coef * x[d];
      gr[d] += lx;
      atomicAdd(&a.adj[int64_t(AJ_GR + d) * ld + pb], -lx);
    }
  }
  for (int d = 0; d < DIM; ++d) gr[d] = gsum<G>(gr[d]);
  if (lane == 0)
    for (int d = 0; d < DIM; ++d) atomicAdd(&a.adj[int64_t(AJ_GR + d) * ld + pa], gr[d]);
}

// ---- VJP of the diffusion term (circuit2.f90:347-397, fab / fw / n2w) -----------------------
// dT_a/dt = sum_b w_ab (T_b rho_b - T_a rho_a),  w_ab = m_b / (rho_a rho_b) c_ab,
// c_ab the kernel.f90:377-539 contraction K_bar : Hessian_a, linear in the
// conductivity (K = difcond I, or difcond times the b-field's diagonal or
// full b b^T).  With positions fixed the map T -> dT/dt is linear, so
//   dT_a/dt's adjoint mu_a adds  -mu_a rho_a sum_b w_ab  to T_a and
//   mu_a w_ab rho_b  to T_b (the source row of an image), and
//   mu_a dT_a/dt / difcond  to the conductivity.
__device__ __forceinline__ void tensor3(double dc, const double* ub, int full, double K[3][3]) {
  for (int x = 0; x < 3; ++x)
    for (int y = 0; y < 3; ++y) K[x][y] = (x == y || full) ? dc * ub[x] * ub[y] : 0.0;
}

template <int K, int DIM, int G>
__global__ void __launch_bounds__(TPB)
k_adj_diff(AdjArgs a) {
  const int64_t c = (blockIdx.x * int64_t(blockDim.x) + threadIdx.x) / G;
  const int lane = threadIdx.x & (G - 1);
  double gdc = 0.0;
  if (c < a.nc) {
    const int64_t k = a.centre_k[c];
    const int64_t pa = a.centre_p[c];
    const double* cols = a.cols;
    const int64_t ld = a.ld;
    auto CA = [&](int f) { return cols[f * ld + pa]; };
    const double xa[3] = {a.sx[k], a.sy[k], a.sz[k]};
    const double iha = 1.0 / CA(es_h), rhoa = CA(es_den);
    double Ka = iha;
    for (int d = 0; d < DIM; ++d) Ka *= iha;
    Ka *= a.wcv;
    const double mu = AJ(a, AJ_LDT, pa);
    const double dc = a.difcond;
    double kta[3][3], ktb[3][3], uba[3] = {0, 0, 0}, ubb[3] = {0, 0, 0};
    const double Ba[3] = {CA(es_bx), CA(es_by), CA(es_bz)};
    const double b2a = Ba[0] * Ba[0] + Ba[1] * Ba[1] + Ba[2] * Ba[2];
    if (b2a != 0.0) {
      const double ib = 1.0 / sqrt(b2a);
      for (int x = 0; x < 3; ++x) uba[x] = Ba[x] * ib;
    }
    const double one[3] = {1.0, 1.0, 1.0};
    if (a.difiso == 1) {
      tensor3(dc, one, 0, kta);
      tensor3(dc, one, 0, ktb);
    } else {
      tensor3(dc, uba, a.full_tensor, kta);
    }
    double diag = 0.0;
    const int n = a.ncnt[c];
    const int32_t* __restrict__ row = a.nl + a.rowoff[c];
    for (int l = lane; l < n; l += G) {
      const int64_t j = row[l];
      const int64_t pb = a.ssrc[j];
      auto CB = [&](int f) { return cols[f * ld + pb]; };
      const double x[3] = {xa[0] - a.sx[j], xa[1] - a.sy[j], xa[2] - a.sz[j]};
      double r2 = x[0] * x[0];
      if (DIM >= 2) r2 += x[1] * x[1];
      if (DIM == 3) r2 += x[2] * x[2];
      const double invr = 1.0 / sqrt(r2);
      const double r = r2 * invr;
      double fa, dfa, ddfa;
      kshape_all<K, double>(r * iha, fa, dfa, ddfa);
      const double ga = (Ka * invr) * dfa;
      if (a.difiso == 0) {
        const double Bb[3] = {CB(es_bx), CB(es_by), CB(es_bz)};
        const double b2 = Bb[0] * Bb[0] + Bb[1] * Bb[1] + Bb[2] * Bb[2];
        if (b2 != 0.0) {  // a zero B_b keeps the previous unit vector (circuit2.f90:220-224)
          const double ib = 1.0 / sqrt(b2);
          for (int q = 0; q < 3; ++q) ubb[q] = Bb[q] * ib;
        }
        tensor3(dc, ubb, a.full_tensor, ktb);
      }
      double rr = 0.0, tr = 0.0;
      for (int p = 0; p < DIM; ++p) {
        tr += 0.5 * (kta[p][p] + ktb[p][p]);
        for (int q = 0; q < DIM; ++q) rr += 0.5 * (kta[p][q] + ktb[p][q]) * x[p] * x[q];
      }
      rr = rr * (invr * invr);
      double contr;
      if (a.ddw == esd_n2w) {
        contr = Ka * iha * ddfa * rr + ga * (tr - rr);
      } else {
        const double f2 = (a.ddw == esd_fab) ? -ga : 0.5 * a.fwc * Ka * iha * fa;
        contr = f2 * (double(DIM + 2) * rr - tr);
      }
      const double rhob = CB(es_den);
      const double w = CB(es_m) / (rhob * rhoa) * contr;
      diag += w;
      atomicAdd(&AJ(a, AJ_GT, pb), mu * w * rhob);
    }
    diag = gsum<G>(diag);
    if (lane == 0) {
      atomicAdd(&AJ(a, AJ_GT, pa), -mu * rhoa * diag);
      if (dc != 0.0) gdc = mu * CA(es_ddt) / dc;
    }
  }
  for (int o = 16; o > 0; o >>= 1) gdc += __shfl_xor_sync(0xffffffffu, gdc, o);
  if ((threadIdx.x & 31) == 0 && gdc != 0.0) atomicAdd(&a.gpar[2], gdc);
}

// ---- step adjoints -------------------------------------------------------------------------
// before the force VJP: the adjoints of the new a, du and zeroed sums
__global__ void k_adj_prep(AdjArgs a, double dt, int first) {
  const int64_t p = blockIdx.x * int64_t(blockDim.x) + threadIdx.x;
  if (p >= a.nreal) return;
  const double hdt = 0.5 * dt;
  for (int d = 0; d < 3; ++d)
    AJ(a, AJ_LA + d, p) = AJ(a, AJ_LAS + d, p) + (first ? 0.0 : hdt * AJ(a, AJ_LV + d, p));
  AJ(a, AJ_LDU, p) = AJ(a, AJ_LDUS, p) + (first ? 0.0 : hdt * AJ(a, AJ_LU, p));
  for (int col = AJ_GR; col <= AJ_GU; ++col) AJ(a, col, p) = 0.0;
  if (a.diff) {  // T follows u's integrator (main.f90:323-362)
    AJ(a, AJ_LDT, p) = AJ(a, AJ_LDTS, p) + (first ? 0.0 : hdt * AJ(a, AJ_LT, p));
    AJ(a, AJ_GT, p) = 0.0;
  }
}

// after it: back through the corrector and the predictor (main.f90:323-362)
//   r' = r + dt v + dt^2 a / 2, v' = v + dt a, u' = u + dt du
//   v'' = v' + dt (a_new - a) / 2, u'' = u' + dt (du_new - du) / 2
// or, for the first force evaluation (first = 1), only add the VJP.
__global__ void k_adj_integrate(AdjArgs a, double dt, int first) {
  const int64_t p = blockIdx.x * int64_t(blockDim.x) + threadIdx.x;
  if (p >= a.nreal) return;
  if (first) {
    for (int d = 0; d < 3; ++d) {
      AJ(a, AJ_LR + d, p) += AJ(a, AJ_GR + d, p);
      AJ(a, AJ_LV + d, p) += AJ(a, AJ_GV + d, p);
      AJ(a, AJ_LAS + d, p) = 0.0;
    }
    AJ(a, AJ_LU, p) += AJ(a, AJ_GU, p);
    AJ(a, AJ_LDUS, p) = 0.0;
    if (a.diff) {
      AJ(a, AJ_LT, p) += AJ(a, AJ_GT, p);
      AJ(a, AJ_LDTS, p) = 0.0;
    }
    return;
  }
  const double hdt = 0.5 * dt;
  for (int d = 0; d < 3; ++d) {
    const double lr1 = AJ(a, AJ_LR + d, p) + AJ(a, AJ_GR + d, p);  // adjoint of r'
    const double lv0 = AJ(a, AJ_LV + d, p);                         // adjoint of v''
    const double lv1 = lv0 + AJ(a, AJ_GV + d, p);                   // adjoint of v'
    AJ(a, AJ_LR + d, p) = lr1;
    AJ(a, AJ_LV + d, p) = lv1 + dt * lr1;
    AJ(a, AJ_LAS + d, p) = -hdt * lv0 + hdt * dt * lr1 + dt * lv1;
  }
  const double lu0 = AJ(a, AJ_LU, p);
  const double lu1 = lu0 + AJ(a, AJ_GU, p);
  AJ(a, AJ_LU, p) = lu1;
  AJ(a, AJ_LDUS, p) = -hdt * lu0 + dt * lu1;
  if (a.diff) {
    const double lt0 = AJ(a, AJ_LT, p);
    const double lt1 = lt0 + AJ(a, AJ_GT, p);
    AJ(a, AJ_LT, p) = lt1;
    AJ(a, AJ_LDTS, p) = -hdt * lt0 + dt * lt1;
  }
}

template <int K, int DIM, int G>
void adj_pairs_g(const AdjArgs& a, cudaStream_t s) {
  const int nb = nblocks(a.nc * G);
  if (a.diff) {  // positions fixed: only the diffusion term depends on the state
    k_adj_diff<K, DIM, G><<<nb, TPB, 0, s>>>(a);
    note_launch();
    return;
  }
  k_adj_c2<K, DIM, G><<<nb, TPB, 0, s>>>(a);
  k_adj_c1_sum<K, DIM, G><<<nb, TPB, 0, s>>>(a);
  k_adj_particle<<<nblocks(a.nreal), TPB, 0, s>>>(a, DIM);
  k_adj_c1_scatter<K, DIM, G><<<nb, TPB, 0, s>>>(a);
  note_launch(4);
}
template <int K, int DIM>
void adj_pairs_k(int G, const AdjArgs& a, cudaStream_t s) {
  if (G == 4) adj_pairs_g<K, DIM, 4>(a, s);
  else adj_pairs_g<K, DIM, 8>(a, s);
}
template <int K>
void adj_pairs_d(int dim, int G, const AdjArgs& a, cudaStream_t s) {
  if (dim == 1) adj_pairs_k<K, 1>(G, a, s);
  else if (dim == 2) adj_pairs_k<K, 2>(G, a, s);
  else adj_pairs_k<K, 3>(G, a, s);
}

// rows in the caller's order (ncomp per row) <-> ncomp columns of ld rows
__global__ void k_adj_gather(const double* __restrict__ in, int ncomp,
                             const int32_t* __restrict__ orig, int64_t n,
                             double* __restrict__ out, int64_t ld) {
  const int64_t p = blockIdx.x * int64_t(blockDim.x) + threadIdx.x;
  if (p >= n) return;
  for (int d = 0; d < ncomp; ++d) out[d * ld + p] = in[int64_t(orig[p]) * ncomp + d];
}
__global__ void k_adj_scatter(const double* __restrict__ in, int64_t ld,
                              const int32_t* __restrict__ orig, int64_t n,
                              double* __restrict__ out, int ncomp) {
  const int64_t p = blockIdx.x * int64_t(blockDim.x) + threadIdx.x;
  if (p >= n) return;
  for (int d = 0; d < ncomp; ++d) out[int64_t(orig[p]) * ncomp + d] = in[d * ld + p];
}

}  // namespace

void launch_adj_gather(const double* in, int ncomp, const int32_t* orig, int64_t n, double* out,
                       int64_t ld, cudaStream_t s) {
  k_adj_gather<<<nblocks(n), TPB, 0, s>>>(in, ncomp, orig, n, out, ld);
  note_launch();
}
void launch_adj_scatter(const double* in, int64_t ld, const int32_t* orig, int64_t n,
                        double* out, int ncomp, cudaStream_t s) {
  k_adj_scatter<<<nblocks(n), TPB, 0, s>>>(in, ld, orig, n, out, ncomp);
  note_launch();
}

void launch_adj_step(int kernel, int dim, int G, const AdjArgs& a, double dt, int first,
                     cudaStream_t s) {
  k_adj_prep<<<nblocks(a.nreal), TPB, 0, s>>>(a, dt, first);
  if (kernel == SPH_KERNEL_M4) adj_pairs_d<KM4>(dim, G, a, s);
  else if (kernel == SPH_KERNEL_M6) adj_pairs_d<KM6>(dim, G, a, s);
  else adj_pairs_d<KGAUSS>(dim, G, a, s);
  k_adj_integrate<<<nblocks(a.nreal), TPB, 0, s>>>(a, dt, first);
  note_launch(2);
}

}  // namespace sph
