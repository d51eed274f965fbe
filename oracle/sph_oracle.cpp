/*
 * sph_oracle.cpp — CPU FP64 OpenMP restatement of the reference SPH step.
 *
 * TEST INFRASTRUCTURE ONLY.  This library is the parity oracle for the CUDA
 * engine and the timed CPU baseline; only tests/, __graft_entry__.smoke()
 * and bench.py's cpu_baseline / --impl reference legs load it.  The product
 * path (libsph.so) never links or calls it.
 *
 * Parity pinning: the reference (Fortran 2008, gfortran + HDF5) cannot be
 * built in this image, and its sources hold no per-particle golden vectors.
 * This restatement is pinned by (a) the reference's own STS coefficient
 * known-answer test (sts_integrator.f90:53-69), (b) brute-force O(N^2)
 * neighbour sets, (c) analytic kernel identities and (d) analytic solutions
 * (Sod exact Riemann, diffusion decay).  Per-particle parity is therefore
 * "partially pinned": the formulas below follow the cited reference lines,
 * but no reference binary output checks them.
 *
 * It exports the same C-ABI as the engine (include/sph_abi.h) so a harness
 * can load either library.  Arithmetic follows the reference statement by
 * statement in FP64 without FMA contraction (build with -ffp-contract=off;
 * the reference's x86-64 build has no FMA either, playground/Makefile:92-93).
 *
 * Deliberate deviations (all switchable or documented):
 *  - the neighbour cap maxneibnum (kernel/base_m6.f90:16) is only enforced
 *    when SPH_P_NEIB_CAP_CHECK = 1 (3D M6 at hfac 1.2 overflows it);
 *  - AV alpha/beta and the Newton tolerance / iteration cap are parameters
 *    (defaults 1, 2, 1e-8, 100 as circuit2.f90:565-566, circuit1.f90:104,114);
 *  - SPH_P_FULL_TENSOR = 1 replaces the diagonal anisotropic tensor
 *    (circuit2.f90:203-205) by k_par * b b^T;
 *  - timestep.f90:40-166 leaves dthydro/dtdiff/dtfld undefined when their
 *    equation is off; here they are 0 / +inf / +inf;
 *  - the neighbour search is a uniform cell grid instead of the kd-tree
 *    (utils/kdtree2.f90); the inclusion predicate is the kd-tree's
 *    (kdtree2.f90:1673-1678) bit for bit.
 */
#include "../include/sph_abi.h"

#include <omp.h>

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <limits>
#include <functional>
#include <string>
#include <vector>

namespace {

// ---- enums (playground/src/const.f90) ------------------------------------
enum : int {
  ec_dim = 1, ec_eqs = 2, ec_ddw = 3, ec_ics = 4, ec_adden = 5, ec_artts = 6,
  ec_coordsys = 7, ec_disotropic = 8, ec_dcondconst = 9, ec_muzero = 10,
  ec_tfinish = 11, ec_npics = 12, ec_hfac = 13, ec_silent = 14,
  ec_resolution = 15, ec_spacing = 16, ec_xmin = 17, ec_xmax = 18,
  ec_ymin = 19, ec_ymax = 20, ec_zmin = 21, ec_zmax = 22, ec_bordsize = 23,
  ec_padding = 24, ec_realpn = 25, ec_fixedpn = 26, ec_gamma = 27,
  ec_lastprint = 28, ec_usedumps = 29, ec_dtprint = 30, ec_process = 31,
  ec_au = 32, ec_placement = 33, ec_eqonhydro = 34, ec_eqondiff = 35,
  ec_eqonfluxlim = 36, ec_eqonradexch = 37, ec_eqonsts = 38, ec_udist = 39,
  ec_umass = 40, ec_utime = 41, ec_uvelocity = 42, ec_udensity = 43,
  ec_upressure = 44, ec_uacceller = 45, ec_time = 46, ec_molecularmass = 47,
  ec_ststype = 48, ec_stsfixeds = 49
};
enum : int {  // 0-based store columns (const.f90:69-103 minus one)
  es_rx = 0, es_ry, es_rz, es_vx, es_vy, es_vz, es_ax, es_ay, es_az, es_m,
  es_den, es_h, es_dh, es_p, es_u, es_du, es_t, es_kappa, es_dtdx, es_dtdy,
  es_dtdz, es_ddt, es_bx, es_by, es_bz, es_dbx, es_dby, es_dbz, es_c, es_om,
  es_type, es_vfld
};
constexpr int ES = SPH_ES_TOTAL;
enum : int { ept_empty = 0, ept_real = 1, ept_fixed = 2, ept_fixedreal = 21,
             ept_fixedmirror = 22, ept_periodic = 3 };
enum : int { ett_sin3 = 100, ett_mti = 101, ett_shock12 = 102, ett_pulse = 103,
             ett_ring = 104, ett_soundwave = 105, ett_hydroshock = 106,
             ett_alfvenwave = 107, ett_OTvortex = 108, ett_boilingtank = 109,
             ett_mtilowres = 110, ett_fld_gauss = 111 };
enum : int { ebc_all = 200, ebc_x = 201, ebc_y = 202, ebc_z = 203 };
enum : int { eeq_hydro = 300, eeq_diffusion = 301, eeq_magnetohydro = 302,
             eeq_magnetohydrodiffusion = 303, eeq_hydrodiffusion = 304,
             eeq_kd2 = 305, eeq_hyrad = 306, eeq_manual = 307 };
enum : int { esd_fab = 400, esd_n2w = 401, esd_fw = 402, esd_2nw_ds = 403,
             esd_2nw_sd = 404 };
enum : int { epc_backcompatibility = 600, epc_fullyperiodic = 601,
             epc_borderless = 602 };
enum : int { ests_auto = 0, ests_fixeds = 1 };

const double pi = 4.0 * std::atan(1.0);             // const.f90:4
const double eps0 = std::numeric_limits<double>::epsilon();  // const.f90:5
const double lightspeed = 2.997924e10;              // const.f90:6
const double Rg = 8.314e7;                          // const.f90:7
const double sigmaB = 5.67051e-5;                   // const.f90:8

thread_local std::string g_err;

int fail(int code, const std::string& msg) {
  g_err = msg;
  return code;
}

// x**n for integer n: binary exponentiation, the same multiplication order
// gfortran uses for an integer power.
inline double powi(double x, int m) {
  unsigned n = m < 0 ? unsigned(-m) : unsigned(m);
  double y = (n % 2) ? x : 1.0;
  while (n >>= 1) {
    x = x * x;
    if (n % 2) y = y * x;
  }
  return m < 0 ? 1.0 / y : y;
}

// ---- kernel bases (kernel/base_m4.f90, base_m6.f90, base_gauss.f90) ------
struct KernelBase {
  int id = SPH_KERNEL_M6;
  double knorm[3];
  double fwcl[3];
  int maxneib[3];
  double krad;
  double cn_hydro, cn_2nw, cn_fab, cn_n2w;  // cnarr, base_*.f90 initkernelbase
};

KernelBase make_kernel(int id) {
  KernelBase k;
  k.id = id;
  if (id == SPH_KERNEL_M6) {  // base_m6.f90:13-33
    k.knorm[0] = 1. / 120.; k.knorm[1] = 7. / (478. * pi); k.knorm[2] = 1. / (120. * pi);
    k.fwcl[0] = 4.; k.fwcl[1] = 9.31505 / 2.25; k.fwcl[2] = 9.6429 / 2.25;
    k.maxneib[0] = 50; k.maxneib[1] = 10000; k.maxneib[2] = 150;
    k.krad = 3.;
    k.cn_hydro = 0.3; k.cn_2nw = 1.1; k.cn_fab = 0.2; k.cn_n2w = 0.4;
  } else if (id == SPH_KERNEL_M4) {  // base_m4.f90:12-32
    k.knorm[0] = 2. / 3.; k.knorm[1] = 10. / (7. * pi); k.knorm[2] = 1. / pi;
    k.fwcl[0] = 6.; k.fwcl[1] = 6.3226; k.fwcl[2] = 6.66400;
    k.maxneib[0] = 35; k.maxneib[1] = 250; k.maxneib[2] = 150;
    k.krad = 2.;
    k.cn_hydro = 0.1; k.cn_2nw = 0.96; k.cn_fab = 0.15; k.cn_n2w = 0.2;
  } else {  // base_gauss.f90:15-36
    k.knorm[0] = 1. / std::sqrt(pi); k.knorm[1] = 1. / pi; k.knorm[2] = 1. / std::pow(pi, 1.5);
    k.fwcl[0] = 4.; k.fwcl[1] = 4.; k.fwcl[2] = 4.;
    k.maxneib[0] = 100; k.maxneib[1] = 5000; k.maxneib[2] = 50000;
    k.krad = 10.;
    k.cn_hydro = 0.55; k.cn_2nw = 1.25; k.cn_fab = 0.24; k.cn_n2w = 0.50;
  }
  return k;
}

// Error flag raised inside OpenMP loops (first one wins).
struct ErrFlag {
  int code = 0;
  void set(int c) {
#pragma omp critical(sph_oracle_err)
    if (code == 0) code = c;
  }
};

// f, f', f'' of the kernel shape (base_*.f90 kf/kdf/kddf).
inline double kf(int id, double q, ErrFlag& e) {
  if (!(q >= 0.)) { e.set(std::isnan(q) ? SPH_ERR_Q_NAN : SPH_ERR_Q_NEG); return 0.; }
  if (id == SPH_KERNEL_M6) {
    if (q >= 3.) return 0.;
    if (q >= 2.) return powi(3. - q, 5);
    if (q >= 1.) return powi(3. - q, 5) - 6. * powi(2. - q, 5);
    return powi(3. - q, 5) - 6. * powi(2. - q, 5) + 15. * powi(1. - q, 5);
  } else if (id == SPH_KERNEL_M4) {
    if (q >= 2.) return 0.;
    if (q >= 1.) return 0.25 * powi(2. - q, 3);
    return 0.25 * powi(2. - q, 3) - powi(1. - q, 3);
  }
  return std::exp(-q * q);
}
inline double kdf(int id, double q, ErrFlag& e) {
  if (!(q >= 0.)) { e.set(std::isnan(q) ? SPH_ERR_Q_NAN : SPH_ERR_Q_NEG); return 0.; }
  if (id == SPH_KERNEL_M6) {
    if (q >= 3.) return 0.;
    if (q >= 2.) return -5. * powi(3. - q, 4);
    if (q >= 1.) return -5. * powi(3. - q, 4) + 30. * powi(2. - q, 4);
    return -5. * powi(3. - q, 4) + 30. * powi(2. - q, 4) - 75. * powi(1. - q, 4);
  } else if (id == SPH_KERNEL_M4) {
    if (q >= 2.) return 0.;
    if (q >= 1.) return -0.75 * powi(2. - q, 2);
    return -0.75 * powi(2. - q, 2) + 3 * powi(1. - q, 2);
  }
  return -2. * std::exp(-q * q) * q;
}
inline double kddf(int id, double q, ErrFlag& e) {
  if (!(q >= 0.)) { e.set(std::isnan(q) ? SPH_ERR_Q_NAN : SPH_ERR_Q_NEG); return 0.; }
  if (id == SPH_KERNEL_M6) {
    if (q >= 3.) return 0.;
    if (q >= 2.) return 20. * powi(3. - q, 3);
    if (q >= 1.) return 20. * powi(3. - q, 3) - 120. * powi(2. - q, 3);
    return 20. * powi(3. - q, 3) - 120. * powi(2. - q, 3) + 300. * powi(1. - q, 3);
  } else if (id == SPH_KERNEL_M4) {
    if (q >= 2.) return 0.;
    if (q >= 1.) return 1.5 * (2. - q);
    return 1.5 * (2. - q) - 6 * (1. - q);
  }
  return -2 * std::exp(-q * q) + 4 * std::exp(-q * q) * q * q;
}

struct Vec3 {
  double x[3];
  double& operator[](int i) { return x[i]; }
  double operator[](int i) const { return x[i]; }
};
inline double dot3(const double* a, const double* b) {
  // Fortran dot_product: sequential sum from zero.
  double s = 0.;
  s = s + a[0] * b[0];
  s = s + a[1] * b[1];
  s = s + a[2] * b[2];
  return s;
}

// ---- the oracle engine -----------------------------------------------------
struct Oracle {
  KernelBase kb;
  int dim = 3;
  double wCv = 0, fwc = 0, krad = 0;
  double cnhydro = 0, cnd2 = 0, cnfld = 0;
  int ddw = esd_fab;
  std::vector<double> st;  // 1-based: st[k] = statevars(k); extras after 49

  std::vector<double> store;  // rows x ES, row-major; reals, fixed, ghosts
  int64_t nrows = 0, realpn = 0, fixedpn = 0, periodpn = 0;
  std::vector<int64_t> crossref;  // ghost -> source row (0-based)
  std::vector<int> gcode;         // ghost image code
  std::vector<int64_t> ibx1, ibx2, iby1, iby2, ibz1, ibz2;

  std::vector<int64_t> noff, nidx;  // neighbour lists (reference numbering)

  std::vector<double> hk, hkp1, dk, dkp1, ok, okp1, epsv;

  // time loop
  bool started = false, stopped = false;
  double ltout = 0., dtout = 0.;
  int64_t iterc = 0;
  std::vector<double> tr, tv, ta, tdu, tdh, tddt, tdb;
  std::vector<double> sY0, sYjm1, sYjm2, sYj, sDY0, sDYjm1;

  int64_t cnt[SPH_CNT_TOTAL] = {0};
  double timers[SPH_T_TOTAL] = {0};

  double& S(int64_t row, int f) { return store[row * ES + f]; }
  double S(int64_t row, int f) const { return store[row * ES + f]; }
  int ival(int k) const { return int(st[k]); }

  // eqSet (state.f90:117-149)
  bool eq_hydro = false, eq_magneto = false, eq_diff = false, eq_fld = false,
       eq_radexch = false, eq_sts = false;
  int eqset() {
    eq_hydro = eq_magneto = eq_diff = eq_fld = eq_radexch = eq_sts = false;
    switch (ival(ec_eqs)) {
      case eeq_hydro: eq_hydro = true; break;
      case eeq_magnetohydro: eq_hydro = eq_magneto = true; break;
      case eeq_diffusion: eq_diff = true; break;
      case eeq_hyrad: eq_fld = eq_hydro = eq_radexch = true; break;
      case eeq_magnetohydrodiffusion: eq_hydro = eq_magneto = eq_diff = true; break;
      case eeq_hydrodiffusion: eq_hydro = eq_diff = true; break;
      case eeq_manual:
        eq_diff = ival(ec_eqondiff) == 1;
        eq_hydro = ival(ec_eqonhydro) == 1;
        eq_fld = ival(ec_eqonfluxlim) == 1;
        eq_radexch = ival(ec_eqonradexch) == 1;
        eq_sts = ival(ec_eqonsts) == 1;
        break;
      default: break;
    }
    return SPH_OK;
  }

  // initkernel (kernel.f90:91-152) + initkernelbase
  int initkernel() {
    dim = ival(ec_dim);
    if (dim < 1 || dim > 3) return fail(SPH_ERR_ARG, "Dimmention is wrong");
    wCv = kb.knorm[dim - 1];
    fwc = kb.fwcl[dim - 1];
    krad = kb.krad;
    cnhydro = kb.cn_hydro;
    ddw = ival(ec_ddw);
    if (ival(ec_coordsys) == 2)
      return fail(SPH_ERR_UNSUPPORTED, "cylindric coordinates: Fab_cylindric does not exist (kernel.f90:137)");
    if (ddw == esd_n2w) cnd2 = kb.cn_n2w;
    else if (ddw == esd_fab) cnd2 = kb.cn_fab;
    else if (ddw == esd_2nw_ds || ddw == esd_2nw_sd) cnd2 = kb.cn_2nw;
    else if (ddw == esd_fw) cnd2 = kb.cn_fab;
    else cnd2 = kb.cn_fab;  // kernel.f90:128-133 (Brookshaw by default)
    cnfld = cnd2;
    return SPH_OK;
  }

  // ---- kernel wrappers (kernel.f90:178-290) --------------------------------
  double get_w(double r, double h, ErrFlag& e) const {
    double q = r / h;
    double f = kf(kb.id, q, e);
    return wCv * f / powi(h, dim);
  }
  void nw(const double* rab, double dr, double h, double* o, ErrFlag& e) const {
    double q = dr / h;
    double df = kdf(kb.id, q, e);
    double hd2 = powi(h, dim + 2);
    for (int k = 0; k < 3; ++k) o[k] = wCv * df * rab[k] / hd2 / q;
  }
  double get_dw_dh(double r, double h, ErrFlag& e) const {
    double q = r / h;
    double f = kf(kb.id, q, e);
    double df = kdf(kb.id, q, e);
    return -wCv / powi(h, dim + 1) * (dim * f + q * df);
  }
  double fab(double dr, double h, ErrFlag& e) const {
    double q = dr / h;
    double df = kdf(kb.id, q, e);
    return wCv * df * dr / powi(h, dim + 2) / q;
  }
  double fw(double dr, double h, ErrFlag& e) const {
    double q = dr / h;
    double f = kf(kb.id, q, e);
    return fwc * wCv * f / powi(h, dim + 2);
  }
  double gab(double dr, double h, ErrFlag& e) const {
    double q = dr / h;
    double df = kdf(kb.id, q, e);
    return -2. * wCv * df / powi(h, dim + 2) / q;
  }
  // hessian_ddw_cart / hessian_fab_cart / hessian_fw_cart (kernel.f90:377-539)
  void hessian(const double* rab, double h, double Hes[3][3], ErrFlag& e) const {
    double r2 = dot3(rab, rab);
    double r11 = rab[0] * rab[0] / r2, r12 = rab[0] * rab[1] / r2,
           r13 = rab[0] * rab[2] / r2, r22 = rab[1] * rab[1] / r2,
           r23 = rab[1] * rab[2] / r2, r33 = rab[2] * rab[2] / r2;
    double cstart = wCv / powi(h, dim + 2);
    for (int a = 0; a < 3; ++a)
      for (int b = 0; b < 3; ++b) Hes[a][b] = 0.;
    double dr = std::sqrt(r2);
    if (ddw == esd_n2w) {
      double q = dr / h;
      double ddf = kddf(kb.id, q, e);
      double df = kdf(kb.id, q, e);
      double dfq = df / q;
      Hes[0][0] = cstart * (ddf * r11 + dfq * (1 - r11));
      if (dim != 1) {
        Hes[0][1] = cstart * (ddf * r12 - dfq * r12);
        Hes[1][0] = Hes[0][1];
        Hes[1][1] = cstart * (ddf * r22 + dfq * (1 - r22));
        if (dim == 3) {
          Hes[0][2] = cstart * (ddf * r13 - dfq * r13);
          Hes[2][0] = Hes[0][2];
          Hes[1][2] = cstart * (ddf * r23 - dfq * r23);
          Hes[2][1] = Hes[1][2];
          Hes[2][2] = cstart * (ddf * r33 + dfq * (1 - r33));
        }
      }
    } else {
      double f2 = (ddw == esd_fw) ? fw(dr, h, e) : gab(dr, h, e);
      f2 = 0.5 * f2;
      double d2 = dim + 2;
      Hes[0][0] = (d2 * r11 - 1) * f2;
      if (dim != 1) {
        Hes[0][1] = d2 * r12 * f2;
        Hes[1][0] = Hes[0][1];
        Hes[1][1] = (d2 * r22 - 1) * f2;
        if (dim == 3) {
          Hes[0][2] = d2 * r13 * f2;
          Hes[2][0] = Hes[0][2];
          Hes[1][2] = d2 * r23 * f2;
          Hes[2][1] = Hes[1][2];
          Hes[2][2] = (d2 * r33 - 1) * f2;
        }
      }
    }
  }

  // ---- boundary conditions (BC.f90:70-475) ----------------------------------
  void clear_periodic() {
    store.resize(size_t(nrows) * ES);
    periodpn = 0;
    crossref.clear();
    gcode.clear();
    ibx1.clear(); ibx2.clear(); iby1.clear(); iby2.clear(); ibz1.clear(); ibz2.clear();
  }
  double xmin, xmax, ymin, ymax, zmin, zmax, bordersize, padding;
  double boxmin[3], boxmax[3];
  void init_borders() {  // BC.f90:46-68
    bordersize = st[ec_bordsize];
    padding = st[ec_padding];
    xmin = st[ec_xmin]; xmax = st[ec_xmax];
    ymin = st[ec_ymin]; ymax = st[ec_ymax];
    zmin = st[ec_zmin]; zmax = st[ec_zmax];
    boxmax[0] = xmax - bordersize; boxmax[1] = ymax - bordersize; boxmax[2] = zmax - bordersize;
    boxmin[0] = xmin + bordersize; boxmin[1] = ymin + bordersize; boxmin[2] = zmin + bordersize;
  }
  void reflect(int refdir) {  // BC.f90:102-194
    const double emin[3] = {xmin, ymin, zmin}, emax[3] = {xmax, ymax, zmax};
    bool ax[3] = {false, false, false};
    if (refdir == ebc_all) { ax[0] = true; ax[1] = dim > 1; ax[2] = dim == 3; }
    else if (refdir == ebc_x) ax[0] = true;
    else if (refdir == ebc_y) ax[1] = dim > 1;
    else if (refdir == ebc_z) ax[2] = dim == 3;
    for (int64_t i = 0; i < realpn; ++i) {
      double dxmin[3], dxmax[3];
      for (int k = 0; k < 3; ++k) {
        dxmin[k] = emin[k] - S(i, es_rx + k);
        dxmax[k] = S(i, es_rx + k) - emax[k];
      }
      for (int k = 0; k < 3; ++k) {
        if (!ax[k]) continue;
        if (dxmax[k] > 0) S(i, es_rx + k) = emin[k] + dxmax[k];
        if (dxmin[k] > 0) S(i, es_rx + k) = emax[k] - dxmin[k];
      }
    }
  }
  void find_inside_border() {  // BC.f90:196-309
    double pmin[3] = {xmin, ymin, zmin}, pmax[3] = {xmax, ymax, zmax};
    if (padding == 0) {
      pmin[0] = xmin + padding / 10; pmin[1] = ymin + padding / 10; pmin[2] = zmin + padding / 10;
      pmax[0] = xmax - padding / 10; pmax[1] = ymax - padding / 10; pmax[2] = zmax - padding / 10;
    }
    std::vector<int64_t>* lo[3] = {&ibx1, &iby1, &ibz1};
    std::vector<int64_t>* hi[3] = {&ibx2, &iby2, &ibz2};
    int64_t storesize = int64_t(store.size() / ES);
    for (int64_t i = 0; i < storesize; ++i) {
      int t = int(S(i, es_type));
      if (t != ept_real && t != ept_fixed && t != ept_fixedreal) continue;
      for (int k = 0; k < dim; ++k) {
        double ra = S(i, es_rx + k);
        if (ra < boxmin[k]) {
          if (ra > pmin[k]) lo[k]->push_back(i);
        } else if (ra > boxmax[k]) {
          if (ra < pmax[k]) hi[k]->push_back(i);
        }
      }
    }
  }
  int64_t self_getcrossref(int64_t j) const {
    return j < nrows ? j : crossref[j - nrows];
  }
  int64_t add_ghost(int64_t pi, int axis, int sign) {
    int64_t k = nrows + periodpn;
    store.resize(size_t(k + 1) * ES, 0.);
    for (int c = 0; c < 3; ++c) S(k, es_rx + c) = S(pi, es_rx + c);
    const double emin[3] = {xmin, ymin, zmin}, emax[3] = {xmax, ymax, zmax};
    if (sign > 0) S(k, es_rx + axis) = emax[axis] + (S(k, es_rx + axis) - emin[axis]);
    else S(k, es_rx + axis) = emin[axis] + (S(k, es_rx + axis) - emax[axis]);
    S(k, es_type) = ept_periodic;
    int parent_code = pi < nrows ? 13 : gcode[pi - nrows];
    int64_t root = pi;
    while (root >= nrows) root = crossref[root - nrows];  // BC.f90:398-400
    crossref.push_back(root);
    int step = axis == 0 ? 1 : (axis == 1 ? 3 : 9);
    gcode.push_back(parent_code + sign * step);
    ++periodpn;
    return k;
  }
  void create_periodic_border(int side) {  // BC.f90:311-475
    if (side == ebc_all || side == ebc_x) {
      for (int pass = 0; pass < 2; ++pass) {
        std::vector<int64_t> lst = pass == 0 ? ibx1 : ibx2;
        for (int64_t pi : lst) {
          int64_t k = add_ghost(pi, 0, pass == 0 ? +1 : -1);
          if (dim > 1) {
            if (S(k, es_ry) < boxmin[1]) iby1.push_back(k);
            else if (S(k, es_ry) > boxmax[1]) iby2.push_back(k);
            if (dim == 3) {
              if (S(k, es_rz) < boxmin[2]) ibz1.push_back(k);
              else if (S(k, es_rz) > boxmax[2]) ibz2.push_back(k);
            }
          }
        }
      }
    }
    if (dim > 1) {
      if (side == ebc_all || side == ebc_y) {
        for (int pass = 0; pass < 2; ++pass) {
          std::vector<int64_t> lst = pass == 0 ? iby1 : iby2;
          for (int64_t pi : lst) {
            int64_t k = add_ghost(pi, 1, pass == 0 ? +1 : -1);
            if (dim == 3) {
              if (S(k, es_rz) < boxmin[2]) ibz1.push_back(k);
              else if (S(k, es_rz) > boxmax[2]) ibz2.push_back(k);
            }
          }
        }
      }
      if (dim == 3 && (side == ebc_all || side == ebc_z)) {
        for (int pass = 0; pass < 2; ++pass) {
          std::vector<int64_t> lst = pass == 0 ? ibz1 : ibz2;
          for (int64_t pi : lst) add_ghost(pi, 2, pass == 0 ? +1 : -1);
        }
      }
    }
  }

  // ---- neighbour search: uniform grid + the kd-tree predicate --------------
  int find_neighbours() {
    double t0 = omp_get_wtime();
    int64_t sn = nrows + periodpn;
    double hmin = std::numeric_limits<double>::infinity();
    double lo[3] = {1e300, 1e300, 1e300}, hi[3] = {-1e300, -1e300, -1e300};
    for (int64_t i = 0; i < realpn; ++i) hmin = std::min(hmin, S(i, es_h));
    for (int64_t i = 0; i < sn; ++i)
      for (int k = 0; k < 3; ++k) {
        lo[k] = std::min(lo[k], S(i, es_rx + k));
        hi[k] = std::max(hi[k], S(i, es_rx + k));
      }
    if (!(hmin > 0)) hmin = 1e-300;
    double L = krad * hmin * std::max(1e-3, st[SPH_P_CELL_FACTOR]);
    int64_t nc[3];
    const int64_t cell_cap = std::max<int64_t>(4 * sn, 1 << 16);
    for (;;) {
      // cells per axis checked against the cap one axis at a time, so the
      // product cannot overflow (a tiny h_min in a large box would need
      // ~1e9 cells per axis)
      int64_t tot = 1;
      bool ok = true;
      for (int k = 0; k < 3 && ok; ++k) {
        const double e = (hi[k] - lo[k]) / L;
        if (!(e < 1e9)) { ok = false; break; }
        nc[k] = int64_t(std::floor(e)) + 1;
        if (tot > cell_cap / nc[k]) ok = false;
        else tot *= nc[k];
      }
      if (ok) break;
      L *= 1.5;
    }
    auto cell_of = [&](int k, double x) {
      int64_t c = int64_t(std::floor((x - lo[k]) / L));
      return std::min(std::max<int64_t>(c, 0), nc[k] - 1);
    };
    int64_t ncell = nc[0] * nc[1] * nc[2];
    std::vector<int64_t> cstart(ncell + 1, 0), order(sn);
    std::vector<int64_t> cid(sn);
    for (int64_t i = 0; i < sn; ++i) {
      cid[i] = cell_of(0, S(i, es_rx)) + nc[0] * (cell_of(1, S(i, es_ry)) + nc[1] * cell_of(2, S(i, es_rz)));
      cstart[cid[i] + 1]++;
    }
    for (int64_t c = 0; c < ncell; ++c) cstart[c + 1] += cstart[c];
    {
      std::vector<int64_t> fill(cstart.begin(), cstart.end() - 1);
      for (int64_t i = 0; i < sn; ++i) order[fill[cid[i]]++] = i;
    }
    std::vector<std::vector<int64_t>> lists(realpn);
    ErrFlag e;
    int64_t cand = 0;
    const bool capcheck = st[SPH_P_NEIB_CAP_CHECK] != 0;
    const int cap = kb.maxneib[dim - 1];
#pragma omp parallel for schedule(dynamic, 256) reduction(+ : cand)
    for (int64_t i = 0; i < realpn; ++i) {
      double qv[3] = {S(i, es_rx), S(i, es_ry), S(i, es_rz)};
      double kh = krad * S(i, es_h);
      double ballsize = kh * kh;  // neighboursearch.f90:126
      double R = std::sqrt(ballsize) * (1 + 1e-12) + 1e-300;
      int64_t c0[3], c1[3];
      for (int k = 0; k < 3; ++k) { c0[k] = cell_of(k, qv[k] - R); c1[k] = cell_of(k, qv[k] + R); }
      auto& out = lists[i];
      for (int64_t cz = c0[2]; cz <= c1[2]; ++cz)
        for (int64_t cy = c0[1]; cy <= c1[1]; ++cy)
          for (int64_t cx = c0[0]; cx <= c1[0]; ++cx) {
            int64_t c = cx + nc[0] * (cy + nc[1] * cz);
            for (int64_t p = cstart[c]; p < cstart[c + 1]; ++p) {
              int64_t j = order[p];
              ++cand;
              // kdtree2.f90:1673-1678: sd = sd + (data(k,j) - qv(k))**2
              double sd = 0.0;
              double d0 = S(j, es_rx) - qv[0];
              sd = sd + d0 * d0;
              double d1 = S(j, es_ry) - qv[1];
              sd = sd + d1 * d1;
              double d2 = S(j, es_rz) - qv[2];
              sd = sd + d2 * d2;
              if (sd > ballsize) continue;
              if (j != i) out.push_back(j);  // neighboursearch.f90:190
            }
          }
      std::sort(out.begin(), out.end());
      if (capcheck && int64_t(out.size()) + 1 > cap) e.set(SPH_ERR_NEIB_OVERFLOW);
    }
    noff.assign(realpn + 1, 0);
    for (int64_t i = 0; i < realpn; ++i) noff[i + 1] = noff[i] + int64_t(lists[i].size());
    nidx.resize(noff[realpn]);
    for (int64_t i = 0; i < realpn; ++i)
      std::copy(lists[i].begin(), lists[i].end(), nidx.begin() + noff[i]);
    cnt[SPH_CNT_NEIB_PAIRS] += noff[realpn];
    cnt[SPH_CNT_SEARCHES]++;
    {
      int64_t mx = 0;
      for (int64_t i = 0; i < realpn; ++i) mx = std::max(mx, noff[i + 1] - noff[i]);
      cnt[SPH_CNT_NEIB_MAX] = mx;
    }
    cnt[SPH_CNT_CANDIDATES] += cand;
    cnt[SPH_CNT_GHOSTS] = periodpn;
    timers[SPH_T_NEIGHBOURS] += 1e3 * (omp_get_wtime() - t0);
    if (e.code) return fail(e.code, "KDTree neibsearch result was truncated (neighboursearch.f90:131)");
    return SPH_OK;
  }

  // ---- circuit1 (circuit1.f90:53-305) ---------------------------------------
  int c1() {
    double t0 = omp_get_wtime();
    int rc = ival(ec_adden) == 1 ? c1advanced() : c1simple();
    if (ival(ec_adden) != 1) {
      int64_t rows = int64_t(store.size() / ES);
      for (int64_t i = 0; i < rows; ++i) S(i, es_om) = 1.;  // circuit1.f90:62
    }
    timers[SPH_T_CIRCUIT1] += 1e3 * (omp_get_wtime() - t0);
    return rc;
  }
  int c1advanced() {
    const int64_t totreal = nrows;
    const double hfac = st[ec_hfac];
    const double allowerror = st[SPH_P_NEWTON_TOL];
    const int maxiter = int(st[SPH_P_NEWTON_MAXITER]);
    hk.resize(totreal); hkp1.resize(totreal); dk.resize(totreal);
    dkp1.resize(totreal); ok.resize(totreal); okp1.resize(totreal); epsv.resize(totreal);
    for (int64_t i = 0; i < totreal; ++i) {
      hkp1[i] = S(i, es_h); dkp1[i] = S(i, es_den); okp1[i] = S(i, es_om); epsv[i] = 0.;
    }
    for (int64_t i = 0; i < realpn; ++i) epsv[i] = 1.;
    int iter = 0;
    ErrFlag e;
    auto maxeps = [&]() {
      double m = -std::numeric_limits<double>::max();
      bool any = false;
      for (int64_t i = 0; i < totreal; ++i)
        if (epsv[i] > 0) { m = any ? std::max(m, epsv[i]) : epsv[i]; any = true; }
      return any ? m : -std::numeric_limits<double>::max();
    };
    const bool dT = eq_diff || eq_fld;
    int64_t pairs = 0, csweeps = 0;
    while (maxeps() > allowerror && iter < maxiter) {
      ++iter;
      hk = hkp1; dk = dkp1; ok = okp1;
#pragma omp parallel for schedule(dynamic, 256) reduction(+ : pairs, csweeps)
      for (int64_t i = 0; i < realpn; ++i) {
        if (!(epsv[i] > allowerror)) continue;
        ++csweeps;
        double ma = S(i, es_m), ha0 = S(i, es_h);
        double ra[3] = {S(i, es_rx), S(i, es_ry), S(i, es_rz)};
        double ta = S(i, es_t);
        double ha = hk[i], rhoa = dk[i], oma = ok[i];
        double dtadx[3] = {0., 0., 0.};
        double dsum = 0., osum = 0.;
        for (int64_t l = noff[i]; l < noff[i + 1]; ++l) {
          int64_t j = nidx[l];
          int64_t rj = self_getcrossref(j);
          double r[3];
          for (int k = 0; k < 3; ++k) r[k] = ra[k] - S(j, es_rx + k);
          double r2 = dot3(r, r);
          double dr = std::sqrt(r2);
          double mb = S(rj, es_m), tb = S(rj, es_t);
          double rhob = dk[rj], hb = hk[rj], omb = ok[rj];
          double dwdh = get_dw_dh(dr, ha, e);
          double w = get_w(dr, ha, e);
          dsum = dsum + mb * w;
          osum = osum + mb * dwdh;
          if (dT) {
            double nwa[3];
            if (ddw == esd_2nw_sd) {
              double nwb[3];
              nw(r, dr, ha, nwa, e);
              nw(r, dr, hb, nwb, e);
              for (int k = 0; k < 3; ++k)
                dtadx[k] = dtadx[k] + mb * (ta * rhoa / oma / rhoa / rhoa * nwa[k] +
                                            tb * rhoa / omb / rhob / rhob * nwb[k]);
            } else {
              nw(r, dr, ha, nwa, e);
              for (int k = 0; k < 3; ++k)
                dtadx[k] = dtadx[k] + mb / rhoa / oma * (tb * rhob - ta * rhoa) * nwa[k];
            }
          }
        }
        pairs += noff[i + 1] - noff[i];
        double w0 = get_w(0., ha, e), dwdh0 = get_dw_dh(0., ha, e);
        dsum = dsum + ma * w0;
        osum = osum + ma * dwdh0;
        osum = 1. - osum * (-ha / (dim * dsum));  // Price 2008 form, :196
        double dfdh = -dim * dsum * osum / ha;
        double fh = ma * powi(hfac / ha, dim) - dsum;
        double hn = ha - fh / dfdh;
        if (hn <= 0.) e.set(SPH_ERR_H_NEG);
        epsv[i] = std::fabs(hn - ha) / ha0;
        dkp1[i] = dsum; okp1[i] = osum; hkp1[i] = hn;
        for (int k = 0; k < 3; ++k) S(i, es_dtdx + k) = dtadx[k];
      }
      if (e.code) break;
    }
    for (int64_t i = 0; i < realpn; ++i) {
      S(i, es_h) = hkp1[i]; S(i, es_den) = dkp1[i]; S(i, es_om) = okp1[i];
    }
    cnt[SPH_CNT_C1_PAIRS] += pairs;
    cnt[SPH_CNT_C1_SWEEPS] += iter;
    cnt[SPH_CNT_C1_CENTRE_SWEEPS] += csweeps;
    if (e.code == SPH_ERR_H_NEG) return fail(e.code, "Negative smoothing length in c1 advanced");
    if (e.code) return fail(e.code, e.code == SPH_ERR_Q_NAN ? "q is nan" : "q is negative");
    return SPH_OK;
  }
  int c1simple() {
    const int64_t totreal = nrows;
    const double hfac = st[ec_hfac];
    dk.resize(totreal); hk.resize(totreal);
    for (int64_t i = 0; i < totreal; ++i) { dk[i] = S(i, es_den); hk[i] = S(i, es_h); }
    ErrFlag e;
    int64_t pairs = 0;
#pragma omp parallel for schedule(dynamic, 256) reduction(+ : pairs)
    for (int64_t i = 0; i < realpn; ++i) {
      double dtadx[3] = {0., 0., 0.};
      double ra[3] = {S(i, es_rx), S(i, es_ry), S(i, es_rz)};
      double ha = S(i, es_h), ma = S(i, es_m), rhoa = S(i, es_den), ta = S(i, es_t);
      double dsum = 0.;
      for (int64_t l = noff[i]; l < noff[i + 1]; ++l) {
        int64_t j = nidx[l];
        int64_t rj = self_getcrossref(j);
        double hb = S(rj, es_h), mb = S(rj, es_m), rhob = S(rj, es_den), tb = S(rj, es_t);
        double r[3];
        for (int k = 0; k < 3; ++k) r[k] = ra[k] - S(j, es_rx + k);
        double dr = std::sqrt(dot3(r, r));
        double w = get_w(dr, ha, e);
        dsum = dsum + mb * w;
        if (eq_diff) {
          double nwa[3], nwb[3];
          if (ddw == esd_2nw_ds) {
            nw(r, dr, ha, nwa, e);
            for (int k = 0; k < 3; ++k) dtadx[k] = dtadx[k] + mb / rhoa * (tb - ta) * nwa[k];
          } else if (ddw == esd_2nw_sd) {
            nw(r, dr, ha, nwa, e);
            nw(r, dr, hb, nwb, e);
            for (int k = 0; k < 3; ++k)
              dtadx[k] = dtadx[k] + mb * (ta / rhoa / rhoa * nwa[k] + tb / rhob / rhob * nwb[k]);
          }
        }
      }
      pairs += noff[i + 1] - noff[i];
      double w0 = get_w(0., ha, e);
      dsum = dsum + ma * w0;
      dk[i] = dsum;
      hk[i] = hfac * std::pow(ma / dsum, 1. / dim);
      for (int k = 0; k < 3; ++k) S(i, es_dtdx + k) = dtadx[k];
    }
    for (int64_t i = 0; i < realpn; ++i) {
      S(i, es_den) = dk[i]; S(i, es_h) = hk[i]; S(i, es_om) = 1.;
    }
    cnt[SPH_CNT_C1_PAIRS] += pairs;
    cnt[SPH_CNT_C1_SWEEPS] += 1;
    cnt[SPH_CNT_C1_CENTRE_SWEEPS] += realpn;
    if (e.code) return fail(e.code, e.code == SPH_ERR_Q_NAN ? "q is nan" : "q is negative");
    return SPH_OK;
  }

  // ---- EOS (eos.f90:21-45) ----------------------------------------------------
  void eos_adiabatic() {
    double gamma = st[ec_gamma];
    for (int64_t i = 0; i < realpn; ++i) {
      S(i, es_p) = (gamma - 1.) * S(i, es_den) * S(i, es_u);
      S(i, es_c) = std::sqrt(gamma * S(i, es_p) / S(i, es_den));
    }
  }
  void eos_isothermal() {
    double c0 = S(0, es_c);
    for (int64_t i = 0; i < realpn; ++i) S(i, es_p) = S(i, es_den) * c0 * c0;
  }

  // ---- circuit2 (circuit2.f90:58-505, 520-575) --------------------------------
  int c2() {
    double t0 = omp_get_wtime();
    const double mhdmuzero = st[ec_muzero];
    const int difiso = ival(ec_disotropic);
    const double difcond = st[ec_dcondconst];
    const int s_adden = ival(ec_adden), s_artts = ival(ec_artts);
    const double s_au = st[ec_au];
    const double alpha = st[SPH_P_AV_ALPHA], beta = st[SPH_P_AV_BETA];
    const bool fullt = st[SPH_P_FULL_TENSOR] != 0;
    if (eq_diff && eq_fld && difiso != 1)
      return fail(SPH_ERR_FLD_ANISO, "There is no anisotropic for FLD");
    if (eq_diff && !(ddw == esd_fw || ddw == esd_fab || ddw == esd_n2w ||
                     ddw == esd_2nw_ds || ddw == esd_2nw_sd))
      return fail(SPH_ERR_DDW, "second deriv id not found");
    ErrFlag e;
    int64_t pairs = 0;
#pragma omp parallel for schedule(dynamic, 256) reduction(+ : pairs)
    for (int64_t i = 0; i < realpn; ++i) {
      double rhoa = S(i, es_den);
      double ra[3] = {S(i, es_rx), S(i, es_ry), S(i, es_rz)};
      double ba[3] = {S(i, es_bx), S(i, es_by), S(i, es_bz)};
      double uba[3] = {0., 0., 0.}, ubb[3] = {0., 0., 0.};
      {
        double bb2 = dot3(ba, ba);
        if (bb2 != 0) for (int k = 0; k < 3; ++k) uba[k] = ba[k] / std::sqrt(bb2);
      }
      double va[3] = {S(i, es_vx), S(i, es_vy), S(i, es_vz)};
      double ha = S(i, es_h), ca = S(i, es_c), pa = S(i, es_p), ua = S(i, es_u);
      double oma = S(i, es_om), ta = S(i, es_t);
      double kappaa = S(i, es_kappa);
      double dtadx[3] = {S(i, es_dtdx), S(i, es_dtdy), S(i, es_dtdz)};
      double dva[3] = {0, 0, 0}, dua = 0., dha = 0., ddta = 0., dba[3] = {0, 0, 0};
      double drhoadt = 0.;
      double kta[3][3] = {{0}}, ktb[3][3] = {{0}};
      double MPa[3][3] = {{0}};
      double Mc1 = dot3(ba, ba);
      if (eq_magneto) {
        for (int li = 0; li < 3; ++li) {
          MPa[li][li] = (0.5 * Mc1 - ba[li] * ba[li]) / mhdmuzero;
          for (int lj = 0; lj < 3; ++lj)
            if (li != lj) MPa[li][lj] = -ba[li] * ba[lj] / mhdmuzero;
        }
      }
      if (eq_diff) {
        if (eq_fld) {
          double g = std::sqrt(dot3(dtadx, dtadx));
          double fld_ra = g / (kappaa * rhoa * ta * rhoa);
          double lambdaa = (2. + fld_ra) / (6. + 3. * fld_ra + fld_ra * fld_ra);
          double fldda = lightspeed * lambdaa / kappaa / rhoa;
          kta[0][0] = kta[1][1] = kta[2][2] = fldda;
          S(i, es_vfld) = fldda / ((ta * rhoa) / g);
        } else if (difiso == 1) {
          kta[0][0] = kta[1][1] = kta[2][2] = difcond;
          ktb[0][0] = ktb[1][1] = ktb[2][2] = difcond;
        } else if (fullt) {
          for (int a = 0; a < 3; ++a)
            for (int b = 0; b < 3; ++b) kta[a][b] = difcond * uba[a] * uba[b];
        } else {
          for (int li = 0; li < 3; ++li) kta[li][li] = difcond * uba[li] * uba[li];
        }
      }
      for (int64_t l = noff[i]; l < noff[i + 1]; ++l) {
        int64_t j = nidx[l];
        int64_t rj = self_getcrossref(j);
        double rb[3] = {S(j, es_rx), S(j, es_ry), S(j, es_rz)};
        double bb[3] = {S(rj, es_bx), S(rj, es_by), S(rj, es_bz)};
        {
          double bb2 = dot3(bb, bb);
          // circuit2.f90:220-224: a zero B_b leaves ubb from the previous
          // neighbour (the reference assigns uba there).
          if (bb2 != 0) for (int k = 0; k < 3; ++k) ubb[k] = bb[k] / std::sqrt(bb2);
        }
        double vb[3] = {S(rj, es_vx), S(rj, es_vy), S(rj, es_vz)};
        double rhob = S(rj, es_den), hb = S(rj, es_h), cb = S(rj, es_c), pb = S(rj, es_p);
        double ub = S(rj, es_u), omb = S(rj, es_om), tb = S(rj, es_t), mb = S(rj, es_m);
        double kappab = S(rj, es_kappa);
        double dtbdx[3] = {S(rj, es_dtdx), S(rj, es_dtdy), S(rj, es_dtdz)};
        double qa = 0., qb = 0., qc = 0.;
        double rab[3], vab[3], urab[3];
        for (int k = 0; k < 3; ++k) rab[k] = ra[k] - rb[k];
        double r2 = dot3(rab, rab);
        double dr = std::sqrt(r2);
        for (int k = 0; k < 3; ++k) { vab[k] = va[k] - vb[k]; urab[k] = rab[k] / dr; }
        double nwa[3], nwb[3];
        nw(rab, dr, ha, nwa, e);
        nw(rab, dr, hb, nwb, e);
        if (s_adden == 1) drhoadt = drhoadt + mb * dot3(vab, nwa);
        if (s_artts == 1) {
          double faba = fab(dr, ha, e), fabb = fab(dr, hb, e);
          // art_viscosity (:558-575)
          double dvr = dot3(vab, urab);
          if (dvr < 0) {
            double vsig = alpha * ca + beta * std::fabs(dvr);
            qa = -0.5 * rhoa * vsig * dvr;
            vsig = alpha * cb + beta * std::fabs(dvr);
            qb = -0.5 * rhob * vsig * dvr;
          }
          for (int k = 0; k < 3; ++k)
            dva[k] = dva[k] - mb * (qa * nwa[k] / (rhoa * rhoa) / oma + qb * nwb[k] / (rhob * rhob) / omb);
          if (s_au != -1) {
            // art_termcond (:520-529)
            double vsigu = std::sqrt(std::fabs(pa - pb) / (0.5 * (rhoa + rhob)));
            qc = vsigu * (ua - ub) * 0.5 * (faba / oma / rhoa + fabb / omb / rhob);
            qc = s_au * qc;
          }
          dua = dua + mb * (+dot3(vab, urab) * qa * faba / oma / rhoa + qc + 0.);
        }
        if (eq_hydro) {
          for (int k = 0; k < 3; ++k)
            dva[k] = dva[k] - mb * ((pa * nwa[k]) / ((rhoa * rhoa) * oma) + (pb * nwb[k]) / ((rhob * rhob) * omb));
          double pnwa[3] = {pa * nwa[0], pa * nwa[1], pa * nwa[2]};
          dua = dua + mb * dot3(vab, pnwa) / (rhoa * rhoa) / oma;
        }
        if (eq_diff) {
          if (eq_fld) {
            double g = std::sqrt(dot3(dtbdx, dtbdx));
            double fld_rb = g / (kappab * rhob * rhob * tb);
            double lambdab = (2. + fld_rb) / (6. + 3. * fld_rb + fld_rb * fld_rb);
            double flddb = lightspeed * lambdab / kappab / rhob;
            for (int a = 0; a < 3; ++a) for (int b = 0; b < 3; ++b) ktb[a][b] = 0.;
            ktb[0][0] = ktb[1][1] = ktb[2][2] = flddb;
          } else if (difiso == 0) {
            if (fullt) {
              for (int a = 0; a < 3; ++a)
                for (int b = 0; b < 3; ++b) ktb[a][b] = difcond * ubb[a] * ubb[b];
            } else {
              for (int li = 0; li < 3; ++li) ktb[li][li] = difcond * ubb[li] * ubb[li];
            }
          }
          if (ddw == esd_fw || ddw == esd_fab || ddw == esd_n2w) {
            double ktab[3][3], Hesa[3][3];
            for (int a = 0; a < 3; ++a)
              for (int b = 0; b < 3; ++b) ktab[a][b] = (kta[a][b] + ktb[a][b]) / 2.;
            hessian(rab, ha, Hesa, e);
            double contr = dot3(ktab[0], Hesa[0]) + dot3(ktab[1], Hesa[1]) + dot3(ktab[2], Hesa[2]);
            ddta = ddta + mb / rhob / rhoa * (tb * rhob - ta * rhoa) * contr;
          } else if (ddw == esd_2nw_ds) {
            double odda = 1. / oma / rhoa / rhoa, oddb = 1. / omb / rhob / rhob;
            double kdta[3], kdtb[3];
            for (int k = 0; k < 3; ++k) { kdta[k] = dot3(kta[k], dtadx); kdtb[k] = dot3(ktb[k], dtbdx); }
            ddta = ddta + mb * (dot3(kdta, nwa) * odda + dot3(kdtb, nwb) * oddb);
          } else {  // esd_2nw_sd
            double kdta[3], kdtb[3], dd[3];
            for (int k = 0; k < 3; ++k) { kdta[k] = dot3(kta[k], dtadx); kdtb[k] = dot3(ktb[k], dtbdx); }
            for (int k = 0; k < 3; ++k) dd[k] = kdtb[k] - kdta[k];
            ddta = ddta + mb / oma / rhoa / rhoa * (dot3(dd, nwa));
          }
        }
        if (eq_magneto) {
          double MPb[3][3] = {{0}};
          double odda = 1. / oma / rhoa / rhoa;
          (void)odda;
          double Mc2 = dot3(bb, bb);
          for (int li = 0; li < 3; ++li) {
            MPb[li][li] = (0.5 * Mc2 - bb[li] * bb[li]) / mhdmuzero;
            for (int lj = 0; lj < 3; ++lj)
              if (li != lj) MPb[li][lj] = -bb[li] * bb[lj] / mhdmuzero;
          }
          double dvat[3], dvbt[3];
          for (int k = 0; k < 3; ++k) { dvat[k] = dot3(MPa[k], nwa); dvbt[k] = dot3(MPb[k], nwb); }
          for (int k = 0; k < 3; ++k)
            dva[k] = dva[k] - mb * (dvat[k] / ((rhoa * rhoa) * oma) + dvbt[k] / ((rhob * rhob) * omb)) - 0.;
          dua = dua + mb * 0.;
          double banwa = dot3(ba, nwa), vabnwa = dot3(vab, nwa);
          for (int k = 0; k < 3; ++k)
            dba[k] = dba[k] - 1. / (rhoa * oma) * mb * (vab[k] * banwa - bb[k] * vabnwa);
        }
      }
      pairs += noff[i + 1] - noff[i];
      if (s_adden == 1) dha = -dim * ha / rhoa * drhoadt / oma;
      S(i, es_ax) = dva[0]; S(i, es_ay) = dva[1]; S(i, es_az) = dva[2];
      S(i, es_dh) = dha;
      S(i, es_ddt) = ddta;
      S(i, es_dbx) = dba[0]; S(i, es_dby) = dba[1]; S(i, es_dbz) = dba[2];
      S(i, es_du) = dua;
    }
    cnt[SPH_CNT_C2_PAIRS] += pairs;
    timers[SPH_T_CIRCUIT2] += 1e3 * (omp_get_wtime() - t0);
    if (e.code) return fail(e.code, e.code == SPH_ERR_Q_NAN ? "q is nan" : "q is negative");
    return SPH_OK;
  }

  // ---- iterate (iterator.f90:44-179) ----------------------------------------
  int neighbours_and_density(int eos_kind) {
    int rc = find_neighbours();
    if (rc) return rc;
    rc = c1();
    if (rc) return rc;
    if (eos_kind == 1) eos_adiabatic();
    else if (eos_kind == 2) eos_isothermal();
    return SPH_OK;
  }
  int build_ghosts_for(int ipc, int ivt) {
    double t0 = omp_get_wtime();
    init_borders();
    if (ipc == epc_fullyperiodic) {
      clear_periodic(); reflect(ebc_all); find_inside_border(); create_periodic_border(ebc_all);
    } else if (ipc == epc_borderless) {
      clear_periodic();
    } else if (ipc == epc_backcompatibility) {
      switch (ivt) {
        case ett_shock12:
          clear_periodic(); find_inside_border(); create_periodic_border(ebc_y); break;
        case ett_pulse: case ett_ring: case ett_fld_gauss: clear_periodic(); break;
        case ett_soundwave: case ett_OTvortex:
          clear_periodic(); reflect(ebc_all); find_inside_border(); create_periodic_border(ebc_all); break;
        case ett_hydroshock:
          clear_periodic(); reflect(ebc_y); reflect(ebc_z); find_inside_border();
          create_periodic_border(ebc_y); create_periodic_border(ebc_z); break;
        case ett_mti: case ett_mtilowres:
          clear_periodic(); reflect(ebc_x); find_inside_border(); create_periodic_border(ebc_x); break;
        default: return fail(SPH_ERR_PROCESS, "Task type was not set");
      }
    } else {
      return fail(SPH_ERR_PROCESS, "Process type was not set");
    }
    timers[SPH_T_GHOSTS] += 1e3 * (omp_get_wtime() - t0);
    return SPH_OK;
  }
  int eos_kind() const {
    int ipc = ival(ec_process), ivt = ival(ec_ics);
    if (ipc != epc_backcompatibility) return 1;
    if (ivt == ett_pulse || ivt == ett_ring || ivt == ett_fld_gauss) return 0;
    if (ivt == ett_soundwave) return 2;
    return 1;
  }
  int density_pass() {
    eqset();
    int rc = initkernel();
    if (rc) return rc;
    rc = build_ghosts_for(ival(ec_process), ival(ec_ics));
    if (rc) return rc;
    return neighbours_and_density(eos_kind());
  }
  int iterate() {
    int rc = density_pass();
    if (rc) return rc;
    rc = c2();
    if (rc) return rc;
    int ivt = ival(ec_ics);
    if (ival(ec_process) == epc_backcompatibility) {
      if (ivt == ett_mti)
        for (int64_t i = 0; i < realpn; ++i) S(i, es_ay) = S(i, es_ay) - 1.;
      if (ivt == ett_mtilowres)
        for (int64_t i = 0; i < realpn; ++i) S(i, es_ay) = S(i, es_ay) - std::erf(S(i, es_ry) * 8.);
    }
    cnt[SPH_CNT_ITERATES]++;
    cnt[SPH_CNT_CENTRES] += realpn;
    return SPH_OK;
  }

  // ---- timestep (timestep.f90:40-166) -----------------------------------------
  void calctimestep(double& dthydro, double& dtdiff, double& dtfld, double& dtfinal) {
    const int64_t n = ival(ec_realpn);
    double dt = std::numeric_limits<double>::max();  // huge()
    dthydro = 0.;
    dtdiff = std::numeric_limits<double>::infinity();
    dtfld = std::numeric_limits<double>::infinity();
    auto minv = [&](int f) { double m = S(0, f); for (int64_t i = 1; i < n; ++i) m = std::min(m, S(i, f)); return m; };
    auto maxv = [&](int f) { double m = S(0, f); for (int64_t i = 1; i < n; ++i) m = std::max(m, S(i, f)); return m; };
    if (eq_hydro) {
      dthydro = cnhydro * minv(es_h) / maxv(es_c);
      dt = std::min(dt, dthydro);
    }
    if (eq_magneto) {
      double mb = std::max(std::max(maxv(es_bx), maxv(es_by)), maxv(es_bz));
      double dt1 = .1 * minv(es_h) / maxv(es_c) / mb;
      dt = std::min(dt, dt1);
    }
    if (eq_diff) {
      double mh = minv(es_h);
      dtdiff = cnd2 * minv(es_den) * minv(es_c) * (mh * mh) / maxv(es_kappa);
      dt = std::min(dt, dtdiff);
    }
    if (eq_fld) {
      double minden = S(0, es_den), minkappa = S(0, es_kappa), minh = S(0, es_h);
      double maxlambda = 0.0;
      for (int64_t i = 0; i < n; ++i) {
        double nta[3] = {S(i, es_dtdx), S(i, es_dtdy), S(i, es_dtdz)};
        double ka = S(i, es_kappa), da = S(i, es_den), ta = S(i, es_t), ha = S(i, es_h);
        if (minden > da) minden = da;
        if (minkappa > ka) minkappa = ka;
        if (minh > ha) minh = ha;
        double fld_ra = std::sqrt(dot3(nta, nta)) / (ka * da * da * ta);
        double lambdaa = (2. + fld_ra) / (6. + 3 * fld_ra + fld_ra * fld_ra);
        if (maxlambda < lambdaa) maxlambda = lambdaa;
      }
      dtfld = cnfld * minh * minh * minden * minkappa / lightspeed / maxlambda;
      dt = std::min(dt, dtfld);
    }
    dtfinal = dt;
  }

  // ---- STS (sts_integrator.f90:10-124) ------------------------------------------
  static double sb(int j) { return j <= 2 ? 1. / 3. : (double(j * j + j) - 2.) / (2. * j * (j + 1.)); }
  static double sa(int j) { return 1 - sb(j); }
  static double smu(int j) { return (2. * j - 1.) / j * sb(j) / sb(j - 1); }
  static double snu(int j) { return -((j - 1.) / j * sb(j) / sb(j - 2)); }
  static double sw(int s) { return 4. / (double(s * s + s) - 2.); }
  static double smu_hat(int j, int s) { return j == 1 ? sb(1) * sw(s) : smu(j) * sw(s); }
  static double sgm_hat(int j, int s) { return -sa(j - 1) * smu_hat(j, s); }

  int sts_integrate(int s, double dt) {
    double t0 = omp_get_wtime();
    int64_t rows = nrows;
    sY0.resize(rows); sYjm1.resize(rows); sYjm2.resize(rows); sYj.resize(rows);
    sDY0.resize(rows); sDYjm1.resize(rows);
    for (int64_t i = 0; i < rows; ++i) sY0[i] = S(i, es_t);
    int rc = iterate();
    if (rc) return rc;
    for (int64_t i = 0; i < rows; ++i) {
      sDY0[i] = S(i, es_ddt);
      sYjm2[i] = sY0[i];
      sYjm1[i] = sY0[i] + smu_hat(1, s) * dt * sDY0[i];
      sYj[i] = sYjm1[i];
    }
    for (int j = 2; j <= s; ++j) {
      for (int64_t i = 0; i < rows; ++i) S(i, es_t) = sYjm1[i];
      rc = iterate();
      if (rc) return rc;
      double mu = smu(j), nu = snu(j), mh = smu_hat(j, s), gh = sgm_hat(j, s);
      for (int64_t i = 0; i < rows; ++i) {
        sDYjm1[i] = S(i, es_ddt);
        sYj[i] = mu * sYjm1[i] + nu * sYjm2[i] + (1. - mu - nu) * sY0[i] + mh * dt * sDYjm1[i] + gh * dt * sDY0[i];
        sYjm2[i] = sYjm1[i];
        sYjm1[i] = sYj[i];
      }
    }
    for (int64_t i = 0; i < rows; ++i) S(i, es_t) = sYj[i];
    timers[SPH_T_STS] += 1e3 * (omp_get_wtime() - t0);
    return SPH_OK;
  }

  // ---- pre-run check (preruncheck.f90:13-60) ---------------------------------------
  int check_vars_ready() {
    int s_tt = ival(ec_eqs);
    double mhdmprs = st[ec_muzero];
    if (mhdmprs <= 0. && (s_tt == eeq_magnetohydro || s_tt == eeq_magnetohydrodiffusion))
      return fail(SPH_ERR_IC_MUZERO, "mhd_magneticconstant <= 0");
    if (ival(ec_disotropic) > 0 && st[ec_dcondconst] <= 0)
      return fail(SPH_ERR_IC_DIFFCOND, "diff_conductivity <= 0");
    for (int64_t i = 0; i < nrows; ++i) {
      if (int(S(i, es_type)) == ept_empty) continue;
      if (S(i, es_den) <= 0.) return fail(SPH_ERR_IC_DENSITY, "density <= 0");
      if (S(i, es_c) <= 0.) return fail(SPH_ERR_IC_CSOUND, "csound <= 0");
      if (S(i, es_h) <= 0.) return fail(SPH_ERR_IC_H, "smoothing length <= 0");
      if (S(i, es_p) <= 0.) return fail(SPH_ERR_IC_PRESSURE, "pressure <= 0");
      if (S(i, es_u) <= 0.) return fail(SPH_ERR_IC_ENERGY, "internal energy <= 0");
    }
    return SPH_OK;
  }

  // number of integrated rows: reals + trailing fixedreal (main.f90:181-184)
  int64_t n_integrated() const {
    int64_t n = realpn;
    for (int64_t i = std::max<int64_t>(realpn - 1, 0); i < nrows; ++i)
      if (int(S(i, es_type)) == ept_fixedreal) ++n;
    return n;
  }

  // ---- time loop (main.f90:216-373) ---------------------------------------------
  int start_run() {
    eqset();
    int rc = initkernel();
    if (rc) return rc;
    double t = st[ec_time];
    dtout = st[ec_dtprint];
    double tfinish = st[ec_tfinish];
    stopped = false;
    if (tfinish > 0.) {
      rc = check_vars_ready();
      if (rc) return rc;
      if (ival(ec_eqs) != eeq_kd2) {
        rc = iterate();
        if (rc) return rc;
      } else {
        stopped = true;
      }
    } else {
      stopped = true;
    }
    ltout = 0.;
    if (dtout > 0) while (ltout < t) ltout = ltout + dtout;
    started = true;
    return SPH_OK;
  }
  // one pass of the while loop body; returns SPH_OK and sets `done` when the
  // loop condition fails.
  // update_radenergy (rad_exchange.f90:9-68) with the implicit solve of
  // :111-126: Newton on the gas energy at fixed u + xi
  int update_radenergy(int64_t n, double dt) {
    const double gamma = st[ec_gamma], gmw = st[ec_molecularmass];
    const double a = 4. * sigmaB / lightspeed;
    const double cv1 = (gamma - 1.) * gmw / Rg;
    int bad = 0;
#pragma omp parallel for schedule(static) reduction(| : bad)
    for (int64_t i = 0; i < n; ++i) {
      const double kappa = S(i, es_kappa);
      const double ack = 4. * sigmaB * kappa;
      const double rhoi = S(i, es_den), ui = S(i, es_u), dudt = S(i, es_du), xii = S(i, es_t);
      const double etot = ui + xii;
      double unew = ui, uold = 2. * ui;
      for (int iter = 0; std::fabs(unew - uold) > 1e-16 && iter < 10; ++iter) {
        uold = unew;
        const double uc = unew * cv1;
        const double uc2 = uc * uc;
        const double u3 = (unew * unew) * unew;
        const double cv2 = cv1 * cv1;
        const double fu = ((unew / dt - ui / dt) - dudt) - ack * (rhoi * (etot - unew) / a - uc2 * uc2);
        const double dfu = 1. / dt + ack * (rhoi / a + 4. * (u3 * (cv2 * cv2)));
        unew = unew - fu / dfu;
      }
      S(i, es_u) = unew;
      S(i, es_t) = etot - unew;
      if (!(S(i, es_t) > 0.) || !(S(i, es_u) > 0.)) bad = 1;
    }
    if (bad) return fail(SPH_ERR_RAD_NEGATIVE, "radiation or thermal energy is negative after exchange");
    return SPH_OK;
  }

  // ---- one leapfrog step in parts (the split step of include/sph_abi.h):
  // the predictor and corrector of one_step (main.f90:323-362) without STS
  // or radiation exchange, and circuit2 alone on the lists of the last
  // density pass
  bool split_ok() {
    eqset();
    if (eq_sts || eq_radexch)
      return fail(SPH_ERR_UNSUPPORTED, "split step: leapfrog without STS or radiation exchange only") == 0;
    return true;
  }
  int split_predict(double dt) {
    if (!split_ok()) return SPH_ERR_UNSUPPORTED;
    const int64_t n = n_integrated();
    tr.resize(3 * n); tv.resize(3 * n); ta.resize(3 * n); tdu.resize(n); tdh.resize(n);
    tddt.resize(n); tdb.resize(3 * n);
    for (int64_t i = 0; i < n; ++i) {
      for (int k = 0; k < 3; ++k) {
        tr[3 * i + k] = S(i, es_rx + k); tv[3 * i + k] = S(i, es_vx + k);
        ta[3 * i + k] = S(i, es_ax + k); tdb[3 * i + k] = S(i, es_dbx + k);
      }
      tdu[i] = S(i, es_du); tdh[i] = S(i, es_dh); tddt[i] = S(i, es_ddt);
    }
    for (int64_t i = 0; i < n; ++i) {
      for (int k = 0; k < 3; ++k) {
        S(i, es_rx + k) = S(i, es_rx + k) + dt * tv[3 * i + k] + 0.5 * dt * dt * ta[3 * i + k];
        S(i, es_vx + k) = tv[3 * i + k] + dt * ta[3 * i + k];
      }
      S(i, es_u) = S(i, es_u) + dt * tdu[i];
      S(i, es_h) = S(i, es_h) + dt * tdh[i];
      S(i, es_t) = S(i, es_t) + dt * tddt[i];
      for (int k = 0; k < 3; ++k) S(i, es_bx + k) = S(i, es_bx + k) + dt * tdb[3 * i + k];
    }
    return SPH_OK;
  }
  int split_forces() {
    if (noff.empty()) return fail(SPH_ERR_STATE, "sph_forces needs the lists of a density pass");
    int rc = c2();
    if (rc) return rc;
    cnt[SPH_CNT_ITERATES]++;
    return SPH_OK;
  }
  int split_correct(double dt) {
    if (!split_ok()) return SPH_ERR_UNSUPPORTED;
    const int64_t n = n_integrated();
    if (int64_t(tdu.size()) != n) return fail(SPH_ERR_STATE, "sph_correct without sph_predict");
    for (int64_t i = 0; i < n; ++i) {
      for (int k = 0; k < 3; ++k)
        S(i, es_vx + k) = S(i, es_vx + k) + 0.5 * dt * (S(i, es_ax + k) - ta[3 * i + k]);
      S(i, es_u) = S(i, es_u) + 0.5 * dt * (S(i, es_du) - tdu[i]);
      S(i, es_h) = S(i, es_h) + 0.5 * dt * (S(i, es_dh) - tdh[i]);
      for (int k = 0; k < 3; ++k)
        S(i, es_bx + k) = S(i, es_bx + k) + 0.5 * dt * (S(i, es_dbx + k) - tdb[3 * i + k]);
      S(i, es_t) = S(i, es_t) + 0.5 * dt * (S(i, es_ddt) - tddt[i]);
    }
    st[ec_time] = st[ec_time] + dt;
    cnt[SPH_CNT_STEPS]++;
    return SPH_OK;
  }

  int one_step(double tfinish, bool& done) {
    double t = st[ec_time];
    if (!((t < tfinish + eps0) && !stopped)) { done = true; return SPH_OK; }
    done = false;
    double dthydro, dtdiff, dtfld, dt;
    double t0 = omp_get_wtime();
    calctimestep(dthydro, dtdiff, dtfld, dt);
    timers[SPH_T_TIMESTEP] += 1e3 * (omp_get_wtime() - t0);
    bool do_sts = false;
    int sts_s = 0;
    if (eq_sts) {
      double sts_dt_min = std::min(dtdiff, dtfld);
      int sts_type = ival(ec_ststype);
      if (sts_type == ests_fixeds) {
        sts_s = ival(ec_stsfixeds);
        dthydro = (sts_s * sts_s + sts_s - 2.) * 0.25 * sts_dt_min;
        dt = dthydro;
        do_sts = true;
      } else if (sts_type == ests_auto) {
        if (dthydro > 0.) {
          double sts_classic = dthydro / sts_dt_min;
          sts_s = int(0.5 * std::sqrt(9. + 16. * sts_classic)) + 1;
          if (sts_classic > 1. && 2 * sts_s <= sts_classic) { dt = dthydro; do_sts = true; }
        }
      }
    }
    if (t + dt > tfinish) { dt = tfinish - t; stopped = true; }
    if (dtout > 0) {
      if (t >= ltout) { while (ltout <= t) ltout = ltout + dtout; }
      if (t + dt > ltout) {
        if (dtout < dt) ltout = ltout - dtout + dt;
        else dt = ltout - t;
      }
    }
    const int64_t n = n_integrated();
    t0 = omp_get_wtime();
    tr.resize(3 * n); tv.resize(3 * n); ta.resize(3 * n); tdu.resize(n); tdh.resize(n);
    tddt.resize(n); tdb.resize(3 * n);
    for (int64_t i = 0; i < n; ++i) {
      for (int k = 0; k < 3; ++k) {
        tr[3 * i + k] = S(i, es_rx + k); tv[3 * i + k] = S(i, es_vx + k);
        ta[3 * i + k] = S(i, es_ax + k); tdb[3 * i + k] = S(i, es_dbx + k);
      }
      tdu[i] = S(i, es_du); tdh[i] = S(i, es_dh);
      if (!do_sts) tddt[i] = S(i, es_ddt);
    }
    for (int64_t i = 0; i < n; ++i) {  // predictor, main.f90:333-342
      for (int k = 0; k < 3; ++k) {
        S(i, es_rx + k) = S(i, es_rx + k) + dt * tv[3 * i + k] + 0.5 * dt * dt * ta[3 * i + k];
        S(i, es_vx + k) = tv[3 * i + k] + dt * ta[3 * i + k];
      }
      S(i, es_u) = S(i, es_u) + dt * tdu[i];
      S(i, es_h) = S(i, es_h) + dt * tdh[i];
      if (!do_sts) S(i, es_t) = S(i, es_t) + dt * tddt[i];
      for (int k = 0; k < 3; ++k) S(i, es_bx + k) = S(i, es_bx + k) + dt * tdb[3 * i + k];
    }
    timers[SPH_T_PREDICT] += 1e3 * (omp_get_wtime() - t0);
    int rc = iterate();
    if (rc) return rc;
    t0 = omp_get_wtime();
    for (int64_t i = 0; i < n; ++i) {  // corrector, main.f90:348-362
      for (int k = 0; k < 3; ++k)
        S(i, es_vx + k) = S(i, es_vx + k) + 0.5 * dt * (S(i, es_ax + k) - ta[3 * i + k]);
      S(i, es_u) = S(i, es_u) + 0.5 * dt * (S(i, es_du) - tdu[i]);
      S(i, es_h) = S(i, es_h) + 0.5 * dt * (S(i, es_dh) - tdh[i]);
      for (int k = 0; k < 3; ++k)
        S(i, es_bx + k) = S(i, es_bx + k) + 0.5 * dt * (S(i, es_dbx + k) - tdb[3 * i + k]);
      if (!do_sts) S(i, es_t) = S(i, es_t) + 0.5 * dt * (S(i, es_ddt) - tddt[i]);
    }
    timers[SPH_T_CORRECT] += 1e3 * (omp_get_wtime() - t0);
    if (do_sts) {
      rc = sts_integrate(sts_s, dt);
      if (rc) return rc;
    }
    if (eq_radexch) {  // main.f90:367-369
      rc = update_radenergy(n, dt);
      if (rc) return rc;
    }
    st[ec_time] = t + dt;
    ++iterc;
    cnt[SPH_CNT_STEPS]++;
    return SPH_OK;
  }
};

// ---- closing error evaluation (main.f90:374-402, errcalc.f90) -----------
// Exact Sod density for errcalc.f90:26-44 (the reference calls SPLASH's
// exact_shock there); restated from the Riemann problem's equations
// (Toro ch. 4): p* by bisection of f_L(p) + f_R(p) + (u_R - u_L) = 0, then
// the wave pattern sampled at (x - x0) / t.
double sod_density(double x, double t, double g, double rl, double pl, double rr, double pr) {
  const double ul = 0.0, ur = 0.0, x0 = 0.0;
  if (!(t > 0.0)) return x < x0 ? rl : rr;
  const double cl = std::sqrt(g * pl / rl), cr = std::sqrt(g * pr / rr);
  const double z = (g - 1.0) / (2.0 * g);
  auto fk = [&](double p, double rk, double pk, double ck) {
    if (p > pk) {
      const double A = 2.0 / ((g + 1.0) * rk), B = (g - 1.0) / (g + 1.0) * pk;
      return (p - pk) * std::sqrt(A / (p + B));
    }
    return 2.0 * ck / (g - 1.0) * (std::pow(p / pk, z) - 1.0);
  };
  double lo = 0.0, hi = 10.0 * std::max(pl, pr);
  for (int it = 0; it < 200; ++it) {
    const double pm = 0.5 * (lo + hi);
    if (fk(pm, rl, pl, cl) + fk(pm, rr, pr, cr) + (ur - ul) > 0.0) hi = pm;
    else lo = pm;
  }
  const double p = 0.5 * (lo + hi);
  const double u = 0.5 * (ul + ur) + 0.5 * (fk(p, rr, pr, cr) - fk(p, rl, pl, cl));
  const double gg = (g - 1.0) / (g + 1.0);
  const double s = (x - x0) / t;
  if (s <= u) {
    if (p > pl) {
      const double sl = ul - cl * std::sqrt((g + 1.0) / (2.0 * g) * p / pl + z);
      return s <= sl ? rl : rl * ((p / pl + gg) / (gg * p / pl + 1.0));
    }
    if (s <= ul - cl) return rl;
    if (s <= u - cl * std::pow(p / pl, z))
      return rl * std::pow(2.0 / (g + 1.0) + (g - 1.0) / ((g + 1.0) * cl) * (ul - s),
                           2.0 / (g - 1.0));
    return rl * std::pow(p / pl, 1.0 / g);
  }
  if (p > pr) {
    const double sr = ur + cr * std::sqrt((g + 1.0) / (2.0 * g) * p / pr + z);
    return s >= sr ? rr : rr * ((p / pr + gg) / (gg * p / pr + 1.0));
  }
  if (s >= ur + cr) return rr;
  if (s >= u + cr * std::pow(p / pr, z))
    return rr * std::pow(2.0 / (g + 1.0) - (g - 1.0) / ((g + 1.0) * cr) * (ur - s),
                         2.0 / (g - 1.0));
  return rr * std::pow(p / pr, 1.0 / g);
}

// err_i of the real particles for the run's initial condition type, and
// L1 = sum err / realpn, summed in row order as Fortran's sum() does
int errcalc(const Oracle& o, double* err, double* l1) {
  const int64_t n = o.realpn;
  const int dim = o.ival(ec_dim), diso = o.ival(ec_disotropic), ivt = o.ival(ec_ics);
  const double t = o.st[ec_time];
  if (o.ival(ec_eqs) == eeq_kd2)
    return fail(SPH_ERR_UNSUPPORTED, "the Taylor (chi) error of equations = kd2 is not built");
  std::vector<double> e(size_t(n), 0.0);  // main.f90:202
  switch (ivt) {
    case ett_shock12:  // errcalc.f90:140-170
      for (int64_t i = 0; i < n; ++i) {
        const double tt = (diso == 1 || o.S(i, es_bx) == 1.) ? t : 1e-15;
        const double tr = 2., tl = 1.;
        const double exact = (tr + tl) / 2. + (tr - tl) / 2. * std::erf(o.S(i, es_rx) / std::sqrt(4 * tt));
        e[i] = std::fabs(exact - o.S(i, es_t));
      }
      break;
    case ett_ring:  // errcalc.f90:99-138
      for (int64_t i = 0; i < n; ++i) {
        const double x1 = o.S(i, es_rx), x2 = o.S(i, es_ry);
        const double rho = std::sqrt(x1 * x1 + x2 * x2);
        const double phi = std::atan2(x2, x1);
        const double exact = std::exp(-0.5 * ((rho - 0.3) * (rho - 0.3) / (0.05 * 0.05) +
                                              (phi * phi) / (0.5 * 0.5 + 2. * 1. * t / rho / rho)));
        e[i] = std::fabs(exact - o.S(i, es_t));
      }
      break;
    case ett_pulse: {  // errcalc.f90:46-97
      const double eps = 0.1, dcnd = o.st[ec_dcondconst];
      const double pifac = std::pow(2 * pi, -dim / 2.);
      const double ekt = eps * eps + 2 * dcnd * t;
      const double ektd2 = std::pow(ekt, dim / 2.);
      const double ektsq = std::pow(ekt, 1. / 2.);
      const double epsdm1 = powi(eps, dim - 1);
      for (int64_t i = 0; i < n; ++i) {
        const double x1 = o.S(i, es_rx), x2 = o.S(i, es_ry), x3 = o.S(i, es_rz);
        double exact;
        if (diso == 1) exact = pifac / ektd2 * std::exp(-0.5 * ((x1 * x1 + x2 * x2 + x3 * x3) / ekt));
        else exact = pifac / epsdm1 / ektsq * std::exp(-0.5 * (x1 * x1 / ekt + (x2 * x2 + x3 * x3) / eps / eps));
        e[i] = std::fabs(exact - o.S(i, es_t));
      }
      break;
    }
    case ett_sin3:  // errcalc.f90:172-197: filled only when ivt == 1, never for sin3
      break;
    case ett_soundwave:  // errcalc.f90:220-236
      for (int64_t i = 0; i < n; ++i)
        e[i] = std::fabs(1. + 0.005 * std::sin(pi * (o.S(i, es_rx) - t)) - o.S(i, es_den));
      break;
    case ett_hydroshock:  // errcalc.f90:26-44
      for (int64_t i = 0; i < n; ++i)
        e[i] = std::fabs(o.S(i, es_den) - sod_density(o.S(i, es_rx), t, 1.4, 1., 1., 1. / 8., 0.1));
      break;
    case ett_alfvenwave:  // errcalc.f90:198-218
      for (int64_t i = 0; i < n; ++i) {
        const double x1 = (o.S(i, es_rx) + 2 * o.S(i, es_ry) + 2 * o.S(i, es_rz)) / 3.;
        const double b2 = (o.S(i, es_by) - 2 * o.S(i, es_bx)) / std::sqrt(5.);
        e[i] = std::fabs(0.1 * std::sin(2. * pi * (x1 - t)) - b2);
      }
      break;
    case ett_OTvortex: case ett_mti: case ett_boilingtank: case ett_mtilowres: case -1:
      break;  // main.f90:377, 394-395
    default:
      return fail(SPH_ERR_UNSUPPORTED, "Task type was not sen in L2 error evaluation");
  }
  double sum = 0.0;
  for (int64_t i = 0; i < n; ++i) sum += e[i];
  if (err) std::copy(e.begin(), e.end(), err);
  if (l1) *l1 = n > 0 ? sum / double(n) : 0.0;
  return SPH_OK;
}

}  // namespace

struct sph_handle {
  Oracle o;
};

extern "C" {

const char* sph_last_error(void) { return g_err.c_str(); }

int sph_create(const double* state49, const double* store, int64_t n_rows,
               int kernel_id, int precision_mode, sph_handle** out) {
  if (!state49 || !store || !out || n_rows <= 0) return fail(SPH_ERR_ARG, "null argument");
  if (kernel_id < 0 || kernel_id > 2) return fail(SPH_ERR_ARG, "bad kernel id");
  if (precision_mode != SPH_PREC_FP64 && precision_mode != SPH_PREC_FP32_COMP)
    return fail(SPH_ERR_ARG, "bad precision mode");
  auto* h = new sph_handle();
  Oracle& o = h->o;
  o.kb = make_kernel(kernel_id);
  o.st.assign(SPH_P_LAST + 1, 0.);
  for (int k = 1; k <= SPH_EC_TOTAL; ++k) o.st[k] = state49[k - 1];
  o.st[SPH_P_AV_ALPHA] = 1.;
  o.st[SPH_P_AV_BETA] = 2.;
  o.st[SPH_P_NEWTON_TOL] = 1e-8;
  o.st[SPH_P_NEWTON_MAXITER] = 100;
  o.st[SPH_P_CELL_FACTOR] = 0.5;
  o.st[SPH_P_REORDER_EVERY] = 8;
  o.realpn = int64_t(o.st[ec_realpn]);
  o.fixedpn = int64_t(o.st[ec_fixedpn]);
  if (o.fixedpn < 0) o.fixedpn = 0;
  if (o.realpn <= 0 || o.realpn + o.fixedpn != n_rows) {
    delete h;
    return fail(SPH_ERR_ARG, "n_rows must equal realpn + fixedpn");
  }
  o.nrows = n_rows;
  o.store.assign(store, store + n_rows * ES);
  *out = h;
  return SPH_OK;
}

int sph_set_param(sph_handle* h, int index, double value) {
  if (!h || index < 1 || index > SPH_P_LAST) return fail(SPH_ERR_ARG, "bad param index");
  if ((index == ec_realpn || index == ec_fixedpn) && value != h->o.st[index])
    return fail(SPH_ERR_ARG, "particle counts are fixed by the store");
  h->o.st[index] = value;
  return SPH_OK;
}

int sph_get_param(sph_handle* h, int index, double* value) {
  if (!h || !value || index < 1 || index > SPH_P_LAST) return fail(SPH_ERR_ARG, "bad param index");
  *value = h->o.st[index];
  return SPH_OK;
}

int sph_set_store(sph_handle* h, const double* store, int64_t n_rows) {
  if (!h || !store || n_rows != h->o.nrows) return fail(SPH_ERR_ARG, "row count mismatch");
  h->o.clear_periodic();
  std::copy(store, store + n_rows * ES, h->o.store.begin());
  return SPH_OK;
}

int sph_iterate(sph_handle* h) {
  if (!h) return fail(SPH_ERR_ARG, "null handle");
  return h->o.iterate();
}

int sph_density(sph_handle* h) {
  if (!h) return fail(SPH_ERR_ARG, "null handle");
  return h->o.density_pass();
}

int sph_timestep(sph_handle* h, double* dt) {
  if (!h || !dt) return fail(SPH_ERR_ARG, "null argument");
  Oracle& o = h->o;
  o.eqset();
  int rc = o.initkernel();
  if (rc) return rc;
  double dthydro, dtdiff, dtfld;
  o.calctimestep(dthydro, dtdiff, dtfld, *dt);
  return SPH_OK;
}

int sph_predict(sph_handle* h, double dt) {
  if (!h) return fail(SPH_ERR_ARG, "null handle");
  return h->o.split_predict(dt);
}

int sph_forces(sph_handle* h) {
  if (!h) return fail(SPH_ERR_ARG, "null handle");
  return h->o.split_forces();
}

int sph_correct(sph_handle* h, double dt) {
  if (!h) return fail(SPH_ERR_ARG, "null handle");
  return h->o.split_correct(dt);
}

static int oracle_fields(const int* fields, int nf) {
  if (!fields || nf < 1 || nf > ES) return fail(SPH_ERR_ARG, "1 to 32 fields");
  for (int k = 0; k < nf; ++k)
    if (fields[k] < 1 || fields[k] > ES) return fail(SPH_ERR_ARG, "bad field index");
  return SPH_OK;
}

int sph_get_columns(sph_handle* h, const int* fields, int nf, double* buf) {
  if (!h || !buf) return fail(SPH_ERR_ARG, "null argument");
  int rc = oracle_fields(fields, nf);
  if (rc) return rc;
  Oracle& o = h->o;
  for (int k = 0; k < nf; ++k)
    for (int64_t i = 0; i < o.nrows; ++i) buf[k * o.nrows + i] = o.S(i, fields[k] - 1);
  return SPH_OK;
}

int sph_set_columns(sph_handle* h, const int* fields, int nf, const double* buf) {
  if (!h || !buf) return fail(SPH_ERR_ARG, "null argument");
  int rc = oracle_fields(fields, nf);
  if (rc) return rc;
  Oracle& o = h->o;
  for (int k = 0; k < nf; ++k)
    for (int64_t i = 0; i < o.nrows; ++i) o.S(i, fields[k] - 1) = buf[k * o.nrows + i];
  return SPH_OK;
}

int sph_step(sph_handle* h, int nsteps) {
  if (!h || nsteps < 0) return fail(SPH_ERR_ARG, "bad argument");
  Oracle& o = h->o;
  if (!o.started) {
    int rc = o.start_run();
    if (rc) return rc;
  }
  if (o.ival(ec_eqs) != eeq_kd2) o.stopped = false;
  for (int s = 0; s < nsteps; ++s) {
    bool done = false;
    int rc = o.one_step(o.st[ec_tfinish], done);
    if (rc) return rc;
    if (done) break;
  }
  return SPH_OK;
}

int sph_run_to(sph_handle* h, double tfinish) {
  if (!h) return fail(SPH_ERR_ARG, "null handle");
  Oracle& o = h->o;
  o.st[ec_tfinish] = tfinish;
  if (!o.started) {
    int rc = o.start_run();
    if (rc) return rc;
  }
  if (o.ival(ec_eqs) != eeq_kd2) o.stopped = false;
  for (;;) {
    bool done = false;
    int rc = o.one_step(tfinish, done);
    if (rc) return rc;
    if (done) break;
  }
  return SPH_OK;
}

int sph_get_store(sph_handle* h, double* out, int64_t cap_rows) {
  if (!h || !out || cap_rows < h->o.nrows) return fail(SPH_ERR_ARG, "buffer too small");
  std::copy(h->o.store.begin(), h->o.store.begin() + h->o.nrows * ES, out);
  return SPH_OK;
}

int sph_errcalc(sph_handle* h, double* err_out, int64_t cap, double* l1_out) {
  if (!h) return fail(SPH_ERR_ARG, "null handle");
  if (err_out && cap < h->o.realpn) return fail(SPH_ERR_ARG, "err_out holds fewer than realpn values");
  return errcalc(h->o, err_out, l1_out);
}

int sph_get_state(sph_handle* h, double* out49) {
  if (!h || !out49) return fail(SPH_ERR_ARG, "null argument");
  for (int k = 1; k <= SPH_EC_TOTAL; ++k) out49[k - 1] = h->o.st[k];
  return SPH_OK;
}

int sph_get_neighbours(sph_handle* h, int64_t* offsets, int64_t* pairs, int64_t cap) {
  if (!h || !offsets) return fail(SPH_ERR_ARG, "null argument");
  Oracle& o = h->o;
  if (o.noff.empty()) return fail(SPH_ERR_STATE, "no neighbour search yet");
  for (int64_t i = 0; i <= o.realpn; ++i) offsets[i] = o.noff[i];
  if (!pairs || cap < o.noff[o.realpn]) return fail(SPH_ERR_ARG, "pairs buffer too small");
  for (int64_t i = 0; i < o.realpn; ++i) {
    std::vector<int64_t> v;
    for (int64_t l = o.noff[i]; l < o.noff[i + 1]; ++l) {
      int64_t j = o.nidx[l];
      int64_t rj = j < o.nrows ? j : o.crossref[j - o.nrows];
      int64_t code = j < o.nrows ? 13 : o.gcode[j - o.nrows];
      v.push_back((rj << 5) | code);
    }
    std::sort(v.begin(), v.end());
    std::copy(v.begin(), v.end(), pairs + o.noff[i]);
  }
  return SPH_OK;
}

// Order-independent digest of each row's set (count, sum of a 64-bit mix of
// the sph_get_neighbours encoding), as the CUDA engine computes it.
static inline uint64_t mix64(uint64_t z) {
  z += 0x9e3779b97f4a7c15ull;
  z = (z ^ (z >> 30)) * 0xbf58476d1ce4e5b9ull;
  z = (z ^ (z >> 27)) * 0x94d049bb133111ebull;
  return z ^ (z >> 31);
}
int sph_get_neighbour_digest(sph_handle* h, uint64_t* out, int64_t n) {
  if (!h || !out) return fail(SPH_ERR_ARG, "null argument");
  Oracle& o = h->o;
  if (o.noff.empty()) return fail(SPH_ERR_STATE, "no neighbour search yet");
  if (n < o.realpn) return fail(SPH_ERR_ARG, "digest buffer shorter than the real rows");
#pragma omp parallel for schedule(static)
  for (int64_t i = 0; i < o.realpn; ++i) {
    uint64_t s = 0;
    for (int64_t l = o.noff[i]; l < o.noff[i + 1]; ++l) {
      const int64_t j = o.nidx[l];
      const int64_t rj = j < o.nrows ? j : o.crossref[j - o.nrows];
      const int64_t code = j < o.nrows ? 13 : o.gcode[j - o.nrows];
      s += mix64(uint64_t((rj << 5) | code));
    }
    out[2 * i] = uint64_t(o.noff[i + 1] - o.noff[i]);
    out[2 * i + 1] = s;
  }
  return SPH_OK;
}

// Reference numbering of the last neighbour lists (ghost rows numbered in the
// order createPeriodicBorder appends them).  Oracle-only helper for tests.
int sphref_get_neighbours_raw(sph_handle* h, int64_t* offsets, int64_t* idx, int64_t cap,
                              int64_t* crossref_out, int32_t* code_out, int64_t ghost_cap,
                              int64_t* n_ghosts) {
  if (!h || !offsets || !n_ghosts) return fail(SPH_ERR_ARG, "null argument");
  Oracle& o = h->o;
  *n_ghosts = o.periodpn;
  for (int64_t i = 0; i <= o.realpn; ++i) offsets[i] = o.noff[i];
  if (idx && cap >= o.noff[o.realpn]) std::copy(o.nidx.begin(), o.nidx.end(), idx);
  if (crossref_out && code_out && ghost_cap >= o.periodpn) {
    std::copy(o.crossref.begin(), o.crossref.end(), crossref_out);
    std::copy(o.gcode.begin(), o.gcode.end(), code_out);
  }
  return SPH_OK;
}

// Ghost rows (positions) of the last iterate; oracle-only helper for tests.
int sphref_get_ghost_positions(sph_handle* h, double* xyz, int64_t cap) {
  if (!h || !xyz) return fail(SPH_ERR_ARG, "null argument");
  Oracle& o = h->o;
  if (cap < o.periodpn) return fail(SPH_ERR_ARG, "buffer too small");
  for (int64_t g = 0; g < o.periodpn; ++g)
    for (int k = 0; k < 3; ++k) xyz[3 * g + k] = o.S(o.nrows + g, es_rx + k);
  return SPH_OK;
}

// STS coefficients (sts_integrator.f90:10-51), exported for the KAT.
double sphref_sts_coef(int which, int j, int s) {
  switch (which) {
    case 0: return Oracle::smu(j);
    case 1: return Oracle::snu(j);
    case 2: return Oracle::smu_hat(j, s);
    case 3: return Oracle::sgm_hat(j, s);
    case 4: return Oracle::sb(j);
    default: return 0.;
  }
}

// Kernel shape / wrappers for analytic identity tests.
double sphref_kernel_eval(int kernel_id, int dim, int what, double r, double h) {
  Oracle o;
  o.kb = make_kernel(kernel_id);
  o.dim = dim;
  o.wCv = o.kb.knorm[dim - 1];
  o.fwc = o.kb.fwcl[dim - 1];
  o.krad = o.kb.krad;
  ErrFlag e;
  switch (what) {
    case 0: return o.get_w(r, h, e);
    case 1: return o.get_dw_dh(r, h, e);
    case 2: return o.fab(r, h, e);
    case 3: return o.gab(r, h, e);
    case 4: return o.fw(r, h, e);
    case 5: return kf(kernel_id, r / h, e);
    case 6: return kdf(kernel_id, r / h, e);
    case 7: return kddf(kernel_id, r / h, e);
    case 8: return o.krad;
    default: return 0.;
  }
}

int sph_get_counters(sph_handle* h, int64_t* out, int n) {
  if (!h || !out) return fail(SPH_ERR_ARG, "null argument");
  for (int k = 0; k < n && k < SPH_CNT_TOTAL; ++k) out[k] = h->o.cnt[k];
  return SPH_OK;
}

int sph_reset_counters(sph_handle* h) {
  if (!h) return fail(SPH_ERR_ARG, "null argument");
  for (auto& c : h->o.cnt) c = 0;
  for (auto& t : h->o.timers) t = 0.;
  return SPH_OK;
}

int sph_get_timers(sph_handle* h, double* out_ms, int n) {
  if (!h || !out_ms) return fail(SPH_ERR_ARG, "null argument");
  for (int k = 0; k < n && k < SPH_T_TOTAL; ++k) out_ms[k] = h->o.timers[k];
  return SPH_OK;
}

void sph_destroy(sph_handle* h) { delete h; }

// Batches: the reference runs the instances of a sweep one after another
// (runner/anisotropic/000_anisopaper_v1_gls_kxx.py through CleanRun /
// ContinueRun, core.py:152-156), and so does the oracle.
struct sph_batch {
  std::vector<sph_handle*> h;
  std::vector<int> status;
};

int sph_batch_create(int n_inst, sph_handle* const* handles, sph_batch** out) {
  if (!out || !handles || n_inst <= 0) return fail(SPH_ERR_ARG, "bad batch arguments");
  for (int i = 0; i < n_inst; ++i) {
    if (!handles[i]) return fail(SPH_ERR_ARG, "null handle in batch");
    for (int j = 0; j < i; ++j)
      if (handles[j] == handles[i]) return fail(SPH_ERR_ARG, "handle twice in batch");
  }
  auto* b = new sph_batch();
  b->h.assign(handles, handles + n_inst);
  b->status.assign(n_inst, 0);
  *out = b;
  return SPH_OK;
}

static int batch_each(sph_batch* b, const std::function<int(sph_handle*)>& fn) {
  int first = SPH_OK;
  std::string msg;
  for (size_t i = 0; i < b->h.size(); ++i) {
    b->status[i] = fn(b->h[i]);
    if (b->status[i] && !first) {
      first = b->status[i];
      msg = "instance " + std::to_string(i) + ": " + g_err;
    }
  }
  return first ? fail(first, msg) : SPH_OK;
}

int sph_batch_step(sph_batch* b, int nsteps) {
  if (!b || nsteps < 0) return fail(SPH_ERR_ARG, "bad argument");
  return batch_each(b, [nsteps](sph_handle* h) { return sph_step(h, nsteps); });
}

int sph_batch_run_to(sph_batch* b, double tfinish) {
  if (!b) return fail(SPH_ERR_ARG, "null batch");
  return batch_each(b, [tfinish](sph_handle* h) { return sph_run_to(h, tfinish); });
}

int sph_batch_status(sph_batch* b, int* status, int n) {
  if (!b || !status) return fail(SPH_ERR_ARG, "null argument");
  for (int i = 0; i < n && i < int(b->status.size()); ++i) status[i] = b->status[i];
  return SPH_OK;
}

void sph_batch_destroy(sph_batch* b) { delete b; }

}  // extern "C"
