// sph_engine.cu — the C-ABI of include/sph_abi.h and the host-side
// orchestration of one SPH step on the device:
//   iterate  (iterator.f90:44-179): reflect -> periodic images -> cell keys ->
//            radix sort -> cell ranges -> neighbour lists -> circuit1 (+EOS)
//            -> circuit2
//   step     (main.f90:241-373): timestep -> predictor -> iterate ->
//            corrector -> STS stages
// Everything runs on one CUDA stream per handle.  The host reads back a few
// scalars per iterate (image count and bounding box, the largest neighbour
// count, the Newton "still active" flag on the Jacobi path, the timestep
// reductions) and nothing else.
#include <algorithm>
#include <atomic>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <limits>
#include <map>
#include <mutex>
#include <string>
#include <vector>

#include "sph_internal.h"

#include <chrono>

using namespace sph;

namespace {

thread_local std::string g_err;
std::atomic<long long> g_launches{0};

int fail(int code, const std::string& msg) {
  g_err = msg;
  return code;
}

#define CK(call)                                                                     \
  do {                                                                               \
    cudaError_t e_ = (call);                                                         \
    if (e_ != cudaSuccess)                                                           \
      return fail(SPH_ERR_CUDA, std::string(#call) + ": " + cudaGetErrorString(e_)); \
  } while (0)

#define RC(call)             \
  do {                       \
    int rc_ = (call);        \
    if (rc_) return rc_;     \
  } while (0)

// state slots (const.f90:14-66)
enum : int {
  ec_dim = 1, ec_eqs = 2, ec_ddw = 3, ec_ics = 4, ec_adden = 5, ec_artts = 6,
  ec_coordsys = 7, ec_disotropic = 8, ec_dcondconst = 9, ec_muzero = 10,
  ec_tfinish = 11, ec_hfac = 13, ec_xmin = 17, ec_xmax = 18, ec_ymin = 19,
  ec_ymax = 20, ec_zmin = 21, ec_zmax = 22, ec_bordsize = 23, ec_padding = 24,
  ec_realpn = 25, ec_fixedpn = 26, ec_gamma = 27, ec_dtprint = 30,
  ec_process = 31, ec_au = 32, ec_eqonhydro = 34, ec_eqondiff = 35,
  ec_eqonfluxlim = 36, ec_eqonradexch = 37, ec_eqonsts = 38, ec_time = 46,
  ec_molecularmass = 47,
  ec_ststype = 48, ec_stsfixeds = 49
};
enum : int { eeq_hydro = 300, eeq_diffusion = 301, eeq_magnetohydro = 302,
             eeq_magnetohydrodiffusion = 303, eeq_hydrodiffusion = 304,
             eeq_kd2 = 305, eeq_hyrad = 306, eeq_manual = 307 };
enum : int { epc_backcompatibility = 600, epc_fullyperiodic = 601, epc_borderless = 602 };
enum : int { ett_sin3 = 100, ett_mti = 101, ett_shock12 = 102, ett_pulse = 103, ett_ring = 104,
             ett_soundwave = 105, ett_hydroshock = 106, ett_alfvenwave = 107, ett_OTvortex = 108,
             ett_boilingtank = 109, ett_mtilowres = 110, ett_fld_gauss = 111, e_none = -1 };

const double kPi = 4.0 * std::atan(1.0);

// kernel bases (kernel/base_m4.f90:12-32, base_m6.f90:13-33, base_gauss.f90:15-36)
struct KBase {
  double knorm[3], fwcl[3];
  int maxneib[3];
  double krad, cn_hydro, cn_2nw, cn_fab, cn_n2w;
};
KBase kbase(int id) {
  KBase k;
  if (id == SPH_KERNEL_M6) {
    k = {{1. / 120., 7. / (478. * kPi), 1. / (120. * kPi)}, {4., 9.31505 / 2.25, 9.6429 / 2.25},
         {50, 10000, 150}, 3., 0.3, 1.1, 0.2, 0.4};
  } else if (id == SPH_KERNEL_M4) {
    k = {{2. / 3., 10. / (7. * kPi), 1. / kPi}, {6., 6.3226, 6.66400}, {35, 250, 150},
         2., 0.1, 0.96, 0.15, 0.2};
  } else {
    k = {{1. / std::sqrt(kPi), 1. / kPi, 1. / std::pow(kPi, 1.5)}, {4., 4., 4.},
         {100, 5000, 50000}, 10., 0.55, 1.25, 0.24, 0.50};
  }
  return k;
}

// device allocations made by DevBuf::ensure on this thread's current handle
thread_local int64_t* t_alloc_count = nullptr;

// Device memory of all handles of the process, cached: a block given back
// (a handle destroyed, a buffer outgrown) waits in its device's free list
// for the next request of a similar size instead of going back to the
// driver.  cudaMalloc and cudaFree cost tens of microseconds each and
// cudaFree waits for the whole device; a batch's instances start with
// about 80 buffers each.  A block is given back only when no work of its
// handle can still use it (the handle's stream synchronised, or the device
// for an outgrown buffer); a request the driver cannot serve first returns
// the device's cached blocks to it.  At most kCacheMax bytes wait per device.
class DevCache {
 public:
  static DevCache& get() {
    static DevCache* c = new DevCache();  // (never destroyed: handles may outlive statics)
    return *c;
  }
  cudaError_t take(size_t want, void** p, size_t* got, int* dev) {
    cudaGetDevice(dev);
    {
      std::lock_guard<std::mutex> lk(mu_);
      auto& f = free_[*dev];
      auto it = f.lower_bound(want);
      // a cached block at most 1.5x the request (no large block for a small one)
      if (it != f.end() && it->first <= want + want / 2) {
        *p = it->second;
        *got = it->first;
        cached_[*dev] -= it->first;
        f.erase(it);
        return cudaSuccess;
      }
    }
    cudaError_t e = cudaMalloc(p, want);
    if (e != cudaSuccess) {
      cudaGetLastError();
      release(*dev);
      e = cudaMalloc(p, want);
    }
    if (e == cudaSuccess) *got = want;
    return e;
  }
  void give(void* p, size_t bytes, int dev) {
    {
      std::lock_guard<std::mutex> lk(mu_);
      if (cached_[dev] + bytes <= kCacheMax) {
        free_[dev].insert({bytes, p});
        cached_[dev] += bytes;
        return;
      }
    }
    int cur = 0;
    cudaGetDevice(&cur);
    if (cur != dev) cudaSetDevice(dev);
    cudaFree(p);
    if (cur != dev) cudaSetDevice(cur);
  }

 private:
  static constexpr size_t kCacheMax = size_t(16) << 30;
  void release(int dev) {
    std::multimap<size_t, void*> f;
    {
      std::lock_guard<std::mutex> lk(mu_);
      f.swap(free_[dev]);
      cached_[dev] = 0;
    }
    for (auto& b : f) cudaFree(b.second);
  }
  std::mutex mu_;
  std::map<int, std::multimap<size_t, void*>> free_;
  std::map<int, size_t> cached_;
};

struct DevBuf {
  void* p = nullptr;
  size_t bytes = 0;
  int dev = 0;
  ~DevBuf() {
    if (p) DevCache::get().give(p, bytes, dev);
  }
  int ensure(size_t b) {
    if (b <= bytes && p) return SPH_OK;
    if (p) {
      // work queued before this call may still use the old block
      cudaDeviceSynchronize();
      DevCache::get().give(p, bytes, dev);
    }
    p = nullptr;
    bytes = 0;
    // 25% headroom: sizes that follow the image count move by a few rows
    // between steps and must not trigger a new block every time
    size_t nb = std::max<size_t>(b + b / 4, 256);
    if (t_alloc_count) ++*t_alloc_count;
    static const bool log_allocs = std::getenv("SPH_ALLOC_LOG") != nullptr;
    if (log_allocs) std::fprintf(stderr, "sph: device allocation of %zu bytes\n", nb);
    cudaError_t e = DevCache::get().take(nb, &p, &bytes, &dev);
    if (e != cudaSuccess) {
      p = nullptr;
      bytes = 0;
      return fail(SPH_ERR_OOM, std::string("cudaMalloc: ") + cudaGetErrorString(e));
    }
    return SPH_OK;
  }
  template <class T> T* as() const { return static_cast<T*>(p); }
};

struct Mode {
  bool ghosts = false;
  int periodic[3] = {0, 0, 0};
  int reflect[3] = {0, 0, 0};
  int eos_kind = 1;
  int mti = 0;  // 1 mti, 2 mtilowres
};

}  // namespace

namespace sph {
int sph_fail(int code, const std::string& msg) { return fail(code, msg); }
void note_launch(int n) { g_launches += n; }
long long launches_so_far() { return g_launches; }
}  // namespace sph

// Jacobi sweeps of circuit1 that a device-resident step runs before it asks
// the host (a step whose particles need more is redone on the host path)
constexpr int kDrsSweeps = 6;
constexpr int kSkinShort = 4, kSkinPause0 = 8, kSkinPauseMax = 128;
// centres searched afresh above which the search's own kernel takes them
constexpr int64_t kFewCentres = 65536;
// fresh searches of a served iterate (centres x widening) as a share of all
// centres, above which the iterate searches plainly instead
constexpr double kSkinDirtyShare = 0.15;

struct sph_handle {
  int dev = 0;  // the device current at sph_create
  int kernel_id = SPH_KERNEL_M6;
  int prec = SPH_PREC_FP64;
  KBase kb;
  std::vector<double> st;  // 1-based
  int64_t nrows = 0, nreal = 0, nfixed = 0, n_int = 0;
  cudaStream_t s = nullptr;

  // canonical store, SoA columns of length nrows
  DevBuf cols, cols_alt, orig, orig_alt, staging;
  // predictor saves, STS stages, circuit1 iterates
  DevBuf save, stsY, hkp1, dkp1, okp1, epsb;
  // images
  DevBuf gcount, goff, gx, gy, gz, gsrc, gcode, scan_tmp;
  int64_t nghost = 0;
  // sort + cells
  DevBuf keys, keys_alt, vals, vals_alt, sort_tmp, cstart;
  DevBuf cell_count, cell_ctr;  // the counting sort's counts and counters
  // sorted arrays
  DevBuf sx, sy, sz, s32, ssrc, cflag, cpos, centre_k, centre_p;
  DevBuf hk_s, dk_s, ok_s;
  DevBuf pk[11], qk[7], qunit;
  // neighbours: one row per centre inside nl, rows sized from each
  // particle's previous count (CSR with slack)
  DevBuf nl, ncnt, rowoff, rowcap, rowcap64, count_prev, h_prev, scan64_tmp, overflow;
  // adjoint: per-row adjoint columns, d/d(alpha, beta), checkpoints of the
  // particle table (the run's initial state, every k-th step, the final one)
  // and the states of the segment being replayed
  DevBuf adj, adj_par, adj_ckpt, adj_seg, adj_io;
  // device-resident steps (SPH_P_GRAPH): the per-step plan, clock and error
  // word on the device, the table saved at the start of a step (restored
  // when the step has to be redone on the host path), the capacities the
  // step is planned for, and the captured CUDA graph of one step
  DevBuf drs_plan, drs_clock, drs_err, drs_save;
  // a batch's device loop: the clock saved at the start of the instance's
  // step (restored when the step is redone on the host path), and a count
  // of parameter changes (a captured loop holds the values it saw)
  DevBuf bclk_save;
  long long param_gen = 0;
  // between sph_predict and sph_correct of a split step: the rows keep their
  // physical order (the predictor's saves are per physical row)
  bool in_split_step = false;
  // the start-up iterate of an instance joining the batch device loop, which
  // searches afresh every iterate: lists built then would serve none
  bool skin_suspended = false;
  DevBuf colbuf;  // staging of sph_get_columns / sph_set_columns
  // A table upload or download crosses PCIe in kXferChunks pieces on the
  // copy stream xs while the compute stream transposes the piece before
  // (upload: after) it; xfer_ev orders the two
  static constexpr int kXferChunks = 8;
  cudaStream_t xs = nullptr;
  std::vector<cudaEvent_t> xfer_ev;
  DevBuf dl_inv;  // the inverse of orig for a download
  int xfer_setup() {
    if (!xs) CK(cudaStreamCreateWithFlags(&xs, cudaStreamNonBlocking));
    while (xfer_ev.size() < size_t(kXferChunks + 1)) {
      cudaEvent_t e = nullptr;
      CK(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
      xfer_ev.push_back(e);
    }
    return SPH_OK;
  }
  int64_t xfer_rows() const { return ((nrows + kXferChunks - 1) / kXferChunks + 31) / 32 * 32; }
  // skin lists (SPH_P_SKIN): the lists of the last skin search (CSR like nl),
  // the records' positions and the centres' h at that search, the rows'
  // image signatures then; per record the largest displacement since; per
  // cell the dilated marks of fast / moving records; per centre the gap of its
  // list at the search, the largest change of h since, its way (filter,
  // search afresh, keep), the fresh-search flag, its scan and those centres
  DevBuf skin_nl, skin_rowoff, skin_rowcap, skin_rowcap64, skin_cnt, skin_count_prev,
      skin_h_prev, skin_bx, skin_by, skin_bz, skin_hb, skin_sig, skin_dsp, skin_fcell,
      skin_mcell, skin_ctmp, skin_gap, skin_hdev, skin_mode, skin_dflag, skin_dpos, skin_dlist,
      skin_hrec, skin_ways, skin_wpos, skin_flist;
  // the rows of the centres searched afresh, laid out anew every skin-list
  // iterate after the end of the table's fixed part (skin_end[0]): their
  // capacities and the scan of those
  DevBuf skin_end, skin_dcap, skin_doff;
  DevBuf skin_gate;  // the iterate's checks and mark windows (k_skin_gate)
  // rows renamed: spare signatures, the two permutations, the old types, a flag
  DevBuf skin_sig_alt, skin_inv, skin_perm, skin_type, skin_flag;
  int64_t skin_nl_size = 0;
  int skin_est = 0;
  bool skin_valid = false;  // the skin lists describe the records of the current sort
  double skin_s = 0.;        // their fraction s (radius (1 + s) krad h)
  double skin_tau = 0.;      // displacement up to which a record is slow
  double skin_eps = 0.;      // displacement up to which a record is still
  double skin_hmin = 0.;     // h_min at their search
  int skin_age = 0;          // iterates served since their search
  // lists that serve fewer than kSkinShort iterates cost more than they save
  // (their search is dearer than a plain one): after such lists the next
  // skin_pause iterates search plainly, a pause that doubles while lists
  // keep ending early (up to kSkinPauseMax) and resets when they last
  int skin_pause = 0, skin_pause_len = 0;
  bool skin_live = false;  // lists built and not yet replaced by a plain search
  bool skin_trace = std::getenv("SPH_SKIN_TRACE") != nullptr;
  int64_t kept_pairs = 0;    // neighbour pairs of the rows kept (counted as found)
  const DevPlan* dplan = nullptr;  // set while a device-resident step is built
  // skin lists of the device-resident step (DevSkin, device memory): they
  // share the host lists' buffers; dlists_ok = nothing on the host has
  // touched the records, rows or lists since the last device-resident run
  // (else the next one starts without lists)
  DevBuf dskin;
  bool dlists_ok = false;
  DevBuf c1_iter;  // the sweep count of the device-resident Newton loop
  // the device-resident STS loop: its stage index and the coefficients of
  // stages 2 .. s (mu, nu, muhat, gmhat), for the s they were made for
  DevBuf sts_j, sts_coef;
  int sts_coef_s = 0;
  std::vector<cudaStream_t> cap_s;  // capture the bodies of conditional nodes, one per level
  int cap_depth = 0;
  int64_t nghost_cap = 0, nall_cap = 0;
  int end_bit_cap = 0;
  // captured steps, one per table pointer pair: a row reorder swaps the
  // table with its spare, so two captures serve a reordering run
  struct GraphSlot {
    cudaGraph_t g = nullptr;
    cudaGraphExec_t x = nullptr;
    const void* k_cols = nullptr;
    const void* k_orig = nullptr;
  };
  GraphSlot gslot[2];
  int gslot_next = 0;
  bool graph_dirty = true;        // every capture is stale (parameters, sizes, buffers)
  int64_t graph_alloc_mark = -1;  // allocations seen when the graph was captured
  DevPlan* h_plan = nullptr;      // pinned read-back of the last device plan
  int adj_nsteps = -1, adj_every = 0, adj_ncp = 0;
  bool adj_initial_force = false;
  double adj_dt = 0., adj_t0 = 0.;
  int64_t nl_size = 0;
  int est_count = 0;
  // scalars
  DevBuf status, red, dcnt, maxcnt, ctrl, ciso;
  unsigned long long* h_red = nullptr;  // pinned
  double* h_ctrl = nullptr;             // pinned
  int32_t* h_i32 = nullptr;             // pinned scratch

  Grid grid{};
  PackGeom pgeom{};
  double mref = 1.0;
  bool have_order = false;
  bool rows_in_order = false;  // the rows are in the order of the current sort
  int steps_since_reorder = 0;

  // time loop state (main.f90)
  bool started = false, stopped = false;
  double ltout = 0., dtout = 0.;

  int64_t cnt_host[SPH_CNT_TOTAL] = {0};
  int64_t host_max_sweeps = 0;  // Newton sweeps of the Jacobi path
  long long launch_base = 0;    // g_launches at create / reset
  double timers[SPH_T_TOTAL] = {0};
  std::vector<std::pair<int, std::pair<cudaEvent_t, cudaEvent_t>>> pending_ev;
  std::vector<cudaEvent_t> ev_pool;

  // equation set (state.f90:117-149)
  bool eq_hydro = false, eq_magneto = false, eq_diff = false, eq_fld = false,
       eq_radexch = false, eq_sts = false;

  int ival(int k) const { return int(st[k]); }

  double* col(int f) const { return cols.as<double>() + int64_t(f) * nrows; }

  // ---- timing -------------------------------------------------------------------
  cudaEvent_t get_event() {
    if (!ev_pool.empty()) {
      cudaEvent_t e = ev_pool.back();
      ev_pool.pop_back();
      return e;
    }
    cudaEvent_t e;
    cudaEventCreate(&e);
    return e;
  }
  struct Phase {
    sph_handle* h;
    int slot;
    cudaEvent_t a = nullptr, b = nullptr;
    Phase(sph_handle* hh, int sl) : h(hh), slot(sl) {
      const double mode = h->st[SPH_P_TIMING];
      if (!h->dplan && (mode == 1 || (mode == 2 && sl == SPH_T_STEP))) {
        a = h->get_event();
        b = h->get_event();
        cudaEventRecord(a, h->s);
      }
    }
    ~Phase() {
      if (a) {
        cudaEventRecord(b, h->s);
        h->pending_ev.push_back({slot, {a, b}});
      }
    }
  };
  void collect_timers() {
    for (auto& pe : pending_ev) {
      float ms = 0.f;
      cudaEventSynchronize(pe.second.second);
      if (cudaEventElapsedTime(&ms, pe.second.first, pe.second.second) == cudaSuccess)
        timers[pe.first] += ms;
      ev_pool.push_back(pe.second.first);
      ev_pool.push_back(pe.second.second);
    }
    pending_ev.clear();
  }

  // ---- configuration ------------------------------------------------------------------
  void eqset() {
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
  }
  int dim() const { return ival(ec_dim); }
  static int lanes_ok(int g) { return (g == 4 || g == 8 || g == 16 || g == 32) ? g : 0; }
  int lanes_search() const {
    int g = lanes_ok(int(st[SPH_P_LANES_SEARCH]));
    return g ? g : (dim() == 3 ? 8 : 8);
  }
  int lanes_pair() const {
    int g = lanes_ok(int(st[SPH_P_LANES_PAIR]));
    return g ? g : (dim() == 3 ? 8 : 4);
  }

  int params(Params& P) {
    eqset();
    int d = dim();
    if (d < 1 || d > 3) return fail(SPH_ERR_ARG, "Dimmention is wrong");
    if (ival(ec_coordsys) == 2)
      return fail(SPH_ERR_UNSUPPORTED, "cylindric coordinates: Fab_cylindric does not exist (kernel.f90:137)");
    P.dim = d;
    P.kernel = kernel_id;
    P.krad = kb.krad;
    P.wCv = kb.knorm[d - 1];
    P.fwc = kb.fwcl[d - 1];
    P.hfac = st[ec_hfac];
    P.alpha = st[SPH_P_AV_ALPHA];
    P.beta = st[SPH_P_AV_BETA];
    P.au = st[ec_au];
    P.gamma = st[ec_gamma];
    P.muzero = st[ec_muzero];
    P.difcond = st[ec_dcondconst];
    P.difiso = ival(ec_disotropic);
    P.ddw = ival(ec_ddw);
    P.full_tensor = st[SPH_P_FULL_TENSOR] != 0;
    P.eq_hydro = eq_hydro; P.eq_magneto = eq_magneto; P.eq_diff = eq_diff; P.eq_fld = eq_fld;
    P.adden = ival(ec_adden);
    P.artts = ival(ec_artts);
    P.tol = st[SPH_P_NEWTON_TOL];
    P.maxiter = std::max(0, int(st[SPH_P_NEWTON_MAXITER]));
    P.eos_kind = 1;
    P.c_iso = 0.;
    if (eq_diff && eq_fld && P.difiso != 1)
      return fail(SPH_ERR_FLD_ANISO, "There is no anisotropic for FLD");
    if (eq_diff && !(P.ddw == esd_fw || P.ddw == esd_fab || P.ddw == esd_n2w ||
                     P.ddw == esd_2nw_ds || P.ddw == esd_2nw_sd))
      return fail(SPH_ERR_DDW, "second deriv id not found");
    return SPH_OK;
  }
  // cnd2 (kernel.f90:108-134)
  double cnd2() const {
    int ddw = ival(ec_ddw);
    if (ddw == esd_n2w) return kb.cn_n2w;
    if (ddw == esd_2nw_ds || ddw == esd_2nw_sd) return kb.cn_2nw;
    return kb.cn_fab;
  }

  int mode(Mode& m) {
    int ipc = ival(ec_process), ivt = ival(ec_ics), d = dim();
    auto all = [&](int* a) { for (int k = 0; k < d; ++k) a[k] = 1; };
    if (ipc == epc_fullyperiodic) {
      m.ghosts = true; all(m.periodic); all(m.reflect);
    } else if (ipc == epc_borderless) {
    } else if (ipc == epc_backcompatibility) {
      switch (ivt) {
        case ett_shock12: m.ghosts = true; if (d > 1) m.periodic[1] = 1; break;
        case ett_pulse: case ett_ring: case ett_fld_gauss: m.eos_kind = 0; break;
        case ett_soundwave: m.ghosts = true; all(m.periodic); all(m.reflect); m.eos_kind = 2; break;
        case ett_OTvortex: m.ghosts = true; all(m.periodic); all(m.reflect); break;
        case ett_hydroshock:
          m.ghosts = true;
          if (d > 1) { m.periodic[1] = m.reflect[1] = 1; }
          if (d > 2) { m.periodic[2] = m.reflect[2] = 1; }
          break;
        case ett_mti: case ett_mtilowres:
          m.ghosts = true; m.periodic[0] = m.reflect[0] = 1; m.mti = ivt == ett_mti ? 1 : 2; break;
        default: return fail(SPH_ERR_PROCESS, "Task type was not set");
      }
    } else {
      return fail(SPH_ERR_PROCESS, "Process type was not set");
    }
    return SPH_OK;
  }

  BoxGeom box(const Mode& m) const {
    BoxGeom g;
    double bs = st[ec_bordsize], pad = st[ec_padding];
    g.emin[0] = st[ec_xmin]; g.emax[0] = st[ec_xmax];
    g.emin[1] = st[ec_ymin]; g.emax[1] = st[ec_ymax];
    g.emin[2] = st[ec_zmin]; g.emax[2] = st[ec_zmax];
    for (int k = 0; k < 3; ++k) {
      g.boxmin[k] = g.emin[k] + bs;  // BC.f90:63-64
      g.boxmax[k] = g.emax[k] - bs;
      g.pmin[k] = g.emin[k];         // BC.f90:210-223 (padding/10 only when padding == 0)
      g.pmax[k] = g.emax[k];
      if (pad == 0) { g.pmin[k] = g.emin[k] + pad / 10; g.pmax[k] = g.emax[k] - pad / 10; }
      g.periodic[k] = m.periodic[k];
      g.reflect[k] = m.reflect[k];
    }
    return g;
  }

  // ---- allocation -----------------------------------------------------------------------
  int alloc_base() {
    RC(cols.ensure(sizeof(double) * NCOL * nrows));
    RC(cols_alt.ensure(sizeof(double) * NCOL * nrows));
    RC(orig.ensure(sizeof(int32_t) * nrows));
    RC(orig_alt.ensure(sizeof(int32_t) * nrows));
    RC(staging.ensure(sizeof(double) * NCOL * nrows));
    RC(dl_inv.ensure(sizeof(int32_t) * nrows));
    RC(xfer_setup());  // (the table transfers' copy stream and events)
    RC(save.ensure(sizeof(double) * 9 * nrows));
    RC(hkp1.ensure(sizeof(double) * nrows));
    RC(dkp1.ensure(sizeof(double) * nrows));
    RC(okp1.ensure(sizeof(double) * nrows));
    RC(epsb.ensure(sizeof(double) * nrows));
    RC(gcount.ensure(sizeof(int32_t) * (nrows + 1)));
    RC(goff.ensure(sizeof(int32_t) * (nrows + 1)));
    RC(status.ensure(sizeof(int)));
    RC(red.ensure(sizeof(unsigned long long) * RED_TOTAL));
    RC(dcnt.ensure(sizeof(unsigned long long) * DC_TOTAL));
    RC(maxcnt.ensure(sizeof(int32_t)));
    RC(overflow.ensure(sizeof(int32_t)));
    RC(count_prev.ensure(sizeof(int32_t) * nrows));
    RC(h_prev.ensure(sizeof(float) * nrows));
    RC(rowoff.ensure(sizeof(int64_t) * nreal));
    RC(rowcap.ensure(sizeof(int32_t) * nreal));
    RC(rowcap64.ensure(sizeof(int64_t) * nreal));
    RC(ncnt.ensure(sizeof(int32_t) * nreal));
    RC(scan64_tmp.ensure(scan64_temp_bytes(nreal)));
    RC(ctrl.ensure(sizeof(double) * 8));
    RC(ciso.ensure(sizeof(double)));
    CK(cudaMemsetAsync(status.p, 0, sizeof(int), s));
    CK(cudaMemsetAsync(dcnt.p, 0, sizeof(unsigned long long) * DC_TOTAL, s));
    CK(cudaMemsetAsync(ctrl.p, 0, sizeof(double) * 8, s));
    CK(cudaMemsetAsync(save.p, 0, sizeof(double) * 9 * nrows, s));
    size_t sb = scan_temp_bytes(nrows + 1);
    RC(scan_tmp.ensure(sb));
    return SPH_OK;
  }
  int alloc_all(int64_t nall) {
    RC(keys.ensure(sizeof(uint32_t) * nall));
    RC(keys_alt.ensure(sizeof(uint32_t) * nall));
    RC(vals.ensure(sizeof(int32_t) * nall));
    RC(vals_alt.ensure(sizeof(int32_t) * nall));
    RC(sort_tmp.ensure(sort_temp_bytes(nall)));
    RC(sx.ensure(sizeof(double) * nall));
    RC(sy.ensure(sizeof(double) * nall));
    RC(sz.ensure(sizeof(double) * nall));
    RC(s32.ensure(sizeof(float4) * nall));
    RC(ssrc.ensure(sizeof(int32_t) * nall));
    RC(cflag.ensure(sizeof(int32_t) * (nall + 1)));
    RC(cpos.ensure(sizeof(int32_t) * (nall + 1)));
    RC(centre_k.ensure(sizeof(int32_t) * std::max<int64_t>(nreal, 1)));
    RC(centre_p.ensure(sizeof(int32_t) * std::max<int64_t>(nreal, 1)));
    RC(hk_s.ensure(sizeof(double) * nall));
    RC(dk_s.ensure(sizeof(double) * nall));
    RC(ok_s.ensure(sizeof(double) * nall));
    size_t sb = scan_temp_bytes(nall + 1);
    if (sb > scan_tmp.bytes) RC(scan_tmp.ensure(sb));
    if (prec == SPH_PREC_FP64) {
      for (int i = 0; i < 11; ++i) RC(pk[i].ensure(sizeof(double2) * nall));
    } else {
      for (int i = 0; i < 7; ++i) RC(qk[i].ensure(sizeof(float4) * nall));
      RC(qunit.ensure(sizeof(float)));
    }
    return SPH_OK;
  }
  PackBufs packs() const {
    PackBufs pb;
    for (int i = 0; i < 11; ++i) pb.p[i] = pk[i].as<double2>();
    for (int i = 0; i < 7; ++i) pb.q[i] = qk[i].as<float4>();
    pb.unit = qunit.as<float>();
    return pb;
  }

  int check_status() {
    int code = 0;
    CK(cudaMemcpyAsync(h_i32, status.p, sizeof(int), cudaMemcpyDeviceToHost, s));
    CK(cudaStreamSynchronize(s));
    code = h_i32[0];
    if (code) {
      CK(cudaMemsetAsync(status.p, 0, sizeof(int), s));
      const char* msg = "device error";
      switch (code) {
        case SPH_ERR_Q_NAN: msg = "q is nan"; break;
        case SPH_ERR_Q_NEG: msg = "q is negative"; break;
        case SPH_ERR_H_NEG: msg = "Negative smoothing length in c1 advanced"; break;
        case SPH_ERR_RAD_NEGATIVE: msg = "radiation or thermal energy is negative after exchange"; break;
        default: break;
      }
      return fail(code, msg);
    }
    return SPH_OK;
  }

  // what names rows under skin lists, after old row perm[i] became row i
  // (inv[perm[i]] = i)
  int rename_rows(const int32_t* perm, const int32_t* inv) {
    RC(skin_sig_alt.ensure(sizeof(uint8_t) * nrows));
    launch_rows_renamed(perm, inv, nrows + nghost, nrows, nghost, nreal, vals_alt.as<int32_t>(),
                        ssrc.as<int32_t>(), gsrc.as<int32_t>(), centre_p.as<int32_t>(),
                        skin_sig.as<uint8_t>(), skin_sig_alt.as<uint8_t>(), s);
    std::swap(skin_sig.p, skin_sig_alt.p);
    std::swap(skin_sig.bytes, skin_sig_alt.bytes);
    std::swap(skin_sig.dev, skin_sig_alt.dev);
    return SPH_OK;
  }

  // ---- physical re-ordering of the rows (locality of the pair loops) ---------------------
  int reorder_rows() {
    if (!have_order || in_split_step || rows_in_order) return SPH_OK;
    dlists_ok = false;  // (the device-resident lists are not renamed)
    // perm = real rows in cell order, then the fixed rows as they are
    int32_t* perm = cpos.as<int32_t>();
    CK(cudaMemcpyAsync(perm, centre_p.p, sizeof(int32_t) * nreal, cudaMemcpyDeviceToDevice, s));
    if (nfixed > 0) {
      std::vector<int32_t> tail(nfixed);
      for (int64_t i = 0; i < nfixed; ++i) tail[i] = int32_t(nreal + i);
      CK(cudaMemcpyAsync(perm + nreal, tail.data(), sizeof(int32_t) * nfixed,
                         cudaMemcpyHostToDevice, s));
      CK(cudaStreamSynchronize(s));
    }
    launch_reorder(cols.as<double>(), cols_alt.as<double>(), orig.as<int32_t>(),
                   orig_alt.as<int32_t>(), perm, nrows, nrows, nrows, s);
    std::swap(cols.p, cols_alt.p);
    std::swap(cols.bytes, cols_alt.bytes);
    std::swap(cols.dev, cols_alt.dev);
    std::swap(orig.p, orig_alt.p);
    std::swap(orig.bytes, orig_alt.bytes);
    std::swap(orig.dev, orig_alt.dev);
    if (skin_valid) {
      // the skin lists name records, which stay; what names rows follows
      RC(skin_inv.ensure(sizeof(int32_t) * nrows));
      launch_inverse(perm, nrows, skin_inv.as<int32_t>(), s);
      RC(rename_rows(perm, skin_inv.as<int32_t>()));
      rows_in_order = true;  // (until a sort puts them in another order)
    } else {
      have_order = false;
    }
    steps_since_reorder = 0;
    CK(cudaGetLastError());
    return SPH_OK;
  }

  // ---- neighbour tables ------------------------------------------------------------------------
  // One CSR table: rows sized from each centre's count in the table's last
  // pass, scaled for the change of h since (k_rowcap); a pass in which a row
  // overflows is re-run with the counts it just measured.
  struct Table {
    DevBuf *nl, *rowoff, *rowcap, *rowcap64, *ncnt, *count_prev, *h_prev;
    int64_t* nl_size;
    int* est;
  };
  Table exact_table() {
    return {&nl, &rowoff, &rowcap, &rowcap64, &ncnt, &count_prev, &h_prev, &nl_size, &est_count};
  }
  Table skin_table() {
    return {&skin_nl, &skin_rowoff, &skin_rowcap, &skin_rowcap64, &skin_cnt, &skin_count_prev,
            &skin_h_prev, &skin_nl_size, &skin_est};
  }
  NeibArgs neib_args(const Table& T, const Params& P) {
    NeibArgs na{};
    na.nc = nreal;
    na.centre_k = centre_k.as<int32_t>();
    na.centre_p = centre_p.as<int32_t>();
    na.sx = sx.as<double>(); na.sy = sy.as<double>(); na.sz = sz.as<double>();
    na.s32 = s32.as<float4>();
    na.shift = pgeom.shift;
    na.hcol = col(es_h);
    na.krad = P.krad;
    na.g = grid;
    na.cstart = cstart.as<int32_t>();
    na.rowoff = T.rowoff->as<int64_t>();
    na.rowcap = T.rowcap->as<int32_t>();
    na.nl_size = *T.nl_size;
    na.nl = T.nl->as<int32_t>();
    na.ncnt = T.ncnt->as<int32_t>();
    na.orig = orig.as<int32_t>();
    na.count_prev = T.count_prev->as<int32_t>();
    na.h_prev = T.h_prev->as<float>();
    na.maxcnt = maxcnt.as<int32_t>();
    na.overflow = overflow.as<int32_t>();
    na.dcnt = dcnt.as<unsigned long long>();
    return na;
  }
  // runs `pass` (which fills the table's rows given its NeibArgs) until no
  // row overflows; `exact`: the table the pair passes read (its longest row
  // is reported and checked against the reference's maxneib cap)
  // pass(na, attempt)
  template <class Pass>
  int fill_table(const Table& T, const Params& P, bool exact, Pass pass) {
    const int d = P.dim;
    for (int attempt = 0; attempt < 4; ++attempt) {
      Phase ph(this, SPH_T_NEIGHBOURS);
      launch_rowcap(nreal, centre_p.as<int32_t>(), orig.as<int32_t>(),
                    T.count_prev->as<int32_t>(), T.h_prev->as<float>(), col(es_h), d, 1.2f,
                    T.rowcap64->as<int64_t>(), T.rowcap->as<int32_t>(), s);
      exclusive_scan64(scan64_tmp.p, scan64_tmp.bytes, T.rowcap64->as<int64_t>(),
                       T.rowoff->as<int64_t>(), nreal, s);
      // (table sizes are multiples of 4 like the rows: a row that fits ends
      // on a 16-byte boundary inside the table)
      if (*T.nl_size <= 0) {
        *T.nl_size = ((int64_t(*T.est) * 12 / 10 + 8) * nreal * 5 / 4 + 3) & ~int64_t(3);
        RC(T.nl->ensure(sizeof(int32_t) * *T.nl_size));
      }
      if (attempt > 0) {
        // a re-run: size the table for the rows computed from the new counts
        CK(cudaMemcpyAsync(h_i32 + 2, T.rowcap->as<int32_t>() + (nreal - 1), sizeof(int32_t),
                           cudaMemcpyDeviceToHost, s));
        CK(cudaMemcpyAsync(reinterpret_cast<int64_t*>(h_red + RED_TOTAL),
                           T.rowoff->as<int64_t>() + (nreal - 1), sizeof(int64_t),
                           cudaMemcpyDeviceToHost, s));
        CK(cudaStreamSynchronize(s));
        int64_t total = reinterpret_cast<int64_t*>(h_red + RED_TOTAL)[0] + h_i32[2];
        if (total > *T.nl_size) {
          *T.nl_size = (total + total / 4 + 3) & ~int64_t(3);
          RC(T.nl->ensure(sizeof(int32_t) * *T.nl_size));
        }
      }
      CK(cudaMemsetAsync(maxcnt.p, 0, sizeof(int32_t), s));
      CK(cudaMemsetAsync(overflow.p, 0, sizeof(int32_t), s));
      NeibArgs na = neib_args(T, P);
      pass(na, attempt);
      CK(cudaMemcpyAsync(h_i32, maxcnt.p, sizeof(int32_t), cudaMemcpyDeviceToHost, s));
      CK(cudaMemcpyAsync(h_i32 + 1, overflow.p, sizeof(int32_t), cudaMemcpyDeviceToHost, s));
      CK(cudaStreamSynchronize(s));
      CK(cudaGetLastError());
      int mc = h_i32[0];
      if (h_i32[1] & 2)
        return fail(SPH_ERR_TIMEOUT, "neighbour search: a bulk copy into shared memory did not "
                                     "complete within its wait limit");
      if (exact) {
        cnt_host[SPH_CNT_NEIB_MAX] = mc;
        if (st[SPH_P_NEIB_CAP_CHECK] != 0 && mc + 1 > kb.maxneib[d - 1])
          return fail(SPH_ERR_NEIB_OVERFLOW, "KDTree neibsearch result was truncated (neighboursearch.f90:131)");
      }
      if (!h_i32[1]) break;
      // count_prev now holds the exact counts, so the next attempt fits
      if (attempt == 3) return fail(SPH_ERR_NEIB_OVERFLOW, "neighbour list capacity");
    }
    return SPH_OK;
  }

  // ---- skin lists (SPH_P_SKIN) -----------------------------------------------------------------
  // The search runs with radius (1 + s) krad h and leaves its lists; the
  // following iterates serve the pair passes from them (k_skin_* in
  // sph_grid.cu: filter with the FP64 predicate, fresh search of the
  // centres the filter cannot vouch for) until the records have moved too
  // far, an image set changes or too many centres need the fresh search.
  double skin_fraction() const {
    if (skin_suspended) return 0.0;
    const double v = st[SPH_P_SKIN];
    return v > 0 ? std::min(v, 1.0) : 0.0;
  }
  // the buffers of both paths' lists (the device-resident step needs no more)
  int skin_alloc_common(int64_t nall) {
    RC(skin_rowoff.ensure(sizeof(int64_t) * nreal));
    RC(skin_rowcap.ensure(sizeof(int32_t) * nreal));
    RC(skin_rowcap64.ensure(sizeof(int64_t) * nreal));
    RC(skin_cnt.ensure(sizeof(int32_t) * nreal));
    RC(skin_count_prev.ensure(sizeof(int32_t) * nrows));
    RC(skin_h_prev.ensure(sizeof(float) * nrows));
    RC(skin_hb.ensure(sizeof(double) * nreal));
    RC(skin_sig.ensure(sizeof(uint8_t) * nrows));
    RC(skin_bx.ensure(sizeof(double) * nall));
    RC(skin_by.ensure(sizeof(double) * nall));
    RC(skin_bz.ensure(sizeof(double) * nall));
    RC(skin_dsp.ensure(sizeof(float) * nall));
    RC(skin_hrec.ensure(sizeof(double) * nall));
    return SPH_OK;
  }
  int skin_alloc(int64_t nall) {
    RC(skin_alloc_common(nall));
    RC(skin_gate.ensure(sizeof(int) * 4));
    RC(skin_dflag.ensure(sizeof(int32_t) * (nreal + 1)));
    RC(skin_dpos.ensure(sizeof(int32_t) * (nreal + 1)));
    RC(skin_dlist.ensure(sizeof(int32_t) * nreal));
    RC(skin_gap.ensure(sizeof(float) * nreal));
    RC(skin_hdev.ensure(sizeof(double) * nreal));
    RC(skin_mode.ensure(sizeof(uint8_t) * nreal));
    RC(skin_ways.ensure(sizeof(int64_t) * (nreal + 1)));
    RC(skin_wpos.ensure(sizeof(int64_t) * (nreal + 1)));
    RC(skin_flist.ensure(sizeof(int32_t) * nreal));
    RC(skin_end.ensure(sizeof(int64_t)));
    // (renaming rows: re-sorts and uploads allocate nothing while lists serve)
    RC(skin_sig_alt.ensure(sizeof(uint8_t) * nrows));
    RC(skin_inv.ensure(sizeof(int32_t) * nrows));
    RC(skin_perm.ensure(sizeof(int32_t) * nrows));
    RC(skin_type.ensure(sizeof(double) * nrows));
    RC(skin_flag.ensure(sizeof(int32_t)));
    RC(skin_dcap.ensure(sizeof(int64_t) * (nreal + 1)));
    RC(skin_doff.ensure(sizeof(int64_t) * (nreal + 1)));
    RC(scan64_tmp.ensure(scan64_temp_bytes(nreal + 1)));
    return SPH_OK;
  }
  SkinFilterArgs filter_args(const NeibArgs& na, bool keep, bool gaps) {
    SkinFilterArgs f{};
    f.nc = nreal;
    f.mode = skin_mode.as<uint8_t>();
    f.keep = keep ? 1 : 0;
    f.gap = gaps ? skin_gap.as<float>() : nullptr;
    // a distance between two FP32 images: per axis each image within one
    // unit of the binade's last place (shift 2^-23) of its position
    f.eimg = float(2.0 * std::sqrt(3.0) * pgeom.shift * 1.1920928955078125e-7);
    f.centre_k = na.centre_k;
    f.centre_p = na.centre_p;
    f.skin_off = skin_rowoff.as<int64_t>();
    f.skin_cnt = skin_cnt.as<int32_t>();
    f.skin_nl = skin_nl.as<int32_t>();
    f.sx = na.sx; f.sy = na.sy; f.sz = na.sz;
    f.s32 = na.s32;
    f.shift = na.shift;
    f.hcol = na.hcol;
    f.krad = na.krad;
    f.rowoff = na.rowoff;
    f.rowcap = na.rowcap;
    f.nl_size = na.nl_size;
    f.nl = na.nl;
    f.ncnt = na.ncnt;
    f.orig = na.orig;
    f.count_prev = na.count_prev;
    f.h_prev = na.h_prev;
    f.maxcnt = na.maxcnt;
    f.overflow = na.overflow;
    f.dcnt = na.dcnt;
    return f;
  }
  // after the sort: the skin search, what later iterates compare against,
  // and the exact lists from the skin lists (every centre filters)
  int skin_build(const Mode& m, const Params& P, double skin, double hmin) {
    const int d = P.dim;
    const int64_t nall = nrows + nghost;
    RC(skin_alloc(nall));
    const double kfac = 1.0 + skin;
    if (skin_est <= 0) {
      skin_est = int(est_count * std::pow(kfac, double(d))) + 8;
      launch_fill_i32(skin_count_prev.as<int32_t>(), nrows, skin_est, s);
      CK(cudaMemsetAsync(skin_h_prev.p, 0, sizeof(float) * nrows, s));
    }
    const bool staged = st[SPH_P_SEARCH_STAGED] != 0;
    RC(fill_table(skin_table(), P, false, [&](NeibArgs& na, int) {
      na.kfac = kfac;
      na.skin_search = 1;
      launch_neighbours(d, lanes_search(), staged, na, s);
      cnt_host[SPH_CNT_SEARCHES]++;
    }));
    {
      Phase ph(this, SPH_T_NEIGHBOURS);
      CK(cudaMemcpyAsync(skin_bx.p, sx.p, sizeof(double) * nall, cudaMemcpyDeviceToDevice, s));
      CK(cudaMemcpyAsync(skin_by.p, sy.p, sizeof(double) * nall, cudaMemcpyDeviceToDevice, s));
      CK(cudaMemcpyAsync(skin_bz.p, sz.p, sizeof(double) * nall, cudaMemcpyDeviceToDevice, s));
      SlotInit si{};
      si.off[si.n] = RED_SKIN_HMAXB; si.val[si.n++] = dkey(0.0);
      launch_init_slots(red.as<unsigned long long>(), si, s);
      launch_gather_h(nreal, centre_p.as<int32_t>(), col(es_h), skin_hb.as<double>(),
                      red.as<unsigned long long>(), RED_SKIN_HMAXB, s);
      BoxGeom gg = box(m);
      if (!m.ghosts) for (int k = 0; k < 3; ++k) gg.periodic[k] = 0;
      launch_skin_sig(cols.as<double>(), nrows, gg, d, skin_sig.as<uint8_t>(), s);
      CK(cudaMemsetAsync(skin_dsp.p, 0, sizeof(float) * nall, s));
      CK(cudaMemsetAsync(skin_hdev.p, 0, sizeof(double) * nreal, s));
      CK(cudaMemsetAsync(skin_mode.p, 0, sizeof(uint8_t) * nreal, s));
      CK(cudaMemsetAsync(skin_dflag.p, 0, sizeof(int32_t) * (nreal + 1), s));
    }
    skin_tau = 0.25 * skin * P.krad * hmin;
    skin_eps = 1e-4 * P.krad * hmin;
    skin_hmin = hmin;
    RC(fill_table(exact_table(), P, true, [&](NeibArgs& na, int) {
      launch_skin_filter(filter_args(na, false, true), s);
    }));
    launch_table_end(rowoff.as<int64_t>(), rowcap.as<int32_t>(), nreal, skin_end.as<int64_t>(), s);
    skin_valid = true;
    skin_live = true;
    skin_s = skin;
    skin_age = 0;
    cnt_host[SPH_CNT_SKIN_BUILDS]++;
    return SPH_OK;
  }
  FewArgs few_args(const NeibArgs& na, const int32_t* list, int64_t n, double reach) {
    FewArgs f{};
    f.n = n;
    f.list = list;
    f.centre_k = na.centre_k;
    f.centre_p = na.centre_p;
    f.sx = na.sx; f.sy = na.sy; f.sz = na.sz;
    f.s32 = na.s32;
    f.shift = na.shift;
    f.hcol = na.hcol;
    f.krad = na.krad;
    f.g = na.g;
    f.cstart = na.cstart;
    f.reach = reach;
    f.rowoff = na.rowoff;
    f.rowcap = na.rowcap;
    f.nl_size = na.nl_size;
    f.nl = na.nl;
    f.ncnt = na.ncnt;
    f.orig = na.orig;
    f.count_prev = na.count_prev;
    f.h_prev = na.h_prev;
    f.maxcnt = na.maxcnt;
    f.overflow = na.overflow;
    f.dcnt = na.dcnt;
    return f;
  }
  // The exact table of a skin-list iterate.  The kept rows stay where they
  // are; the filtered ones are written in place; the centres searched afresh
  // (skin_dlist, ndirty of them) get rows laid out anew after the table's
  // fixed part.  A filter row that overflows joins the centres searched
  // afresh (for good: mode 1); when their rows find no room either, the
  // whole table is laid out anew and every row written.
  int skin_fill(const Params& P, int64_t ndirty, int64_t nfilter, double reach) {
    const int d = P.dim;
    Table T = exact_table();
    // the centres searched afresh (skin_dlist): a lane group each when they
    // are few (the search's shared streams would leave most SMs idle), the
    // search's own groups of consecutive centres when they are many
    auto search_dirty = [&](const NeibArgs& na, int64_t nd, double rch) {
      if (nd <= 0) return;
      if (nd < kFewCentres) {
        launch_search_few(d, few_args(na, skin_dlist.as<int32_t>(), nd, rch), s);
      } else {
        NeibArgs nb = na;
        nb.cmap = skin_dlist.as<int32_t>();
        nb.nc = nd;
        nb.reach = rch;
        launch_neighbours(d, lanes_search(), st[SPH_P_SEARCH_STAGED] != 0, nb, s);
        cnt_host[SPH_CNT_SEARCHES]++;
      }
    };
    auto dyn = [&](int64_t nd) {
      launch_dyn_rows(nd, skin_dlist.as<int32_t>(), centre_p.as<int32_t>(), orig.as<int32_t>(),
                      count_prev.as<int32_t>(), h_prev.as<float>(), col(es_h), d,
                      skin_dcap.as<int64_t>(), skin_doff.as<int64_t>(), scan64_tmp.p,
                      scan64_tmp.bytes, skin_end.as<int64_t>(), rowoff.as<int64_t>(),
                      rowcap.as<int32_t>(), s);
    };
    auto read_flags = [&](int& mc, int& ov) -> int {
      CK(cudaMemcpyAsync(h_i32, maxcnt.p, sizeof(int32_t), cudaMemcpyDeviceToHost, s));
      CK(cudaMemcpyAsync(h_i32 + 1, overflow.p, sizeof(int32_t), cudaMemcpyDeviceToHost, s));
      CK(cudaStreamSynchronize(s));
      CK(cudaGetLastError());
      mc = h_i32[0];
      ov = h_i32[1];
      if (ov & 2)
        return fail(SPH_ERR_TIMEOUT, "neighbour search: a bulk copy into shared memory did not "
                                     "complete within its wait limit");
      return SPH_OK;
    };
    int mc = 0, ov = 0;
    {
      Phase ph(this, SPH_T_NEIGHBOURS);
      CK(cudaMemsetAsync(maxcnt.p, 0, sizeof(int32_t), s));
      CK(cudaMemsetAsync(overflow.p, 0, sizeof(int32_t), s));
      dyn(ndirty);
      NeibArgs na = neib_args(T, P);
      SkinFilterArgs fa = filter_args(na, true, false);
      fa.list = skin_flist.as<int32_t>();  // (the centres that filter)
      fa.nc = nfilter;
      launch_skin_filter(fa, s);
      search_dirty(na, ndirty, reach);
      RC(read_flags(mc, ov));
    }
    int mc_all = mc;
    if (ov) {
      // overflowed filter rows join the fresh searches; all of those anew
      Phase ph(this, SPH_T_NEIGHBOURS);
      launch_overflow_to_search(nreal, ncnt.as<int32_t>(), rowoff.as<int64_t>(),
                                rowcap.as<int32_t>(), nl_size, skin_mode.as<uint8_t>(),
                                skin_dflag.as<int32_t>(), s);
      exclusive_scan(scan_tmp.p, scan_tmp.bytes, skin_dflag.as<int32_t>(),
                     skin_dpos.as<int32_t>(), nreal + 1, s);
      launch_skin_compact(nreal, skin_dflag.as<int32_t>(), skin_dpos.as<int32_t>(),
                          skin_dlist.as<int32_t>(), s);
      CK(cudaMemcpyAsync(h_i32 + 3, skin_dpos.as<int32_t>() + nreal, sizeof(int32_t),
                         cudaMemcpyDeviceToHost, s));
      CK(cudaStreamSynchronize(s));
      ndirty = h_i32[3];
      CK(cudaMemsetAsync(overflow.p, 0, sizeof(int32_t), s));
      dyn(ndirty);
      NeibArgs na = neib_args(T, P);
      search_dirty(na, ndirty, reach);
      RC(read_flags(mc, ov));
      mc_all = std::max(mc_all, mc);
    }
    if (ov) {
      // no room after the fixed part: lay the whole table out anew
      RC(fill_table(T, P, true, [&](NeibArgs& na, int) {
        launch_skin_filter(filter_args(na, false, false), s);
        search_dirty(na, ndirty, reach);
      }));
      launch_table_end(rowoff.as<int64_t>(), rowcap.as<int32_t>(), nreal,
                       skin_end.as<int64_t>(), s);
      cnt_host[SPH_CNT_SKIN_RELAYOUTS]++;
      mc_all = int(cnt_host[SPH_CNT_NEIB_MAX]);
    }
    cnt_host[SPH_CNT_NEIB_MAX] = mc_all;
    if (st[SPH_P_NEIB_CAP_CHECK] != 0 && mc_all + 1 > kb.maxneib[d - 1])
      return fail(SPH_ERR_NEIB_OVERFLOW, "KDTree neibsearch result was truncated (neighboursearch.f90:131)");
    cnt_host[SPH_CNT_SKIN_DIRTY] += ndirty;
    return SPH_OK;
  }
  // an iterate served from the skin lists; served = false (nothing changed
  // but the periodic wrap and the records' positions, which the fresh
  // search redoes) when they no longer can serve it
  int skin_reuse(const Mode& m, const Params& P, bool& served) {
    served = false;
    const int d = P.dim;
    const int64_t nall = nrows + nghost;
    BoxGeom g = box(m);
    {
      Phase ph(this, SPH_T_GHOSTS);
      if (m.ghosts) launch_reflect(cols.as<double>(), nrows, nreal, g, s);
    }
    BoxGeom gg = g;
    if (!m.ghosts) for (int k = 0; k < 3; ++k) gg.periodic[k] = 0;
    const float tau = float(skin_tau), eps = float(skin_eps);
    unsigned long long* rb = red.as<unsigned long long>();
    {
      Phase ph(this, SPH_T_NEIGHBOURS);
      SlotInit si{};
      for (int k = 0; k < 3; ++k) {
        si.off[si.n] = RED_LO_X + k; si.val[si.n++] = dkey(1e308);
        si.off[si.n] = RED_HI_X + k; si.val[si.n++] = dkey(-1e308);
      }
      si.off[si.n] = RED_SKIN_D; si.val[si.n++] = dkey(0.0);
      si.off[si.n] = RED_SKIN_HMAX; si.val[si.n++] = dkey(0.0);
      launch_init_slots(rb, si, s);
      // (the signature flag and the four counts are plain integers)
      CK(cudaMemsetAsync(rb + RED_SKIN_SIG, 0, 5 * sizeof(unsigned long long), s));
      launch_skin_refresh(vals_alt.as<int32_t>(), nall, nrows, nreal, cols.as<double>(),
                          gsrc.as<int32_t>(), gcode.as<int8_t>(), gg, d, skin_sig.as<uint8_t>(),
                          skin_bx.as<double>(), skin_by.as<double>(), skin_bz.as<double>(),
                          sx.as<double>(), sy.as<double>(), sz.as<double>(), s32.as<float4>(),
                          pgeom, skin_dsp.as<float>(), tau, eps, skin_hrec.as<double>(), rb, s);
      // the checks and the marks' windows on the device, then the marks and
      // every centre's way: the iterate asks the host once, after the ways
      // (when a check failed, the host ends the lists and drops the ways)
      SkinGateIn gi{};
      gi.dcap = P.krad * skin_hmin;
      gi.krad = P.krad;
      gi.tau = skin_tau;
      gi.kfac = 1.0 + skin_s;
      gi.invL = grid.invL;
      gi.pg = pgeom;
      int* gate = skin_gate.as<int>();
      launch_skin_gate(rb, gi, gate, s);
      const int64_t ncell = int64_t(grid.nx) * grid.ny * grid.nz;
      RC(skin_fcell.ensure(size_t(ncell)));
      RC(skin_mcell.ensure(size_t(ncell)));
      RC(skin_ctmp.ensure(size_t(ncell)));
      launch_skin_marks(nall, skin_dsp.as<float>(), tau, eps, keys_alt.as<uint32_t>(),
                        sx.as<double>(), sy.as<double>(), sz.as<double>(), grid, d, gate + 1,
                        skin_fcell.as<uint8_t>(), skin_mcell.as<uint8_t>(),
                        skin_ctmp.as<uint8_t>(), s);
      launch_skin_classify(nreal, centre_k.as<int32_t>(), skin_hrec.as<double>(),
                           skin_hb.as<double>(), skin_hdev.as<double>(), skin_gap.as<float>(),
                           P.krad, 1.0 + skin_s, tau, eps, skin_dsp.as<float>(),
                           keys_alt.as<uint32_t>(), skin_fcell.as<uint8_t>(),
                           skin_mcell.as<uint8_t>(), skin_mode.as<uint8_t>(),
                           skin_ways.as<int64_t>(), skin_wpos.as<int64_t>(),
                           skin_dlist.as<int32_t>(), skin_flist.as<int32_t>(), scan64_tmp.p,
                           scan64_tmp.bytes, ncnt.as<int32_t>(), rb + RED_SKIN_NKEPT, s);
      CK(cudaMemcpyAsync(h_red, rb, sizeof(unsigned long long) * RED_TOTAL,
                         cudaMemcpyDeviceToHost, s));
      CK(cudaMemcpyAsync(h_red + RED_TOTAL, skin_wpos.as<int64_t>() + nreal, sizeof(int64_t),
                         cudaMemcpyDeviceToHost, s));
      CK(cudaMemcpyAsync(h_i32 + 8, gate, 3 * sizeof(int), cudaMemcpyDeviceToHost, s));
      CK(cudaStreamSynchronize(s));
      CK(cudaGetLastError());
    }
    const double D = dkey_inv(h_red[RED_SKIN_D]);
    const unsigned long long nfast = h_red[RED_SKIN_NFAST], nmove = h_red[RED_SKIN_NMOVE];
    // (SPH_SKIN_TRACE in the environment: why lists end, on stderr)
    auto end_lists = [&](const char* why) {
      if (skin_trace)
        std::fprintf(stderr, "skin lists end after %d iterates: %s (D %.3g, fast %llu, moving %llu)\n",
                     skin_age, why, D, nfast, nmove);
      return SPH_OK;
    };
    switch (h_i32[8]) {
      case 0: break;
      case 1: return end_lists("an image set changed");
      case 2: return end_lists("records moved a search radius");
      case 3: return end_lists("h");
      case 4: return end_lists("a record left the FP32 binade");
      default: return end_lists("a search radius spans too many cells");
    }
    const int64_t counts = reinterpret_cast<const int64_t*>(h_red + RED_TOTAL)[0];
    const int64_t ndirty = counts & 0xffffffffll, nfilter = counts >> 32;
    const int64_t nkept = int64_t(h_red[RED_SKIN_NKEPT]);
    // Their search over cells of step b, its range widened by D, costs
    // several times a search's share per centre (measured on the 128^3
    // Sedov blast: about 20 ns a centre against 1 ns); the iterate is
    // served only while that stays well below a plain search (images, sort
    // and search) with the widening of the smallest radius
    const double rmin = P.krad * skin_hmin;
    const double widen = std::pow((rmin + D) / rmin, double(d));
    if (double(ndirty) * widen > kSkinDirtyShare * double(nreal))
      return end_lists("too many centres to search afresh");
    const double reach_d = D * (1.0 + 1e-9);
    RC(skin_fill(P, ndirty, nfilter, reach_d));
    ++skin_age;
    cnt_host[SPH_CNT_SKIN_REUSES]++;
    cnt_host[SPH_CNT_SKIN_KEPT] += nkept;
    kept_pairs += int64_t(h_red[RED_SKIN_NKEPT_PAIRS]);
    served = true;
    return SPH_OK;
  }

  // ---- neighbour phase: images, grid, sort, lists --------------------------------------------
  int neighbour_phase(const Mode& m, const Params& P) {
    double skin = skin_fraction();
    if (skin > 0 && skin_valid && skin == skin_s) {
      bool served = false;
      RC(skin_reuse(m, P, served));
      if (served) return SPH_OK;
    }
    skin_valid = false;
    dlists_ok = false;
    if (skin_live) {
      // the lists ended (here or by a change of the table or parameters);
      // short-lived ones start a pause of plain searches
      skin_live = false;
      if (skin_age < kSkinShort) {
        skin_pause_len = skin_pause_len ? std::min(2 * skin_pause_len, kSkinPauseMax) : kSkinPause0;
        skin_pause = skin_pause_len;
      } else {
        skin_pause_len = 0;
      }
    }
    if (skin > 0 && skin_pause > 0) {  // lists ended early: plain searches for now
      --skin_pause;
      skin = 0.0;
    }
    const int d = P.dim;
    BoxGeom g = box(m);
    {
      Phase ph(this, SPH_T_GHOSTS);
      if (m.ghosts) launch_reflect(cols.as<double>(), nrows, nreal, g, s);
      // reduction slots: lo (min), hi (max), hmin
      SlotInit si{};
      for (int k = 0; k < 3; ++k) {
        si.off[si.n] = RED_LO_X + k; si.val[si.n++] = dkey(1e308);
        si.off[si.n] = RED_HI_X + k; si.val[si.n++] = dkey(-1e308);
      }
      si.off[si.n] = RED_HMIN; si.val[si.n++] = dkey(1e308);
      launch_init_slots(red.as<unsigned long long>(), si, s);
      BoxGeom gg = g;
      if (!m.ghosts) for (int k = 0; k < 3; ++k) gg.periodic[k] = 0;
      launch_ghost_count(cols.as<double>(), nrows, nreal, gg, d, gcount.as<int32_t>(),
                         red.as<unsigned long long>(), s);
      CK(cudaMemsetAsync(gcount.as<int32_t>() + nrows, 0, sizeof(int32_t), s));
      exclusive_scan(scan_tmp.p, scan_tmp.bytes, gcount.as<int32_t>(), goff.as<int32_t>(),
                     nrows + 1, s);
      CK(cudaMemcpyAsync(h_i32, goff.as<int32_t>() + nrows, sizeof(int32_t),
                         cudaMemcpyDeviceToHost, s));
      CK(cudaMemcpyAsync(h_red, red.p, sizeof(unsigned long long) * (RED_HMIN + 1),
                         cudaMemcpyDeviceToHost, s));
      CK(cudaStreamSynchronize(s));
      nghost = h_i32[0];
      RC(gx.ensure(sizeof(double) * std::max<int64_t>(nghost, 1)));
      RC(gy.ensure(sizeof(double) * std::max<int64_t>(nghost, 1)));
      RC(gz.ensure(sizeof(double) * std::max<int64_t>(nghost, 1)));
      RC(gsrc.ensure(sizeof(int32_t) * std::max<int64_t>(nghost, 1)));
      RC(gcode.ensure(sizeof(int8_t) * std::max<int64_t>(nghost, 1)));
      if (nghost > 0)
        launch_ghost_write(cols.as<double>(), nrows, gg, d, goff.as<int32_t>(), gx.as<double>(),
                           gy.as<double>(), gz.as<double>(), gsrc.as<int32_t>(),
                           gcode.as<int8_t>(), nullptr, s);
    }
    const int64_t nall = nrows + nghost;
    RC(alloc_all(nall));
    // grid: cell edge krad * h_min * factor, at most 1024 cells per axis
    double lo[3], hi[3];
    for (int k = 0; k < 3; ++k) {
      lo[k] = dkey_inv(h_red[RED_LO_X + k]);
      hi[k] = dkey_inv(h_red[RED_HI_X + k]);
    }
    double hmin = dkey_inv(h_red[RED_HMIN]);
    if (!(hmin > 0) || !std::isfinite(hmin)) return fail(SPH_ERR_IC_H, "smoothing length <= 0");
    for (int k = 0; k < 3; ++k)
      if (!std::isfinite(lo[k]) || !std::isfinite(hi[k])) return fail(SPH_ERR_Q_NAN, "q is nan");
    double cf = st[SPH_P_CELL_FACTOR] > 0 ? st[SPH_P_CELL_FACTOR] : 0.4;
    double L = P.krad * hmin * cf;
    int64_t ncell = 0;
    const int64_t ncell_cap = std::min<int64_t>(std::max<int64_t>(8 * nall, 1 << 20),
                                                int64_t(1) << 31);
    int n3[3];
    for (int guard = 0;; ++guard) {
      double e[3];
      for (int k = 0; k < 3; ++k) e[k] = (hi[k] - lo[k]) / L;
      if (grid_dims(e, ncell_cap, n3, &ncell)) break;
      L *= 1.25;
      if (guard > 400) return fail(SPH_ERR_GRID, "cell grid would not fit");
    }
    grid.ox = lo[0]; grid.oy = lo[1]; grid.oz = lo[2];
    grid.L = L; grid.invL = 1.0 / L;
    grid.nx = n3[0]; grid.ny = n3[1]; grid.nz = n3[2];
    int end_bit = 1;
    while ((int64_t(1) << end_bit) < ncell) ++end_bit;
    // FP32 position packing: one binade [2^E, 2^(E+1)) over the whole extent
    // (with skin lists, and room of one search radius on every side for the
    // records to move before the next sort)
    const double mg = skin > 0 ? P.krad * hmin : 0.0;
    double ext = std::max(hi[0] - lo[0], std::max(hi[1] - lo[1], hi[2] - lo[2])) + 2.0 * mg;
    double sh = 1.0;
    if (ext > 0) {
      while (sh < ext * 1.0001) sh *= 2.0;
      while (sh * 0.5 >= ext * 1.0001) sh *= 0.5;
    }
    pgeom.ox = lo[0] - mg; pgeom.oy = lo[1] - mg; pgeom.oz = lo[2] - mg;
    pgeom.shift = sh;
    pgeom.mref = mref;
    {
      Phase ph(this, SPH_T_SORT);
      launch_keys(cols.as<double>(), nrows, gx.as<double>(), gy.as<double>(), gz.as<double>(),
                  nghost, grid, keys.as<uint32_t>(), vals.as<int32_t>(), s);
      // the cell count follows 1 / h_min^d, which drifts from step to step:
      // room for four times the current count (at most the cap) keeps the
      // reallocation out of the steady state
      const size_t cells = size_t(std::min<int64_t>(4 * (ncell + 1), ncell_cap + 1));
      if (sizeof(int32_t) * size_t(ncell + 1) > cstart.bytes)
        RC(cstart.ensure(sizeof(int32_t) * cells));
      if (sizeof(int32_t) * size_t(ncell + 1) > cell_count.bytes)
        RC(cell_count.ensure(sizeof(int32_t) * cells));
      const size_t sb = scan_temp_bytes(ncell + 1);
      if (sb > scan_tmp.bytes) RC(scan_tmp.ensure(sb));
      RC(cell_ctr.ensure(2 * sizeof(int32_t)));
      // counting sort by cell (vals serves as its list of crowded cells);
      // a cell of more than 4096 records takes the library's radix sort
      if (!cell_sort(keys.as<uint32_t>(), nall, ncell, cell_count.as<int32_t>(),
                     cstart.as<int32_t>(), vals_alt.as<int32_t>(), keys_alt.as<uint32_t>(),
                     vals.as<int32_t>(), cell_ctr.as<int32_t>(), scan_tmp.p, scan_tmp.bytes,
                     h_i32 + 5, s)) {
        sort_pairs(sort_tmp.p, sort_tmp.bytes, keys.as<uint32_t>(), keys_alt.as<uint32_t>(),
                   vals.as<int32_t>(), vals_alt.as<int32_t>(), nall, end_bit, s);
        launch_cell_starts(keys_alt.as<uint32_t>(), nall, ncell, cstart.as<int32_t>(), s);
      }
      launch_sorted_gather(vals_alt.as<int32_t>(), nall, nrows, nreal, cols.as<double>(),
                           gx.as<double>(), gy.as<double>(), gz.as<double>(), gsrc.as<int32_t>(),
                           sx.as<double>(), sy.as<double>(), sz.as<double>(), ssrc.as<int32_t>(),
                           cflag.as<int32_t>(), s32.as<float4>(), pgeom, s);
      CK(cudaMemsetAsync(cflag.as<int32_t>() + nall, 0, sizeof(int32_t), s));
      exclusive_scan(scan_tmp.p, scan_tmp.bytes, cflag.as<int32_t>(), cpos.as<int32_t>(),
                     nall + 1, s);
      launch_centres(vals_alt.as<int32_t>(), cflag.as<int32_t>(), cpos.as<int32_t>(), nall,
                     centre_k.as<int32_t>(), centre_p.as<int32_t>(), s);
    }
    // neighbour lists: rows sized from each particle's previous count; a row
    // that overflows (or a table that is too small) re-runs the search with
    // the counts it just measured
    if (est_count <= 0) {
      double kh = P.krad * P.hfac;
      double est = d == 3 ? 4.0 / 3.0 * kPi * kh * kh * kh : (d == 2 ? kPi * kh * kh : 2 * kh);
      est_count = int(est * 1.3) + 8;
      if (st[SPH_P_NEIB_CAP] > 0) est_count = int(st[SPH_P_NEIB_CAP]);
      launch_fill_i32(count_prev.as<int32_t>(), nrows, est_count, s);
      CK(cudaMemsetAsync(h_prev.p, 0, sizeof(float) * nrows, s));
    }
    if (skin > 0) {
      RC(skin_build(m, P, skin, hmin));
    } else {
      const bool staged = st[SPH_P_SEARCH_STAGED] != 0;
      RC(fill_table(exact_table(), P, true, [&](NeibArgs& na, int) {
        launch_neighbours(d, lanes_search(), staged, na, s);
        cnt_host[SPH_CNT_SEARCHES]++;
      }));
    }
    have_order = true;
    rows_in_order = false;
    cnt_host[SPH_CNT_GHOSTS] = nghost;
    return SPH_OK;
  }

  // ---- circuit1 + EOS ----------------------------------------------------------------------
  int circuit1(const Mode& m, Params& P) {
    const int64_t nall = nrows + nghost;
    PackBufs pb = packs();
    P.eos_kind = m.eos_kind;
    if (m.eos_kind == 2) {
      // c of row 1 (eos.f90:43): find the physical row whose original index is 0
      std::vector<int32_t> og(nrows);
      CK(cudaMemcpyAsync(og.data(), orig.p, sizeof(int32_t) * nrows, cudaMemcpyDeviceToHost, s));
      CK(cudaStreamSynchronize(s));
      int64_t p0 = std::find(og.begin(), og.end(), 0) - og.begin();
      CK(cudaMemcpyAsync(h_ctrl + 7, col(es_c) + p0, sizeof(double), cudaMemcpyDeviceToHost, s));
      CK(cudaStreamSynchronize(s));
      P.c_iso = h_ctrl[7];
    }
    {
      Phase pk(this, SPH_T_PACK);
      const int groups = PACK_POS | ((eq_diff || eq_fld) ? PACK_TEMP : 0);
      if (dplan)
        launch_pack_dev(prec, groups, nall_cap, ssrc.as<int32_t>(), sx.as<double>(),
                        sy.as<double>(), sz.as<double>(), cols.as<double>(), nrows, dplan, pb, s);
      else
        launch_pack(prec, groups, nall, ssrc.as<int32_t>(), sx.as<double>(), sy.as<double>(),
                    sz.as<double>(), cols.as<double>(), nrows, pgeom, pb, s);
    }
    Phase ph(this, SPH_T_CIRCUIT1);
    C1Args a{};
    a.nc = nreal;
    a.rowoff = rowoff.as<int64_t>();
    a.G = lanes_pair();
    a.centre_k = centre_k.as<int32_t>();
    a.centre_p = centre_p.as<int32_t>();
    a.nl = nl.as<int32_t>();
    a.ncnt = ncnt.as<int32_t>();
    a.cols = cols.as<double>();
    a.ld = nrows;
    a.hk_s = hk_s.as<double>();
    a.dk_s = dk_s.as<double>();
    a.ok_s = ok_s.as<double>();
    a.hkp1 = hkp1.as<double>();
    a.dkp1 = dkp1.as<double>();
    a.okp1 = okp1.as<double>();
    a.eps = epsb.as<double>();
    a.mref = mref;
    a.status = status.as<int>();
    a.dcnt = dcnt.as<unsigned long long>();
    a.red = red.as<unsigned long long>();
    a.active_slot = RED_C1_ACTIVE;
    a.gate = nullptr;
    const bool advanced = ival(ec_adden) == 1;
    if (advanced && P.maxiter == 0) {  // zero sweeps: h, rho, Omega stay (circuit1.f90:114)
      launch_eos(cols.as<double>(), nrows, nreal, P, s);
      CK(cudaGetLastError());
      return SPH_OK;
    }
    if (advanced && !eq_diff && !eq_fld) {
      launch_c1_newton(prec, kernel_id, P.dim, a, pb, P, s);
      CK(cudaGetLastError());
      return SPH_OK;
    }
    // Jacobi sweeps (circuit1.f90:105-211) / direct summation (:237-301)
    a.simple = advanced ? 0 : 1;
    CK(cudaMemcpyAsync(hkp1.p, col(es_h), sizeof(double) * nrows, cudaMemcpyDeviceToDevice, s));
    CK(cudaMemcpyAsync(dkp1.p, col(es_den), sizeof(double) * nrows, cudaMemcpyDeviceToDevice, s));
    CK(cudaMemcpyAsync(okp1.p, col(es_om), sizeof(double) * nrows, cudaMemcpyDeviceToDevice, s));
    launch_set_col(epsb.as<double>(), nrows, 1.0, s);
    int iter = 0;
    if (dplan) {
      // device-resident step: the sweeps as a while node, as many as the
      // particles need (up to kDrsSweeps) without looking at the host; a
      // particle still active after the last of fewer than maxiter sweeps
      // sets the error word, which sends the step back to the host path
      unsigned long long* rb = red.as<unsigned long long>();
      a.active_slot = RED_C1_ACTIVE;
      a.gate = nullptr;
      auto sweep = [&]() {
        launch_c1_snapshot(nall_cap, ssrc.as<int32_t>(), hkp1.as<double>(), dkp1.as<double>(),
                           okp1.as<double>(), hk_s.as<double>(), dk_s.as<double>(),
                           ok_s.as<double>(), s, dplan, nullptr);
        launch_fill_u64(rb + RED_C1_ACTIVE, 1, 0ull, s);
        launch_c1_sweep(prec, kernel_id, P.dim, a, pb, P, s);
      };
      if (a.simple) {
        a.first = 1;
        sweep();
        iter = 1;
      } else {
        const int sweeps = std::max(1, std::min(P.maxiter, kDrsSweeps));
        int* itd = c1_iter.as<int>();
        a.iter_dev = itd;
        RC(capture_cond(
            cudaGraphCondTypeWhile,
            [&](cudaGraphConditionalHandle hw) { launch_sweeps_init(itd, hw, s); },
            [&](cudaGraphConditionalHandle hw) {
              sweep();
              launch_sweeps_ctl(itd, rb + RED_C1_ACTIVE, sweeps, P.maxiter, drs_err.as<int>(), hw,
                                s);
              return SPH_OK;
            }));
        a.iter_dev = nullptr;
        iter = sweeps;
      }
    } else
    for (;;) {
      ++iter;
      a.first = iter == 1;
      launch_c1_snapshot(nall, ssrc.as<int32_t>(), hkp1.as<double>(), dkp1.as<double>(),
                         okp1.as<double>(), hk_s.as<double>(), dk_s.as<double>(),
                         ok_s.as<double>(), s);
      launch_fill_u64(red.as<unsigned long long>() + RED_C1_ACTIVE, 1, 0ull, s);
      launch_c1_sweep(prec, kernel_id, P.dim, a, pb, P, s);
      if (a.simple) break;
      CK(cudaMemcpyAsync(h_red + RED_C1_ACTIVE, red.as<unsigned long long>() + RED_C1_ACTIVE,
                         sizeof(unsigned long long), cudaMemcpyDeviceToHost, s));
      CK(cudaStreamSynchronize(s));
      CK(cudaGetLastError());
      if (!h_red[RED_C1_ACTIVE] || iter >= P.maxiter) break;
    }
    launch_c1_finalize(nrows, nreal, cols.as<double>(), nrows, hkp1.as<double>(),
                       dkp1.as<double>(), okp1.as<double>(), a.simple, P, s);
    host_max_sweeps = std::max<int64_t>(host_max_sweeps, iter);
    CK(cudaGetLastError());
    return SPH_OK;
  }

  int circuit2(const Mode& m, const Params& P) {
    const int64_t nall = nrows + nghost;
    PackBufs pb = packs();
    // the positions (PACK_POS) were packed for circuit1 in this iterate and
    // have not moved; h, rho, Omega, P, c and grad T are new
    int groups = PACK_HYDRO | ((eq_diff || eq_magneto) ? PACK_EXTRA : 0);
    pb.kp_wcv = P.wCv;
    pb.kp_alpha = P.alpha;
    pb.kp_au = P.au;
    pb.kp_dim = P.dim;
    {
      Phase pk(this, SPH_T_PACK);
      if (dplan)
        launch_pack_dev(prec, groups, nall_cap, ssrc.as<int32_t>(), sx.as<double>(),
                        sy.as<double>(), sz.as<double>(), cols.as<double>(), nrows, dplan, pb, s);
      else
        launch_pack(prec, groups, nall, ssrc.as<int32_t>(), sx.as<double>(), sy.as<double>(),
                    sz.as<double>(), cols.as<double>(), nrows, pgeom, pb, s);
    }
    Phase ph(this, SPH_T_CIRCUIT2);
    C2Args a{};
    a.nc = nreal;
    a.rowoff = rowoff.as<int64_t>();
    a.G = lanes_pair();
    a.centre_k = centre_k.as<int32_t>();
    a.centre_p = centre_p.as<int32_t>();
    a.nl = nl.as<int32_t>();
    a.ncnt = ncnt.as<int32_t>();
    a.cols = cols.as<double>();
    a.ld = nrows;
    a.mref = mref;
    a.status = status.as<int>();
    a.dcnt = dcnt.as<unsigned long long>();
    launch_c2(prec, kernel_id, P.dim, a, pb, P, s);
    if (m.mti) launch_apply_mti(cols.as<double>(), nrows, orig.as<int32_t>(), nrows, nreal,
                                m.mti == 2, s);
    CK(cudaGetLastError());
    return SPH_OK;
  }

  // the integrator's mode: which of B and T an equation moves this run
  int lf_mode(bool do_sts) {
    eqset();
    return (do_sts ? LF_STS : 0) | (eq_magneto ? 0 : LF_NO_B) | ((eq_diff || eq_fld) ? 0 : LF_NO_T);
  }

  // iterate() (iterator.f90:44-179); full = false stops after circuit1 + EOS
  int iterate(bool full) {
    if (dplan) return iterate_dev(full);
    Params P{};
    RC(params(P));
    Mode m;
    RC(mode(m));
    RC(neighbour_phase(m, P));
    RC(circuit1(m, P));
    if (full) RC(circuit2(m, P));
    RC(check_status());
    cnt_host[SPH_CNT_ITERATES] += full ? 1 : 0;
    cnt_host[SPH_CNT_CENTRES] += nreal;
    return SPH_OK;
  }

  // ---- device-resident step ------------------------------------------------------------------
  // The classic step asks the host four or five times per iterate (image
  // count and bounding box, list overflow, Newton sweeps, status) and once
  // per step (dt).  The device-resident step plans all of that on the device
  // (k_plan, k_dt), runs the sort and the passes over capacities fixed on the
  // host, and reports problems through one error word read after the step:
  // a capacity that was too small, a list row that overflowed, or Newton
  // sweeps beyond kDrsSweeps send the step back to the host path from the
  // table saved at its start.  With no host round trip inside, one step is
  // captured as a CUDA graph and replayed.

  // Adds an if node after the work captured so far on s: `pre(handle)`
  // captures the kernel that sets the handle, then `body` is captured into
  // the node's body graph (its launches go to s while it runs).
  template <class Pre, class Body>
  int capture_if(Pre&& pre, Body&& body) {
    return capture_cond(cudaGraphCondTypeIf, pre, body);
  }
  // the same with a while node: the body runs again while the handle is
  // non-zero after it (a kernel in the body sets it)
  template <class Pre, class Body>
  int capture_cond(cudaGraphConditionalNodeType type, Pre&& pre, Body&& body) {
    cudaStreamCaptureStatus cs;
    cudaGraph_t g = nullptr;
    const cudaGraphNode_t* deps = nullptr;
    size_t nd = 0;
    CK(cudaStreamGetCaptureInfo(s, &cs, nullptr, &g, &deps, &nd));
    if (cs != cudaStreamCaptureStatusActive) return fail(SPH_ERR_STATE, "if node outside a capture");
    cudaGraphConditionalHandle hnd;
    CK(cudaGraphConditionalHandleCreate(&hnd, g, 0, 0));
    pre(hnd);
    CK(cudaStreamGetCaptureInfo(s, &cs, nullptr, &g, &deps, &nd));
    cudaGraphNodeParams cp{};
    cp.type = cudaGraphNodeTypeConditional;
    cp.conditional.handle = hnd;
    cp.conditional.type = type;
    cp.conditional.size = 1;
    cudaGraphNode_t node;
    CK(cudaGraphAddNode(&node, g, deps, nd, &cp));
    CK(cudaStreamUpdateCaptureDependencies(s, &node, 1, cudaStreamSetCaptureDependencies));
    // (one capture stream per nesting level: the levels above still capture)
    if (int(cap_s.size()) <= cap_depth) {
      cudaStream_t ns = nullptr;
      CK(cudaStreamCreateWithFlags(&ns, cudaStreamNonBlocking));
      cap_s.push_back(ns);
    }
    cudaStream_t bs = cap_s[cap_depth];
    CK(cudaStreamBeginCaptureToGraph(bs, cp.conditional.phGraph_out[0], nullptr, nullptr, 0,
                                     cudaStreamCaptureModeThreadLocal));
    cudaStream_t outer = s;
    s = bs;
    ++cap_depth;
    const int rc = body(hnd);
    --cap_depth;
    s = outer;
    cudaGraph_t out;
    const cudaError_t e = cudaStreamEndCapture(bs, &out);
    if (rc) return rc;
    if (e != cudaSuccess) return fail(SPH_ERR_CUDA, std::string("if node body: ") + cudaGetErrorString(e));
    return SPH_OK;
  }

  // The device-resident step's neighbour phase.  Without skin lists: images,
  // sort, centres and the search, every iterate (search_dev).  With them
  // (SPH_P_SKIN > 0): the records' positions refreshed in the lists' sorted
  // order, every centre checked against its list, and the search only when
  // the device decides so (an if node: a skin search, or a plain one in a
  // pause after short-lived lists); every centre's row is then its list's
  // records that pass the FP64 predicate.  No host decision either way.
  int neighbour_phase_dev(const Mode& m, const Params& P) {
    skin_valid = false;  // (the host path's lists)
    const double skin = skin_fraction();
    if (!(skin > 0)) return search_dev(m, P, false);
    const int d = P.dim;
    BoxGeom g = box(m);
    if (m.ghosts) launch_reflect(cols.as<double>(), nrows, nreal, g, s);
    BoxGeom gg = g;
    if (!m.ghosts) for (int k = 0; k < 3; ++k) gg.periodic[k] = 0;
    unsigned long long* rb = red.as<unsigned long long>();
    DevSkin* ds = dskin.as<DevSkin>();
    DevPlan* plan = drs_plan.as<DevPlan>();
    SlotInit si{};
    for (int k = 0; k < 3; ++k) {
      si.off[si.n] = RED_LO_X + k; si.val[si.n++] = dkey(1e308);
      si.off[si.n] = RED_HI_X + k; si.val[si.n++] = dkey(-1e308);
    }
    si.off[si.n] = RED_SKIN_D; si.val[si.n++] = dkey(0.0);
    si.off[si.n] = RED_SKIN_HMAX; si.val[si.n++] = dkey(0.0);
    si.off[si.n] = RED_DSKIN_FAIL; si.val[si.n++] = 0ull;
    si.off[si.n] = RED_SKIN_SIG; si.val[si.n++] = 0ull;
    launch_init_slots(rb, si, s);
    launch_skin_refresh(vals_alt.as<int32_t>(), nall_cap, nrows, nreal, cols.as<double>(),
                        gsrc.as<int32_t>(), gcode.as<int8_t>(), gg, d, skin_sig.as<uint8_t>(),
                        skin_bx.as<double>(), skin_by.as<double>(), skin_bz.as<double>(),
                        sx.as<double>(), sy.as<double>(), sz.as<double>(), s32.as<float4>(),
                        PackGeom{}, skin_dsp.as<float>(), 0.f, 0.f, skin_hrec.as<double>(), rb, s,
                        plan, ds);
    launch_dskin_check(nreal, centre_p.as<int32_t>(), col(es_h), skin_hb.as<double>(), P.krad, ds,
                       rb, s);
    RC(capture_if(
        [&](cudaGraphConditionalHandle hs) {
          launch_dskin_decide(ds, rb, plan, P.krad, skin, kSkinShort, kSkinPause0, kSkinPauseMax,
                              hs, dcnt.as<unsigned long long>(), s);
        },
        [&](cudaGraphConditionalHandle) { return search_dev(m, P, true); }));
    // every centre's row from its skin list
    SkinFilterArgs f{};
    f.nc = nreal;
    f.centre_k = centre_k.as<int32_t>();
    f.centre_p = centre_p.as<int32_t>();
    f.skin_off = skin_rowoff.as<int64_t>();
    f.skin_cnt = skin_cnt.as<int32_t>();
    f.skin_nl = skin_nl.as<int32_t>();
    f.sx = sx.as<double>(); f.sy = sy.as<double>(); f.sz = sz.as<double>();
    f.s32 = s32.as<float4>();
    f.hcol = col(es_h);
    f.krad = P.krad;
    f.rowoff = rowoff.as<int64_t>();
    f.rowcap = rowcap.as<int32_t>();
    f.nl_size = nl_size;
    f.nl = nl.as<int32_t>();
    f.ncnt = ncnt.as<int32_t>();
    f.orig = orig.as<int32_t>();
    f.count_prev = count_prev.as<int32_t>();
    f.h_prev = h_prev.as<float>();
    f.maxcnt = maxcnt.as<int32_t>();
    f.overflow = overflow.as<int32_t>();
    f.dcnt = dcnt.as<unsigned long long>();
    f.plan = plan;
    f.skin_cap = skin_rowcap.as<int32_t>();
    f.skin_size = skin_nl_size;
    launch_skin_filter(f, s);
    CK(cudaGetLastError());
    return SPH_OK;
  }

  // images, keys, sort, centres and the search of the device-resident step;
  // skin: the search of skin lists (radius factor from the device, into the
  // skin table), what later iterates compare against, and the layout of the
  // rows filtered from them (the positions are already wrapped)
  int search_dev(const Mode& m, const Params& P, bool skin) {
    const int d = P.dim;
    BoxGeom g = box(m);
    if (m.ghosts && !skin) launch_reflect(cols.as<double>(), nrows, nreal, g, s);
    SlotInit si{};
    for (int k = 0; k < 3; ++k) {
      si.off[si.n] = RED_LO_X + k; si.val[si.n++] = dkey(1e308);
      si.off[si.n] = RED_HI_X + k; si.val[si.n++] = dkey(-1e308);
    }
    si.off[si.n] = RED_HMIN; si.val[si.n++] = dkey(1e308);
    launch_init_slots(red.as<unsigned long long>(), si, s);
    BoxGeom gg = g;
    if (!m.ghosts) for (int k = 0; k < 3; ++k) gg.periodic[k] = 0;
    launch_ghost_count(cols.as<double>(), nrows, nreal, gg, d, gcount.as<int32_t>(),
                       red.as<unsigned long long>(), s);
    CK(cudaMemsetAsync(gcount.as<int32_t>() + nrows, 0, sizeof(int32_t), s));
    exclusive_scan(scan_tmp.p, scan_tmp.bytes, gcount.as<int32_t>(), goff.as<int32_t>(),
                   nrows + 1, s);
    PlanIn pin{};
    pin.nrows = nrows;
    pin.nghost_cap = nghost_cap;
    pin.nall_cap = nall_cap;
    pin.krad = P.krad;
    pin.cf = st[SPH_P_CELL_FACTOR] > 0 ? st[SPH_P_CELL_FACTOR] : 0.4;
    pin.mref = mref;
    pin.end_bit_cap = end_bit_cap;
    DevPlan* plan = drs_plan.as<DevPlan>();
    launch_plan(red.as<unsigned long long>(), goff.as<int32_t>() + nrows, pin, plan,
                drs_err.as<int>(), s);
    launch_ghost_write_cap(cols.as<double>(), nrows, gg, d, goff.as<int32_t>(), nghost_cap,
                           gx.as<double>(), gy.as<double>(), gz.as<double>(),
                           gsrc.as<int32_t>(), gcode.as<int8_t>(), s);
    launch_keys_dev(cols.as<double>(), nrows, gx.as<double>(), gy.as<double>(), gz.as<double>(),
                    plan, nall_cap, keys.as<uint32_t>(), vals.as<int32_t>(), s);
    sort_pairs(sort_tmp.p, sort_tmp.bytes, keys.as<uint32_t>(), keys_alt.as<uint32_t>(),
               vals.as<int32_t>(), vals_alt.as<int32_t>(), nall_cap, end_bit_cap, s);
    launch_cell_starts_dev(keys_alt.as<uint32_t>(), nall_cap, plan, cstart.as<int32_t>(), s);
    launch_sorted_gather_dev(vals_alt.as<int32_t>(), nall_cap, nrows, nreal, cols.as<double>(),
                             gx.as<double>(), gy.as<double>(), gz.as<double>(),
                             gsrc.as<int32_t>(), sx.as<double>(), sy.as<double>(),
                             sz.as<double>(), ssrc.as<int32_t>(), cflag.as<int32_t>(),
                             s32.as<float4>(), plan, s);
    exclusive_scan(scan_tmp.p, scan_tmp.bytes, cflag.as<int32_t>(), cpos.as<int32_t>(),
                   nall_cap + 1, s);
    launch_centres(vals_alt.as<int32_t>(), cflag.as<int32_t>(), cpos.as<int32_t>(), nall_cap,
                   centre_k.as<int32_t>(), centre_p.as<int32_t>(), s);
    // (the skin table's rows: their last counts, plain or skin, with room
    // for a skin search after a plain one)
    const float slack = skin ? float(1.2 * std::pow(1.0 + skin_fraction(), double(d))) : 1.2f;
    DevBuf& t_cap = skin ? skin_rowcap : rowcap;
    DevBuf& t_cap64 = skin ? skin_rowcap64 : rowcap64;
    DevBuf& t_off = skin ? skin_rowoff : rowoff;
    DevBuf& t_cp = skin ? skin_count_prev : count_prev;
    DevBuf& t_hp = skin ? skin_h_prev : h_prev;
    launch_rowcap(nreal, centre_p.as<int32_t>(), orig.as<int32_t>(), t_cp.as<int32_t>(),
                  t_hp.as<float>(), col(es_h), d, slack, t_cap64.as<int64_t>(),
                  t_cap.as<int32_t>(), s);
    exclusive_scan64(scan64_tmp.p, scan64_tmp.bytes, t_cap64.as<int64_t>(), t_off.as<int64_t>(),
                     nreal, s);
    NeibArgs na{};
    na.plan = plan;
    na.nc = nreal;
    na.centre_k = centre_k.as<int32_t>();
    na.centre_p = centre_p.as<int32_t>();
    na.sx = sx.as<double>(); na.sy = sy.as<double>(); na.sz = sz.as<double>();
    na.s32 = s32.as<float4>();
    na.hcol = col(es_h);
    na.krad = P.krad;
    na.cstart = cstart.as<int32_t>();
    na.rowoff = t_off.as<int64_t>();
    na.rowcap = t_cap.as<int32_t>();
    na.nl_size = skin ? skin_nl_size : nl_size;
    na.nl = skin ? skin_nl.as<int32_t>() : nl.as<int32_t>();
    na.ncnt = skin ? skin_cnt.as<int32_t>() : ncnt.as<int32_t>();
    na.orig = orig.as<int32_t>();
    na.count_prev = t_cp.as<int32_t>();
    na.h_prev = t_hp.as<float>();
    na.maxcnt = maxcnt.as<int32_t>();
    na.overflow = overflow.as<int32_t>();
    na.dcnt = dcnt.as<unsigned long long>();
    if (skin) {
      DevSkin* ds = dskin.as<DevSkin>();
      na.kfac_dev = &ds->kfac;
      na.skin_search = 1;
    }
    launch_neighbours(d, lanes_search(), st[SPH_P_SEARCH_STAGED] != 0, na, s);
    if (skin) {
      // what the next iterates compare against: positions, centres' h and
      // the rows' image signatures of this search; no displacement yet
      unsigned long long* rb = red.as<unsigned long long>();
      CK(cudaMemcpyAsync(skin_bx.p, sx.p, sizeof(double) * nall_cap, cudaMemcpyDeviceToDevice, s));
      CK(cudaMemcpyAsync(skin_by.p, sy.p, sizeof(double) * nall_cap, cudaMemcpyDeviceToDevice, s));
      CK(cudaMemcpyAsync(skin_bz.p, sz.p, sizeof(double) * nall_cap, cudaMemcpyDeviceToDevice, s));
      launch_gather_h(nreal, centre_p.as<int32_t>(), col(es_h), skin_hb.as<double>(), rb,
                      RED_SKIN_HMAXB, s);
      launch_skin_sig(cols.as<double>(), nrows, gg, d, skin_sig.as<uint8_t>(), s);
      CK(cudaMemsetAsync(skin_dsp.p, 0, sizeof(float) * nall_cap, s));
      launch_dskin_built(dskin.as<DevSkin>(), rb, s);
      // the rows filtered from the lists: their last counts
      launch_rowcap(nreal, centre_p.as<int32_t>(), orig.as<int32_t>(), count_prev.as<int32_t>(),
                    h_prev.as<float>(), col(es_h), d, 1.2f, rowcap64.as<int64_t>(),
                    rowcap.as<int32_t>(), s);
      exclusive_scan64(scan64_tmp.p, scan64_tmp.bytes, rowcap64.as<int64_t>(),
                       rowoff.as<int64_t>(), nreal, s);
    }
    CK(cudaGetLastError());
    return SPH_OK;
  }

  int iterate_dev(bool full) {
    Params P{};
    RC(params(P));
    Mode m;
    RC(mode(m));
    RC(neighbour_phase_dev(m, P));
    RC(circuit1(m, P));
    if (full) RC(circuit2(m, P));
    return SPH_OK;
  }

  // can this handle's step run without the host?  (sets the reason when not)
  bool drs_eligible(const char** why) {
    eqset();
    Mode m;
    if (mode(m) != SPH_OK) { *why = "mode"; return false; }
    if (!started) { *why = "not started"; return false; }
    if (eq_radexch) { *why = "radiation exchange"; return false; }
    if (eq_sts && ival(ec_ststype) != 1) { *why = "STS with automatic stages"; return false; }
    if (m.eos_kind == 2) { *why = "isothermal EOS"; return false; }
    if (st[SPH_P_NEIB_CAP_CHECK] != 0) { *why = "neighbour cap check"; return false; }
    if (nl_size <= 0 || nghost < 0) { *why = "no search yet"; return false; }
    return true;
  }

  // capacities of the device-resident step, from the last host-planned one
  int drs_prepare() {
    skin_valid = false;  // its capacities may move the sorted arrays
    const int64_t want_ghost = nghost + nghost / 4 + 1024;
    if (want_ghost > nghost_cap || nall_cap != nrows + nghost_cap) {
      nghost_cap = std::max(want_ghost, nghost_cap);
      nall_cap = nrows + nghost_cap;
      graph_dirty = true;
    }
    RC(gx.ensure(sizeof(double) * nghost_cap));
    RC(gy.ensure(sizeof(double) * nghost_cap));
    RC(gz.ensure(sizeof(double) * nghost_cap));
    RC(gsrc.ensure(sizeof(int32_t) * nghost_cap));
    RC(gcode.ensure(sizeof(int8_t) * nghost_cap));
    RC(alloc_all(nall_cap));
    const int64_t cap = std::min<int64_t>(std::max<int64_t>(8 * nall_cap, 1 << 20),
                                          int64_t(1) << 31);
    RC(cstart.ensure(sizeof(int32_t) * size_t(cap + 1)));
    int eb = 1;
    while (eb < 32 && (int64_t(1) << eb) <= cap) ++eb;
    if (eb != end_bit_cap) { end_bit_cap = eb; graph_dirty = true; }
    RC(drs_plan.ensure(sizeof(DevPlan)));
    RC(drs_clock.ensure(sizeof(DevClock)));
    RC(drs_err.ensure(sizeof(int)));
    RC(c1_iter.ensure(sizeof(int)));
    RC(drs_save.ensure(sizeof(double) * NCOL * size_t(nrows)));
    RC(bclk_save.ensure(sizeof(DevClock)));
    if (eq_sts) {
      RC(stsY.ensure(sizeof(double) * 6 * nrows));
      RC(sts_coef_upload(ival(ec_stsfixeds)));
    }
    const double skin = skin_fraction();
    if (skin > 0) {
      // the device-resident lists: the host lists' buffers at the device
      // step's capacities, the skin table sized for the rows search_dev lays
      // out (last counts x 1.2 (1 + s)^d, counts up to (1 + s)^d those of
      // the exact rows)
      RC(skin_alloc_common(nall_cap));
      RC(dskin.ensure(sizeof(DevSkin)));
      const double kf = std::pow(1.0 + skin, double(dim()));
      const int64_t need = int64_t(double(nl_size) * kf * kf * 1.05) + 16 * nreal;
      if (need > skin_nl_size) {
        RC(skin_nl.ensure(sizeof(int32_t) * size_t(need)));
        skin_nl_size = need;
      }
      if (skin_est <= 0) {
        skin_est = int(est_count * kf) + 8;
        launch_fill_i32(skin_count_prev.as<int32_t>(), nrows, skin_est, s);
        CK(cudaMemsetAsync(skin_h_prev.p, 0, sizeof(float) * nrows, s));
      }
    }
    return SPH_OK;
  }
  // before a device-resident run: it starts without lists when the host has
  // touched the records, rows or lists since the last one
  int dlists_reset(cudaStream_t st_) {
    if (skin_fraction() > 0 && !dlists_ok)
      CK(cudaMemsetAsync(dskin.p, 0, sizeof(DevSkin), st_));
    return SPH_OK;
  }

  // the work of one step, with every size and decision on the device
  int step_body_dev() {
    CK(cudaMemsetAsync(drs_err.p, 0, sizeof(int), s));
    CK(cudaMemsetAsync(overflow.p, 0, sizeof(int32_t), s));
    Params P{};
    RC(params(P));
    unsigned long long* r = red.as<unsigned long long>();
    SlotInit si{};
    const int slot[8] = {RED_TS_HMIN, RED_TS_CMAX, RED_TS_DENMIN, RED_TS_CMIN,
                         RED_TS_KAPMAX, RED_TS_BMAX, RED_TS_KAPMIN, RED_TS_LAMMAX};
    const double init[8] = {1e308, -1e308, 1e308, 1e308, -1e308, -1e308, 1e308, -1e308};
    for (int k = 0; k < 8; ++k) { si.off[k] = slot[k]; si.val[k] = dkey(init[k]); }
    si.n = 8;
    launch_init_slots(r, si, s);
    launch_timestep_reduce(cols.as<double>(), nrows, orig.as<int32_t>(), nrows,
                           int64_t(st[ec_realpn]), P, r, s);
    DtIn di{};
    di.eq_hydro = eq_hydro; di.eq_magneto = eq_magneto; di.eq_diff = eq_diff; di.eq_fld = eq_fld;
    di.sts_fixed = eq_sts ? 1 : 0;
    di.sts_s = ival(ec_stsfixeds);
    di.cn_hydro = kb.cn_hydro;
    di.cnd2 = cnd2();
    launch_dt(r, di, drs_clock.as<DevClock>(), ctrl.as<double>(), s);
    const bool do_sts = eq_sts;
    launch_predict(cols.as<double>(), nrows, orig.as<int32_t>(), nrows, n_int, save.as<double>(),
                   ctrl.as<double>(), lf_mode(do_sts), s);
    RC(iterate(true));
    launch_correct(cols.as<double>(), nrows, orig.as<int32_t>(), nrows, n_int, save.as<double>(),
                   ctrl.as<double>(), lf_mode(do_sts), s);
    if (do_sts) RC(sts_integrate(ival(ec_stsfixeds), 0.0));
    launch_clock_advance(drs_clock.as<DevClock>(), s);
    return SPH_OK;
  }

  static void drop_slot(GraphSlot& q) {
    if (q.x) cudaGraphExecDestroy(q.x);
    if (q.g) cudaGraphDestroy(q.g);
    q = GraphSlot{};
  }

  void drop_graph() {
    for (auto& q : gslot) drop_slot(q);
    graph_dirty = true;
  }

  // one step of the time loop without host round trips (falls back to
  // one_step when the handle does not qualify or the step must be redone)
  int one_step_graph(double tfinish, bool& done) {
    double t = st[ec_time];
    if (!((t < tfinish + std::numeric_limits<double>::epsilon()) && !stopped)) {
      done = true;
      return SPH_OK;
    }
    const char* why = nullptr;
    if (!drs_eligible(&why)) {
      static const bool log = std::getenv("SPH_GRAPH_LOG") != nullptr;
      if (log) std::fprintf(stderr, "sph: step on the host path: %s\n", why);
      return one_step(tfinish, done);
    }
    done = false;
    int reorder_every = int(st[SPH_P_REORDER_EVERY]);
    if (reorder_every > 0 && steps_since_reorder >= reorder_every) RC(reorder_rows());
    RC(drs_prepare());
    // buffers the graph was captured with may have moved since
    if (cnt_host[SPH_CNT_ALLOCS] != graph_alloc_mark) graph_dirty = true;
    if (graph_dirty) {
      drop_graph();
      graph_dirty = false;
      graph_alloc_mark = cnt_host[SPH_CNT_ALLOCS];
    }
    RC(copy_table(drs_save.p, cols.p));
    DevClock clk{};
    clk.t = t;
    clk.ltout = ltout;
    clk.dtout = dtout;
    clk.tfinish = tfinish;
    clk.stopped = stopped ? 1 : 0;
    std::memcpy(h_ctrl + 1, &clk, sizeof(DevClock));
    CK(cudaMemcpyAsync(drs_clock.p, h_ctrl + 1, sizeof(DevClock), cudaMemcpyHostToDevice, s));
    GraphSlot* gs = nullptr;
    for (auto& q : gslot)
      if (q.x && q.k_cols == cols.p && q.k_orig == orig.p) gs = &q;
    if (!gs) {
      gs = &gslot[gslot_next];
      gslot_next ^= 1;
      drop_slot(*gs);
      dplan = drs_plan.as<DevPlan>();
      cudaError_t e = cudaStreamBeginCapture(s, cudaStreamCaptureModeThreadLocal);
      int rc = e == cudaSuccess ? step_body_dev() : SPH_ERR_CUDA;
      cudaError_t e2 = cudaStreamEndCapture(s, &gs->g);
      dplan = nullptr;
      if (rc || e != cudaSuccess || e2 != cudaSuccess) {
        cudaGetLastError();
        drop_graph();
        if (!rc) rc = fail(SPH_ERR_CUDA, "step capture failed");
        return rc;
      }
      if (cudaGraphInstantiate(&gs->x, gs->g, 0) != cudaSuccess) {
        cudaGetLastError();
        drop_graph();
        return fail(SPH_ERR_CUDA, "graph instantiation failed");
      }
      gs->k_cols = cols.p;
      gs->k_orig = orig.p;
    }
    RC(dlists_reset(s));
    CK(cudaGraphLaunch(gs->x, s));
    // one read-back per step: the clock, the error words
    CK(cudaMemcpyAsync(h_ctrl + 1, drs_clock.p, sizeof(DevClock), cudaMemcpyDeviceToHost, s));
    CK(cudaMemcpyAsync(h_i32 + 4, drs_err.p, sizeof(int), cudaMemcpyDeviceToHost, s));
    CK(cudaMemcpyAsync(h_i32 + 5, overflow.p, sizeof(int32_t), cudaMemcpyDeviceToHost, s));
    CK(cudaMemcpyAsync(h_i32 + 6, status.p, sizeof(int), cudaMemcpyDeviceToHost, s));
    CK(cudaMemcpyAsync(h_plan, drs_plan.p, sizeof(DevPlan), cudaMemcpyDeviceToHost, s));
    CK(cudaStreamSynchronize(s));
    CK(cudaGetLastError());
    std::memcpy(&clk, h_ctrl + 1, sizeof(DevClock));
    if (h_i32[4] || h_i32[5] || h_i32[6]) {
      // redo this step on the host path from the saved table
      RC(copy_table(cols.p, drs_save.p));
      CK(cudaMemsetAsync(status.p, 0, sizeof(int), s));
      cnt_host[SPH_CNT_GRAPH_REDOS]++;
      return one_step(tfinish, done);
    }
    st[ec_time] = clk.t;
    ltout = clk.ltout;
    stopped = clk.stopped != 0;
    have_order = true;
    rows_in_order = false;
    nghost = h_plan->nghost;  // the host view of the last search, as after a host step
    grid = h_plan->grid;
    pgeom = h_plan->pg;
    cnt_host[SPH_CNT_STEPS]++;
    cnt_host[SPH_CNT_ITERATES] += eq_sts ? 1 + ival(ec_stsfixeds) : 1;
    // (with skin lists the device counts its searches)
    if (!(skin_fraction() > 0)) cnt_host[SPH_CNT_SEARCHES] += eq_sts ? 1 + ival(ec_stsfixeds) : 1;
    dlists_ok = true;
    steps_since_reorder++;
    cnt_host[SPH_CNT_GRAPH_STEPS]++;
    return SPH_OK;
  }

  // ---- one instance of a batch's device loop -------------------------------------------------
  // The body of the instance's if node: the reorder decision of one_step
  // (every SPH_P_REORDER_EVERY steps, as the rows of the last search), the
  // reorder itself in place, the table saved for a redo, the device-resident
  // step of one_step_graph, and the check of its error words.  Captured with
  // the capacities of drs_prepare.
  int batch_step_body(BatchInst* b) {
    launch_inst_begin(b, drs_clock.as<DevClock>(), bclk_save.as<DevClock>(), s);
    launch_reorder_gated(b, cols.as<double>(), cols_alt.as<double>(), orig.as<int32_t>(),
                         orig_alt.as<int32_t>(), centre_p.as<int32_t>(), nreal, nrows,
                         skin_fraction() > 0 ? dskin.as<DevSkin>() : nullptr, s);
    RC(copy_table(drs_save.p, cols.p));
    RC(step_body_dev());
    launch_inst_end(b, drs_err.as<int>(), overflow.as<int32_t>(), status.as<int>(), s);
    return SPH_OK;
  }
  // host view of the clock before a device loop
  void upload_clock(double tfinish) {
    DevClock clk{};
    clk.t = st[ec_time];
    clk.ltout = ltout;
    clk.dtout = dtout;
    clk.tfinish = tfinish;
    clk.stopped = stopped ? 1 : 0;
    std::memcpy(h_ctrl + 1, &clk, sizeof(DevClock));
  }
  // host view after a device loop ran `steps` steps of this instance
  void adopt_loop(const DevClock& clk, const DevPlan& plan, long long steps, int since) {
    steps_since_reorder = since;
    if (steps <= 0) return;
    st[ec_time] = clk.t;
    ltout = clk.ltout;
    stopped = clk.stopped != 0;
    have_order = true;
    rows_in_order = false;
    nghost = plan.nghost;
    grid = plan.grid;
    pgeom = plan.pg;
    const long long per = eq_sts ? 1 + ival(ec_stsfixeds) : 1;
    cnt_host[SPH_CNT_STEPS] += steps;
    cnt_host[SPH_CNT_ITERATES] += steps * per;
    if (!(skin_fraction() > 0)) cnt_host[SPH_CNT_SEARCHES] += steps * per;
    cnt_host[SPH_CNT_GRAPH_STEPS] += steps;
  }

  // ---- closing error evaluation (main.f90:374-402) ---------------------------------------------
  DevBuf errb, errpart;
  int errcalc(double* err_out, int64_t cap, double* l1) {
    if (err_out && cap < nreal) return fail(SPH_ERR_ARG, "err_out holds fewer than realpn values");
    if (ival(ec_eqs) == eeq_kd2)
      return fail(SPH_ERR_UNSUPPORTED, "the Taylor (chi) error of equations = kd2 is not built");
    ErrCalcIn in{};
    in.dim = dim();
    in.diso = ival(ec_disotropic);
    in.t = st[ec_time];
    switch (ival(ec_ics)) {
      case ett_shock12: in.kind = EK_SHOCK12; break;
      case ett_ring: in.kind = EK_RING; break;
      case ett_pulse: {
        // the constants of errcalc.f90:66-71, in its operation order
        in.kind = EK_PULSE;
        const double eps = 0.1, dcnd = st[ec_dcondconst];
        in.pifac = std::pow(2.0 * kPi, -in.dim / 2.0);
        in.ekt = eps * eps + 2.0 * dcnd * in.t;
        in.ektd2 = std::pow(in.ekt, in.dim / 2.0);
        in.ektsq = std::pow(in.ekt, 1.0 / 2.0);
        in.epsdm1 = 1.0;
        for (int k = 1; k < in.dim; ++k) in.epsdm1 *= eps;
        break;
      }
      // err_sinxet fills err only when the type equals 1 (errcalc.f90:185),
      // which ett_sin3 (100) never does: err stays 0
      case ett_sin3: in.kind = EK_ZERO; break;
      case ett_soundwave: in.kind = EK_SOUNDWAVE; break;
      case ett_hydroshock:
        // exact_shock(1, t, 1.4, 0., 1., 1./8., 1., 0.1, 0., 0., ...)
        // (errcalc.f90:38): the standard Sod states, gamma 1.4 whatever
        // the run's gamma
        in.kind = EK_HYDROSHOCK;
        in.fan = riemann_fan(1.4, 1.0, 0.0, 1.0, 1.0 / 8.0, 0.0, 0.1, 0.0);
        break;
      case ett_alfvenwave: in.kind = EK_ALFVEN; break;
      case ett_OTvortex: case ett_mti: case ett_boilingtank: case ett_mtilowres: case e_none:
        in.kind = EK_ZERO;  // no calculator: err as allocated, zero
        break;
      default:
        return fail(SPH_ERR_UNSUPPORTED, "Task type was not sen in L2 error evaluation");
    }
    const int64_t np = errcalc_parts(nreal);
    RC(errb.ensure(sizeof(double) * nreal));
    RC(errpart.ensure(sizeof(double) * (np + 1)));
    double* part = errpart.as<double>();
    double* sum = part + np;
    launch_errcalc(cols.as<double>(), nrows, orig.as<int32_t>(), nrows, nreal, in,
                   errb.as<double>(), part, sum, s);
    CK(cudaGetLastError());
    double total = 0.0;
    CK(cudaMemcpyAsync(h_ctrl + 15, sum, sizeof(double), cudaMemcpyDeviceToHost, s));
    if (err_out)
      CK(cudaMemcpyAsync(err_out, errb.p, sizeof(double) * nreal, cudaMemcpyDeviceToHost, s));
    CK(cudaStreamSynchronize(s));
    total = h_ctrl[15];
    if (l1) *l1 = nreal > 0 ? total / double(nreal) : 0.0;
    return SPH_OK;
  }

  // ---- pre-run check (preruncheck.f90:13-60) -------------------------------------------------
  int check_vars_ready() {
    int s_tt = ival(ec_eqs);
    if (st[ec_muzero] <= 0. && (s_tt == eeq_magnetohydro || s_tt == eeq_magnetohydrodiffusion))
      return fail(SPH_ERR_IC_MUZERO, "mhd_magneticconstant <= 0");
    if (ival(ec_disotropic) > 0 && st[ec_dcondconst] <= 0)
      return fail(SPH_ERR_IC_DIFFCOND, "diff_conductivity <= 0");
    std::vector<double> h(NCOL * nrows);
    CK(cudaMemcpyAsync(h.data(), cols.p, sizeof(double) * NCOL * nrows, cudaMemcpyDeviceToHost, s));
    CK(cudaStreamSynchronize(s));
    auto C = [&](int f, int64_t i) { return h[size_t(f) * nrows + i]; };
    for (int64_t i = 0; i < nrows; ++i) {
      if (int(C(es_type, i)) == ept_empty) continue;
      if (C(es_den, i) <= 0.) return fail(SPH_ERR_IC_DENSITY, "density <= 0");
      if (C(es_c, i) <= 0.) return fail(SPH_ERR_IC_CSOUND, "csound <= 0");
      if (C(es_h, i) <= 0.) return fail(SPH_ERR_IC_H, "smoothing length <= 0");
      if (C(es_p, i) <= 0.) return fail(SPH_ERR_IC_PRESSURE, "pressure <= 0");
      if (C(es_u, i) <= 0.) return fail(SPH_ERR_IC_ENERGY, "internal energy <= 0");
    }
    return SPH_OK;
  }

  // ---- time loop (main.f90:216-373) ------------------------------------------------------------
  int start_run() {
    eqset();
    double t = st[ec_time];
    dtout = st[ec_dtprint];
    double tfinish = st[ec_tfinish];
    stopped = false;
    if (tfinish > 0.) {
      RC(check_vars_ready());
      if (ival(ec_eqs) != eeq_kd2) RC(iterate(true));
      else stopped = true;
    } else {
      stopped = true;
    }
    ltout = 0.;
    if (dtout > 0) while (ltout < t) ltout = ltout + dtout;
    started = true;
    return SPH_OK;
  }

  int timestep(double& dthydro, double& dtdiff, double& dtfld, double& dt) {
    Phase ph(this, SPH_T_TIMESTEP);
    Params P{};
    RC(params(P));
    unsigned long long* r = red.as<unsigned long long>();
    SlotInit si{};
    const int slot[8] = {RED_TS_HMIN, RED_TS_CMAX, RED_TS_DENMIN, RED_TS_CMIN,
                         RED_TS_KAPMAX, RED_TS_BMAX, RED_TS_KAPMIN, RED_TS_LAMMAX};
    const double init[8] = {1e308, -1e308, 1e308, 1e308, -1e308, -1e308, 1e308, -1e308};
    for (int k = 0; k < 8; ++k) { si.off[k] = slot[k]; si.val[k] = dkey(init[k]); }
    si.n = 8;
    launch_init_slots(r, si, s);
    launch_timestep_reduce(cols.as<double>(), nrows, orig.as<int32_t>(), nrows,
                           int64_t(st[ec_realpn]), P, r, s);
    CK(cudaMemcpyAsync(h_red + RED_TS_HMIN, r + RED_TS_HMIN,
                       sizeof(unsigned long long) * (RED_TS_LAMMAX - RED_TS_HMIN + 1),
                       cudaMemcpyDeviceToHost, s));
    CK(cudaStreamSynchronize(s));
    CK(cudaGetLastError());
    // every earlier phase has completed at this point; the event pairs are
    // read at the end of the call unless many have piled up
    if (pending_ev.size() > 4096) collect_timers();
    double hmin = dkey_inv(h_red[RED_TS_HMIN]), cmax = dkey_inv(h_red[RED_TS_CMAX]);
    double denmin = dkey_inv(h_red[RED_TS_DENMIN]), cmin = dkey_inv(h_red[RED_TS_CMIN]);
    double kapmax = dkey_inv(h_red[RED_TS_KAPMAX]), bmax = dkey_inv(h_red[RED_TS_BMAX]);
    double kapmin = dkey_inv(h_red[RED_TS_KAPMIN]), lammax = dkey_inv(h_red[RED_TS_LAMMAX]);
    dt = std::numeric_limits<double>::max();
    dthydro = 0.;
    dtdiff = std::numeric_limits<double>::infinity();
    dtfld = std::numeric_limits<double>::infinity();
    if (eq_hydro) {
      dthydro = kb.cn_hydro * hmin / cmax;
      dt = std::min(dt, dthydro);
    }
    if (eq_magneto) dt = std::min(dt, .1 * hmin / cmax / bmax);
    if (eq_diff) {
      dtdiff = cnd2() * denmin * cmin * (hmin * hmin) / kapmax;
      dt = std::min(dt, dtdiff);
    }
    if (eq_fld) {
      dtfld = cnd2() * hmin * hmin * denmin * kapmin / kLightspeed / lammax;
      dt = std::min(dt, dtfld);
    }
    return SPH_OK;
  }

  // sts_integrator.f90:10-51: the stage coefficients
  static double sts_b(int j) { return j <= 2 ? 1. / 3. : (double(j * j + j) - 2.) / (2. * j * (j + 1.)); }
  static double sts_mu(int j) { return (2. * j - 1.) / j * sts_b(j) / sts_b(j - 1); }
  static double sts_nu(int j) { return -((j - 1.) / j * sts_b(j) / sts_b(j - 2)); }
  static double sts_w(int s_) { return 4. / (double(s_ * s_ + s_) - 2.); }
  static double sts_mu_hat(int j, int s_) { return j == 1 ? sts_b(1) * sts_w(s_) : sts_mu(j) * sts_w(s_); }
  static double sts_gm_hat(int j, int s_) { return -(1 - sts_b(j - 1)) * sts_mu_hat(j, s_); }
  int sts_coef_upload(int sts_s) {
    RC(sts_j.ensure(sizeof(int)));
    if (sts_s < 2 || (sts_coef.p && sts_coef_s == sts_s)) return SPH_OK;
    std::vector<double> c(4 * size_t(sts_s - 1));
    for (int j = 2; j <= sts_s; ++j) {
      double* q = c.data() + 4 * (j - 2);
      q[0] = sts_mu(j); q[1] = sts_nu(j); q[2] = sts_mu_hat(j, sts_s); q[3] = sts_gm_hat(j, sts_s);
    }
    RC(sts_coef.ensure(sizeof(double) * c.size()));
    CK(cudaMemcpy(sts_coef.p, c.data(), sizeof(double) * c.size(), cudaMemcpyHostToDevice));
    sts_coef_s = sts_s;
    return SPH_OK;
  }
  int sts_integrate(int sts_s, double dt) {
    // sts_integrator.f90:87-124; coefficients :10-51
    auto mu = [](int j) { return sts_mu(j); };
    auto nu = [](int j) { return sts_nu(j); };
    auto mu_hat = [](int j, int s_) { return sts_mu_hat(j, s_); };
    auto gm_hat = [](int j, int s_) { return sts_gm_hat(j, s_); };
    RC(stsY.ensure(sizeof(double) * 6 * nrows));
    double* Y = stsY.as<double>();
    {
      Phase ph(this, SPH_T_STS);
      launch_sts_stage(0, cols.as<double>(), nrows, nrows, Y, 0, 0, 0, 0, 0, ctrl.as<double>(), s);
    }
    RC(iterate(true));
    {
      Phase ph(this, SPH_T_STS);
      launch_sts_stage(1, cols.as<double>(), nrows, nrows, Y, mu_hat(1, sts_s), 0, 0, 0, 0,
                       ctrl.as<double>(), s);
    }
    if (dplan && sts_s >= 2) {
      // the device-resident step: stages 2 .. s as a while node over one
      // captured iterate (coefficients uploaded with the step's buffers)
      int* jd = sts_j.as<int>();
      const double* coef = sts_coef.as<double>();
      RC(capture_cond(
          cudaGraphCondTypeWhile,
          [&](cudaGraphConditionalHandle hw) { launch_sts_loop_init(jd, sts_s, hw, s); },
          [&](cudaGraphConditionalHandle hw) {
            RC(iterate(true));
            launch_sts_stage_dev(cols.as<double>(), nrows, nrows, Y, coef, jd, ctrl.as<double>(), s);
            launch_sts_loop_ctl(jd, sts_s, hw, s);
            return SPH_OK;
          }));
    } else
    for (int j = 2; j <= sts_s; ++j) {
      RC(iterate(true));
      Phase ph(this, SPH_T_STS);
      launch_sts_stage(2, cols.as<double>(), nrows, nrows, Y, mu(j), nu(j), mu_hat(j, sts_s),
                       gm_hat(j, sts_s), 0, ctrl.as<double>(), s);
    }
    {
      Phase ph(this, SPH_T_STS);
      launch_sts_stage(3, cols.as<double>(), nrows, nrows, Y, 0, 0, 0, 0, 0, ctrl.as<double>(), s);
    }
    CK(cudaGetLastError());
    return SPH_OK;
  }

  // One leapfrog step with a given dt (main.f90:323-362 without the
  // timestep and output logic): the differentiated forward map.  With
  // `stop_before_correct` the step ends after the force pass, leaving the
  // buffers of that pass for the adjoint kernels.
  int fixed_step(double dt, bool stop_before_correct = false) {
    h_ctrl[0] = dt;
    CK(cudaMemcpyAsync(ctrl.p, h_ctrl, sizeof(double), cudaMemcpyHostToDevice, s));
    {
      Phase ph(this, SPH_T_PREDICT);
      launch_predict(cols.as<double>(), nrows, orig.as<int32_t>(), nrows, n_int, save.as<double>(),
                     ctrl.as<double>(), lf_mode(false), s);
    }
    RC(iterate(true));
    if (stop_before_correct) return SPH_OK;
    return fixed_step_correct(dt);
  }
  // the rest of fixed_step after its force pass
  int fixed_step_correct(double dt) {
    {
      Phase ph(this, SPH_T_CORRECT);
      launch_correct(cols.as<double>(), nrows, orig.as<int32_t>(), nrows, n_int, save.as<double>(),
                     ctrl.as<double>(), lf_mode(false), s);
    }
    st[ec_time] += dt;
    cnt_host[SPH_CNT_STEPS]++;
    return SPH_OK;
  }
  size_t table_bytes() const { return sizeof(double) * NCOL * size_t(nrows); }
  int copy_table(void* dst, const void* src) {
    if (dst == cols.p) skin_valid = dlists_ok = false;  // the records' positions jump
    CK(cudaMemcpyAsync(dst, src, table_bytes(), cudaMemcpyDeviceToDevice, s));
    return SPH_OK;
  }
  double* ckpt(int i) { return adj_ckpt.as<double>() + size_t(i) * NCOL * nrows; }
  double* seg(int i) { return adj_seg.as<double>() + size_t(i) * NCOL * nrows; }
  // What the VJP of a step reads from its force pass, kept per step of a
  // segment while the segment is replayed, so that the backward sweep does
  // not run each step's forward a second time: the table after the force
  // pass, the sorted records, the centres and the neighbour lists.  Slots
  // are sized at the sweep's start; a step whose pass outgrew them (more
  // images, longer lists) is recomputed instead.
  DevBuf adj_mid;
  size_t adj_mid_slot = 0;
  int64_t adj_mid_nall = 0, adj_mid_nl = 0;
  std::vector<char> adj_mid_ok;
  std::vector<int64_t> adj_mid_used;  // per slot: the pass's record count and list size
  int64_t adj_mid_restored = 0;
  struct MidPart { DevBuf* b; size_t bytes; };
  void mid_parts(MidPart (&p)[9], int64_t nall, int64_t nl) {
    p[0] = {&cols, table_bytes()};
    p[1] = {&sx, sizeof(double) * size_t(nall)};
    p[2] = {&sy, sizeof(double) * size_t(nall)};
    p[3] = {&sz, sizeof(double) * size_t(nall)};
    p[4] = {&ssrc, sizeof(int32_t) * size_t(nall)};
    p[5] = {&centre_k, sizeof(int32_t) * size_t(nreal)};
    p[6] = {&centre_p, sizeof(int32_t) * size_t(nreal)};
    p[7] = {&rowoff, sizeof(int64_t) * size_t(nreal)};
    p[8] = {&ncnt, sizeof(int32_t) * size_t(nreal)};
    (void)nl;
  }
  static size_t mid_round(size_t b) { return (b + 255) & ~size_t(255); }
  size_t mid_slot_bytes(int64_t nall, int64_t nl) {
    MidPart p[9];
    mid_parts(p, nall, nl);
    size_t t = mid_round(sizeof(int32_t) * size_t(nl));
    for (auto& q : p) t += mid_round(q.bytes);
    return t;
  }
  // copy the pass's buffers into slot i (to) or back (from); false: the
  // pass does not fit the slot
  int mid_copy(int i, bool save, bool* fits) {
    int64_t nall = nrows + nghost, nlu = nl_size;
    if (save) {
      adj_mid_used[2 * size_t(i)] = nall;
      adj_mid_used[2 * size_t(i) + 1] = nlu;
    } else {
      nall = adj_mid_used[2 * size_t(i)];
      nlu = adj_mid_used[2 * size_t(i) + 1];
    }
    *fits = nall <= adj_mid_nall && nlu <= adj_mid_nl;
    if (!*fits) return SPH_OK;
    char* base = adj_mid.as<char>() + size_t(i) * adj_mid_slot;
    MidPart p[9];
    mid_parts(p, nall, nlu);
    size_t off = 0;
    auto cp = [&](void* dev, size_t bytes, size_t cap) -> int {
      void* slot = base + off;
      CK(cudaMemcpyAsync(save ? slot : dev, save ? dev : slot, bytes, cudaMemcpyDeviceToDevice, s));
      off += mid_round(cap);
      return SPH_OK;
    };
    MidPart cap[9];
    mid_parts(cap, adj_mid_nall, adj_mid_nl);
    for (int k = 0; k < 9; ++k) RC(cp(p[k].b->p, p[k].bytes, cap[k].bytes));
    RC(cp(nl.p, sizeof(int32_t) * size_t(nlu), sizeof(int32_t) * size_t(adj_mid_nl)));
    return SPH_OK;
  }

  // the hydro subset the adjoint kernels differentiate
  // which adjoint applies: the hydro one, or (adj_diff) the diffusion one
  bool adj_diff = false;
  int adjoint_supported() {
    eqset();
    adj_diff = false;
    if (eq_diff && !eq_hydro) {
      // pure diffusion: positions stay where they are (v = 0, no force), so
      // dT/dt is linear in T and in the conductivity
      if (eq_fld || eq_sts || eq_radexch || eq_magneto)
        return fail(SPH_ERR_UNSUPPORTED, "adjoint: diffusion without FLD, STS or MHD");
      const int ddw = ival(ec_ddw);
      if (ddw != esd_fab && ddw != esd_fw && ddw != esd_n2w)
        return fail(SPH_ERR_UNSUPPORTED, "adjoint: diffusion with ddw = fab, fw or n2w");
      if (nfixed > 0) return fail(SPH_ERR_UNSUPPORTED, "adjoint: fixed particles");
      if (!(st[SPH_P_FIXED_DT] > 0)) return fail(SPH_ERR_ARG, "adjoint: set SPH_P_FIXED_DT > 0");
      std::vector<double> v(3 * size_t(nrows));
      CK(cudaMemcpyAsync(v.data(), cols.as<double>() + size_t(es_vx) * nrows,
                         sizeof(double) * 3 * nrows, cudaMemcpyDeviceToHost, s));
      CK(cudaStreamSynchronize(s));
      for (double x : v)
        if (x != 0.0) return fail(SPH_ERR_UNSUPPORTED, "adjoint: diffusion needs v = 0 (fixed positions)");
      adj_diff = true;
      return SPH_OK;
    }
    if (ival(ec_eqs) != eeq_hydro || eq_magneto || eq_diff || eq_fld || eq_sts || eq_radexch)
      return fail(SPH_ERR_UNSUPPORTED, "adjoint: equations must be hydro or diffusion");
    if (ival(ec_adden) != 1)
      return fail(SPH_ERR_UNSUPPORTED, "adjoint: needs the Newton h-iteration (adden = yes)");
    if (ival(ec_artts) == 1 && st[ec_au] != -1.0 && st[ec_au] != 0.0)
      return fail(SPH_ERR_UNSUPPORTED,
                  "adjoint: artificial conductivity (au) is not differentiated; set au = 0 or -1");
    if (nfixed > 0) return fail(SPH_ERR_UNSUPPORTED, "adjoint: fixed particles");
    Mode m;
    RC(mode(m));
    if (m.eos_kind != 1 || m.mti) return fail(SPH_ERR_UNSUPPORTED, "adjoint: adiabatic EOS only");
    if (!(st[SPH_P_FIXED_DT] > 0)) return fail(SPH_ERR_ARG, "adjoint: set SPH_P_FIXED_DT > 0");
    return SPH_OK;
  }

  int adjoint_forward(int nsteps, int every) {
    RC(adjoint_supported());
    if (nsteps < 1 || every < 1) return fail(SPH_ERR_ARG, "adjoint: nsteps and every must be >= 1");
    st[SPH_P_REORDER_EVERY] = 0;  // rows stay put: checkpoints are row images
    st[SPH_P_SKIN] = 0;           // every iterate searches afresh (the replays' lists are
                                  // then those of the recorded steps, in the same order)
    // The adjoint differentiates the converged density pass (h a function of
    // the positions alone).  The stored rho and Omega are those of the last
    // Newton iterate before its update of h, so with the parity tolerance
    // (one sweep from the predicted h) they would still depend, to first
    // order, on that starting h; a tolerance of 1e-12 adds the sweep that
    // makes the dependence second order (Newton converges quadratically).
    st[SPH_P_NEWTON_TOL] = std::min(st[SPH_P_NEWTON_TOL], 1e-12);
    adj_dt = st[SPH_P_FIXED_DT];
    adj_nsteps = nsteps;
    adj_every = every;
    adj_ncp = (nsteps - 1) / every + 1;  // states at 0, k, 2k, ... below nsteps
    // slots: [0] before the initial force pass, [1 + i] at step i k, [ncp + 1] final
    RC(adj_ckpt.ensure(table_bytes() * size_t(adj_ncp + 2)));
    RC(adj_seg.ensure(table_bytes() * size_t(every)));
    adj_initial_force = !started;
    RC(copy_table(ckpt(0), cols.p));
    if (!started) {
      eqset();
      dtout = 0.;
      RC(check_vars_ready());
      RC(iterate(true));
      ltout = 0.;
      stopped = false;
      started = true;
    }
    adj_t0 = st[ec_time];
    for (int n = 0; n < nsteps; ++n) {
      if (n % every == 0) RC(copy_table(ckpt(1 + n / every), cols.p));
      RC(fixed_step(adj_dt));
    }
    RC(copy_table(ckpt(adj_ncp + 1), cols.p));
    CK(cudaStreamSynchronize(s));
    return SPH_OK;
  }

  AdjArgs adj_args() {
    Params P{};
    params(P);
    AdjArgs a{};
    a.nc = nreal;
    a.nreal = nreal;
    a.centre_k = centre_k.as<int32_t>();
    a.centre_p = centre_p.as<int32_t>();
    a.nl = nl.as<int32_t>();
    a.rowoff = rowoff.as<int64_t>();
    a.ncnt = ncnt.as<int32_t>();
    a.ssrc = ssrc.as<int32_t>();
    a.sx = sx.as<double>();
    a.sy = sy.as<double>();
    a.sz = sz.as<double>();
    a.cols = cols.as<double>();
    a.ld = nrows;
    a.adj = adj.as<double>();
    a.gpar = adj_par.as<double>();
    a.wcv = P.wCv;
    a.alpha = P.alpha;
    a.beta = P.beta;
    a.gamma = P.gamma;
    a.artts = P.artts == 1;
    a.hydro = P.eq_hydro != 0;
    a.diff = adj_diff ? 1 : 0;
    a.ddw = P.ddw;
    a.difiso = P.difiso;
    a.full_tensor = P.full_tensor;
    a.difcond = P.difcond;
    a.fwc = P.fwc;
    return a;
  }

  // dL/dv(T), dL/du(T), dL/dr(T) (original row order; NULL = 0) -> dL/d(r0,
  // v0, u0) and dL/d(alpha, beta) by the checkpointed adjoint sweep
  // (and dL/dT(T) -> dL/dT0, dL/d difcond for the diffusion adjoint; g_par
  // then has npar = 3 slots: alpha, beta, difcond)
  int adjoint_backward(const double* dl_dv, const double* dl_du, const double* dl_dr,
                       double* g_r0, double* g_v0, double* g_u0, double* g_par,
                       const double* dl_dT = nullptr, double* g_T0 = nullptr, int npar = 2) {
    if (adj_nsteps < 1) return fail(SPH_ERR_ARG, "adjoint: no forward run recorded");
    const int d = dim();
    RC(adj.ensure(sizeof(double) * AJ_TOTAL * size_t(nrows)));
    RC(adj_par.ensure(sizeof(double) * 3));
    RC(adj_io.ensure(sizeof(double) * 3 * size_t(nrows)));
    CK(cudaMemsetAsync(adj.p, 0, sizeof(double) * AJ_TOTAL * size_t(nrows), s));
    CK(cudaMemsetAsync(adj_par.p, 0, sizeof(double) * 3, s));
    auto load = [&](const double* host, int col, int ncomp) -> int {
      if (!host) return SPH_OK;
      CK(cudaMemcpyAsync(adj_io.p, host, sizeof(double) * ncomp * nrows, cudaMemcpyHostToDevice, s));
      launch_adj_gather(adj_io.as<double>(), ncomp, orig.as<int32_t>(), nrows,
                        adj.as<double>() + size_t(col) * nrows, nrows, s);
      return SPH_OK;
    };
    RC(load(dl_dv, AJ_LV, 3));
    RC(load(dl_du, AJ_LU, 1));
    RC(load(dl_dr, AJ_LR, 3));
    RC(load(dl_dT, AJ_LT, 1));
    const int G = lanes_pair();
    // per-step slots of the force passes when they fit a quarter of the free
    // device memory (at most 16 GB): 25 % room for more images and longer lists
    bool mid_on = false;
    adj_mid_restored = 0;
    {
      adj_mid_nall = (nrows + nghost) + (nghost + 3) / 4 + 1024;
      adj_mid_nl = nl_size + nl_size / 4 + 1024;
      adj_mid_slot = mid_slot_bytes(adj_mid_nall, adj_mid_nl);
      const size_t want = adj_mid_slot * size_t(adj_every);
      size_t free_b = 0, total_b = 0;
      if (cudaMemGetInfo(&free_b, &total_b) != cudaSuccess) {
        cudaGetLastError();
        free_b = 0;
      }
      if (want <= std::min(free_b / 4, size_t(16) << 30)) {
        RC(adj_mid.ensure(want));
        mid_on = true;
      }
      adj_mid_ok.assign(size_t(adj_every), 0);
      adj_mid_used.assign(2 * size_t(adj_every), 0);
      // (SPH_ADJ_TRACE in the environment: the slots' use, on stderr)
      static const bool trace = std::getenv("SPH_ADJ_TRACE") != nullptr;
      if (trace)
        std::fprintf(stderr, "adjoint backward: %s, %d slots of %.1f MB, free %.1f GB\n",
                     mid_on ? "force passes kept" : "force passes recomputed", adj_every,
                     adj_mid_slot / 1e6, free_b / 1e9);
    }
    for (int sgi = adj_ncp - 1; sgi >= 0; --sgi) {
      const int n0 = sgi * adj_every, n1 = std::min(adj_nsteps, n0 + adj_every);
      // replay the segment, keeping the state before every step and (where
      // it fits) what the step's VJP reads from its force pass
      RC(copy_table(cols.p, ckpt(1 + sgi)));
      for (int n = n0; n < n1; ++n) {
        RC(copy_table(seg(n - n0), cols.p));
        st[ec_time] = adj_t0 + n * adj_dt;
        if (!mid_on) {
          RC(fixed_step(adj_dt));
          continue;
        }
        RC(fixed_step(adj_dt, true));
        bool fits = false;
        RC(mid_copy(n - n0, true, &fits));
        adj_mid_ok[size_t(n - n0)] = fits ? 1 : 0;
        RC(fixed_step_correct(adj_dt));
      }
      for (int n = n1 - 1; n >= n0; --n) {
        bool fits = mid_on && adj_mid_ok[size_t(n - n0)];
        if (fits) RC(mid_copy(n - n0, false, &fits));
        adj_mid_restored += fits ? 1 : 0;
        if (!fits) {
          RC(copy_table(cols.p, seg(n - n0)));
          st[ec_time] = adj_t0 + n * adj_dt;
          RC(fixed_step(adj_dt, true));
        }
        launch_adj_step(kernel_id, d, G, adj_args(), adj_dt, 0, s);
      }
    }
    if (adj_initial_force) {
      RC(copy_table(cols.p, ckpt(0)));
      RC(iterate(true));
      launch_adj_step(kernel_id, d, G, adj_args(), adj_dt, 1, s);
    }
    auto store = [&](double* host, int col, int ncomp) -> int {
      if (!host) return SPH_OK;
      launch_adj_scatter(adj.as<double>() + size_t(col) * nrows, nrows, orig.as<int32_t>(), nrows,
                         adj_io.as<double>(), ncomp, s);
      CK(cudaMemcpyAsync(host, adj_io.p, sizeof(double) * ncomp * nrows, cudaMemcpyDeviceToHost, s));
      CK(cudaStreamSynchronize(s));
      return SPH_OK;
    };
    RC(store(g_v0, AJ_LV, 3));
    RC(store(g_u0, AJ_LU, 1));
    RC(store(g_r0, AJ_LR, 3));
    RC(store(g_T0, AJ_LT, 1));
    if (g_par) {
      CK(cudaMemcpyAsync(h_ctrl + 1, adj_par.p, sizeof(double) * 3, cudaMemcpyDeviceToHost, s));
      CK(cudaStreamSynchronize(s));
      for (int k = 0; k < npar && k < 3; ++k) g_par[k] = h_ctrl[1 + k];
    }
    if (std::getenv("SPH_ADJ_TRACE"))
      std::fprintf(stderr, "adjoint backward: %lld of %d steps from kept force passes\n",
                   (long long)adj_mid_restored, adj_nsteps);
    // back to the state at the end of the forward run
    RC(copy_table(cols.p, ckpt(adj_ncp + 1)));
    st[ec_time] = adj_t0 + adj_nsteps * adj_dt;
    RC(check_status());
    CK(cudaStreamSynchronize(s));
    return SPH_OK;
  }

  int one_step(double tfinish, bool& done) {
    double t = st[ec_time];
    if (!((t < tfinish + std::numeric_limits<double>::epsilon()) && !stopped)) {
      done = true;
      return SPH_OK;
    }
    done = false;
    int reorder_every = int(st[SPH_P_REORDER_EVERY]);
    // with skin lists the rows keep their order while the lists serve, and
    // are re-sorted before the search that replaces lists near their end
    if (reorder_every > 0 && steps_since_reorder >= reorder_every) RC(reorder_rows());
    double dthydro, dtdiff, dtfld, dt;
    RC(timestep(dthydro, dtdiff, dtfld, dt));
    bool do_sts = false;
    int sts_s = 0;
    if (eq_sts) {
      double sts_dt_min = std::min(dtdiff, dtfld);
      int sts_type = ival(ec_ststype);
      if (sts_type == 1) {
        sts_s = ival(ec_stsfixeds);
        dthydro = (sts_s * sts_s + sts_s - 2.) * 0.25 * sts_dt_min;
        dt = dthydro;
        do_sts = true;
      } else if (sts_type == 0) {
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
    h_ctrl[0] = dt;
    CK(cudaMemcpyAsync(ctrl.p, h_ctrl, sizeof(double), cudaMemcpyHostToDevice, s));
    {
      Phase ph(this, SPH_T_PREDICT);
      launch_predict(cols.as<double>(), nrows, orig.as<int32_t>(), nrows, n_int, save.as<double>(),
                     ctrl.as<double>(), lf_mode(do_sts), s);
    }
    RC(iterate(true));
    {
      Phase ph(this, SPH_T_CORRECT);
      launch_correct(cols.as<double>(), nrows, orig.as<int32_t>(), nrows, n_int, save.as<double>(),
                     ctrl.as<double>(), lf_mode(do_sts), s);
    }
    if (do_sts) RC(sts_integrate(sts_s, dt));
    if (eq_radexch) {  // main.f90:367-369
      launch_radexch(cols.as<double>(), nrows, orig.as<int32_t>(), nrows, n_int, dt,
                     st[ec_gamma], st[ec_molecularmass], status.as<int>(), s);
      RC(check_status());
    }
    st[ec_time] = t + dt;
    cnt_host[SPH_CNT_STEPS]++;
    steps_since_reorder++;
    CK(cudaGetLastError());
    return SPH_OK;
  }

  void destroy() {
    if (s) cudaStreamSynchronize(s);
    for (auto& pe : pending_ev) {
      cudaEventDestroy(pe.second.first);
      cudaEventDestroy(pe.second.second);
    }
    for (auto e : ev_pool) cudaEventDestroy(e);
    drop_graph();
    if (h_plan) cudaFreeHost(h_plan);
    if (h_red) cudaFreeHost(h_red);
    if (h_ctrl) cudaFreeHost(h_ctrl);
    if (h_i32) cudaFreeHost(h_i32);
    for (auto c : cap_s) cudaStreamDestroy(c);
    for (auto e : xfer_ev) cudaEventDestroy(e);
    if (xs) {
      cudaStreamSynchronize(xs);
      cudaStreamDestroy(xs);
    }
    if (s) cudaStreamDestroy(s);
  }
};

// ---- batches stepped by one device loop ----------------------------------------------------------
// A batch of instances (config-3 sweeps: lattices x second-derivative
// methods, run one Context after another by the reference's runners) steps
// as one CUDA graph: a while node whose body is a gate kernel, one if node
// per instance holding that instance's device-resident step, and a control
// kernel.  The gate opens the if nodes of the instances whose time loop has
// not ended (t < tfinish + eps and not stopped, main.f90:241); the if nodes
// of one iteration are independent branches, so the instances' steps run
// side by side on the device; the control kernel ends the loop when no
// instance runs, when one set an error word, or after kLoopCap iterations
// (a bound on every launch).  The host relaunches the loop until every
// instance is done; an instance whose step set an error word (a capacity or
// list row too small, Newton beyond its fixed sweeps) gets its table and
// clock back and redoes that step on the host path, as one_step_graph does.
namespace sph {

constexpr int kLoopCap = 128;

struct BatchGraph {
  cudaStream_t s = nullptr;
  cudaGraph_t g = nullptr;
  cudaGraphExec_t x = nullptr;
  std::vector<sph_handle*> members;
  struct Mark { long long allocs, params; int64_t nall_cap; int end_bit; };
  std::vector<Mark> marks;
  DevBuf bi, ifh, iter;
  std::vector<BatchInst> hbi;
  void drop() {
    if (x) cudaGraphExecDestroy(x);
    if (g) cudaGraphDestroy(g);
    x = nullptr;
    g = nullptr;
  }
  ~BatchGraph() {
    if (s) cudaStreamSynchronize(s);  // (its buffers go back to the cache)
    drop();
    if (s) cudaStreamDestroy(s);
  }
  static Mark mark_of(const sph_handle* h) {
    return {h->cnt_host[SPH_CNT_ALLOCS], h->param_gen, h->nall_cap, h->end_bit_cap};
  }
  bool stale(const std::vector<sph_handle*>& hs) const {
    if (!x || hs != members) return true;
    for (size_t i = 0; i < hs.size(); ++i) {
      const Mark m = mark_of(hs[i]);
      const Mark& o = marks[i];
      if (m.allocs != o.allocs || m.params != o.params || m.nall_cap != o.nall_cap ||
          m.end_bit != o.end_bit)
        return true;
    }
    return false;
  }
  // the while node, its body (gate -> if nodes -> control) and each
  // instance's step captured into its if node's body
  int build(const std::vector<sph_handle*>& hs) {
    drop();
    const int n = int(hs.size());
    if (!s) CK(cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking));
    RC(bi.ensure(sizeof(BatchInst) * n));
    RC(ifh.ensure(sizeof(cudaGraphConditionalHandle) * n));
    RC(iter.ensure(sizeof(int)));
    BatchInst* dbi = bi.as<BatchInst>();
    auto bad = [&](cudaError_t e, const char* what) {
      cudaGetLastError();
      drop();
      return fail(SPH_ERR_CUDA, std::string("batch loop: ") + what + ": " + cudaGetErrorString(e));
    };
    cudaError_t e = cudaGraphCreate(&g, 0);
    if (e != cudaSuccess) return bad(e, "graph");
    cudaGraphConditionalHandle wh;
    e = cudaGraphConditionalHandleCreate(&wh, g, 1, cudaGraphCondAssignDefault);
    if (e != cudaSuccess) return bad(e, "while handle");
    cudaGraphNodeParams wp{};
    wp.type = cudaGraphNodeTypeConditional;
    wp.conditional.handle = wh;
    wp.conditional.type = cudaGraphCondTypeWhile;
    wp.conditional.size = 1;
    cudaGraphNode_t wnode;
    e = cudaGraphAddNode(&wnode, g, nullptr, 0, &wp);
    if (e != cudaSuccess) return bad(e, "while node");
    cudaGraph_t body = wp.conditional.phGraph_out[0];
    // gate
    cudaGraphNode_t gate_node = nullptr;
    {
      e = cudaStreamBeginCaptureToGraph(s, body, nullptr, nullptr, 0, cudaStreamCaptureModeThreadLocal);
      if (e != cudaSuccess) return bad(e, "gate capture");
      launch_batch_gate(dbi, n, ifh.as<cudaGraphConditionalHandle>(), s);
      cudaGraph_t out;
      e = cudaStreamEndCapture(s, &out);
      if (e != cudaSuccess) return bad(e, "gate capture end");
      size_t nn = 0;
      e = cudaGraphGetNodes(body, nullptr, &nn);
      if (e != cudaSuccess || nn != 1) return bad(e, "gate node");
      e = cudaGraphGetNodes(body, &gate_node, &nn);
      if (e != cudaSuccess) return bad(e, "gate node");
    }
    // one if node per instance, after the gate
    std::vector<cudaGraphConditionalHandle> hh(n);
    std::vector<cudaGraphNode_t> ifn(n);
    for (int i = 0; i < n; ++i) {
      sph_handle* h = hs[i];
      e = cudaGraphConditionalHandleCreate(&hh[i], body, 0, 0);
      if (e != cudaSuccess) return bad(e, "if handle");
      cudaGraphNodeParams ip{};
      ip.type = cudaGraphNodeTypeConditional;
      ip.conditional.handle = hh[i];
      ip.conditional.type = cudaGraphCondTypeIf;
      ip.conditional.size = 1;
      e = cudaGraphAddNode(&ifn[i], body, &gate_node, 1, &ip);
      if (e != cudaSuccess) return bad(e, "if node");
      cudaGraph_t ib = ip.conditional.phGraph_out[0];
      h->dplan = h->drs_plan.as<DevPlan>();
      e = cudaStreamBeginCaptureToGraph(h->s, ib, nullptr, nullptr, 0,
                                        cudaStreamCaptureModeThreadLocal);
      int rc = e == cudaSuccess ? h->batch_step_body(dbi + i) : SPH_ERR_CUDA;
      cudaGraph_t out;
      cudaError_t e2 = e == cudaSuccess ? cudaStreamEndCapture(h->s, &out) : e;
      h->dplan = nullptr;
      if (rc || e != cudaSuccess || e2 != cudaSuccess) {
        cudaGetLastError();
        drop();
        return rc ? rc : fail(SPH_ERR_CUDA, std::string("batch loop: step capture: ") +
                                                cudaGetErrorString(e != cudaSuccess ? e : e2));
      }
    }
    // control, after every if node
    {
      e = cudaStreamBeginCaptureToGraph(s, body, ifn.data(), nullptr, ifn.size(),
                                        cudaStreamCaptureModeThreadLocal);
      if (e != cudaSuccess) return bad(e, "control capture");
      launch_batch_ctl(dbi, n, wh, iter.as<int>(), kLoopCap, s);
      cudaGraph_t out;
      e = cudaStreamEndCapture(s, &out);
      if (e != cudaSuccess) return bad(e, "control capture end");
    }
    CK(cudaMemcpyAsync(ifh.p, hh.data(), sizeof(cudaGraphConditionalHandle) * n,
                       cudaMemcpyHostToDevice, s));
    CK(cudaStreamSynchronize(s));
    const auto ti = std::chrono::steady_clock::now();
    e = cudaGraphInstantiate(&x, g, 0);
    if (e != cudaSuccess) return bad(e, "instantiate");
    static const bool trace = std::getenv("SPH_BATCH_TRACE") != nullptr;
    if (trace)
      std::fprintf(stderr, "batch loop instantiated in %.1f ms\n",
                   std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - ti)
                       .count());
    members = hs;
    marks.clear();
    for (auto* h : hs) marks.push_back(mark_of(h));
    return SPH_OK;
  }
};

void batch_graph_destroy(BatchGraph* bg) { delete bg; }

// Step the instances of a batch to tfinish (use_state: each instance's own
// tfinish) for at most `limit` steps each through the device loop.  *used =
// false (and nothing done) when an instance cannot take device-resident
// steps; the caller then runs the batch on host workers.
int batch_graph_run(BatchGraph** pbg, sph_handle* const* hs_in, int n, double tfinish,
                    bool use_state, long long limit, std::vector<int>& status,
                    std::vector<std::string>& msg, bool* used) {
  *used = false;
  std::vector<sph_handle*> hs(hs_in, hs_in + n);
  for (auto* h : hs)
    if (handle_device(h) != handle_device(hs[0])) return SPH_OK;
  CK(cudaSetDevice(handle_device(hs[0])));
  std::vector<double> tf(n);
  std::vector<long long> done_steps(n, 0);
  // start every instance (the start-up iterate of main.f90 runs on the
  // host path), then check that each can take device-resident steps
  for (int i = 0; i < n; ++i) {
    sph_handle* h = hs[i];
    t_alloc_count = &h->cnt_host[SPH_CNT_ALLOCS];
    if (!use_state) h->st[ec_tfinish] = tfinish;
    tf[i] = h->st[ec_tfinish];
    int rc = SPH_OK;
    if (!h->started) rc = h->start_run();
    if (!rc && h->ival(ec_eqs) != eeq_kd2) h->stopped = false;
    t_alloc_count = nullptr;
    if (rc) {
      status[i] = rc;
      msg[i] = g_err;
    }
  }
  for (int i = 0; i < n; ++i) {
    const char* why = nullptr;
    if (!status[i] && !hs[i]->drs_eligible(&why)) {
      // host workers instead (the instances keep their start)
      std::fill(status.begin(), status.end(), 0);
      return SPH_OK;
    }
  }
  *used = true;
  if (!*pbg) *pbg = new BatchGraph();
  BatchGraph* bg = *pbg;
  auto runs = [&](int i) {
    const sph_handle* h = hs[i];
    return status[i] == 0 && done_steps[i] < limit &&
           h->st[ec_time] < tf[i] + std::numeric_limits<double>::epsilon() && !h->stopped;
  };
  for (int guard = 0;; ++guard) {
    // the loop's members: every instance without an error (buffers of
    // finished instances stay valid; their if nodes stay closed)
    std::vector<int> live;
    for (int i = 0; i < n; ++i) {
      if (status[i]) continue;
      t_alloc_count = &hs[i]->cnt_host[SPH_CNT_ALLOCS];
      int rc = hs[i]->drs_prepare();
      t_alloc_count = nullptr;
      if (rc) {
        status[i] = rc;
        msg[i] = g_err;
        continue;
      }
      live.push_back(i);
    }
    bool any = false;
    for (int i : live) any |= runs(i);
    if (!any) break;
    std::vector<sph_handle*> lh;
    for (int i : live) lh.push_back(hs[i]);
    // (SPH_BATCH_TRACE in the environment: the loop's build times, on stderr)
    static const bool trace = std::getenv("SPH_BATCH_TRACE") != nullptr;
    if (bg->stale(lh)) {
      const auto t0 = std::chrono::steady_clock::now();
      RC(bg->build(lh));
      if (trace)
        std::fprintf(stderr, "batch loop built for %zu instances in %.1f ms\n", lh.size(),
                     std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0)
                         .count());
    }
    const int m = int(live.size());
    BatchInst* dbi = bg->bi.as<BatchInst>();
    bg->hbi.assign(m, BatchInst{});
    for (int k = 0; k < m; ++k) {
      const int i = live[k];
      sph_handle* h = hs[i];
      BatchInst& b = bg->hbi[k];
      b.clk = h->drs_clock.as<DevClock>();
      b.every = std::max(0, int(h->st[SPH_P_REORDER_EVERY]));
      b.since = h->steps_since_reorder;
      b.limit = runs(i) ? limit - done_steps[i] : 0;
      h->upload_clock(tf[i]);
      CK(cudaMemcpyAsync(h->drs_clock.p, h->h_ctrl + 1, sizeof(DevClock), cudaMemcpyHostToDevice,
                         bg->s));
      RC(h->dlists_reset(bg->s));
    }
    CK(cudaMemcpyAsync(dbi, bg->hbi.data(), sizeof(BatchInst) * m, cudaMemcpyHostToDevice, bg->s));
    CK(cudaMemsetAsync(bg->iter.p, 0, sizeof(int), bg->s));
    // the instances' own streams may still hold work (uploads, a host step)
    for (auto* h : lh) CK(cudaStreamSynchronize(h->s));
    CK(cudaGraphLaunch(bg->x, bg->s));
    CK(cudaMemcpyAsync(bg->hbi.data(), dbi, sizeof(BatchInst) * m, cudaMemcpyDeviceToHost, bg->s));
    CK(cudaStreamSynchronize(bg->s));
    CK(cudaGetLastError());
    for (int k = 0; k < m; ++k) {
      const int i = live[k];
      sph_handle* h = hs[i];
      const BatchInst& b = bg->hbi[k];
      if (b.steps <= 0 && !b.failed) continue;
      DevClock clk{}, saved{};
      CK(cudaMemcpy(&clk, h->drs_clock.p, sizeof(DevClock), cudaMemcpyDeviceToHost));
      CK(cudaMemcpy(&saved, h->bclk_save.p, sizeof(DevClock), cudaMemcpyDeviceToHost));
      CK(cudaMemcpy(h->h_plan, h->drs_plan.p, sizeof(DevPlan), cudaMemcpyDeviceToHost));
      done_steps[i] += b.steps;
      if (!b.failed) {
        h->adopt_loop(clk, *h->h_plan, b.steps, b.since);
        h->dlists_ok = true;
        continue;
      }
      // the steps before the failed one stand; the failed one is redone on
      // the host path from the table and the clock saved at its start
      h->adopt_loop(saved, *h->h_plan, b.steps, b.since);
      h->st[ec_time] = saved.t;
      h->ltout = saved.ltout;
      h->stopped = saved.stopped != 0;
      t_alloc_count = &h->cnt_host[SPH_CNT_ALLOCS];
      int rc = h->copy_table(h->cols.p, h->drs_save.p);
      if (!rc && cudaMemsetAsync(h->status.p, 0, sizeof(int), h->s) != cudaSuccess)
        rc = fail(SPH_ERR_CUDA, "status reset");
      h->cnt_host[SPH_CNT_GRAPH_REDOS]++;
      bool done = false;
      if (!rc) rc = h->one_step(tf[i], done);
      if (!rc && !done) done_steps[i] += 1;
      t_alloc_count = nullptr;
      if (rc) {
        status[i] = rc;
        msg[i] = g_err;
      }
    }
    if (guard > 1000000) return fail(SPH_ERR_STATE, "batch loop did not finish");
  }
  for (auto* h : hs) h->collect_timers();
  return SPH_OK;
}

}  // namespace sph

extern "C" {

// counts the device allocations of one C-ABI call on its handle
struct AllocScope {
  explicit AllocScope(sph_handle* h) { t_alloc_count = h ? &h->cnt_host[SPH_CNT_ALLOCS] : nullptr; }
  ~AllocScope() { t_alloc_count = nullptr; }
};

const char* sph_last_error(void) { return g_err.c_str(); }

int sph_create(const double* state49, const double* store, int64_t n_rows, int kernel_id,
               int precision_mode, sph_handle** out) {
  if (!state49 || !store || !out || n_rows <= 0) return fail(SPH_ERR_ARG, "null argument");
  if (kernel_id < 0 || kernel_id > 2) return fail(SPH_ERR_ARG, "bad kernel id");
  if (precision_mode != SPH_PREC_FP64 && precision_mode != SPH_PREC_FP32_COMP)
    return fail(SPH_ERR_ARG, "bad precision mode");
  if (n_rows > int64_t(INT32_MAX) / 8) return fail(SPH_ERR_ARG, "too many rows");
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) {
    cudaGetLastError();
    return fail(SPH_ERR_CUDA, "no CUDA device");
  }
  auto* h = new sph_handle();
  cudaGetDevice(&h->dev);
  h->kernel_id = kernel_id;
  h->prec = precision_mode;
  h->kb = kbase(kernel_id);
  h->st.assign(SPH_P_LAST + 1, 0.);
  for (int k = 1; k <= SPH_EC_TOTAL; ++k) h->st[k] = state49[k - 1];
  h->st[SPH_P_AV_ALPHA] = 1.;
  h->st[SPH_P_AV_BETA] = 2.;
  h->st[SPH_P_NEWTON_TOL] = 1e-8;
  h->st[SPH_P_NEWTON_MAXITER] = 100;
  h->st[SPH_P_CELL_FACTOR] = 0.4;
  h->st[SPH_P_REORDER_EVERY] = 8;
  h->st[SPH_P_SKIN] = 0.1;
  h->nreal = int64_t(h->st[ec_realpn]);
  h->nfixed = std::max<int64_t>(0, int64_t(h->st[ec_fixedpn]));
  if (h->nreal <= 0 || h->nreal + h->nfixed != n_rows) {
    delete h;
    return fail(SPH_ERR_ARG, "n_rows must equal realpn + fixedpn");
  }
  h->nrows = n_rows;
  // integrated rows: reals + fixedreal rows after them (main.f90:181-184)
  h->n_int = h->nreal;
  for (int64_t i = std::max<int64_t>(h->nreal - 1, 0); i < n_rows; ++i)
    if (int(store[i * NCOL + es_type]) == ept_fixedreal) h->n_int++;
  // mass scale for the packed streams
  double msum = 0.;
  for (int64_t i = 0; i < n_rows; ++i) msum += std::fabs(store[i * NCOL + es_m]);
  h->mref = msum > 0 ? store[0 * NCOL + es_m] : 1.0;
  if (!(h->mref > 0)) h->mref = msum / n_rows > 0 ? msum / n_rows : 1.0;
  int rc = SPH_OK;
  if (cudaStreamCreateWithFlags(&h->s, cudaStreamNonBlocking) != cudaSuccess) {
    cudaGetLastError();
    delete h;
    return fail(SPH_ERR_CUDA, "cudaStreamCreate failed");
  }
  if (cudaMallocHost(&h->h_red, sizeof(unsigned long long) * (RED_TOTAL + 2)) != cudaSuccess ||
      cudaMallocHost(&h->h_ctrl, sizeof(double) * 16) != cudaSuccess ||
      cudaMallocHost(&h->h_plan, sizeof(DevPlan)) != cudaSuccess ||
      cudaMallocHost(&h->h_i32, sizeof(int32_t) * 16) != cudaSuccess) {
    cudaGetLastError();
    h->destroy();
    delete h;
    return fail(SPH_ERR_OOM, "cudaMallocHost failed");
  }
  rc = h->alloc_base();
  if (!rc) {
    if (cudaMemcpyAsync(h->staging.p, store, sizeof(double) * NCOL * n_rows,
                        cudaMemcpyHostToDevice, h->s) != cudaSuccess)
      rc = fail(SPH_ERR_CUDA, "upload failed");
  }
  if (!rc) {
    launch_upload_store(h->staging.as<double>(), h->cols.as<double>(), h->orig.as<int32_t>(),
                        n_rows, h->s);
    if (cudaStreamSynchronize(h->s) != cudaSuccess || cudaGetLastError() != cudaSuccess)
      rc = fail(SPH_ERR_CUDA, "upload kernel failed");
  }
  if (rc) {
    h->destroy();
    delete h;
    return rc;
  }
  h->launch_base = launches_so_far();
  *out = h;
  return SPH_OK;
}

int sph_set_param(sph_handle* h, int index, double value) {
  if (!h || index < 1 || index > SPH_P_LAST) return fail(SPH_ERR_ARG, "bad param index");
  if ((index == ec_realpn || index == ec_fixedpn) && value != h->st[index])
    return fail(SPH_ERR_ARG, "particle counts are fixed by the store");
  if (h->st[index] != value) {  // a captured step holds the old value
    h->graph_dirty = true;
    h->param_gen++;
    // parameters that cannot change a neighbour set leave skin lists valid
    switch (index) {
      case SPH_P_TIMING: case SPH_P_AV_ALPHA: case SPH_P_AV_BETA: case SPH_P_NEWTON_TOL:
      case SPH_P_NEWTON_MAXITER: case SPH_P_LANES_PAIR: case SPH_P_FIXED_DT: case SPH_P_GRAPH:
      case SPH_P_REORDER_EVERY: case ec_tfinish: case ec_dtprint: case ec_time:
        break;
      default:
        h->skin_valid = h->dlists_ok = false;
    }
  }
  h->st[index] = value;
  if (index == SPH_P_NEIB_CAP && value > 0) h->est_count = 0;
  return SPH_OK;
}

int sph_get_param(sph_handle* h, int index, double* value) {
  if (!h || !value || index < 1 || index > SPH_P_LAST) return fail(SPH_ERR_ARG, "bad param index");
  *value = h->st[index];
  return SPH_OK;
}

int sph_set_store(sph_handle* h, const double* store, int64_t n_rows) {
  AllocScope alloc_scope(h);
  if (!h || !store || n_rows != h->nrows) return fail(SPH_ERR_ARG, "row count mismatch");
  // Skin lists outlive the upload: it puts the rows back in caller order
  // (old row p becomes row orig[p]), so what names rows is renamed; the new
  // positions and h are measured by the next iterate like any move; a
  // changed particle type (the image set) ends the lists.
  const bool keep = h->skin_valid;
  if (keep) {
    RC(h->skin_inv.ensure(sizeof(int32_t) * n_rows));
    RC(h->skin_perm.ensure(sizeof(int32_t) * n_rows));
    RC(h->skin_type.ensure(sizeof(double) * n_rows));
    RC(h->skin_flag.ensure(sizeof(int32_t)));
    CK(cudaMemcpyAsync(h->skin_inv.p, h->orig.p, sizeof(int32_t) * n_rows,
                       cudaMemcpyDeviceToDevice, h->s));
    CK(cudaMemcpyAsync(h->skin_type.p, h->col(es_type), sizeof(double) * n_rows,
                       cudaMemcpyDeviceToDevice, h->s));
    CK(cudaMemsetAsync(h->skin_flag.p, 0, sizeof(int32_t), h->s));
  }
  h->dlists_ok = false;
  {
    // in pieces: piece c crosses PCIe on the copy stream while piece c - 1
    // is transposed (the staging buffer waits for the work queued before)
    RC(h->xfer_setup());
    const int64_t cr = h->xfer_rows();
    CK(cudaEventRecord(h->xfer_ev[sph_handle::kXferChunks], h->s));
    CK(cudaStreamWaitEvent(h->xs, h->xfer_ev[sph_handle::kXferChunks], 0));
    double* stg = h->staging.as<double>();
    for (int c = 0; int64_t(c) * cr < n_rows; ++c) {
      const int64_t a = int64_t(c) * cr, b = std::min(n_rows, a + cr);
      CK(cudaMemcpyAsync(stg + a * NCOL, store + a * NCOL, sizeof(double) * NCOL * (b - a),
                         cudaMemcpyHostToDevice, h->xs));
      CK(cudaEventRecord(h->xfer_ev[c], h->xs));
      CK(cudaStreamWaitEvent(h->s, h->xfer_ev[c], 0));
      launch_upload_rows(stg, h->cols.as<double>(), h->orig.as<int32_t>(), n_rows, a, b, h->s);
    }
  }
  if (keep) {
    launch_inverse(h->skin_inv.as<int32_t>(), n_rows, h->skin_perm.as<int32_t>(), h->s);
    launch_type_changed(h->cols.as<double>(), n_rows, h->skin_type.as<double>(),
                        h->skin_perm.as<int32_t>(), h->skin_flag.as<int32_t>(), h->s);
    RC(h->rename_rows(h->skin_perm.as<int32_t>(), h->skin_inv.as<int32_t>()));
    CK(cudaMemcpyAsync(h->h_i32 + 4, h->skin_flag.p, sizeof(int32_t), cudaMemcpyDeviceToHost, h->s));
  }
  CK(cudaStreamSynchronize(h->s));
  CK(cudaGetLastError());
  if (keep && h->h_i32[4] == 0) {
    h->rows_in_order = false;  // (caller order: the next re-sort restores cell order)
  } else {
    h->have_order = false;
    h->skin_valid = false;
  }
  return SPH_OK;
}

int sph_iterate(sph_handle* h) {
  AllocScope alloc_scope(h);
  if (!h) return fail(SPH_ERR_ARG, "null handle");
  RC(h->reorder_rows());
  int rc = h->iterate(true);
  h->collect_timers();
  return rc;
}

int sph_density(sph_handle* h) {
  AllocScope alloc_scope(h);
  if (!h) return fail(SPH_ERR_ARG, "null handle");
  RC(h->reorder_rows());
  int rc = h->iterate(false);
  h->collect_timers();
  return rc;
}

int sph_step(sph_handle* h, int nsteps) {
  AllocScope alloc_scope(h);
  if (!h || nsteps < 0) return fail(SPH_ERR_ARG, "bad argument");
  int rc = SPH_OK;
  {
    sph_handle::Phase ph(h, SPH_T_STEP);
    if (!h->started) rc = h->start_run();
    if (!rc && h->ival(ec_eqs) != eeq_kd2) h->stopped = false;
    const bool graph = h->st[SPH_P_GRAPH] != 0;
    for (int i = 0; !rc && i < nsteps; ++i) {
      bool done = false;
      rc = graph ? h->one_step_graph(h->st[ec_tfinish], done) : h->one_step(h->st[ec_tfinish], done);
      if (done) break;
    }
  }
  h->collect_timers();
  return rc;
}

int sph_run_to(sph_handle* h, double tfinish) {
  AllocScope alloc_scope(h);
  if (!h) return fail(SPH_ERR_ARG, "null handle");
  h->st[ec_tfinish] = tfinish;
  int rc = SPH_OK;
  {
    sph_handle::Phase ph(h, SPH_T_STEP);
    if (!h->started) rc = h->start_run();
    if (!rc && h->ival(ec_eqs) != eeq_kd2) h->stopped = false;
    const bool graph = h->st[SPH_P_GRAPH] != 0;
    while (!rc) {
      bool done = false;
      rc = graph ? h->one_step_graph(tfinish, done) : h->one_step(tfinish, done);
      if (done) break;
    }
  }
  h->collect_timers();
  return rc;
}

int sph_get_store(sph_handle* h, double* out, int64_t cap_rows) {
  if (!h || !out || cap_rows < h->nrows) return fail(SPH_ERR_ARG, "buffer too small");
  // in pieces of caller rows: piece c is transposed while piece c - 1
  // crosses PCIe on the copy stream
  RC(h->xfer_setup());
  RC(h->dl_inv.ensure(sizeof(int32_t) * size_t(h->nrows)));
  launch_inverse(h->orig.as<int32_t>(), h->nrows, h->dl_inv.as<int32_t>(), h->s);
  const int64_t cr = h->xfer_rows();
  double* stg = h->staging.as<double>();
  for (int c = 0; int64_t(c) * cr < h->nrows; ++c) {
    const int64_t a = int64_t(c) * cr, b = std::min(h->nrows, a + cr);
    launch_download_rows(h->cols.as<double>(), h->dl_inv.as<int32_t>(), stg, h->nrows, a, b,
                         h->s);
    CK(cudaEventRecord(h->xfer_ev[c], h->s));
    CK(cudaStreamWaitEvent(h->xs, h->xfer_ev[c], 0));
    CK(cudaMemcpyAsync(out + a * NCOL, stg + a * NCOL, sizeof(double) * NCOL * (b - a),
                       cudaMemcpyDeviceToHost, h->xs));
  }
  CK(cudaStreamSynchronize(h->xs));
  CK(cudaGetLastError());
  return SPH_OK;
}

int sph_get_state(sph_handle* h, double* out49) {
  if (!h || !out49) return fail(SPH_ERR_ARG, "null argument");
  for (int k = 1; k <= SPH_EC_TOTAL; ++k) out49[k - 1] = h->st[k];
  return SPH_OK;
}

int sph_get_neighbours(sph_handle* h, int64_t* offsets, int64_t* pairs, int64_t cap) {
  if (!h || !offsets) return fail(SPH_ERR_ARG, "null argument");
  if (!h->have_order) return fail(SPH_ERR_STATE, "no neighbour search since the last re-ordering");
  const int64_t nc = h->nreal, nall = h->nrows + h->nghost;
  std::vector<int32_t> cnt(nc), cp(nc), og(h->nrows), sidx(nall), ssrc(nall);
  std::vector<int8_t> gcode(std::max<int64_t>(h->nghost, 1));
  std::vector<int64_t> roff(nc);
  CK(cudaMemcpyAsync(roff.data(), h->rowoff.p, sizeof(int64_t) * nc, cudaMemcpyDeviceToHost, h->s));
  CK(cudaStreamSynchronize(h->s));
  int64_t nl_used = nc > 0 ? roff[nc - 1] + 1 : 1;
  for (int64_t c = 0; c < nc; ++c) nl_used = std::max<int64_t>(nl_used, roff[c] + 1);
  std::vector<int32_t> ncv(nc);
  CK(cudaMemcpyAsync(ncv.data(), h->ncnt.p, sizeof(int32_t) * nc, cudaMemcpyDeviceToHost, h->s));
  CK(cudaStreamSynchronize(h->s));
  for (int64_t c = 0; c < nc; ++c) nl_used = std::max<int64_t>(nl_used, roff[c] + ncv[c]);
  nl_used = std::min<int64_t>(nl_used, h->nl_size);
  std::vector<int32_t> nl(nl_used);
  cudaStream_t s = h->s;
  CK(cudaMemcpyAsync(cnt.data(), h->ncnt.p, sizeof(int32_t) * nc, cudaMemcpyDeviceToHost, s));
  CK(cudaMemcpyAsync(cp.data(), h->centre_p.p, sizeof(int32_t) * nc, cudaMemcpyDeviceToHost, s));
  CK(cudaMemcpyAsync(og.data(), h->orig.p, sizeof(int32_t) * h->nrows, cudaMemcpyDeviceToHost, s));
  CK(cudaMemcpyAsync(sidx.data(), h->vals_alt.p, sizeof(int32_t) * nall, cudaMemcpyDeviceToHost, s));
  CK(cudaMemcpyAsync(ssrc.data(), h->ssrc.p, sizeof(int32_t) * nall, cudaMemcpyDeviceToHost, s));
  if (h->nghost > 0)
    CK(cudaMemcpyAsync(gcode.data(), h->gcode.p, sizeof(int8_t) * h->nghost, cudaMemcpyDeviceToHost, s));
  CK(cudaMemcpyAsync(nl.data(), h->nl.p, sizeof(int32_t) * nl.size(), cudaMemcpyDeviceToHost, s));
  CK(cudaStreamSynchronize(s));
  std::vector<int64_t> cnt_by_orig(nc, 0), centre_of_orig(nc, -1);
  for (int64_t c = 0; c < nc; ++c) {
    int64_t o = og[cp[c]];
    if (o < 0 || o >= nc) return fail(SPH_ERR_STATE, "centre row out of range");
    cnt_by_orig[o] = cnt[c];
    centre_of_orig[o] = c;
  }
  offsets[0] = 0;
  for (int64_t o = 0; o < nc; ++o) offsets[o + 1] = offsets[o] + cnt_by_orig[o];
  if (!pairs || cap < offsets[nc]) return fail(SPH_ERR_ARG, "pairs buffer too small");
  for (int64_t o = 0; o < nc; ++o) {
    int64_t c = centre_of_orig[o];
    int64_t base = offsets[o];
    for (int l = 0; l < cnt[c]; ++l) {
      int64_t q = nl[size_t(roff[c] + l)];
      int64_t u = sidx[q];
      int64_t rj = og[ssrc[q]];
      int64_t code = u < h->nrows ? 13 : gcode[u - h->nrows];
      pairs[base + l] = (rj << 5) | code;
    }
    std::sort(pairs + base, pairs + base + cnt[c]);
  }
  return SPH_OK;
}

int sph_get_neighbour_digest(sph_handle* h, uint64_t* out, int64_t n) {
  if (!h || !out) return fail(SPH_ERR_ARG, "null argument");
  if (!h->have_order) return fail(SPH_ERR_STATE, "no neighbour search since the last re-ordering");
  if (n < h->nreal) return fail(SPH_ERR_ARG, "digest buffer shorter than the real rows");
  const int64_t nc = h->nreal;
  DevBuf d;
  RC(d.ensure(sizeof(unsigned long long) * 2 * std::max<int64_t>(nc, 1)));
  launch_neib_digest(nc, h->centre_p.as<int32_t>(), h->orig.as<int32_t>(),
                     h->rowoff.as<int64_t>(), h->ncnt.as<int32_t>(), h->nl.as<int32_t>(),
                     h->vals_alt.as<int32_t>(), h->ssrc.as<int32_t>(), h->gcode.as<int8_t>(),
                     h->nrows, d.as<unsigned long long>(), h->s);
  CK(cudaGetLastError());
  CK(cudaMemcpyAsync(out, d.p, sizeof(uint64_t) * 2 * nc, cudaMemcpyDeviceToHost, h->s));
  CK(cudaStreamSynchronize(h->s));
  return SPH_OK;
}

// ---- one leapfrog step in parts (a driver that exchanges fields between
// the parts, one domain per GPU) ----
int sph_timestep(sph_handle* h, double* dt) {
  AllocScope alloc_scope(h);
  if (!h || !dt) return fail(SPH_ERR_ARG, "null argument");
  double dthydro = 0., dtdiff = 0., dtfld = 0., d = 0.;
  RC(h->timestep(dthydro, dtdiff, dtfld, d));
  *dt = d;
  return SPH_OK;
}

static int split_step_supported(sph_handle* h) {
  h->eqset();
  if (h->eq_sts || h->eq_radexch)
    return fail(SPH_ERR_UNSUPPORTED,
                "split step: leapfrog without STS or radiation exchange only");
  return SPH_OK;
}

int sph_predict(sph_handle* h, double dt) {
  AllocScope alloc_scope(h);
  if (!h) return fail(SPH_ERR_ARG, "null handle");
  RC(split_step_supported(h));
  h->h_ctrl[0] = dt;
  CK(cudaMemcpyAsync(h->ctrl.p, h->h_ctrl, sizeof(double), cudaMemcpyHostToDevice, h->s));
  launch_predict(h->cols.as<double>(), h->nrows, h->orig.as<int32_t>(), h->nrows, h->n_int,
                 h->save.as<double>(), h->ctrl.as<double>(), h->lf_mode(false), h->s);
  CK(cudaGetLastError());
  h->in_split_step = true;
  return SPH_OK;
}

int sph_forces(sph_handle* h) {
  AllocScope alloc_scope(h);
  if (!h) return fail(SPH_ERR_ARG, "null handle");
  if (!h->have_order) return fail(SPH_ERR_STATE, "sph_forces needs the lists of a density pass");
  Params P{};
  RC(h->params(P));
  Mode m;
  RC(h->mode(m));
  RC(h->circuit2(m, P));
  RC(h->check_status());
  h->cnt_host[SPH_CNT_ITERATES] += 1;
  h->collect_timers();
  return SPH_OK;
}

int sph_correct(sph_handle* h, double dt) {
  AllocScope alloc_scope(h);
  if (!h) return fail(SPH_ERR_ARG, "null handle");
  RC(split_step_supported(h));
  if (!h->in_split_step) return fail(SPH_ERR_STATE, "sph_correct without sph_predict");
  h->h_ctrl[0] = dt;
  CK(cudaMemcpyAsync(h->ctrl.p, h->h_ctrl, sizeof(double), cudaMemcpyHostToDevice, h->s));
  launch_correct(h->cols.as<double>(), h->nrows, h->orig.as<int32_t>(), h->nrows, h->n_int,
                 h->save.as<double>(), h->ctrl.as<double>(), h->lf_mode(false), h->s);
  CK(cudaGetLastError());
  h->in_split_step = false;
  h->st[ec_time] += dt;
  h->cnt_host[SPH_CNT_STEPS]++;
  return SPH_OK;
}

static int column_set(const int* fields, int nf, ColumnSet* fs) {
  if (!fields || nf < 1 || nf > SPH_ES_TOTAL) return fail(SPH_ERR_ARG, "1 to 32 fields");
  fs->n = nf;
  for (int k = 0; k < nf; ++k) {
    if (fields[k] < 1 || fields[k] > SPH_ES_TOTAL) return fail(SPH_ERR_ARG, "bad field index");
    fs->f[k] = fields[k] - 1;
  }
  return SPH_OK;
}

int sph_get_columns(sph_handle* h, const int* fields, int nf, double* out) {
  AllocScope alloc_scope(h);
  if (!h || !out) return fail(SPH_ERR_ARG, "null argument");
  ColumnSet fs{};
  RC(column_set(fields, nf, &fs));
  const size_t bytes = sizeof(double) * size_t(nf) * size_t(h->nrows);
  RC(h->colbuf.ensure(bytes));
  launch_get_columns(h->cols.as<double>(), h->nrows, h->orig.as<int32_t>(), h->nrows, fs,
                     h->colbuf.as<double>(), h->s);
  CK(cudaMemcpyAsync(out, h->colbuf.p, bytes, cudaMemcpyDefault, h->s));
  CK(cudaStreamSynchronize(h->s));
  CK(cudaGetLastError());
  return SPH_OK;
}

int sph_set_columns(sph_handle* h, const int* fields, int nf, const double* in) {
  AllocScope alloc_scope(h);
  if (!h || !in) return fail(SPH_ERR_ARG, "null argument");
  ColumnSet fs{};
  RC(column_set(fields, nf, &fs));
  const size_t bytes = sizeof(double) * size_t(nf) * size_t(h->nrows);
  RC(h->colbuf.ensure(bytes));
  CK(cudaMemcpyAsync(h->colbuf.p, in, bytes, cudaMemcpyDefault, h->s));
  launch_set_columns(h->cols.as<double>(), h->nrows, h->orig.as<int32_t>(), h->nrows, fs,
                     h->colbuf.as<double>(), h->s);
  // skin lists follow moved positions and changed h by themselves (the next
  // iterate measures both); a changed particle type may change the image set
  for (int k = 0; k < fs.n; ++k)
    if (fs.f[k] == es_type) h->skin_valid = h->dlists_ok = false;
  CK(cudaStreamSynchronize(h->s));
  CK(cudaGetLastError());
  return SPH_OK;
}

int sph_get_counters(sph_handle* h, int64_t* out, int n) {
  if (!h || !out) return fail(SPH_ERR_ARG, "null argument");
  unsigned long long d[DC_TOTAL];
  CK(cudaMemcpyAsync(d, h->dcnt.p, sizeof(d), cudaMemcpyDeviceToHost, h->s));
  CK(cudaStreamSynchronize(h->s));
  int64_t all[SPH_CNT_TOTAL];
  for (int k = 0; k < SPH_CNT_TOTAL; ++k) all[k] = h->cnt_host[k];
  all[SPH_CNT_NEIB_PAIRS] = int64_t(d[DC_NEIB_PAIRS]) + h->kept_pairs;
  all[SPH_CNT_C1_PAIRS] = int64_t(d[DC_C1_PAIRS]);
  all[SPH_CNT_C1_SWEEPS] = std::max<int64_t>(int64_t(d[DC_C1_MAXSWEEPS]), h->host_max_sweeps);
  all[SPH_CNT_C2_PAIRS] = int64_t(d[DC_C2_PAIRS]);
  all[SPH_CNT_CANDIDATES] = int64_t(d[DC_CANDIDATES]);
  all[SPH_CNT_C1_CENTRE_SWEEPS] = int64_t(d[DC_C1_CENTRE_SWEEPS]);
  all[SPH_CNT_LAUNCHES] = int64_t(launches_so_far() - h->launch_base);
  all[SPH_CNT_EXACT_TESTS] = int64_t(d[DC_EXACT_TESTS]);
  all[SPH_CNT_SEARCHES] += int64_t(d[DC_SEARCHES]);
  all[SPH_CNT_SKIN_BUILDS] += int64_t(d[DC_SKIN_BUILDS]);
  all[SPH_CNT_SKIN_REUSES] += int64_t(d[DC_SKIN_REUSES]);
  for (int k = 0; k < n && k < SPH_CNT_TOTAL; ++k) out[k] = all[k];
  return SPH_OK;
}

int sph_reset_counters(sph_handle* h) {
  if (!h) return fail(SPH_ERR_ARG, "null argument");
  CK(cudaMemsetAsync(h->dcnt.p, 0, sizeof(unsigned long long) * DC_TOTAL, h->s));
  CK(cudaStreamSynchronize(h->s));
  for (auto& c : h->cnt_host) c = 0;
  for (auto& t : h->timers) t = 0.;
  h->kept_pairs = 0;
  h->host_max_sweeps = 0;
  h->launch_base = launches_so_far();
  return SPH_OK;
}

int sph_get_timers(sph_handle* h, double* out_ms, int n) {
  if (!h || !out_ms) return fail(SPH_ERR_ARG, "null argument");
  h->collect_timers();
  for (int k = 0; k < n && k < SPH_T_TOTAL; ++k) out_ms[k] = h->timers[k];
  return SPH_OK;
}

int sph_errcalc(sph_handle* h, double* err_out, int64_t cap, double* l1_out) {
  AllocScope alloc_scope(h);
  if (!h) return fail(SPH_ERR_ARG, "null handle");
  return h->errcalc(err_out, cap, l1_out);
}

int sph_adjoint_forward(sph_handle* h, int nsteps, int every) {
  AllocScope alloc_scope(h);
  if (!h) return fail(SPH_ERR_ARG, "null handle");
  int rc = h->adjoint_forward(nsteps, every);
  h->collect_timers();
  return rc;
}

int sph_adjoint_backward(sph_handle* h, const double* dl_dv, const double* dl_du,
                         const double* dl_dr, double* g_r0, double* g_v0, double* g_u0,
                         double* g_par) {
  AllocScope alloc_scope(h);
  if (!h) return fail(SPH_ERR_ARG, "null handle");
  int rc = h->adjoint_backward(dl_dv, dl_du, dl_dr, g_r0, g_v0, g_u0, g_par);
  h->collect_timers();
  return rc;
}

int sph_adjoint_backward_diffusion(sph_handle* h, const double* dl_dT, double* g_T0,
                                   double* g_difcond) {
  AllocScope alloc_scope(h);
  if (!h) return fail(SPH_ERR_ARG, "null handle");
  if (!h->adj_diff) return fail(SPH_ERR_STATE, "adjoint: the recorded forward run is not a diffusion run");
  double g[3] = {0, 0, 0};
  int rc = h->adjoint_backward(nullptr, nullptr, nullptr, nullptr, nullptr, nullptr, g, dl_dT,
                               g_T0, 3);
  if (g_difcond) *g_difcond = g[2];
  h->collect_timers();
  return rc;
}

void sph_destroy(sph_handle* h) {
  if (!h) return;
  h->destroy();
  delete h;
}

}  // extern "C"

namespace sph {
int handle_device(const sph_handle* h) { return h->dev; }

int start_for_device_loop(sph_handle* h) {
  if (!h) return sph_fail(SPH_ERR_ARG, "null handle");
  if (h->started) return sph_step(h, 0);
  h->skin_suspended = true;
  const int rc = sph_step(h, 0);
  h->skin_suspended = false;
  return rc;
}
}  // namespace sph
