// sph_internal.h — host-side declarations shared by the engine's translation
// units: device buffers of one handle, the cell grid and the kernel launchers.
#pragma once

#include <cstdint>
#include <string>
#include <vector>
#include <cuda_runtime.h>

#include "sph_device.cuh"

namespace sph {

// Uniform cell grid over all particles (reals, fixed, periodic images).
struct Grid {
  double ox, oy, oz;  // origin (lower corner)
  double L, invL;     // cell edge
  int nx, ny, nz;     // cells per axis
};

// Order-preserving uint64 image of a double, for atomicMin/atomicMax.
__host__ __device__ inline unsigned long long dkey(double v) {
  long long b;
#ifdef __CUDA_ARCH__
  b = __double_as_longlong(v);
#else
  static_assert(sizeof(double) == sizeof(long long), "");
  __builtin_memcpy(&b, &v, sizeof(b));
#endif
  unsigned long long u = (unsigned long long)b;
  return (b >= 0) ? (u | 0x8000000000000000ull) : ~u;
}
__host__ __device__ inline double dkey_inv(unsigned long long u) {
  unsigned long long b = (u & 0x8000000000000000ull) ? (u & 0x7fffffffffffffffull) : ~u;
  double v;
#ifdef __CUDA_ARCH__
  v = __longlong_as_double((long long)b);
#else
  __builtin_memcpy(&v, &b, sizeof(v));
#endif
  return v;
}

// Cells per axis of a uniform grid, n3[k] = floor(e[k]) + 1 with e[k] the
// extent of axis k in cell edges, and their product *ncell.  False when an
// axis would need 1e9 cells or more, or when the product exceeds cap.  The
// product is checked against cap one axis at a time (n > cap / n3 before
// multiplying), so it never overflows: three axes just under 1e9 cells would
// otherwise multiply past 2^63 and wrap to a value that may pass the test.
__host__ __device__ inline bool grid_dims(const double e[3], int64_t cap, int n3[3],
                                          int64_t* ncell) {
  int64_t n = 1;
  for (int k = 0; k < 3; ++k) {
    if (!(e[k] < 1e9) || !(e[k] >= 0.0)) return false;
    n3[k] = int(floor(e[k])) + 1;
    if (n > cap / n3[k]) return false;
    n *= n3[k];
  }
  *ncell = n;
  return true;
}

// Reduction slots (unsigned long long, dkey-encoded min/max).
enum RedSlot : int {
  RED_LO_X = 0, RED_LO_Y, RED_LO_Z, RED_HI_X, RED_HI_Y, RED_HI_Z, RED_HMIN,
  RED_TS_HMIN, RED_TS_CMAX, RED_TS_DENMIN, RED_TS_CMIN, RED_TS_KAPMAX,
  RED_TS_BMAX, RED_TS_KAPMIN, RED_TS_LAMMAX, RED_C1_ACTIVE, RED_C1_ACTIVE2,
  // skin lists: largest displacement and h (dkey max), image signature
  // changed (0/1), records that moved more than tau and eps (plain counts)
  RED_SKIN_D, RED_SKIN_HMAX, RED_SKIN_SIG, RED_SKIN_NFAST, RED_SKIN_NMOVE,
  RED_SKIN_NKEPT,   // rows a skin-list iterate keeps (plain count)
  RED_SKIN_NKEPT_PAIRS,  // their neighbours (plain count)
  RED_SKIN_HMAXB,   // largest h of the centres at the skin search (dkey max)
  RED_DSKIN_FAIL,   // device-resident lists: a centre whose row cannot be filtered (0/1)
  RED_TOTAL
};

// Device counters (unsigned long long, cumulative).
enum DevCnt : int {
  DC_NEIB_PAIRS = 0, DC_C1_PAIRS, DC_C2_PAIRS, DC_CANDIDATES,
  DC_C1_CENTRE_SWEEPS, DC_C1_MAXSWEEPS, DC_EXACT_TESTS,
  // the device-resident step's searches, skin-list builds and iterates served
  DC_SEARCHES, DC_SKIN_BUILDS, DC_SKIN_REUSES, DC_TOTAL
};

// Periodic geometry for the image builder (BC.f90:46-68, 196-475).
struct BoxGeom {
  double emin[3], emax[3];
  double boxmin[3], boxmax[3];
  double pmin[3], pmax[3];
  int periodic[3];  // axes that get periodic images
  int reflect[3];   // axes whose real particles are wrapped
};

// A batch's device loop (sph_engine.cu): step the instances to tfinish
// (use_state: each instance's own tfinish), at most `limit` steps each, as
// one CUDA graph per launch; per-instance codes and messages in status /
// msg.  *used = false when some instance cannot take device-resident steps
// (nothing stepped; the caller runs host workers instead).
struct BatchGraph;
int batch_graph_run(BatchGraph** bg, sph_handle* const* hs, int n, double tfinish,
                    bool use_state, long long limit, std::vector<int>& status,
                    std::vector<std::string>& msg, bool* used);
void batch_graph_destroy(BatchGraph* bg);

// Record an error message for sph_last_error and return `code`.
int sph_fail(int code, const std::string& msg);
// The device a handle was created on.
int handle_device(const sph_handle* h);
// sph_step(h, 0) for an instance about to join the batch device loop: its
// start-up iterate (if it has not run) builds no skin lists, which the
// loop's fresh searches would drop unused.
int start_for_device_loop(sph_handle* h);

// Count of this library's kernel launches (process-wide).
void note_launch(int n = 1);
long long launches_so_far();

// ---- launchers (sph_grid.cu) -----------------------------------------------------
void launch_upload_store(const double* rowmajor, double* cols, int32_t* orig, int64_t n,
                         cudaStream_t s);
void launch_download_store(const double* cols, const int32_t* orig, double* rowmajor,
                           int64_t n, cudaStream_t s);
// the same for rows a .. b - 1 only (a a multiple of 32), so that a table
// crosses PCIe in pieces while the next piece is transposed: upload rows
// in caller order (orig[i] = i); download caller rows through inv, the
// inverse of orig
void launch_upload_rows(const double* rowmajor, double* cols, int32_t* orig, int64_t n, int64_t a,
                        int64_t b, cudaStream_t s);
void launch_download_rows(const double* cols, const int32_t* inv, double* rowmajor, int64_t n,
                          int64_t a, int64_t b, cudaStream_t s);
void launch_reorder(const double* cols_in, double* cols_out, const int32_t* orig_in,
                    int32_t* orig_out, const int32_t* perm, int64_t n, int64_t ld_in,
                    int64_t ld_out, cudaStream_t s);
void launch_reflect(double* cols, int64_t ld, int64_t nreal, BoxGeom g, cudaStream_t s);
void launch_ghost_count(const double* cols, int64_t nrows, int64_t nreal, BoxGeom g,
                        int dim, int32_t* count, unsigned long long* red, cudaStream_t s);
void launch_ghost_write(const double* cols, int64_t nrows, BoxGeom g, int dim,
                        const int32_t* offset, double* gx, double* gy, double* gz,
                        int32_t* gsrc, int8_t* gcode, unsigned long long* red, cudaStream_t s);
void launch_keys(const double* cols, int64_t nrows, const double* gx, const double* gy,
                 const double* gz, int64_t nghost, Grid g, uint32_t* keys, int32_t* vals,
                 cudaStream_t s);
void launch_cell_starts(const uint32_t* keys, int64_t n, int64_t ncell, int32_t* cstart,
                        cudaStream_t s);
struct PackGeom {
  double ox, oy, oz;  // origin subtracted before the binade shift
  double shift;       // 2^E with every (x - origin) in [0, 2^E)
  double mref;        // mass scale (packed m = m / mref)
};
// ---- device-resident step (no host round trip inside a step) ----
// What the host computes between the image count and the sort in the
// classic step, computed by k_plan on the device instead: the image count,
// the cell grid, the FP32 packing frame and the padding key of the
// capacity-sized sort.  err is 0 or an SPH_ERR_* code (SPH_ERR_STATE for a
// capacity that was too small: the step is then redone on the host path).
struct DevPlan {
  int64_t nghost, nall, ncell;
  Grid grid;
  PackGeom pg;
  uint32_t pad_key;
  int err;
};
// Skin lists of the device-resident step (device memory, one per handle).
// Every iterate either serves every centre's row from its skin list (the
// FP64 predicate over the list) or searches afresh; no host decision.
struct DevSkin {
  int live;             // the lists describe the records of the current sort
  int age;              // iterates served since their search
  int pause, pause_len; // plain searches left, length of the last pause
  double kfac;          // radius factor of this iterate's search (1 + s, or 1 in a pause)
  double kfac_b;        // that of the lists' search
  double hmin_b;        // smallest h at that search
};
// the time-loop state of main.f90:241-373 on the device
struct DevClock {
  double t, ltout, dtout, tfinish, dt;
  int stopped;
};
struct PlanIn {
  int64_t nrows, nghost_cap, nall_cap;
  double krad, cf, mref;
  int end_bit_cap;
};
void launch_plan(const unsigned long long* red, const int32_t* nghost_dev, PlanIn in,
                 DevPlan* plan, int* err_out, cudaStream_t s);
// err := code (first error wins) if *v != 0
void launch_flag_if_nonzero(const unsigned long long* v, int* err, int code, cudaStream_t s);
// the device-resident Newton sweeps as a while node: *iter = 0 and the
// handle set before it; after each sweep ++*iter, and the loop goes on while
// a particle stays active and *iter < sweeps (err := SPH_ERR_STATE when one
// is still active after the last of fewer than maxiter sweeps: the host
// loop would sweep on)
void launch_sweeps_init(int* iter, cudaGraphConditionalHandle h, cudaStream_t s);
void launch_sweeps_ctl(int* iter, const unsigned long long* active, int sweeps, int maxiter,
                       int* err, cudaGraphConditionalHandle h, cudaStream_t s);
struct DtIn {
  int eq_hydro, eq_magneto, eq_diff, eq_fld, sts_fixed, sts_s;
  double cn_hydro, cnd2;
};
void launch_dt(const unsigned long long* red, DtIn in, DevClock* clk, double* ctrl, cudaStream_t s);
void launch_clock_advance(DevClock* clk, cudaStream_t s);

// ---- selected columns of the table in caller row order ----
struct ColumnSet {
  int n;
  int f[SPH_ES_TOTAL];  // 0-based store columns
};
void launch_get_columns(const double* cols, int64_t ld, const int32_t* orig, int64_t nrows,
                        ColumnSet fs, double* out, cudaStream_t s);
void launch_set_columns(double* cols, int64_t ld, const int32_t* orig, int64_t nrows,
                        ColumnSet fs, const double* in, cudaStream_t s);

// ---- batches stepped by one device loop (a CUDA graph with a while node) ----
// One record per instance of a batch, in device memory.  The loop's gate
// kernel decides which instances step in an iteration (their if nodes);
// each instance's step begins by deciding its row reorder and ends by
// checking its error words.
struct BatchInst {
  const DevClock* clk;    // the instance's device clock
  int running;            // this iteration steps the instance
  int failed;             // a step set an error word: the host redoes it
  int every, since;       // row-reorder period, steps since the last reorder
  int reorder;            // the current step reorders the rows first
  int since_before;       // `since` before the current step
  long long steps, limit; // steps completed in the loop, the most it may take
};
// t < tfinish + eps and not stopped (the time loop's condition), for an
// instance that has not failed and has steps left
void launch_batch_gate(BatchInst* bi, int n, const cudaGraphConditionalHandle* ifh,
                       cudaStream_t s);
// after every instance of an iteration: continue while some instance runs,
// none failed and fewer than cap iterations ran in this launch
void launch_batch_ctl(const BatchInst* bi, int n, cudaGraphConditionalHandle wh, int* iter,
                      int cap, cudaStream_t s);
void launch_inst_begin(BatchInst* b, const DevClock* clk, DevClock* clk_save, cudaStream_t s);
void launch_inst_end(BatchInst* b, const int* err, const int32_t* overflow, const int* status,
                     cudaStream_t s);
// the rows in the order of the last search (real rows by centre_p, then the
// fixed rows as they are) when b->reorder is set: gathered into the spare
// table, then copied back, so the table keeps its address
void launch_reorder_gated(const BatchInst* b, double* cols, double* cols_alt, int32_t* orig,
                          int32_t* orig_alt, const int32_t* centre_p, int64_t nreal,
                          int64_t nrows, DevSkin* ds, cudaStream_t s);
void launch_keys_dev(const double* cols, int64_t nrows, const double* gx, const double* gy,
                     const double* gz, const DevPlan* plan, int64_t ncap, uint32_t* keys,
                     int32_t* vals, cudaStream_t s);
void launch_cell_starts_dev(const uint32_t* keys, int64_t ncap, const DevPlan* plan,
                            int32_t* cstart, cudaStream_t s);
void launch_sorted_gather_dev(const int32_t* sidx, int64_t ncap, int64_t nrows, int64_t nreal,
                              const double* cols, const double* gx, const double* gy,
                              const double* gz, const int32_t* gsrc, double* sx, double* sy,
                              double* sz, int32_t* ssrc, int32_t* centre_slot, float4* s32,
                              const DevPlan* plan, cudaStream_t s);
void launch_ghost_write_cap(const double* cols, int64_t nrows, BoxGeom g, int dim,
                            const int32_t* offset, int64_t cap, double* gx, double* gy,
                            double* gz, int32_t* gsrc, int8_t* gcode, cudaStream_t s);
void launch_sorted_gather(const int32_t* sidx, int64_t n, int64_t nrows, int64_t nreal,
                          const double* cols, const double* gx, const double* gy,
                          const double* gz, const int32_t* gsrc, double* sx, double* sy,
                          double* sz, int32_t* ssrc, int32_t* centre_slot, float4* s32,
                          PackGeom pg, cudaStream_t s);
void launch_centres(const int32_t* sidx, const int32_t* flag, const int32_t* pos, int64_t n,
                    int32_t* centre_k, int32_t* centre_p, cudaStream_t s);
struct NeibArgs {
  const DevPlan* plan;  // if set: grid and shift from the device plan
  int64_t nc;
  const int32_t* centre_k;
  const int32_t* centre_p;
  const double* sx;
  const double* sy;
  const double* sz;
  const float4* s32;
  double shift;
  const double* hcol;
  double krad;
  Grid g;
  const int32_t* cstart;
  const int64_t* rowoff;  // start of each centre's row in nl
  const int32_t* rowcap;  // slots of each row
  int64_t nl_size;
  int32_t* nl;
  int32_t* ncnt;
  const int32_t* orig;
  int32_t* count_prev;  // per original row: neighbours found by the last search
  float* h_prev;        // per original row: h of that search
  int32_t* maxcnt;
  int32_t* overflow;
  unsigned long long* dcnt;
  // optional: the centres to search are cmap[0 .. nc-1] (indices into
  // centre_k / centre_p / rowoff / rowcap / ncnt) instead of 0 .. nc-1
  const int32_t* cmap;
  // the predicate's radius is kfac * krad * h (0 or 1: krad * h), and the
  // cells searched reach `reach` further (records that moved since they
  // were sorted into their cells)
  double kfac;
  double reach;
  int skin_search;  // a skin search: its pairs are not the neighbour pairs counted
  const double* kfac_dev;  // if set: kfac read from the device (device-resident step)
};
// ---- skin lists (SPH_P_SKIN; sph_grid.cu) ----
// per row: the row's image signature (the periodic sides that hold it; its
// image set is a function of it), 0 for rows that get no images
void launch_skin_sig(const double* cols, int64_t nrows, BoxGeom g, int dim, uint8_t* sig,
                     cudaStream_t s);
// per record (sorted order) from the rows' current positions: sx/sy/sz and
// the FP32 images, the displacement since the skin search (FP64, rounded
// up, kept in dsp as the running maximum, FP32 rounded up) and the slots
// RED_LO_* / RED_HI_* (bounding box), RED_SKIN_D, RED_SKIN_HMAX (real
// rows), RED_SKIN_SIG (a row whose image signature differs from sig_b),
// RED_SKIN_NFAST (displacement > tau) and RED_SKIN_NMOVE (> eps)
// (device-resident step: with plan set, n and pg come from the plan (n the
// launch bound); with gate set, nothing is done unless gate->live)
void launch_skin_refresh(const int32_t* sidx, int64_t n, int64_t nrows, int64_t nreal,
                         const double* cols, const int32_t* gsrc, const int8_t* gcode,
                         BoxGeom g, int dim, const uint8_t* sig_b, const double* bx,
                         const double* by, const double* bz, double* sx, double* sy, double* sz,
                         float4* s32, PackGeom pg, float* dsp, float tau, float eps,
                         double* hrec, unsigned long long* red, cudaStream_t s,
                         const DevPlan* plan = nullptr, const DevSkin* gate = nullptr);
// with the lists live, per centre: can its row come from its skin list?
// Every record now within krad h of the centre was within krad h + 2 D at
// the lists' search (both moved at most D since), and the list holds all
// within kfac_b krad h_b; red[RED_DSKIN_FAIL] = 1 where that fails
void launch_dskin_check(int64_t nc, const int32_t* centre_p, const double* hcol, const double* hb,
                        double krad, const DevSkin* ds, unsigned long long* red, cudaStream_t s);
// the iterate's way: rows from the lists (hsearch = 0) or a search
// (hsearch = 1, radius factor ds->kfac: 1 + skin, or 1 for the plain
// searches of a pause after lists that served fewer than short_age iterates)
void launch_dskin_decide(DevSkin* ds, const unsigned long long* red, const DevPlan* plan,
                         double krad, double skin, int short_age, int pause0, int pause_max,
                         cudaGraphConditionalHandle hsearch, unsigned long long* dcnt,
                         cudaStream_t s);
// after the search: its lists are live when it was a skin search
void launch_dskin_built(DevSkin* ds, const unsigned long long* red, cudaStream_t s);
// The checks of a skin-list iterate on the refreshed records, on the
// device so that the iterate asks the host once: gate[0] = 0 when the
// lists may serve, else why not (1 an image set changed, 2 a record moved
// a search radius dcap, 3 h, 4 a record left the FP32 binade, 5 a window
// spans more than 256 cells); gate[1], gate[2] = the windows wf, wm of the
// marks in cells (0 when gate[0] != 0)
struct SkinGateIn {
  double dcap, krad, tau, kfac, invL;
  PackGeom pg;
};
void launch_skin_gate(const unsigned long long* red, SkinGateIn in, int* gate, cudaStream_t s);
// cell flags of the records that moved more than tau (fast_cell, by their
// position now) and eps (move_cell, may be NULL; by the cell they were
// sorted into), dilated by w[0] / w[1] cells per side along each of dim
// axes (w in device memory; tmp: a spare field of the cell count)
void launch_skin_marks(int64_t n, const float* dsp, float tau, float eps, const uint32_t* keys,
                       const double* sx, const double* sy, const double* sz, Grid g, int dim,
                       const int* w, uint8_t* fast_cell, uint8_t* move_cell, uint8_t* tmp,
                       cudaStream_t s);
// mode[c] = 0 (filter the skin list), 1 (search afresh) or 2 (keep the row)
// for every centre (see sph_grid.cu), near_f / near_m the dilated cell
// flags looked up by the cell keys[k] each centre's record was sorted into,
// h of the centres from hrec (per record); hdev[c] = running maximum of
// |h - hb[c]|.  The centres searched afresh go to dlist, those that filter
// to flist (in centre order); pos[nc] = their counts (low / high 32 bits);
// ways and pos hold nc + 1 entries.  nkept[0..1] += rows kept, their pairs.
void launch_skin_classify(int64_t nc, const int32_t* centre_k, const double* hrec,
                          const double* hb, double* hdev, const float* gap, double krad,
                          double kfac, float tau, float eps, const float* dsp,
                          const uint32_t* keys, const uint8_t* near_f, const uint8_t* near_m,
                          uint8_t* mode, int64_t* ways, int64_t* pos, int32_t* dlist,
                          int32_t* flist, void* scan_tmp, size_t scan_bytes,
                          const int32_t* ncnt, unsigned long long* nkept, cudaStream_t s);
// rows renamed under skin lists (old row perm[i] -> row i, inv[perm[i]] =
// i): sidx / ssrc / gsrc / centre_p renamed through inv, the rows' image
// signatures moved from sig_in to sig_out
void launch_rows_renamed(const int32_t* perm, const int32_t* inv, int64_t nall, int64_t nrows,
                         int64_t nghost, int64_t nreal, int32_t* sidx, int32_t* ssrc,
                         int32_t* gsrc, int32_t* centre_p, const uint8_t* sig_in,
                         uint8_t* sig_out, cudaStream_t s);
// q[p[i]] = i
void launch_inverse(const int32_t* p, int64_t n, int32_t* q, cudaStream_t s);
// *changed = 1 if some row's particle type differs from old_type[perm[row]]
void launch_type_changed(const double* cols, int64_t n, const double* old_type,
                         const int32_t* perm, int32_t* changed, cudaStream_t s);
// rows of the centres list[0 .. nd-1] laid out after *base: capacities
// from their last counts (as k_rowcap), their scan, rowoff / rowcap
void launch_dyn_rows(int64_t nd, const int32_t* list, const int32_t* centre_p,
                     const int32_t* orig, const int32_t* count_prev, const float* h_prev,
                     const double* hcol, int dim, int64_t* cap, int64_t* off, void* scan_tmp,
                     size_t scan_bytes, const int64_t* base, int64_t* rowoff, int32_t* rowcap,
                     cudaStream_t s);
// end[0] = rowoff[n - 1] + rowcap[n - 1]
void launch_table_end(const int64_t* rowoff, const int32_t* rowcap, int64_t n, int64_t* end,
                      cudaStream_t s);
// filter rows (mode 0) whose count exceeds their row become mode 1; dflag[c]
// = 1 for every centre of mode 1
void launch_overflow_to_search(int64_t nc, const int32_t* ncnt, const int64_t* rowoff,
                               const int32_t* rowcap, int64_t nl_size, uint8_t* mode,
                               int32_t* dflag, cudaStream_t s);
// search of the centres list[0 .. n-1], G lanes each (see sph_grid.cu)
struct FewArgs {
  int64_t n;
  const int32_t* list;
  const int32_t* centre_k;
  const int32_t* centre_p;
  const double* sx;
  const double* sy;
  const double* sz;
  const float4* s32;
  double shift;
  const double* hcol;
  double krad;
  Grid g;
  const int32_t* cstart;
  double reach;
  const int64_t* rowoff;
  const int32_t* rowcap;
  int64_t nl_size;
  int32_t* nl;
  int32_t* ncnt;
  const int32_t* orig;
  int32_t* count_prev;
  float* h_prev;
  int32_t* maxcnt;
  int32_t* overflow;
  unsigned long long* dcnt;
};
void launch_search_few(int dim, const FewArgs& a, cudaStream_t s);
// dlist[dpos[c]] = c for every c with dflag[c] != 0
void launch_skin_compact(int64_t nc, const int32_t* dflag, const int32_t* dpos, int32_t* dlist,
                         cudaStream_t s);
// hb[c] = hcol[centre_p[c]], and their maximum into red[slot] (dkey max)
void launch_gather_h(int64_t nc, const int32_t* centre_p, const double* hcol, double* hb,
                     unsigned long long* red, int slot, cudaStream_t s);
struct SkinFilterArgs {
  int64_t nc;           // centres (list == NULL) or list entries
  const int32_t* list;  // optional: the centres to filter
  const uint8_t* mode;  // 0: filter; 1: left to the search; 2: kept when keep != 0
                        // (NULL with list NULL: every centre filters)
  int keep;
  float* gap;           // optional: per centre, the smallest |r - krad h| of its list
  float eimg;           // error bound of a distance between two FP32 images
  const int32_t* centre_k;
  const int32_t* centre_p;
  const int64_t* skin_off;
  const int32_t* skin_cnt;
  const int32_t* skin_nl;
  const double* sx;
  const double* sy;
  const double* sz;
  const float4* s32;
  double shift;
  const double* hcol;
  double krad;
  const int64_t* rowoff;
  const int32_t* rowcap;
  int64_t nl_size;
  int32_t* nl;
  int32_t* ncnt;
  const int32_t* orig;
  int32_t* count_prev;
  float* h_prev;
  int32_t* maxcnt;
  int32_t* overflow;
  unsigned long long* dcnt;
  const DevPlan* plan;  // if set: shift from the device plan
  // if set: each skin row's slots (and skin_size the table's), to which the
  // entries read are clamped (a skin search that overflowed them is redone
  // on the host; its lists are never served)
  const int32_t* skin_cap;
  int64_t skin_size;
};
// each centre's neighbour row = its skin list's records that pass the FP64
// predicate ((dx*dx + dy*dy) + dz*dz) <= (krad*h)^2, in skin-list order
void launch_skin_filter(const SkinFilterArgs& a, cudaStream_t s);

// staged: the candidate runs of a chunk copied into shared memory by bulk
// copies (SPH_P_SEARCH_STAGED); overflow |= 2 if a copy's wait timed out
void launch_neighbours(int dim, int G, bool staged, const NeibArgs& a, cudaStream_t s);
// per centre in original order: out[2 o] = count, out[2 o + 1] = sum of
// mix64((row << 5) | image) over the neighbours (sph_get_neighbour_digest)
void launch_neib_digest(int64_t nc, const int32_t* centre_p, const int32_t* orig,
                        const int64_t* rowoff, const int32_t* ncnt, const int32_t* nl,
                        const int32_t* sidx, const int32_t* ssrc, const int8_t* gcode,
                        int64_t nrows, unsigned long long* out, cudaStream_t s);
void launch_rowcap(int64_t nc, const int32_t* centre_p, const int32_t* orig,
                   const int32_t* count_prev, const float* h_prev, const double* hcol,
                   int dim, float slack, int64_t* rowcap64, int32_t* rowcap,
                   cudaStream_t s);
size_t scan64_temp_bytes(int64_t n);
void exclusive_scan64(void* tmp, size_t tmp_bytes, const int64_t* in, int64_t* out, int64_t n,
                      cudaStream_t s);
// pack groups
// (PACK_TEMP: with PACK_POS, also the temperature stream the circuit1
// sweeps of the diffusion paths read)
enum PackGroup : int { PACK_POS = 1, PACK_HYDRO = 2, PACK_EXTRA = 4, PACK_TEMP = 8 };
struct PackBufs {
  double2* p[11];
  // FP32: q[0] = (x, y, z high parts, m), q[1] = (x, y, z low parts, 1/h),
  // q[2] = (rho / 2, wCv / (h^(d+1) rho^2 Omega), P, alpha c), q[3] = (au u, v), q[4] / q[5] the
  // temperature, diffusion and field quantities (the force pass); q[6] =
  // (x, y, z as 31-bit fixed point over the packing frame, m) (the density
  // pass: one 16-byte record per neighbour)
  float4* q[7];
  // the length of one fixed-point unit (shift 2^-31), written by the pack
  // kernel (the frame may be planned on the device)
  float* unit;
  // the force pass's FP32 factor wCv / h^(d+1), the viscosity's alpha and
  // the conductivity's au (set before its packing)
  double kp_wcv = 0.0, kp_alpha = 0.0, kp_au = 0.0;
  int kp_dim = 0;
};
void launch_pack_dev(int prec, int groups, int64_t ncap, const int32_t* ssrc, const double* sx,
                     const double* sy, const double* sz, const double* cols, int64_t ld,
                     const DevPlan* plan, PackBufs pb, cudaStream_t s);
void launch_pack(int prec, int groups, int64_t n, const int32_t* ssrc, const double* sx,
                 const double* sy, const double* sz, const double* cols, int64_t ld,
                 PackGeom pg, PackBufs pb, cudaStream_t s);
// leapfrog predictor / corrector; mode: LF_STS (the STS integrator moves T),
// LF_NO_B (no equation changes B), LF_NO_T (none changes T)
enum LeapfrogMode : int { LF_STS = 1, LF_NO_B = 2, LF_NO_T = 4 };
void launch_predict(double* cols, int64_t ld, const int32_t* orig, int64_t nrows,
                    int64_t n_int, double* save, const double* ctrl, int mode,
                    cudaStream_t s);
void launch_correct(double* cols, int64_t ld, const int32_t* orig, int64_t nrows,
                    int64_t n_int, const double* save, const double* ctrl, int mode,
                    cudaStream_t s);
void launch_timestep_reduce(const double* cols, int64_t ld, const int32_t* orig,
                            int64_t nrows, int64_t n_ts, Params P,
                            unsigned long long* red, cudaStream_t s);
void launch_fill_u64(unsigned long long* p, int n, unsigned long long v, cudaStream_t s);
// radiation - gas exchange after the corrector (rad_exchange.f90:9-118)
void launch_radexch(double* cols, int64_t ld, const int32_t* orig, int64_t nrows, int64_t n_int,
                    double dt, double gamma, double gmw, int* status, cudaStream_t s);
// up to 8 single reduction slots set in one launch: p[off[i]] = val[i]
struct SlotInit {
  int n;
  int off[12];
  unsigned long long val[12];
};
void launch_init_slots(unsigned long long* p, const SlotInit& in, cudaStream_t s);
void launch_fill_i32(int32_t* p, int64_t n, int32_t v, cudaStream_t s);
void launch_sts_stage(int kind, double* cols, int64_t ld, int64_t n, double* Y, double a0,
                      double a1, double a2, double a3, double a4, const double* ctrl,
                      cudaStream_t s);
// the device-resident step's stages j = 2 .. s as a while node: stage j
// (kind 2) with its coefficients coef[4 (j - 2) + 0..3] (mu, nu, muhat,
// gmhat) for j = *jdev; sts_loop_init sets *jdev = 2 and the handle (2 <= s),
// sts_loop_ctl advances j and sets it again (j <= s)
void launch_sts_stage_dev(double* cols, int64_t ld, int64_t n, double* Y, const double* coef,
                          const int* jdev, const double* ctrl, cudaStream_t s);
void launch_sts_loop_init(int* jdev, int sts_s, cudaGraphConditionalHandle h, cudaStream_t s);
void launch_sts_loop_ctl(int* jdev, int sts_s, cudaGraphConditionalHandle h, cudaStream_t s);
void launch_eos(double* cols, int64_t ld, int64_t nreal, Params P, cudaStream_t s);
void launch_apply_mti(double* cols, int64_t ld, const int32_t* orig, int64_t nrows,
                      int64_t nreal, int lowres, cudaStream_t s);
void launch_set_col(double* col, int64_t n, double v, cudaStream_t s);

// CUB wrappers (sph_grid.cu)
// Counting sort of the records by cell (keys in [0, ncell)): vout / kout the
// record indices and keys in key order, each cell's records in increasing
// index (as a stable sort), cstart[0 .. ncell] the cells' starts; count
// (ncell + 1) and big (ncell) are scratch, ctr two device ints, h_ctr a
// pinned host int; scan_tmp sized for ncell + 1 entries.  Returns false
// (nothing written) when a cell holds more than 4096 records.
bool cell_sort(const uint32_t* keys, int64_t n, int64_t ncell, int32_t* count, int32_t* cstart,
               int32_t* vout, uint32_t* kout, int32_t* big, int32_t* ctr, void* scan_tmp,
               size_t scan_bytes, int32_t* h_ctr, cudaStream_t s);
size_t sort_temp_bytes(int64_t n);
void sort_pairs(void* tmp, size_t tmp_bytes, const uint32_t* kin, uint32_t* kout,
                const int32_t* vin, int32_t* vout, int64_t n, int end_bit, cudaStream_t s);
size_t scan_temp_bytes(int64_t n);
void exclusive_scan(void* tmp, size_t tmp_bytes, const int32_t* in, int32_t* out, int64_t n,
                    cudaStream_t s);

// ---- circuit1 (sph_circuit1.cu) ---------------------------------------------------
struct C1Args {
  int64_t nc;
  const int64_t* rowoff;  // start of each centre's neighbour row in nl
  int G;                  // lanes per centre
  const int32_t* centre_k;
  const int32_t* centre_p;
  const int32_t* nl;
  const int32_t* ncnt;
  double* cols;
  int64_t ld;
  // Jacobi-sweep path
  const double* hk_s;  // snapshots in sorted order
  const double* dk_s;
  const double* ok_s;
  double* hkp1;
  double* dkp1;
  double* okp1;
  double* eps;
  int simple;  // c1simple
  double mref;
  int* status;
  unsigned long long* dcnt;
  unsigned long long* red;
  int active_slot;                  // red slot the sweep marks when a particle stays active
  const unsigned long long* gate;   // if set and zero, the sweep has nothing to do
  int first;                        // the iterate's first sweep
  const int* iter_dev;              // if set: the first sweep is the one where *iter_dev == 0
};
void launch_c1_newton(int prec, int kernel, int dim, const C1Args& a, PackBufs pb, Params P,
                      cudaStream_t s);
void launch_c1_sweep(int prec, int kernel, int dim, const C1Args& a, PackBufs pb, Params P,
                     cudaStream_t s);
void launch_c1_finalize(int64_t nrows, int64_t nreal, double* cols, int64_t ld, const double* hkp1,
                        const double* dkp1, const double* okp1, int simple, Params P,
                        cudaStream_t s);
void launch_c1_snapshot(int64_t n, const int32_t* ssrc, const double* hkp1,
                        const double* dkp1, const double* okp1, double* hk_s, double* dk_s,
                        double* ok_s, cudaStream_t s, const DevPlan* plan = nullptr,
                        const unsigned long long* gate = nullptr);

// ---- circuit2 (sph_circuit2.cu) ---------------------------------------------------
struct C2Args {
  int64_t nc;
  const int64_t* rowoff;
  int G;
  const int32_t* centre_k;
  const int32_t* centre_p;
  const int32_t* nl;
  const int32_t* ncnt;
  double* cols;
  int64_t ld;
  double mref;
  int* status;
  unsigned long long* dcnt;
};
void launch_c2(int prec, int kernel, int dim, const C2Args& a, PackBufs pb, Params P,
               cudaStream_t s);

// ---- adjoint of the hydro step (sph_adjoint.cu) ----
// columns of the per-row adjoint buffer (ld = rows of the particle table):
// state adjoints LR (r), LV (v), LU (u), LAS (a), LDUS (du); the adjoints
// LA, LDU of the new a, du fed to the force VJP; its results GR, GV (r', v'),
// GH, GRHO, GOM, GP, GC, GU (h, rho, Omega, P, c, u); S' (d2 rho^/dh2) and
// the Newton-h coefficients MU, WC.  The diffusion adjoint adds LT (T),
// LDTS (the stored dT/dt), LDT (the new dT/dt fed to its VJP) and GT (T').
enum AdjCol : int {
  AJ_LR = 0, AJ_LV = 3, AJ_LU = 6, AJ_LAS = 7, AJ_LDUS = 10, AJ_LA = 11, AJ_LDU = 14,
  AJ_GR = 15, AJ_GV = 18, AJ_GH = 21, AJ_GRHO = 22, AJ_GOM = 23, AJ_GP = 24, AJ_GC = 25,
  AJ_GU = 26, AJ_SP = 27, AJ_MU = 28, AJ_WC = 29, AJ_LT = 30, AJ_LDTS = 31, AJ_LDT = 32,
  AJ_GT = 33, AJ_TOTAL = 34
};
struct AdjArgs {
  int64_t nc, nreal;
  const int32_t* centre_k;
  const int32_t* centre_p;
  const int32_t* nl;
  const int64_t* rowoff;
  const int32_t* ncnt;
  const int32_t* ssrc;
  const double* sx;
  const double* sy;
  const double* sz;
  const double* cols;
  int64_t ld;
  double* adj;   // AJ_TOTAL columns of ld rows
  double* gpar;  // d/d alpha, d/d beta, d/d difcond
  double wcv, alpha, beta, gamma;
  int artts, hydro;
  // the diffusion adjoint (diff = 1): equations = diffusion with fixed
  // positions, second-derivative method fab / fw / n2w
  int diff, ddw, difiso, full_tensor;
  double difcond, fwc;
};
// one step's adjoint: prep, force VJP (circuit2, Newton-h density, EOS) and
// the integrator's adjoint; first = 1 for the force evaluation of the
// initial state (no integrator step)
void launch_adj_step(int kernel, int dim, int G, const AdjArgs& a, double dt, int first,
                     cudaStream_t s);
// caller-order rows (ncomp per row) to ncomp columns of ld physical rows, and back
void launch_adj_gather(const double* in, int ncomp, const int32_t* orig, int64_t n, double* out,
                       int64_t ld, cudaStream_t s);
void launch_adj_scatter(const double* in, int64_t ld, const int32_t* orig, int64_t n,
                        double* out, int ncomp, cudaStream_t s);

// ---- end-of-run error calculators (errcalc.f90, main.f90:374-402) ---------
enum ErrKind : int { EK_ZERO = 0, EK_SHOCK12, EK_RING, EK_PULSE, EK_SOUNDWAVE,
                     EK_HYDROSHOCK, EK_ALFVEN };
// Exact solution of a 1-D Riemann problem: the star state and the wave
// speeds, solved once on the host; sampled per particle on the device.
struct RiemannFan {
  double gamma, x0;
  double rl, ul, pl, cl, rr, ur, pr, cr;
  double ps, us, rsl, rsr;  // star pressure, velocity, densities left / right of the contact
  int shock_l, shock_r;     // 1: shock, 0: rarefaction
  double sl, sr;            // shock speeds
  double hl, tl, hr, tr;    // rarefaction head / tail speeds
};
RiemannFan riemann_fan(double gamma, double rl, double ul, double pl, double rr, double ur,
                       double pr, double x0);
struct ErrCalcIn {
  int kind, dim, diso;
  double t;
  double pifac, ekt, ektd2, ektsq, epsdm1;  // pulse constants (errcalc.f90:66-71)
  RiemannFan fan;                           // hydroshock (errcalc.f90:38)
};
// err[orig[i]] for the real rows (orig < nreal) of the table; sum of err
// over [0, nreal) in a fixed order into *sum (part: scratch of
// errcalc_parts(nreal) doubles)
int64_t errcalc_parts(int64_t nreal);
void launch_errcalc(const double* cols, int64_t ld, const int32_t* orig, int64_t nrows,
                    int64_t nreal, const ErrCalcIn& in, double* err, double* part, double* sum,
                    cudaStream_t s);

}  // namespace sph
