/*
 * sph_abi.h — C-ABI of the B200 SPH step engine (libsph.so).
 *
 * This is the drop-in boundary that replaces the reference's process
 * boundary: the Python driver used to spawn `./execute` and exchange state
 * through `output/dump_full.h5` (playground/runner/fortdriver/core.py:152-169,
 * 321-326, 465-470).  Here the driver keeps the same two arrays in memory and
 * hands them to the engine through plain pointers:
 *
 *   state[49]  : FP64 state vector, slot k-1 holds statevars(k)
 *                (playground/src/state.f90:36, enum in const.f90:14-66)
 *   store[N*32]: FP64 particle table, row-major, one row of 32 fields per
 *                particle (the Fortran store(32,N) seen from C / h5py as
 *                (N,32); field map const.f90:69-103).  Rows are the real
 *                particles followed by the fixed ones (dumper.f90:33-34).
 *
 * Conventions
 *  - every entry point returns an int status: 0 = ok, >0 = one of SPH_ERR_*,
 *    each mirroring an abort site of the reference (`error stop` / `stop`);
 *  - buffers are caller-owned; a handle owns its device memory and one CUDA
 *    stream; a handle is not thread-safe; no C++ exception crosses the ABI;
 *  - there is no CPU fallback: if no CUDA device is usable, sph_create
 *    returns SPH_ERR_CUDA.
 */
#ifndef SPH_ABI_H
#define SPH_ABI_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ---- sizes of the interchange arrays (const.f90:66, :102) ---------------- */
#define SPH_EC_TOTAL 49
#define SPH_ES_TOTAL 32

/* ---- kernel choice: the reference picks it at compile time with
 *      `make kernel=<k>` (playground/Makefile:14,84-86); here it is a
 *      run-time argument of sph_create. ------------------------------------ */
#define SPH_KERNEL_M4    0   /* kernel/base_m4.f90    */
#define SPH_KERNEL_M6    1   /* kernel/base_m6.f90    */
#define SPH_KERNEL_GAUSS 2   /* kernel/base_gauss.f90 */

/* ---- precision of the pair arithmetic ------------------------------------ */
#define SPH_PREC_FP64      0 /* plain FP64 everywhere (parity mode)          */
#define SPH_PREC_FP32_COMP 1 /* FP32 pair sums, two-sum compensated; FP64
                                Newton h/Omega update, integrator, dt         */

/* ---- parameters beyond the 49 state slots (sph_set_param index) ---------
 * Indices 1..49 address statevars(k) exactly as setStateVal does
 * (state.f90:47-52).  The following extra slots hold values that the
 * reference hard-codes; their defaults reproduce it. */
#define SPH_P_AV_ALPHA        50 /* circuit2.f90:565, default 1              */
#define SPH_P_AV_BETA         51 /* circuit2.f90:566, default 2              */
#define SPH_P_NEWTON_TOL      52 /* circuit1.f90:104, default 1e-8           */
#define SPH_P_NEWTON_MAXITER  53 /* circuit1.f90:114, default 100            */
#define SPH_P_FULL_TENSOR     54 /* 0: diagonal K (circuit2.f90:203-205,371-373),
                                    1: full k_par * b b^T (new)              */
#define SPH_P_NEIB_CAP_CHECK  55 /* 1: abort like neighboursearch.f90:127-131
                                    when n_i+1 > maxneibnum; default 0       */
#define SPH_P_CELL_FACTOR     56 /* cell edge / (krad*h_min), default 0.5    */
#define SPH_P_REORDER_EVERY   57 /* physical re-sort interval in steps (8)   */
#define SPH_P_TIMING          58 /* 1: CUDA-event times per phase and per
                                       call (sph_get_timers); 2: per call only */
#define SPH_P_NEIB_CAP        59 /* neighbour slots per centre (0 = auto)    */
#define SPH_P_LANES_SEARCH    60 /* lanes per centre in the neighbour search
                                    (4, 8, 16, 32; 0 = auto)                  */
#define SPH_P_LANES_PAIR      61 /* lanes per centre in circuit1/circuit2     */
#define SPH_P_FIXED_DT        62 /* dt of sph_adjoint_forward's steps (> 0)   */
#define SPH_P_GRAPH           63 /* 1: sph_step / sph_run_to run each step as a
                                      replayed CUDA graph with no host round trip
                                      inside (a step that cannot be planned on
                                      the device is redone on the host path)   */
#define SPH_P_SEARCH_STAGED   64 /* 1: the neighbour search copies each chunk's
                                      candidate runs into shared memory with
                                      bulk (TMA) copies instead of fetching
                                      them per batch (default 0)               */
#define SPH_P_SKIN            65 /* s in (0, 1]: neighbour lists kept between
                                      iterates as skin lists of radius
                                      (1 + s) krad h; every iterate a centre
                                      keeps its row (nothing near it moved),
                                      refilters its skin list with the FP64
                                      predicate, or (near a fast particle) is
                                      searched afresh, so the sets equal a
                                      fresh search's; the lists are rebuilt
                                      when particles moved too far.  0 = a
                                      fresh search every iterate.  Default 0.1.
                                      (The device-resident steps of SPH_P_GRAPH
                                      and the batch loop keep or rebuild all
                                      lists at once, decided on the device.)   */
#define SPH_P_LAST            65

/* ---- status codes --------------------------------------------------------- */
#define SPH_OK                     0
#define SPH_ERR_ARG                1  /* bad argument / null pointer          */
#define SPH_ERR_CUDA               2  /* CUDA runtime error / no device       */
#define SPH_ERR_Q_NAN              3  /* base_m6.f90:49-50 'q is nan'         */
#define SPH_ERR_Q_NEG              4  /* base_m6.f90:51-52 'q is negative'    */
#define SPH_ERR_H_NEG              5  /* circuit1.f90:202-204                 */
#define SPH_ERR_NEIB_OVERFLOW      6  /* neighboursearch.f90:127-131          */
#define SPH_ERR_IC_DENSITY         7  /* preruncheck.f90:39-42                */
#define SPH_ERR_IC_CSOUND          8  /* preruncheck.f90:43-46                */
#define SPH_ERR_IC_H               9  /* preruncheck.f90:47-50                */
#define SPH_ERR_IC_PRESSURE       10  /* preruncheck.f90:51-54                */
#define SPH_ERR_IC_ENERGY         11  /* preruncheck.f90:55-57                */
#define SPH_ERR_IC_MUZERO         12  /* preruncheck.f90:28-31                */
#define SPH_ERR_IC_DIFFCOND       13  /* preruncheck.f90:32-35                */
#define SPH_ERR_UNSUPPORTED       14  /* option outside this engine's scope   */
#define SPH_ERR_FLD_ANISO         15  /* circuit2.f90:189, :367               */
#define SPH_ERR_DDW               16  /* circuit2.f90:422-423                 */
#define SPH_ERR_PROCESS           17  /* iterator.f90:173-177                 */
#define SPH_ERR_GRID              18  /* cell grid would not fit              */
#define SPH_ERR_OOM               19  /* device allocation failed             */
#define SPH_ERR_TIMEOUT           20  /* a bounded device wait gave up        */
#define SPH_ERR_STATE             21  /* call not valid in this handle state  */
#define SPH_ERR_RAD_NEGATIVE      22  /* rad_exchange.f90:61-64               */

/* ---- work counters (sph_get_counters, cumulative since create/reset) ----- */
#define SPH_CNT_ITERATES        0 /* calls of iterate (iterator.f90:44)       */
#define SPH_CNT_STEPS           1 /* completed time steps                     */
#define SPH_CNT_NEIB_PAIRS      2 /* in-support pairs found (sum over iterates)*/
#define SPH_CNT_C1_PAIRS        3 /* pair evaluations in circuit1 (all sweeps)*/
#define SPH_CNT_C1_SWEEPS       4 /* Newton sweeps (max over particles)       */
#define SPH_CNT_C2_PAIRS        5 /* pair evaluations in circuit2             */
#define SPH_CNT_GHOSTS          6 /* periodic images built (last iterate)     */
#define SPH_CNT_CANDIDATES      7 /* cell-list candidates tested              */
#define SPH_CNT_CENTRES         8 /* real centres processed (sum)             */
#define SPH_CNT_C1_CENTRE_SWEEPS 9 /* sum over particles of their sweeps      */
#define SPH_CNT_LAUNCHES      10 /* kernels of this library launched         */
#define SPH_CNT_NEIB_MAX      11 /* longest neighbour list of the last search */
#define SPH_CNT_SEARCHES      12 /* neighbour-search launches (incl. re-runs
                                    after a list outgrew its slots)          */
#define SPH_CNT_EXACT_TESTS   13 /* candidates decided by the FP64 test      */
#define SPH_CNT_ALLOCS        14 /* device allocations made by this handle    */
#define SPH_CNT_GRAPH_STEPS   15 /* steps run as a device-resident graph      */
#define SPH_CNT_GRAPH_REDOS   16 /* device-resident steps redone on the host  */
#define SPH_CNT_SKIN_BUILDS   17 /* searches that built skin lists          */
#define SPH_CNT_SKIN_REUSES   18 /* iterates served from skin lists          */
#define SPH_CNT_SKIN_DIRTY    19 /* centres searched afresh in those (sum)   */
#define SPH_CNT_SKIN_KEPT     20 /* rows kept unchanged in those (sum)       */
#define SPH_CNT_SKIN_RELAYOUTS 21 /* skin-list iterates that laid the whole
                                     table out anew                          */
#define SPH_CNT_TOTAL          22

/* ---- per-kernel timers (sph_get_timers, milliseconds, cumulative) ------- */
#define SPH_T_PREDICT    0
#define SPH_T_GHOSTS     1
#define SPH_T_SORT       2
#define SPH_T_NEIGHBOURS 3
#define SPH_T_CIRCUIT1   4
#define SPH_T_CIRCUIT2   5
#define SPH_T_CORRECT    6
#define SPH_T_TIMESTEP   7
#define SPH_T_STS        8
#define SPH_T_STEP       9 /* whole sph_step / sph_run_to calls */
#define SPH_T_PACK      10 /* pair-data packing before circuit1 and circuit2
                              (not part of SPH_T_CIRCUIT1 / SPH_T_CIRCUIT2) */
#define SPH_T_TOTAL      11

typedef struct sph_handle sph_handle;

/* Create an engine from the dump pair.  Replaces `./execute` start-up with
 * restore() (main.f90:112-116, dumper.f90:44-66) and initkernel
 * (kernel.f90:91-152).  n_rows = realpn + fixedpn rows of store.  The state
 * vector is validated like preruncheck.f90:13-60 when the run starts. */
int sph_create(const double* state49, const double* store, int64_t n_rows,
               int kernel_id, int precision_mode, sph_handle** out);

/* statevars(k) = value (state.f90:47-52) for k in 1..49, or an SPH_P_* slot. */
int sph_set_param(sph_handle* h, int index, double value);
int sph_get_param(sph_handle* h, int index, double* value);

/* Replace the particle table (same layout as sph_create). */
int sph_set_store(sph_handle* h, const double* store, int64_t n_rows);

/* One iterate(): periodic ghosts, neighbour search, circuit1, EOS, circuit2
 * (iterator.f90:44-179). */
int sph_iterate(sph_handle* h);

/* The density half of iterate(): ghosts, neighbour search, circuit1, EOS. */
int sph_density(sph_handle* h);

/* Advance the time loop of main.f90:241-373 by nsteps steps (the first call
 * also runs the initial iterate of main.f90:216-225). */
int sph_step(sph_handle* h, int nsteps);

/* Run the time loop until statevars(ec_time) reaches tfinish. */
int sph_run_to(sph_handle* h, double tfinish);

/* Read back the particle table (real + fixed rows, original row order) and
 * the state vector, in the dump layout (dumper.f90:26-34). */
int sph_get_store(sph_handle* h, double* out, int64_t cap_rows);
int sph_get_state(sph_handle* h, double* out49);

/* Neighbour sets of the last neighbour search, one row per real centre in
 * original order.  offsets has n_real+1 entries.  Each entry of `pairs` is
 * (rj << 5) | image where rj is the 0-based row of the real/fixed particle
 * the neighbour is (or is an image of, BC.f90:36-44) and image =
 * (sx+1) + 3(sy+1) + 9(sz+1) encodes the periodic shift (13 = no shift).
 * Entries are sorted ascending.  If cap is too small, offsets are filled and
 * SPH_ERR_ARG is returned. */
int sph_get_neighbours(sph_handle* h, int64_t* offsets, int64_t* pairs,
                       int64_t cap);

/* Digest of the same sets for comparisons at full size, where the pair
 * arrays would take gigabytes of host memory (2.1M centres x 178 pairs):
 * out[2 o] = number of neighbours of real row o, out[2 o + 1] = the sum
 * (mod 2^64) of a 64-bit mix of every entry (rj << 5) | image of that row,
 * which does not depend on the order of the row.  n >= n_real rows.
 * Serves the same comparison as sph_get_neighbours (the reference's lists,
 * neighboursearch.f90:74-180). */
int sph_get_neighbour_digest(sph_handle* h, uint64_t* out, int64_t n);

/* ---- one leapfrog step in parts --------------------------------------------
 * The step of sph_step (main.f90:241-373, leapfrog without STS or radiation
 * exchange) split where a domain decomposition exchanges particle fields:
 *   sph_timestep  -> dt = min over this handle's real rows of the equations'
 *                    limits (timestep.f90:40-166; the caller takes the
 *                    global minimum and clips it to tfinish / output times
 *                    as main.f90:273-299 does);
 *   sph_predict   (main.f90:323-342), sph_density (images, search,
 *                    circuit1, EOS), [exchange of rho, h, Omega, P, c],
 *   sph_forces    (circuit2 on the density pass's neighbour lists),
 *                    [exchange of a, du/dt, dh/dt],
 *   sph_correct   (main.f90:348-362; advances the handle's time by dt).
 * Rows keep their physical order from sph_predict to sph_correct.
 * sph_get_columns / sph_set_columns move whole columns of the table
 * (1-based field indices of const.f90, nf of them) in caller row order:
 * buf[k * n_rows + row]; buf may be host or device memory. */
int sph_timestep(sph_handle* h, double* dt);
int sph_predict(sph_handle* h, double dt);
int sph_forces(sph_handle* h);
int sph_correct(sph_handle* h, double dt);
int sph_get_columns(sph_handle* h, const int* fields, int nf, double* buf);
int sph_set_columns(sph_handle* h, const int* fields, int nf, const double* buf);

int sph_get_counters(sph_handle* h, int64_t* out, int n);
int sph_reset_counters(sph_handle* h);
int sph_get_timers(sph_handle* h, double* out_ms, int n);

/* ---- adjoint (gradients of a final-state misfit) ------------------------
 * No counterpart in the reference (its Fortran computes no derivatives).
 * sph_adjoint_forward runs nsteps leapfrog steps of fixed dt
 * (SPH_P_FIXED_DT; main.f90:323-362 without the timestep and output logic)
 * from the handle's state, keeping a copy of the particle table every
 * `every` steps; on a handle that has not stepped yet the initial force
 * pass (main.f90:216-225) is part of the differentiated map.  It lowers the
 * Newton tolerance (SPH_P_NEWTON_TOL) to 1e-12 and stops the physical
 * re-ordering of rows (SPH_P_REORDER_EVERY = 0) on the handle: the
 * differentiated density pass is the converged one.
 * sph_adjoint_backward takes dL/dv, dL/du, dL/dr at the final state (caller
 * row order, n_rows x 3 / n_rows / n_rows x 3; NULL = zero) and returns
 * dL/dr0, dL/dv0 (n_rows x 3), dL/du0 (n_rows) at the initial state and
 * dL/d(alpha, beta) (2 values; SPH_P_AV_ALPHA / SPH_P_AV_BETA), NULL
 * outputs skipped.  It replays each segment from its copy and runs the
 * hand-written adjoint kernels of the force pass (circuit2.f90:294-345), of
 * the Newton-h density pass (circuit1.f90:76-224, by the implicit function
 * theorem at convergence), of the EOS (eos.f90:21-33) and of the
 * integrator.  Differentiated subset: equations = hydro, adden = yes
 * (Newton h), artificial viscosity on or off with au = 0 or -1 (no
 * artificial conductivity), adiabatic EOS,
 * no fixed particles; other set-ups return SPH_ERR_UNSUPPORTED.  The handle
 * is left at the final state of the forward run. */
int sph_adjoint_forward(sph_handle* h, int nsteps, int every);
int sph_adjoint_backward(sph_handle* h, const double* dl_dv, const double* dl_du,
                         const double* dl_dr, double* g_r0, double* g_v0, double* g_u0,
                         double* g_par);
/* The diffusion adjoint: after sph_adjoint_forward on a run with equations
 * = diffusion (fixed positions: v = 0; ddw = fab, fw or n2w; isotropic,
 * diagonal or full b b^T conductivity tensor, circuit2.f90:347-397), maps
 * dL/dT(T) (realpn values, original row order) to dL/dT0 (g_T0) and
 * dL/d difcond (one value, state slot dcondconst), NULL outputs skipped. */
int sph_adjoint_backward_diffusion(sph_handle* h, const double* dl_dT, double* g_T0,
                                   double* g_difcond);

/* ---- end-of-run error (main.f90:374-402, errcalc.f90) --------------------
 * Replaces the engine's closing error evaluation: for the run's initial
 * condition type (state slot ics) at the handle's current time, err_i of
 * every real particle (errcalc.f90: shock12 :140-170 erf profile of T,
 * ring :99-138, pulse :46-97, sin3 :172-197, soundwave :220-236 density,
 * hydroshock :26-44 Sod density of the exact Riemann solution with the
 * reference's fixed gamma 1.4, alfvenwave :198-218) and
 * L1 = sum_i err_i / realpn (main.f90:401-402).  Types without a
 * calculator there (mti, mtilowres, OTvortex, boilingtank, none) give
 * err = 0, L1 = 0; fld_gauss and equations = kd2 (the chi error) return
 * SPH_ERR_UNSUPPORTED.  err_out (cap >= realpn doubles, original row order)
 * may be NULL. */
int sph_errcalc(sph_handle* h, double* err_out, int64_t cap, double* l1_out);

/* ---- batches of instances -----------------------------------------------
 * Many independent runs stepped together (the resolution x method sweeps
 * of the experiment runners, e.g. runner/
 * 000_anisopaper_v1_gls_kxx.py, which run one Context after another through
 * CleanRun / ContinueRun, core.py:152-156).  Each instance keeps its own
 * handle, stream and time loop; a batch runs the instances' steps from one
 * host worker per instance, so their kernels and their host round trips
 * (dt, image counts, list sizes) overlap on the device instead of queueing
 * one run behind the other.  The handles stay owned by the caller and must
 * not be used elsewhere while a batch call runs.  Results equal those of
 * the instances stepped one by one. */
typedef struct sph_batch sph_batch;
int sph_batch_create(int n_inst, sph_handle* const* handles, sph_batch** out);
/* sph_step(h_i, nsteps) for every instance */
int sph_batch_step(sph_batch* b, int nsteps);
/* sph_run_to(h_i, tfinish) for every instance */
int sph_batch_run_to(sph_batch* b, double tfinish);
/* status of every instance's last batch call (0 = ok); the call itself
 * returns the first non-zero status, its message in sph_last_error */
int sph_batch_status(sph_batch* b, int* status, int n);
void sph_batch_destroy(sph_batch* b);

/* ---- allocation-free density ---------------------------------------------
 * No counterpart in the reference.  For callers that cannot allocate device
 * memory (a code running inside another application's fixed device-memory
 * budget, e.g. an in-situ hook handed particle arrays by a host simulation,
 * or a caller that must avoid the device synchronisation of cudaMalloc /
 * cudaFree): rho_i = sum_{j != i, r_ij <= krad h_i} m_j W(r_ij, h_i)
 * + m_i W(0, h_i) over n particles given as device arrays (x, y, z, m, h;
 * y and z may be NULL below 3 dimensions), written to the device array rho.
 * No periodic images.  All intermediate data lives in a fixed static device
 * array of SPH_NOALLOC_SCRATCH_BYTES on every GPU that loads the library;
 * n above SPH_NOALLOC_MAX_PARTICLES is rejected with SPH_ERR_ARG.  The first
 * call on a device looks the array up.  Calls share the array: calls that overlap on the GPU race.  `stream` is a
 * cudaStream_t of the current device (NULL = default stream; a stream of
 * another device is rejected with SPH_ERR_ARG); the call synchronises it. */
#define SPH_NOALLOC_MAX_PARTICLES 262144
#define SPH_NOALLOC_SCRATCH_BYTES (32u << 20)
int sph_density_noalloc(const double* x, const double* y, const double* z,
                        const double* m, const double* h, int64_t n, int dim,
                        int kernel_id, double* rho, void* stream);

/* Last error message (static storage, valid until the next call). */
const char* sph_last_error(void);

void sph_destroy(sph_handle* h);

#ifdef __cplusplus
}
#endif
#endif /* SPH_ABI_H */
