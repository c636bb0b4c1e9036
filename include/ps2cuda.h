/*
 * ps2cuda — B200 (sm_100a) stage-2 gamma estimation for pySTAMPS
 * (the StaMPS ps_est_gamma_quick loop: bin -> CLAP -> resample -> topofit ->
 * gamma convergence).
 *
 * Plain C ABI: host or device pointers and sizes, no C++ or torch types.
 * Every function returns 0 on success or a negative PS2_ERR_* code; the text
 * of the last error of the calling thread is returned by ps2_last_error().
 *
 * Reference interfaces replaced (pySTAMPS, paths within that project):
 *  - ps2_create / ps2_load_patch / ps2_run_to_convergence / ps2_download
 *    replace the body of run_stage2_native_with_options
 *    (crates/pystamps-core/src/native_stage2.rs:208-413): a Rust caller keeps
 *    prepare_stage2_inputs (:415-561) and write_pm1 (:1899-1965) and calls
 *    these in place of the gamma loop (:261-406). The dispatch point is
 *    run_native_stage (2, Patch) in crates/pystamps-core/src/bin/pystamps-native.rs:198-201.
 *  - ps2_grid_accumulate replaces accumulate_weighted_grid (src/lib.rs:1013-1087)
 *    behind the Python registry kernel "stage2_grid_accumulate"
 *    (pystamps/kernels/accelerated.py:410, 429-443).
 *  - ps2_topofit is the native driver's topofit over rows (fit_stage2_rows /
 *    topofit_row / refine_candidate, native_stage2.rs:659-720, 1207-1303):
 *    first-argmax peak rule, the rule of the gamma loop itself.
 *  - ps2_topofit_near_max replaces the registry kernels "stage2_topofit",
 *    "stage2_topofit_row_invariant" and "stage2_topofit_coh_row_invariant"
 *    (pystamps/kernels/accelerated.py:316-380, 411-427, 446-493), i.e.
 *    ported._ps_topofit_single (pystamps/pipeline/ported.py:2355-2431, near-max
 *    tolerance 2e-4) and the PyO3 ps_topofit_batch_* (src/lib.rs:525-586,
 *    1159-1379, tolerance 5e-3): the tolerance is an argument.
 *  - ps2_histogram_with_centers replaces histogram_with_centers
 *    (src/lib.rs:2443-2455) behind "stage2_histogram" (accelerated.py:235-265, 496-509).
 *  - ps2_clap_filter_grid replaces clap_filter_grid_stack
 *    (native_stage2.rs:742-922) / ported._clap_filt_grid_stack_prepared
 *    (pystamps/pipeline/ported.py:1208-1298).
 *  - ps2_random_coherence_histogram replaces random_coherence_histogram
 *    (native_stage2.rs:1310-1512) / the "stage2_topofit_coh_row_invariant" +
 *    "stage2_histogram" registry kernels (accelerated.py:414-427).
 */
#ifndef PS2CUDA_H
#define PS2CUDA_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define PS2_OK 0
#define PS2_ERR_INVALID_ARG (-1)
#define PS2_ERR_CUDA (-2)
#define PS2_ERR_NOT_LOADED (-3)
#define PS2_ERR_UNSUPPORTED (-4)
#define PS2_ERR_OUT_OF_MEMORY (-5)

#define PS2_PRECISION_FP32 0 /* FP32 compute, FP64 only in K refinement and weighting */
#define PS2_PRECISION_FP64 1 /* plain FP64 everywhere (direct sincos, no recurrence) */

#define PS2_COH_BINS 100

typedef struct ps2_ctx ps2_ctx;

/* Prepared stage-2 inputs (the output of prepare_stage2_inputs,
 * native_stage2.rs:415-561). Row-major arrays; complex values are
 * interleaved (re, im) float pairs. */
typedef struct ps2_patch_desc {
  int64_t n_ps;        /* PS candidates (rows) */
  int64_t n_ifg;       /* non-master interferograms (columns) */
  const float* ph_nm;  /* complex64 [n_ps, n_ifg], unit magnitude (0 stays 0) */
  const float* amp;    /* NULL, or f32 [n_ps, n_ifg] magnitudes (SNR weighting only) */
  const float* bperp;  /* f32 [n_ps, n_ifg], or [n_ifg] when bperp_row_invariant */
  int32_t bperp_row_invariant;
  const int64_t* grid_lin; /* [n_ps] 0-based cell (i-1)*n_j + (j-1) */
  int64_t n_i, n_j;        /* grid cells */
  const double* weight0;   /* [n_ps] initial weighting 1/D_A (0 where D_A == 0) */
  const double* low_pass;  /* [n_win_ex * n_win_ex] Butterworth low pass (fftshifted) */
  int64_t n_win_ex;        /* CLAP FFT size, round(clap_win) = 32 */
  int64_t clap_window;     /* CLAP window, round(0.75 * clap_win) = 24 */
  double clap_alpha, clap_beta;
  double n_trial_wraps;    /* trials = -ceil(8*n)..ceil(8*n) */
  const double* nr;        /* [PS2_COH_BINS] random-phase coherence histogram */
  double nr_max_nz_ix;     /* 1-based index of the last non-zero Nr bin */
  int64_t low_coh_thresh;  /* 31 (15 for small baselines) */
  int32_t psquare;         /* 1: P-square weighting, 0: SNR weighting */
  double gamma_change_convergence;
  int64_t gamma_max_iterations;
  int32_t precision;       /* PS2_PRECISION_* */
  int32_t pointers_on_device; /* 1: the array pointers above are device pointers */
} ps2_patch_desc;

typedef struct ps2_iter_stats {
  int64_t i_loop;            /* 1-based iteration that produced these numbers */
  double gamma_change_rms;   /* sqrt(mean((coh - coh_prev)^2)) */
  double gamma_change_delta; /* gamma_change_rms - previous gamma_change_rms */
  int32_t stop;              /* convergence or iteration cap reached */
  int32_t n_invalid;         /* rows with a zero element in conj(ph_patch)*ph_nm */
} ps2_iter_stats;

/* Host buffers for the pm1.mat variables (native_stage2.rs:1899-1965);
 * NULL members are skipped. Row order is the caller's original PS order. */
typedef struct ps2_outputs {
  double* K_ps;        /* [n_ps] rad/m; NaN for invalid rows */
  double* C_ps;        /* [n_ps] */
  double* coh_ps;      /* [n_ps] */
  double* N_opt;       /* [n_ps] */
  float* ph_res;       /* [n_ps, n_ifg] */
  float* ph_patch;     /* complex64 [n_ps, n_ifg] */
  float* ph_grid;      /* complex64 [n_i, n_j, n_ifg] */
  float* ph_weight;    /* complex64 [n_ps, n_ifg] */
  double* coh_ps_save; /* [n_ps] */
  double* Nr;          /* [PS2_COH_BINS] Nr as scaled by the last P-square update */
  double* gamma_change_save;
  int64_t* i_loop;
  double* ph_res_f64;   /* FP64 precision only: [n_ps, n_ifg] */
  double* ph_patch_f64; /* FP64 precision only: complex128 [n_ps, n_ifg] */
  double* ph_grid_f64;  /* FP64 precision only: complex128 [n_i, n_j, n_ifg] */
  double* ph_weight_f64;/* FP64 precision only: complex128 [n_ps, n_ifg] */
} ps2_outputs;

/* ---------------------------------------------------------- context API -- */
int ps2_create(ps2_ctx** out, int device);
void ps2_destroy(ps2_ctx* ctx);
const char* ps2_last_error(void);
/* Uploads and lays out one patch (cell-sorted rows). Copies the inputs; no
 * caller pointer is retained after return. */
int ps2_load_patch(ps2_ctx* ctx, const ps2_patch_desc* desc);
/* Runs n_iter gamma iterations whatever the convergence test says (for
 * timing); stats may be NULL or hold n_iter entries. */
int ps2_iterate(ps2_ctx* ctx, int64_t n_iter, ps2_iter_stats* stats);
/* Runs iterations until the reference's stop rule holds
 * (|delta gamma_change| < gamma_change_convergence or i_loop >= max). The
 * first iteration runs as individual launches; the rest run as one CUDA graph
 * launch (a WHILE conditional node whose body is one iteration), built on the
 * first call after ps2_load_patch. PS2_NO_GRAPH=1 in the environment selects
 * individual launches throughout. */
int ps2_run_to_convergence(ps2_ctx* ctx, ps2_iter_stats* last);
/* Runs ONE gamma iteration under the reference's stop rule: when the rule
 * holds the P-square update is skipped, as the loop does before it ends
 * (native_stage2.rs:307-314); *stats (may be NULL) receives its statistics.
 * For callers that act between iterations (per-iteration pm1 dumps,
 * checkpoints); ps2_run_to_convergence is the fast path. */
int ps2_step(ps2_ctx* ctx, ps2_iter_stats* stats);
/* Resets the loop state of the loaded patch to iteration 1 (K=0, w=weight0). */
int ps2_reset(ps2_ctx* ctx);
int ps2_download(ps2_ctx* ctx, ps2_outputs* out);
/* Device time in milliseconds (CUDA events on the context's stream) of the
 * last ps2_iterate call from its first launch to its last (for
 * ps2_run_to_convergence: the sum of the iterations), and the summed time of
 * each kernel family in it: [0] binning, [1] CLAP windows + overlap-add,
 * [2] topofit, [3] convergence / weighting update. */
int ps2_last_timing(const ps2_ctx* ctx, double* total_ms, double* per_kernel_ms /*[4] or NULL*/);
/* Checkpoint / resume of the gamma loop (the reference has none; its
 * PYSTAMPS_STAGE2_NATIVE_DEBUG_PM dumps, native_stage2.rs:259, 337-356,
 * 385-404, write pm1_iter_NN.mat but cannot restart from them).
 * ps2_export_state copies the loop state after the last iteration (K, weights,
 * coherence, C, N_opt, the P-square table, scaled Nr, the convergence state and
 * iteration count; ph_res with SNR weighting) into a host buffer: call it with
 * buf NULL to get the size in *bytes, then with a buffer of that size. The
 * blob is opaque (the context's cell-sorted row order) and valid for the same
 * patch loaded the same way, in the same precision: ps2_import_state into a
 * context holding that patch restores the state, and ps2_run_to_convergence /
 * ps2_step / ps2_iterate then continue from the next iteration with the same
 * results as an uninterrupted run. Mismatched or truncated states are rejected. */
int ps2_export_state(ps2_ctx* ctx, void* buf, int64_t* bytes);
int ps2_import_state(ps2_ctx* ctx, const void* buf, int64_t bytes);
/* Times the launch shapes of the loaded patch and keeps the fastest for this
 * context and for later loads in the same bucket (interferograms rounded up to
 * a multiple of 8, power-of-two PS count, precision; a process-wide table):
 * the FP32 topofit with 4, 8, 16 and 32 lanes per PS (ms_per_candidate: NULL
 * or [4]; *chosen_lanes the winner), CLAP with 8 or 4 warps per block and as
 * many or one resident block per SM, binning with 16 blocks per SM queued or
 * 3 or 2 (a persistent grid), and the CLAP form (window stack or fused window
 * blocks, each timed with its second pass). The CLAP and binning shapes give
 * bit-identical results (the two CLAP forms wherever their FP64 sums are
 * exact); the lane width changes the order of the topofit's partial sums. */
int ps2_autotune(ps2_ctx* ctx, int32_t* chosen_lanes, double* ms_per_candidate);
/* Reads (get: NULL or [5]) and/or pins (set: NULL or [5]) the launch shapes of
 * the context: topofit lanes per PS (0 = rule from n_ifg, or 4/8/16/32), CLAP
 * warps per block (0 = default, 4 or 8; FP64 runs 4), CLAP resident blocks per
 * SM (0 = as many as fit), binning blocks per SM (0 = 16 queued), CLAP form
 * (0 = each window into a window stack, then the overlap-add pass; 1 = blocks
 * of 4 x 4 windows summed into FP64 partials, then a combine pass: no window
 * stack). For callers that keep their own tuning table. */
int ps2_launch_shapes(ps2_ctx* ctx, int32_t* get, const int32_t* set);
/* Number of kernel launches issued by the last iterate/run call. */
int64_t ps2_last_launch_count(const ps2_ctx* ctx);

/* ------------------------------------------------- stateless kernels ---- */
/* All pointers are host pointers unless stated otherwise. */
int ps2_grid_accumulate(const float* ph_weight, const int64_t* grid_lin, int64_t n_ps, int64_t n_ifg, int64_t n_i,
                        int64_t n_j, float* out /* complex64 [n_i, n_j, n_ifg] */);
int ps2_topofit(const float* cpxphase /* complex64 [n, m] */, const float* bperp /* [n, m] or [m] */,
                int32_t bperp_row_invariant, double n_trial_wraps, int64_t n, int64_t m, double* K, double* C,
                double* coh, float* residual /* complex64 [n, m] or NULL */);
int ps2_clap_filter_grid(const float* ph_grid /* complex64 [n_i, n_j, m] */, int64_t n_i, int64_t n_j, int64_t m,
                         int64_t clap_window, double alpha, double beta, const double* low_pass, int64_t n_win_ex,
                         float* out /* complex64 [n_i, n_j, m] */);
/* The registry's topofit rule over rows: per row only the non-zero columns
 * take part (an all-zero row gives NaN K, C, coh and a zero residual); trial
 * coherences; every local maximum within near_max_tol of the largest is
 * refined and the reference's choice among them is kept
 * (_ps_topofit_near_max_trial_indices / _select_candidate / _refine_candidate,
 * pystamps/pipeline/ported.py:2433-2513). precision PS2_PRECISION_FP32: cpxphase
 * complex64 and bperp f32 (the reference's single-precision path, taken when
 * either input is single precision); PS2_PRECISION_FP64: complex128 and f64.
 * residual: NULL or complex64 [n, m]. Synchronous; host pointers. */
int ps2_topofit_near_max(const void* cpxphase, const void* bperp, int32_t bperp_row_invariant, int32_t precision,
                         double n_trial_wraps, int64_t n, int64_t m, double near_max_tol, double* K, double* C,
                         double* coh, float* residual);
/* Counts of the finite values per centre (f64 [n_centers]): equally spaced
 * centres use the ceil rule, others the nearest-midpoint rule
 * (pystamps/kernels/accelerated.py:235-265). Host pointers. */
int ps2_histogram_with_centers(const double* values, int64_t n, const double* centers, int64_t n_centers,
                               double* out);
/* ---- host-side preparation (prepare_stage2_inputs, native_stage2.rs:447-467,
 * 563-612) ------------------------------------------------------------------
 * Threaded host passes (threads 0 = all cores), no device work.
 * ps2_prepare_phase: ph complex64 [n_ps, n_full] -> ph_nm complex64 [n_ps, m] and
 *   amp f32 [n_ps, m] over the columns cols[m]: amp = |ph| (hypotf), 1 where it
 *   is 0; ph_nm = ph / amp (so a zero stays 0).
 * ps2_prepare_bperp: bperp_mat f64 [n_ps, width] -> f32 [n_ps, m] over cols[m]
 *   (NULL: all width == m columns); *row_invariant = every row equals the
 *   first. */
int ps2_prepare_phase(const float* ph, int64_t n_ps, int64_t n_full, const int64_t* cols, int64_t m, float* ph_nm,
                      float* amp, int threads);
int ps2_prepare_bperp(const double* bperp_mat, int64_t n_ps, int64_t width, const int64_t* cols, int64_t m, float* out,
                      int32_t* row_invariant, int threads);

/* Setup histogram of the coherence of 300,000 (n_rand) random-phase rows, in
 * FP64 on the GPU; the MATLAB v5 uniform generator (seed 2005) runs on the
 * host. ifgday_ix ([n_ifg, 2], 1-based) and n_image are used only when
 * small_baseline != 0. */
int ps2_random_coherence_histogram(const double* bperp_nm, int64_t n_ifg, double n_trial_wraps, int64_t n_rand,
                                   int32_t small_baseline, const int64_t* ifgday_ix, int64_t n_image,
                                   double* nr_out /* [PS2_COH_BINS] */, double* nr_max_nz_ix);

/* CLAP filter for callers that cannot allocate GPU memory: code running under
 * a memory budget owned by another allocator (a framework's caching pool, a
 * Rust or JVM host that hands in pre-allocated buffers), or code that must not
 * call cudaMalloc/cudaFree because they synchronise the device. Same result as
 * ps2_clap_filter_grid, but d_ph_grid and d_out are DEVICE pointers owned by
 * the caller, the work is queued on `stream` (a cudaStream_t, NULL = legacy
 * default stream) and the call returns without waiting. It allocates nothing:
 * its scratch is a fixed 32 MiB array inside the library, which every GPU that
 * loads the library holds until the process exits. Sizes whose scratch
 * (16*G*Mp + 8*W*clap_window^2*Mp bytes + about 13 KiB, G = n_i*n_j, Mp = m rounded
 * up to 4, W = CLAP windows) exceed 32 MiB are rejected with
 * PS2_ERR_UNSUPPORTED. Every call shares that one array: calls whose GPU work
 * overlaps (other streams, other host threads) race on it and must be
 * serialised by the caller. The first call on a device resolves the array's
 * device address (cudaGetSymbolAddress) with that device current; make that
 * first call before any stream capture. low_pass is a host pointer
 * [32*32]; its values (and the window weights) travel to the GPU inside the
 * arguments of a kernel the call queues, so the caller may reuse or free it as
 * soon as the call returns. This entry point has no counterpart in the
 * reference. */
int ps2_clap_filter_grid_noalloc(const float* d_ph_grid, int64_t n_i, int64_t n_j, int64_t m, int64_t clap_window,
                                 double alpha, double beta, const double* low_pass, int64_t n_win_ex, float* d_out,
                                 void* stream);


/* ---- batches ----------------------------------------------------------------
 * Runs every loaded context of `ctxs` (FP32, P-square weighting, one device,
 * each context once) to its own convergence together: each gamma iteration is
 * one launch per step (binning, CLAP, overlap-add, finalize) covering every
 * still-iterating patch, and one persistent topofit launch per lane-width
 * class (4, 8, 16 or 32 lanes per PS, from the patch's interferogram count).
 * A patch that meets its stop rule drops out; each patch's results are those
 * of ps2_run_to_convergence on that context alone (same arithmetic, same
 * per-block partial sums). Work runs on ctxs[0]'s stream after the work
 * already queued on every context's stream. last[p] (optional, [n]) receives
 * each patch's final statistics; ps2_download then reads each context. The
 * reference runs patches one after another
 * (pystamps/pipeline/stages.py:184-221); this batching has no counterpart. */
int ps2_batch_run(ps2_ctx* const* ctxs, int64_t n, ps2_iter_stats* last);

/* ---- stage-3 re-estimate -------------------------------------------------
 * The re-estimate of stage-3 selection (pystamps/pipeline/ported.py:4429-4575,
 * inside stage3_select_ps): for each selected PS, the clap_win x clap_win
 * patch of the stage-2 filtered grid around its cell, with that cell zeroed
 * (and, for the first interferogram, the slc_osf neighbourhood), is
 * CLAP-filtered (_clap_filt_patch, :992-1009) and the value at the cell kept
 * (ph_patch2, 0 where the patch does not fit); then
 * psdph = ph * conj(ph_patch2) is normalised and re-fitted by the reference's
 * stage-3 topofit (_ps_topofit_single, :2355-2431: near-max candidates within
 * 2e-4, each refined, the reference's choice among them) on the fit_ifg
 * columns. Rows with any zero psdph get K = coh = NaN, C = 0. All pointers are
 * host pointers; the call is synchronous. FP32 arithmetic (the reference uses
 * complex128 for the patch filter and complex64 for the fit). */
typedef struct ps3_reestimate_desc {
  int64_t n_sel;            /* selected PS rows */
  int64_t n_ifg;            /* M: interferograms (master column removed) */
  const float* ph;          /* complex64 [n_sel, M]: the selected rows of ph */
  const float* bperp;       /* f32 [n_sel, M]: their bp1.bperp_mat rows */
  const int64_t* grid_ij;   /* [n_sel, 2]: their 1-based pm1.grid_ij cells */
  const float* ph_grid;     /* complex64 [grid_rows, grid_cols, M]: pm1.ph_grid */
  int64_t grid_rows, grid_cols;
  int64_t n_i, n_j;         /* max of pm1.grid_ij over all PS (the patch placement limits) */
  const int64_t* fit_ifg;   /* [n_fit] 0-based columns the fit uses (ifg_index - 1) */
  int64_t n_fit;
  int64_t clap_win;         /* 32 */
  double clap_alpha, clap_beta;
  const double* low_pass;   /* [clap_win * clap_win] pm1.low_pass */
  int64_t slc_osf;
  double n_trial_wraps;     /* pm1.n_trial_wraps */
} ps3_reestimate_desc;

typedef struct ps3_reestimate_out {
  float* ph_patch2;         /* complex64 [n_sel, M] */
  double* K_ps2;            /* [n_sel] */
  double* C_ps2;            /* [n_sel] */
  double* coh_ps2;          /* [n_sel] */
  float* ph_res2;           /* f32 [n_sel, M]: residual angle on fit_ifg columns, 0 elsewhere */
} ps3_reestimate_out;

int ps3_reestimate(const ps3_reestimate_desc* desc, ps3_reestimate_out* out, int device);

/* The same re-estimate from a context that ran stage 2 (ps2_run_to_convergence
 * or ps2_batch_run): the patch's phases, bperp, cells, low-pass, CLAP
 * parameters, trial count and last binned grid are read where they already
 * are in device memory, so only the selection goes in and the results come
 * out. sel: 0-based rows in the caller's order; fit_ifg: 0-based columns.
 * outputs_on_device != 0: the out pointers are device pointers on the
 * context's device. The window is 32 x 32 (parms clap_win, the only stage-3
 * window this library runs) with the context's 32 x 32 low-pass filter.
 * Synchronous; FP32 contexts. */
int ps2_stage3_reestimate(ps2_ctx* ctx, const int64_t* sel, int64_t n_sel, const int64_t* fit_ifg, int64_t n_fit,
                          int64_t slc_osf, ps3_reestimate_out* out, int outputs_on_device);

/* ---- one patch over several GPUs ------------------------------------------
 * A patch split by rows into contiguous cell ranges, one range per rank (one
 * GPU each): every rank loads a context with its rows only (ps2_load_patch of
 * the sub-patch: same n_i, n_j, low-pass, Nr and parameters, rows in their
 * original relative order) and iterates with
 *   ps2_shard_bin(ctx, d_grid)          bin this rank's rows; copy the context's
 *                                       grid (complex [n_i*n_j, Mp], Mp = M
 *                                       rounded up to 4; complex128 for FP64)
 *                                       to the device buffer d_grid
 *   <sum d_grid over the ranks>         cells are disjoint: the sum is the grid
 *                                       of the whole patch, bit for bit
 *   ps2_shard_filter(ctx, d_grid, lo, hi)  copy the summed grid in; CLAP of the
 *                                       windows meeting rows of cells lo..hi-1
 *                                       and overlap-add of cells lo..hi-1
 *   ps2_shard_fit(ctx, stats)           topofit of this rank's rows; stats (host,
 *                                       PS2_SHARD_STATS doubles) = coherence
 *                                       histogram [100], sum of squared changes,
 *                                       invalid rows
 *   <sum stats over the ranks>
 *   ps2_shard_finalize(ctx, stats, n_total, &it)  the stop rule and the P-square
 *                                       update from the summed statistics (the
 *                                       same on every rank); loop while !it.stop
 * Each call is synchronous on the context's stream. The reference iterates one
 * patch on one host (native_stage2.rs:261-406); this split has no counterpart.
 * Per-PS results equal a single-context run; the convergence RMS sums rank
 * totals, so it can differ from it in the last bits. */
#define PS2_SHARD_STATS (PS2_COH_BINS + 2)
int ps2_shard_bin(ps2_ctx* ctx, void* d_grid);
int ps2_shard_filter(ps2_ctx* ctx, const void* d_grid, int64_t cell_lo, int64_t cell_hi);
int ps2_shard_fit(ps2_ctx* ctx, double* stats);
int ps2_shard_finalize(ps2_ctx* ctx, const double* stats, int64_t n_total, ps2_iter_stats* out);

/* ---- differentiable coherence (adjoints) ------------------------------------
 * The gamma map with K given, as a function of the input phases, K and the
 * CLAP parameters, on the loaded patch's geometry (cells, bperp, low-pass,
 * CLAP window):
 *   grid  = sum over each cell of ph * exp(-j K bperp) * w      (the binning)
 *   filt  = CLAP(grid; alpha, beta) + pyramid overlap-add        (the filter)
 *   p     = filt[cell] / |filt[cell]|                            (resample)
 *   coh   = |sum_c conj(p_c) ph_c exp(-j K bperp_c)| / sum_c |conj(p_c) ph_c|
 * which is the coherence topofit reports for that K (ps_topofit's coh0 at
 * K0 = K; crates/pystamps-core/src/native_stage2.rs:1257-1303 and the
 * filter/resample steps :888-1184), without the trial search.
 * All arrays are device pointers in the caller's row order on the context's
 * device: d_ph complex64 [n_ps, n_ifg] (interleaved float pairs), d_K, d_w,
 * d_coh float [n_ps]. Work is queued on `stream` (a cudaStream_t; NULL is
 * the legacy default stream), after the work already queued on the
 * context's own stream, and is asynchronous; calls on different streams must
 * be ordered by the caller. The context's gamma-loop state is untouched.
 * The arithmetic runs in the context's precision (a patch loaded with
 * PS2_PRECISION_FP64 gives FP64 forward and adjoint arithmetic on the same
 * float inputs and outputs). No counterpart in the reference, which has no
 * gradients. */
int ps2_coherence_forward(ps2_ctx* ctx, const float* d_ph, const float* d_K, const float* d_w, double clap_alpha,
                          double clap_beta, float* d_coh, void* stream);

/* Vector-Jacobian product of ps2_coherence_forward: given d_gcoh = dL/dcoh
 * [n_ps], writes dL/dph (complex64 [n_ps, n_ifg], as dL/dRe + j dL/dIm),
 * dL/dK [n_ps] and d_galpha_beta[0..1] = dL/dclap_alpha, dL/dclap_beta (a
 * device double[2]). The forward pass is recomputed; CLAP's window spectra
 * are recomputed per window, not stored. The median of the smoothed spectrum
 * passes its gradient to the elements equal to the 512th and 513th order
 * statistics (half each, split evenly among ties); w is a constant. */
int ps2_coherence_backward(ps2_ctx* ctx, const float* d_ph, const float* d_K, const float* d_w, double clap_alpha,
                           double clap_beta, const float* d_gcoh, float* d_gph, float* d_gK, double* d_galpha_beta,
                           void* stream);

#ifdef __cplusplus
}
#endif
#endif /* PS2CUDA_H */
