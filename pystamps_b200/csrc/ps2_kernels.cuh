// Kernel argument blocks and launchers for the stage-2 loop.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

namespace ps2 {

// e^{-2 pi i k / 32}, k = 0..15, computed on the host in double precision.
struct Twiddles32f {
  float2 w[16];
};
struct Twiddles32d {
  double2 w[16];
};

// --------------------------------------------------------------- binning --
// fill_phase_weight + accumulate_grid (native_stage2.rs:629-657, 722-740):
// grid[cell, c] = sum over the cell's rows s (ascending original row order)
// of ph_nm[s, c] * e^{-j bp K_s} * w_s, summed sequentially.
struct BinArgs {
  const void* ph_nm;     // complex [N, M] (cell-sorted rows)
  const float* bp;       // f32 [N, M] sorted, or [M]
  int bp_row_inv;
  const int32_t* cell_start;  // [G + 1]
  int64_t G;
  int M, Mp, nchunk;
  const void* K;         // real [N] (sorted)
  void* w;               // real [N] (sorted): read (mode 0) or written (mode 1)
  const void* coh;       // real [N] previous coherence (mode 1)
  const double* lut;     // P-square prand_hi table (mode 1)
  int lut_len;
  int mode;              // 0: w given; 1: w = (1 - lut[round(1000 coh)])^2
  void* grid;            // complex [G, Mp]
  int blocks_per_sm;     // launch shape: resident blocks per SM (0: as many as fit)
};

// ------------------------------------------------------------------ CLAP --
struct ClapArgs {
  const void* grid;   // complex [G, Mp]
  int n_i, n_j, M, Mp;
  int n_win;          // 24
  int nwi, nwj;       // window counts per axis
  int alpha_is_one;
  double alpha, beta;
  const double* low_pass;  // [32*32] natural FFT order (device)
  const double* wscaled;   // [n_win*n_win] pyramid weight / 1024 (device)
  double g7[7];            // 7-tap Gaussian of the |H| smoothing
  void* win_out;           // complex [W, n_win*n_win, Mp] (window-stack form)
  void* part;              // complex FP64 [window blocks, box, box, Mp] (fused form; win_out unused)
  int64_t w_lo, w_n;       // windows (window blocks in the fused form) w_lo .. w_lo + w_n - 1 (w_n = 0: all)
  int nw_block;            // launch shape: warps (interferograms) per block, 4 or 8 (0: 8 in FP32, 4 in FP64)
  int blocks_per_sm;       // launch shape: resident blocks per SM (0: as many as fit)
};

struct OverlapArgs {
  const void* win_out;  // complex [W, n_win*n_win, Mp] (window-stack form)
  const void* part;     // complex FP64 block partials of the fused form (win_out unused)
  void* filt;           // complex [G, Mp]
  int n_i, n_j, M, Mp, n_win, n_inc, nwi, nwj;
  int normalize;        // 1 (FP32 stage-2 loop): store f/|f|, the unit patch phase the topofit reads
  int64_t cell_lo, cell_n;  // cells cell_lo .. cell_lo + cell_n - 1 (cell_n = 0: all cells)
};

// --------------------------------------------------------------- topofit --
struct TopoArgs {
  const void* ph_nm;      // complex [N, M] sorted (loop mode)
  const void* filt;       // complex [G, Mp] filtered grid (loop mode)
  const int32_t* cell_of; // [N] (loop mode)
  const void* cpx;        // complex [N, M] (registry mode, replaces ph_nm/filt)
  const float* bp;        // f32 [N, M] or [M]
  int bp_row_inv;
  int64_t N;
  int M, Mp;
  int n_half;             // ceil(8 * n_trial_wraps)
  int zero_mode;          // 0: a zero element invalidates the row; 1: zero columns skipped
  void* K_out;            // real [N]
  void* C_out;            // real [N]
  void* coh_io;           // real [N]: previous coherence in, new coherence out
  uint8_t* nopt;          // [N]
  double* rms_partial;    // [gridDim.x]
  int32_t* hist;          // [100]
  int32_t* n_invalid;     // [1]
  double cutoff0, dbin;
  // optional outputs (written only when non-null)
  void* residual;         // complex [N, M]
  void* ph_res;           // real [N, M]
  void* ph_patch;         // complex [N, M]
  int accumulate_stats;   // 1: rms partials / histogram / invalid count
  int lanes;              // lanes per PS in the FP32 kernel (4, 8, 16, 32); 0: from n_ifg
  int filt_unit;          // 1: filt already holds f/|f| (k_overlap with normalize), FP32 kernel
};

// -------------------------------------------------------------- finalize --
struct FinalizeArgs {
  const double* rms_partial;
  int n_partial;
  int64_t N;
  const int32_t* hist;       // Na
  double* nr_scaled;         // [100] in/out
  double nr_max_nz_ix;
  int low_coh_thresh;
  int psquare;
  double gamma_change_convergence;
  int64_t gamma_max_iterations;
  double g7w[7];             // gausswin(7, 2.5) for the prand smoothing
  double g7sum;
  const double* taps79;      // interp(x, 10) FIR
  double* lut;               // [1001] out
  double* state;             // [4]: gamma_change_save, i_loop, last rms, last delta
  double* stats_out;         // [6] per-iteration record
  int32_t* n_invalid;
  int force_continue;        // iterate past the stop rule (timing runs)
};

// --------------------------------------------------------------- stage 3 --
struct S3ClapArgs {
  const float2* grid;      // stage-2 ph_grid [rows, cols, grid_stride]
  int grid_cols, M, grid_stride;
  const int32_t* jobs;     // [n_jobs][4]: patch origin row, col (0-based; -1: no patch), PS cell in the patch
  int64_t n_jobs;
  int ngroups;             // ceil(M / 4)
  int slc_rad;             // slc_osf - 1
  int alpha_is_one;
  double alpha, beta;
  const double* low_pass;  // [32 * 32]
  double g7[7];
  float2* job_out;         // [n_jobs, M] filtered value at the PS cell
};

struct S3FitArgs {
  const float2* ph;        // [*, M] rows of the selected PS
  const float* bp;         // [*, M], or [M] when bp_row_inv
  const int32_t* row;      // [n_sel] row of each selected PS in ph / bp (NULL: row r)
  int bp_row_inv;
  const int32_t* job_of;   // [n_sel]
  const float2* job_out;   // [n_jobs, M]
  const int32_t* fit;      // [n_fit] columns used by topofit
  int n_fit, M, n_half;
  int64_t n_sel;
  size_t warp_smem;        // bytes of shared memory per warp
  float2* ph_patch2;       // [n_sel, M]
  double* K2;
  double* C2;
  double* coh2;
  float* ph_res2;          // [n_sel, M]
};

// --------------------------------------------------------------- batches --
// One patch of a batch: the single-patch arguments of every step.
struct PatchDev {
  BinArgs bin;        // bin.K = K[0]; mode is set per iteration from fin.state
  ClapArgs clap;
  OverlapArgs ov;
  TopoArgs topo;
  FinalizeArgs fin;
  float* K1;          // K[1]: the K this iteration binned with
  int mpad, nvb;      // topofit column padding and virtual blocks
  int psquare;
  int lanes;
};

struct BatchArgs {
  const PatchDev* patch;      // [P]
  int P;
  int* active;                // [P] 1 while the patch iterates
  int* n_active;              // [1]
  const int64_t* bin_prefix;  // [P + 1] warp-tasks (G * nchunk)
  const int64_t* clap_prefix; // [P + 1] block-tasks (W * Mp / 4)
  const int64_t* ov_prefix;   // [P + 1] elements (G * Mp)
};

// -------------------------------------------------------------- adjoints --
// R-typed arrays are float or double by the context's precision.
struct CohArgs {
  const void* filt;       // complex R [G, Mp]
  const float2* ph;       // [N, M] sorted (the caller's phases)
  const void* K;          // R [N] sorted
  const void* w;          // R [N] sorted (bin backward)
  const float* bp;        // [N, M] sorted or [M]
  int bp_row_inv;
  const int32_t* cell_of; // [N]
  int64_t N;
  int M, Mp;
  float* coh;             // forward out [N]
  const float* gcoh;      // backward in [N]
  void* gph;              // backward out: complex R [N, M]
  void* gK;               // backward out: R [N]
  void* gf;               // backward out: d L / d filt per (PS, ifg), complex R [N, M]
  const void* ggrid;      // bin backward in: complex R [G, Mp]
};

struct ClapBwdArgs {
  ClapArgs f;           // the forward call's arguments (grid = its input)
  const void* gfilt;    // complex R [G, Mp]: d L / d CLAP output
  void* wgrad;          // complex R [W, n_win^2, Mp]: d L / d window input
  double* ab_partial;   // [2 * blocks]: d L / d alpha, d L / d beta per block
};

// ---------------------------------------------------------- launchers -----
cudaError_t launch_bin(const BinArgs& a, bool fp64, int sm_count, cudaStream_t st);
// w[s] = (1 - lut[round(1000 coh[s])])^2 for s < N (a.coh, a.lut, a.lut_len, a.w)
cudaError_t launch_psquare_weights(const BinArgs& a, int64_t N, bool fp64, int sm_count, cudaStream_t st);
cudaError_t launch_clap(const ClapArgs& a, bool fp64, const Twiddles32f& tf, const Twiddles32d& td, int sm_count,
                        cudaStream_t st);
cudaError_t launch_overlap(const OverlapArgs& a, bool fp64, cudaStream_t st);
cudaError_t launch_topofit(const TopoArgs& a, bool fp64, int grid_blocks, cudaStream_t st);
int topofit_grid_blocks(int sm_count, bool fp64);
int topofit_lanes(int M);
cudaError_t launch_finalize(const FinalizeArgs& a, cudaStream_t st);
cudaError_t launch_loop_continue(cudaGraphConditionalHandle h, const double* stats, cudaStream_t st);
cudaError_t launch_coh(const CohArgs& a, int which /*0 fwd, 1 coherence bwd, 2 bin bwd*/, bool fp64,
                       int sm_count, cudaStream_t st);
cudaError_t launch_cell_sum(const CohArgs& a, const int32_t* cell_start, int64_t G, void* out, bool fp64,
                            int sm_count, cudaStream_t st);
cudaError_t launch_clap_bwd(const ClapBwdArgs& b, bool fp64, const Twiddles32f& tf, const Twiddles32d& td,
                            int* blocks_out, cudaStream_t st);
int clap_bwd_max_blocks(int sm_count, bool fp64);
cudaError_t launch_gather_widen(const float* src, double* dst, const int32_t* perm, int64_t n, cudaStream_t st);
// dst[perm[s]] = double(src[s]) for an f32 vector, or 0.0 / 1.0 for a u8 flag vector (flags)
cudaError_t launch_scatter_widen(const void* src, bool flags, double* dst, const int32_t* perm, int64_t n,
                                 cudaStream_t st);
cudaError_t launch_scatter_narrow(const double* src, float* dst, const int32_t* perm, int64_t n, int64_t words,
                                  cudaStream_t st);
cudaError_t launch_reduce_ab(const double* part, int n, double* out, cudaStream_t st);
size_t topofit_smem_bytes(int L, int mpad, int n_half);
// complex FP64 elements of the fused CLAP's window-block partials
int64_t clap_part_elems(int nwi, int nwj, int n_win, int Mp);
// window blocks per axis (4 windows a side) of the fused CLAP
int clap_block_count(int nw_axis);
cudaError_t topofit_geometry(const TopoArgs& a, int grid_cap, int* L_out, int* mpad_out, int* blocks_out);
cudaError_t launch_batch_reset(const BatchArgs& b, cudaStream_t st);
cudaError_t launch_s3_clap(const S3ClapArgs& a, const Twiddles32f& tf, int sm_count, cudaStream_t st);
cudaError_t launch_s3_fit(const S3FitArgs& a, int sm_count, cudaStream_t st);

// ----------------------------------------------------- registry topofit --
// _ps_topofit_single over rows (pystamps/pipeline/ported.py:2355-2431):
// near-max candidates within tol, each refined, the reference's choice.
struct NearMaxArgs {
  const void* cpx;   // complex [n, M] (complex64 or complex128)
  const void* bp;    // real [n, M], or [M] when bp_row_inv
  int bp_row_inv;
  int64_t n;
  int M, n_half;
  double tol;
  double* K;
  double* C;
  double* coh;
  float2* residual;  // complex64 [n, M] or NULL
};
size_t topofit_near_max_smem(bool fp64, int M, int n_half);
cudaError_t launch_topofit_near_max(const NearMaxArgs& a, bool fp64, int sm_count, cudaStream_t st);
// histogram_with_centers (pystamps/kernels/accelerated.py:235-265)
cudaError_t launch_hist_centers(const double* v, int64_t n, const double* mids, int nc, int equal, double d,
                                double cutoff0, unsigned long long* counts, int sm_count, cudaStream_t st);
cudaError_t launch_batch_bin(const BatchArgs& b, int64_t total, int sm_count, cudaStream_t st);
cudaError_t launch_batch_clap(const BatchArgs& b, int64_t total, const Twiddles32f& tf, int sm_count,
                              cudaStream_t st);
cudaError_t launch_batch_overlap(const BatchArgs& b, int64_t total, int sm_count, cudaStream_t st);
cudaError_t launch_batch_topofit(const BatchArgs& b, int L, const int32_t* units, int n_units, size_t smem,
                                 int sm_count, cudaStream_t st);
cudaError_t launch_batch_finalize(const BatchArgs& b, cudaStream_t st);
cudaError_t launch_batch_continue(cudaGraphConditionalHandle h, const int* n_active, cudaStream_t st);
cudaError_t launch_snr_weight(const TopoArgs& t, const float* amp, void* w_out, bool fp64, int sm_count,
                              cudaStream_t st);
cudaError_t launch_random_hist(const double* rnd, int64_t n_rand, const double* bp, int m, const int64_t* ia,
                               const int64_t* ib, int small_baseline, int n_half, double cutoff0, double dbin,
                               double2* phasors, int32_t* hist, int sm_count, cudaStream_t st);  // phasors: [m * (2*n_half+1)]

// layout helpers
cudaError_t launch_gather_rows(const void* src, void* dst, const int32_t* perm, int64_t n, int64_t row_bytes,
                               cudaStream_t st);
cudaError_t launch_scatter_rows(const void* src, void* dst, const int32_t* perm, int64_t n, int64_t row_bytes,
                                cudaStream_t st);
cudaError_t launch_unpad_grid(const void* src, void* dst, int64_t G, int M, int Mp, int elem_bytes, cudaStream_t st);
cudaError_t launch_pad_grid(const void* src, void* dst, int64_t G, int M, int Mp, int elem_bytes, cudaStream_t st);
cudaError_t launch_init_state(const double* w0, const int32_t* perm, int64_t N, void* K, void* w, void* coh,
                              bool fp64, cudaStream_t st);
cudaError_t launch_ph_weight(const BinArgs& a, int64_t N, bool fp64, const int32_t* perm, void* out_orig,
                             cudaStream_t st);

}  // namespace ps2
