// Host side of libps2cuda: the stage-2 context (device-resident patch, the
// gamma loop driver) and the C ABI declared in include/ps2cuda.h.
//
// Layout in HBM (per loaded patch; N PS, M interferograms, G = n_i*n_j cells,
// Mp = M rounded up to a multiple of 4, W CLAP windows):
//   ph_nm   complex64 [N, M]   rows stably sorted by grid cell (counting sort)
//   bp      f32 [N, M] sorted (or [M] when every row has the same baselines)
//   K[2]    real [N]           ping-pong: K used by this iteration's binning /
//                              K written by this iteration's topofit
//   w, coh, C                  real [N], nopt u8 [N]
//   grid    complex [G, Mp]    binned phase (the reference's ph_grid)
//   win     complex [W, 576, Mp] weighted CLAP window outputs
//   filt    complex [G, Mp]    CLAP-filtered grid
// Real/complex are f32/complex64 for PS2_PRECISION_FP32 and f64/complex128
// for PS2_PRECISION_FP64.
#include <cuda_runtime.h>
#include <sched.h>

#include <algorithm>
#include <cmath>
#include <cstdarg>
#include <mutex>
#include <cstdio>
#include <cstring>
#include <cstdlib>
#include <string>
#include <system_error>
#include <thread>
#include <vector>

#include "../../include/ps2cuda.h"
#include "interp10_taps.h"
#include "ps2_kernels.cuh"

using namespace ps2;

namespace {

thread_local std::string g_err;

int set_err(int code, const char* fmt, ...) {
  char buf[512];
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(buf, sizeof(buf), fmt, ap);
  va_end(ap);
  g_err = buf;
  return code;
}

#define CK(call)                                                                                              \
  do {                                                                                                        \
    cudaError_t e__ = (call);                                                                                 \
    if (e__ != cudaSuccess) {                                                                                 \
      return set_err(e__ == cudaErrorMemoryAllocation ? PS2_ERR_OUT_OF_MEMORY : PS2_ERR_CUDA, "%s: %s (%s:%d)", \
                     #call, cudaGetErrorString(e__), __FILE__, __LINE__);                                     \
    }                                                                                                         \
  } while (0)

// Device allocation owned by a context.
struct DevBuf {
  void* p = nullptr;
  size_t bytes = 0;
  DevBuf() = default;
  DevBuf(const DevBuf&) = delete;
  DevBuf& operator=(const DevBuf&) = delete;
  ~DevBuf() { release(); }
  // keeps the current allocation when it is large enough (a context reloads
  // patches without returning to cudaMalloc/cudaFree, which synchronise)
  cudaError_t alloc(size_t n) {
    if (n == 0) n = 16;
    if (p && bytes >= n) return cudaSuccess;
    release();
    cudaError_t e = cudaMalloc(&p, n);
    if (e == cudaSuccess) bytes = n;
    else p = nullptr;
    return e;
  }
  void release() {
    if (p) cudaFree(p);
    p = nullptr;
    bytes = 0;
  }
  template <typename T>
  T* as() const { return static_cast<T*>(p); }
};

// MATLAB rand('state', seed) / v5 uniform generator (native_stage2.rs:1785-1873):
// 32-word subtract-with-borrow lagged-Fibonacci state, xorshift-32 mantissa
// scrambling of the 53-bit result.
class V5Uniform {
 public:
  explicit V5Uniform(uint32_t seed) : j_(seed == 0 ? (1u << 31) : seed) {
    uint32_t s = j_;
    for (int k = 0; k < 32; ++k) {
      uint64_t x = 0;
      for (int b = 0; b < 53; ++b) {
        s = xs32(s);
        x = (x << 1) | ((s >> 19) & 1u);
      }
      st_[k] = static_cast<double>(x) * kUlp;
    }
  }
  double next() {
    double v = st_[(ix_ + 20) & 31] - st_[(ix_ + 5) & 31] - borrow_;
    if (v < 0.0) {
      v += 1.0;
      borrow_ = kUlp;
    } else {
      borrow_ = 0.0;
    }
    st_[ix_] = v;
    ix_ = (ix_ + 1) & 31;
    const uint32_t lo = j_, hi = xs32(lo);
    j_ = hi;
    const uint64_t mask = ((static_cast<uint64_t>(hi) << 32) & ((uint64_t(1) << 52) - 1)) ^ lo;
    if (v == 0.0) return std::ldexp(static_cast<double>(mask), -53);
    uint64_t bits;
    std::memcpy(&bits, &v, 8);
    const int eb = static_cast<int>((bits >> 52) & 0x7ff);
    uint64_t mant = bits & ((uint64_t(1) << 52) - 1);
    int ex;
    if (eb == 0) {
      const int lead = 63 - __builtin_clzll(mant);
      ex = lead - 1073;
      mant <<= (52 - lead);
    } else {
      ex = eb - 1022;
      mant |= (uint64_t(1) << 52);
    }
    return std::ldexp(static_cast<double>(mant ^ mask), ex - 53);
  }

 private:
  static constexpr double kUlp = 1.1102230246251565e-16;  // 2^-53
  static uint32_t xs32(uint32_t v) {
    v ^= v << 13;
    v ^= v >> 17;
    v ^= v << 5;
    return v;
  }
  double st_[32];
  int ix_ = 0;
  double borrow_ = 0.0;
  uint32_t j_;
};

void coh_bin_rule(double* cutoff0, double* d) {
  // centres 0.005 + 0.01*i (native_stage2.rs:510-512), equal-spacing rule (:1593-1607)
  const double c0 = 0.005 + 0.01 * 0.0, c1 = 0.005 + 0.01 * 1.0, c99 = 0.005 + 0.01 * 99.0;
  *d = (c99 - c0) / 99.0;
  *cutoff0 = (c0 + c1) / 2.0;
}

void gauss7(double* g, double* sum) {
  // gausswin(7, 2.5) (native_stage2.rs:1685-1699); the same values are the
  // CLAP |H| smoothing taps (:1044-1053)
  const double sd = (7.0 - 1.0) / (2.0 * 2.5);
  double s = 0.0;
  for (int i = 0; i < 7; ++i) {
    const double x = static_cast<double>(i) - 3.0;
    g[i] = std::exp(-0.5 * (x / sd) * (x / sd));
    s += g[i];
  }
  if (sum) *sum = s;
}

void twiddles(Twiddles32f* tf, Twiddles32d* td) {
  for (int k = 0; k < 16; ++k) {
    const double a = -2.0 * M_PI * k / 32.0;
    td->w[k] = make_double2(std::cos(a), std::sin(a));
    tf->w[k] = make_float2(static_cast<float>(std::cos(a)), static_cast<float>(std::sin(a)));
  }
}

// pyramid overlap weight (clap_window_weight, native_stage2.rs:1014-1037) / n_ex^2
std::vector<double> window_weight_scaled(int n_win, int n_ex) {
  const int h = n_win / 2;
  std::vector<double> out(static_cast<size_t>(n_win) * n_win, 0.0);
  for (int r = 0; r < h; ++r)
    for (int c = 0; c < h; ++c) {
      out[r * n_win + c] = static_cast<double>(r) + static_cast<double>(c) + 1.0e-6;
      out[r * n_win + h + c] = static_cast<double>(r) + static_cast<double>(h - 1 - c) + 1.0e-6;
    }
  for (int r = 0; r < h; ++r)
    for (int c = 0; c < n_win; ++c) out[(h + r) * n_win + c] = out[(h - 1 - r) * n_win + c];
  const double inv = 1.0 / static_cast<double>(n_ex * n_ex);
  for (auto& v : out) v *= inv;
  return out;
}

// Launch shapes chosen by ps2_autotune, kept process-wide per (interferogram
// bucket, PS bucket, precision): the FP32 topofit's lanes per PS, CLAP's warps
// per block and resident blocks per SM, binning's resident blocks per SM
// (0 everywhere: the built-in rules).
struct TuneShape {
  int lanes = 0, clap_nw = 0, clap_bps = 0, bin_bps = 0, clap_fused = 0;
};
std::mutex g_tune_mu;
std::vector<std::pair<int64_t, TuneShape>> g_tune_cache;
int64_t tune_key(int64_t M, int64_t N, bool fp64) {
  int64_t lb = 0;
  while ((int64_t(1) << lb) < N) ++lb;
  return (((M + 7) / 8) * 64 + lb) * 2 + (fp64 ? 1 : 0);
}
bool tune_lookup(int64_t key, TuneShape* out) {
  std::lock_guard<std::mutex> g(g_tune_mu);
  for (auto& kv : g_tune_cache)
    if (kv.first == key) {
      *out = kv.second;
      return true;
    }
  return false;
}
void tune_store(int64_t key, const TuneShape& v) {
  std::lock_guard<std::mutex> g(g_tune_mu);
  for (auto& kv : g_tune_cache)
    if (kv.first == key) {
      kv.second = v;
      return;
    }
  g_tune_cache.emplace_back(key, v);
}

}  // namespace

struct ps2_ctx {
  int device = 0;
  int sm_count = 148;
  cudaStream_t st = nullptr;
  bool loaded = false;
  bool fp64 = false;
  int64_t N = 0, G = 0;
  int M = 0, Mp = 0, n_i = 0, n_j = 0, n_win = 24, n_inc = 6, nwi = 0, nwj = 0, nchunk = 0, n_half = 0;
  int bp_row_inv = 0, psquare = 1, low_coh_thresh = 31, alpha_is_one = 1;
  double alpha = 1.0, beta = 0.3, conv = 0.005, nr_max_nz_ix = 1.0;
  int64_t max_iter = 25;
  double cutoff0 = 0.01, dbin = 0.01;
  double g7[7], g7sum = 0.0;
  Twiddles32f twf;
  Twiddles32d twd;
  DevBuf ph_nm, bp, amp, perm, cell_start, cell_of, w0, K[2], w, coh, C, nopt, grid, win, wpart, filt, low_pass, wscaled,
      taps, lut, nr0, nr_scaled, state, stats, hist, n_invalid, rms_partial, ph_res, scratch, stage;
  // differentiable coherence (ps2_coherence_forward / _backward): own buffers,
  // the loop state above is left untouched
  DevBuf ad_ph, ad_K, ad_w, ad_coh, ad_grid, ad_win, ad_filt, ad_gfilt, ad_gph, ad_gK, ad_gf, ad_part;
  int ad_blocks = 0, ad_blocks64 = 0;
  cudaEvent_t ad_ev = nullptr;
  // stage-3 re-estimate from the loaded patch (ps2_stage3_reestimate): for
  // each row in the caller's order, its cell-sorted position and its cell
  std::vector<int32_t> h_sorted_pos, h_cell;
  int64_t gmax_i = 0, gmax_j = 0;
  // ps2_load_patch: the phase and bperp rows go up on this copy stream while the
  // host sorts the rows by cell
  cudaStream_t cst = nullptr;
  cudaEvent_t ev_ph = nullptr, ev_bp = nullptr;
  DevBuf stage_bp;
  // batches led by this context (ps2_batch_run): per-patch arguments and tables
  DevBuf bt;
  int* h_active = nullptr;  // pinned [1]
  cudaGraph_t loop_graph = nullptr;
  cudaGraphExec_t loop_exec = nullptr;
  bool graph_failed = false;
  bool last_run_graph = false;
  int64_t graph_body_launches = 0;
  int topo_lanes = 0;  // 0: rule from n_ifg; else chosen by ps2_autotune
  int clap_nw = 0, clap_bps = 0, bin_bps = 0;  // launch shapes (0: built-in rules)
  int clap_fused = 0;  // CLAP form: 0 window stack + overlap-add pass, 1 window blocks into partials + combine
  int topo_blocks = 0;
  int64_t iters_done = 0;  // since load/reset
  double* h_stats = nullptr;  // pinned [8]
  ps2_iter_stats last{};
  double last_ms = 0.0, kernel_ms[4] = {0, 0, 0, 0};
  int64_t launches = 0;
  std::vector<cudaEvent_t> evpool;
};

namespace {

size_t rsz(const ps2_ctx* c) { return c->fp64 ? sizeof(double) : sizeof(float); }
size_t csz(const ps2_ctx* c) { return 2 * rsz(c); }

int ensure_events(ps2_ctx* c, size_t n) {
  while (c->evpool.size() < n) {
    cudaEvent_t e;
    CK(cudaEventCreate(&e));
    c->evpool.push_back(e);
  }
  return PS2_OK;
}

BinArgs bin_args(ps2_ctx* c, int mode, const void* K) {
  BinArgs a{};
  a.ph_nm = c->ph_nm.p;
  a.bp = c->bp.as<float>();
  a.bp_row_inv = c->bp_row_inv;
  a.cell_start = c->cell_start.as<int32_t>();
  a.G = c->G;
  a.M = c->M;
  a.Mp = c->Mp;
  a.nchunk = c->nchunk;
  a.K = K;
  a.w = c->w.p;
  a.coh = c->coh.p;
  a.lut = c->lut.as<double>();
  a.lut_len = 1001;
  a.mode = mode;
  a.grid = c->grid.p;
  a.blocks_per_sm = c->bin_bps;
  return a;
}

ClapArgs clap_args(ps2_ctx* c, const void* grid, void* win) {
  ClapArgs a{};
  a.grid = grid;
  a.n_i = c->n_i;
  a.n_j = c->n_j;
  a.M = c->M;
  a.Mp = c->Mp;
  a.n_win = c->n_win;
  a.nwi = c->nwi;
  a.nwj = c->nwj;
  a.alpha_is_one = c->alpha_is_one;
  a.alpha = c->alpha;
  a.beta = c->beta;
  a.low_pass = c->low_pass.as<double>();
  a.wscaled = c->wscaled.as<double>();
  for (int i = 0; i < 7; ++i) a.g7[i] = c->g7[i];
  a.win_out = win;
  a.nw_block = c->clap_nw;
  a.blocks_per_sm = c->clap_bps;
  return a;
}

OverlapArgs overlap_args(ps2_ctx* c, const void* win, void* filt) {
  OverlapArgs o{};
  o.win_out = win;
  o.filt = filt;
  o.n_i = c->n_i;
  o.n_j = c->n_j;
  o.M = c->M;
  o.Mp = c->Mp;
  o.n_win = c->n_win;
  o.n_inc = c->n_inc;
  o.nwi = c->nwi;
  o.nwj = c->nwj;
  return o;
}

// The loop's CLAP in the context's form: windows into the window stack and
// the overlap-add pass, or window blocks into the partials and the combine
// pass (the same sums in another association: the forms agree to the last bit
// wherever the FP64 partial sums are exact, as they are for the window values
// of a patch). The adjoint keeps the window stack its backward pass reads.
ClapArgs clap_args_loop(ps2_ctx* c, const void* grid, int fused) {
  ClapArgs a = clap_args(c, grid, fused ? nullptr : c->win.p);
  if (fused) a.part = c->wpart.p;
  return a;
}

OverlapArgs overlap_args_loop(ps2_ctx* c, void* filt, int fused) {
  OverlapArgs o = overlap_args(c, fused ? nullptr : c->win.p, filt);
  if (fused) o.part = c->wpart.p;
  return o;
}

TopoArgs topo_args(ps2_ctx* c, void* K_out, void* C_out, void* coh_io) {
  TopoArgs t{};
  t.ph_nm = c->ph_nm.p;
  t.filt = c->filt.p;
  t.cell_of = c->cell_of.as<int32_t>();
  t.cpx = nullptr;
  t.bp = c->bp.as<float>();
  t.bp_row_inv = c->bp_row_inv;
  t.N = c->N;
  t.M = c->M;
  t.Mp = c->Mp;
  t.n_half = c->n_half;
  t.zero_mode = 0;
  t.filt_unit = c->fp64 ? 0 : 1;  // the loop's k_overlap stores f/|f| in FP32
  t.K_out = K_out;
  t.C_out = C_out;
  t.coh_io = coh_io;
  t.nopt = c->nopt.as<uint8_t>();
  t.rms_partial = c->rms_partial.as<double>();
  t.hist = c->hist.as<int32_t>();
  t.n_invalid = c->n_invalid.as<int32_t>();
  t.cutoff0 = c->cutoff0;
  t.dbin = c->dbin;
  t.accumulate_stats = 1;
  t.lanes = c->topo_lanes;
  return t;
}

// CLAP window geometry shared by the context and the stateless entry point.
int clap_geometry(int64_t n_i, int64_t n_j, int64_t n_win, int* n_inc, int* nwi, int* nwj) {
  if (n_win < 4 || n_win > 32) return set_err(PS2_ERR_UNSUPPORTED, "CLAP window %lld unsupported (4..32)", (long long)n_win);
  *n_inc = static_cast<int>(std::max<int64_t>(n_win / 4, 1));
  const int64_t a = static_cast<int64_t>(std::ceil(static_cast<double>(n_i) / *n_inc)) - 3;
  const int64_t b = static_cast<int64_t>(std::ceil(static_cast<double>(n_j) / *n_inc)) - 3;
  if (a > 0 && b > 0 && (n_i < n_win || n_j < n_win))
    return set_err(PS2_ERR_INVALID_ARG,
                   "grid %lldx%lld is smaller than the %lld-cell CLAP window but yields windows "
                   "(the reference's window placement underflows for 19-23 cells per side)",
                   (long long)n_i, (long long)n_j, (long long)n_win);
  *nwi = a > 0 && b > 0 ? static_cast<int>(a) : 0;
  *nwj = a > 0 && b > 0 ? static_cast<int>(b) : 0;
  return PS2_OK;
}

int copy_in(ps2_ctx* c, DevBuf& dst, const void* src, size_t bytes, bool on_device) {
  CK(dst.alloc(bytes));
  CK(cudaMemcpyAsync(dst.p, src, bytes, on_device ? cudaMemcpyDeviceToDevice : cudaMemcpyHostToDevice, c->st));
  return PS2_OK;
}

FinalizeArgs finalize_args(ps2_ctx* c, bool force_continue) {
  FinalizeArgs f{};
  f.rms_partial = c->rms_partial.as<double>();
  f.n_partial = c->topo_blocks;  // unlaunched blocks' partials stay zero
  f.N = c->N;
  f.hist = c->hist.as<int32_t>();
  f.nr_scaled = c->nr_scaled.as<double>();
  f.nr_max_nz_ix = c->nr_max_nz_ix;
  f.low_coh_thresh = c->low_coh_thresh;
  f.psquare = c->psquare;
  f.gamma_change_convergence = c->conv;
  f.gamma_max_iterations = c->max_iter;
  for (int i = 0; i < 7; ++i) f.g7w[i] = c->g7[i];
  f.g7sum = c->g7sum;
  f.taps79 = c->taps.as<double>();
  f.lut = c->lut.as<double>();
  f.state = c->state.as<double>();
  f.stats_out = c->stats.as<double>();
  f.n_invalid = c->n_invalid.as<int32_t>();
  f.force_continue = force_continue ? 1 : 0;
  return f;
}

// Queues one gamma iteration on the context's stream. `later` selects the form
// of iterations 2.. (P-square weights from the previous table, or the SNR
// weight kernel); `capturing` queues into a graph without touching counters.
int enqueue_iteration(ps2_ctx* c, bool later, bool force_continue, cudaEvent_t* ev, int64_t* launched_out) {
  const bool fp64 = c->fp64;
  int64_t launched = 0;
  if (ev) CK(cudaEventRecord(ev[0], c->st));
  if (!c->psquare && later) {
    TopoArgs t = topo_args(c, nullptr, nullptr, nullptr);
    t.ph_res = c->ph_res.p;
    CK(launch_snr_weight(t, c->amp.as<float>(), c->w.p, fp64, c->sm_count, c->st));
    ++launched;
  }
  CK(cudaMemsetAsync(c->hist.p, 0, sizeof(int32_t) * PS2_COH_BINS, c->st));
  CK(cudaMemsetAsync(c->n_invalid.p, 0, sizeof(int32_t), c->st));
  CK(cudaMemsetAsync(c->rms_partial.p, 0, sizeof(double) * c->topo_blocks, c->st));
  if (later && c->psquare) {
    // the P-square weights of this iteration, then binning with them (mode 0)
    CK(launch_psquare_weights(bin_args(c, 1, c->K[0].p), c->N, fp64, c->sm_count, c->st));
    ++launched;
  }
  CK(launch_bin(bin_args(c, 0, c->K[0].p), fp64, c->sm_count, c->st));
  ++launched;
  if (ev) CK(cudaEventRecord(ev[1], c->st));
  CK(launch_clap(clap_args_loop(c, c->grid.p, c->clap_fused), fp64, c->twf, c->twd, c->sm_count, c->st));
  OverlapArgs ov = overlap_args_loop(c, c->filt.p, c->clap_fused);
  ov.normalize = fp64 ? 0 : 1;
  CK(launch_overlap(ov, fp64, c->st));
  launched += 2;
  if (ev) CK(cudaEventRecord(ev[2], c->st));
  // K[1] keeps the K this iteration binned with (pm1's ph_weight needs it);
  // topofit then rewrites K[0] in place
  CK(cudaMemcpyAsync(c->K[1].p, c->K[0].p, rsz(c) * c->N, cudaMemcpyDeviceToDevice, c->st));
  TopoArgs t = topo_args(c, c->K[0].p, c->C.p, c->coh.p);
  if (!c->psquare) t.ph_res = c->ph_res.p;
  CK(launch_topofit(t, fp64, c->topo_blocks, c->st));
  ++launched;
  if (ev) CK(cudaEventRecord(ev[3], c->st));
  CK(launch_finalize(finalize_args(c, force_continue), c->st));
  ++launched;
  if (ev) CK(cudaEventRecord(ev[4], c->st));
  if (launched_out) *launched_out = launched;
  return PS2_OK;
}

int run_one_iteration(ps2_ctx* c, bool force_continue, cudaEvent_t* ev) {
  int64_t launched = 0;
  int rc = enqueue_iteration(c, c->iters_done > 0, force_continue, ev, &launched);
  if (rc) return rc;
  c->iters_done += 1;
  c->launches += launched;
  return PS2_OK;
}

void drop_loop_graph(ps2_ctx* c) {
  if (c->loop_exec) cudaGraphExecDestroy(c->loop_exec);
  if (c->loop_graph) cudaGraphDestroy(c->loop_graph);
  c->loop_exec = nullptr;
  c->loop_graph = nullptr;
}

// The loop from iteration 2 on as one graph: a WHILE conditional node whose
// body is one iteration followed by k_loop_continue, which clears the
// condition when finalize raised the stop flag (native_stage2.rs:312-314).
int build_loop_graph(ps2_ctx* c, int64_t* body_launches) {
  cudaGraph_t g = nullptr;
  CK(cudaGraphCreate(&g, 0));
  c->loop_graph = g;
  cudaGraphConditionalHandle h;
  CK(cudaGraphConditionalHandleCreate(&h, g, 1, cudaGraphCondAssignDefault));
  cudaGraphNodeParams p{};
  p.type = cudaGraphNodeTypeConditional;
  p.conditional.handle = h;
  p.conditional.type = cudaGraphCondTypeWhile;
  p.conditional.size = 1;
  cudaGraphNode_t node;
  CK(cudaGraphAddNode(&node, g, nullptr, 0, &p));
  cudaGraph_t body = p.conditional.phGraph_out[0];
  CK(cudaStreamBeginCaptureToGraph(c->st, body, nullptr, nullptr, 0, cudaStreamCaptureModeThreadLocal));
  int64_t launched = 0;
  int rc = enqueue_iteration(c, true, false, nullptr, &launched);
  cudaError_t e2 = rc ? cudaSuccess : launch_loop_continue(h, c->stats.as<double>(), c->st);
  cudaGraph_t captured = nullptr;
  cudaError_t e3 = cudaStreamEndCapture(c->st, &captured);
  if (rc) return rc;
  CK(e2);
  CK(e3);
  CK(cudaGraphInstantiate(&c->loop_exec, g, 0));
  *body_launches = launched + 1;
  return PS2_OK;
}

void fill_stats(const double* h, ps2_iter_stats* s) {
  s->i_loop = static_cast<int64_t>(h[0]);
  s->gamma_change_rms = h[1];
  s->gamma_change_delta = h[2];
  s->stop = h[3] != 0.0 ? 1 : 0;
  s->n_invalid = static_cast<int32_t>(h[4]);
}

int reset_state(ps2_ctx* c) {
  CK(launch_init_state(c->w0.as<double>(), c->perm.as<int32_t>(), c->N, c->K[0].p, c->w.p, c->coh.p, c->fp64, c->st));
  CK(cudaMemsetAsync(c->K[1].p, 0, rsz(c) * c->N, c->st));
  CK(cudaMemcpyAsync(c->nr_scaled.p, c->nr0.p, sizeof(double) * PS2_COH_BINS, cudaMemcpyDeviceToDevice, c->st));
  double st0[4] = {0.0, 1.0, 0.0, 0.0};
  CK(cudaMemcpyAsync(c->state.p, st0, sizeof(st0), cudaMemcpyHostToDevice, c->st));
  CK(cudaStreamSynchronize(c->st));
  c->iters_done = 0;
  c->last = ps2_iter_stats{};
  return PS2_OK;
}

// Checkpoint blob of the gamma loop (ps2_export_state / ps2_import_state).
struct StateHeader {
  char magic[8];  // "PS2LOOP\0"
  int32_t version, fp64, psquare, reserved;
  int64_t N, M, G, iters_done;
  ps2_iter_stats last;
};
constexpr int32_t kStateVersion = 1;

// The loop state after an iteration, in the blob's order: K (current), K
// binned with, w, coh, C (real [N] each), N_opt (u8 [N]), the P-square table
// (f64 [1001]), scaled Nr (f64 [100]), the convergence state (f64 [4]) and the
// last statistics record (f64 [8]); with SNR weighting also ph_res (real [N, M]).
struct StatePart {
  DevBuf* buf;
  size_t bytes;
};
std::vector<StatePart> state_parts(ps2_ctx* c) {
  const size_t R = rsz(c), N = static_cast<size_t>(c->N);
  std::vector<StatePart> v = {{&c->K[0], R * N}, {&c->K[1], R * N}, {&c->w, R * N},
                              {&c->coh, R * N},  {&c->C, R * N},    {&c->nopt, N},
                              {&c->lut, sizeof(double) * 1001},   {&c->nr_scaled, sizeof(double) * PS2_COH_BINS},
                              {&c->state, sizeof(double) * 4},    {&c->stats, sizeof(double) * 8}};
  if (!c->psquare) v.push_back({&c->ph_res, R * N * static_cast<size_t>(c->M)});
  return v;
}
size_t state_bytes(ps2_ctx* c) {
  size_t b = sizeof(StateHeader);
  for (const auto& p : state_parts(c)) b += p.bytes;
  return b;
}

}  // namespace

// ====================================================================== ABI
extern "C" {

const char* ps2_last_error(void) { return g_err.c_str(); }

int ps2_create(ps2_ctx** out, int device) {
  if (!out) return set_err(PS2_ERR_INVALID_ARG, "ps2_create: out is NULL");
  int ndev = 0;
  CK(cudaGetDeviceCount(&ndev));
  if (device < 0 || device >= ndev) return set_err(PS2_ERR_INVALID_ARG, "device %d out of range (%d devices)", device, ndev);
  CK(cudaSetDevice(device));
  ps2_ctx* c = new ps2_ctx();
  c->device = device;
  cudaDeviceProp prop;
  cudaError_t e = cudaGetDeviceProperties(&prop, device);
  if (e != cudaSuccess) {
    delete c;
    return set_err(PS2_ERR_CUDA, "cudaGetDeviceProperties: %s", cudaGetErrorString(e));
  }
  c->sm_count = prop.multiProcessorCount;
  e = cudaStreamCreateWithFlags(&c->st, cudaStreamNonBlocking);
  if (e == cudaSuccess) e = cudaMallocHost(reinterpret_cast<void**>(&c->h_stats), 8 * sizeof(double));
  if (e != cudaSuccess) {
    if (c->st) cudaStreamDestroy(c->st);
    delete c;
    return set_err(PS2_ERR_CUDA, "ps2_create: %s", cudaGetErrorString(e));
  }
  twiddles(&c->twf, &c->twd);
  gauss7(c->g7, &c->g7sum);
  coh_bin_rule(&c->cutoff0, &c->dbin);
  *out = c;
  return PS2_OK;
}

void ps2_destroy(ps2_ctx* c) {
  if (!c) return;
  cudaSetDevice(c->device);
  if (c->st) cudaStreamSynchronize(c->st);
  DevBuf* bufs[] = {&c->ph_nm, &c->bp, &c->amp, &c->perm, &c->cell_start, &c->cell_of, &c->w0, &c->K[0], &c->K[1],
                    &c->w, &c->coh, &c->C, &c->nopt, &c->grid, &c->win, &c->wpart, &c->filt, &c->low_pass, &c->wscaled,
                    &c->taps, &c->lut, &c->nr0, &c->nr_scaled, &c->state, &c->stats, &c->hist, &c->n_invalid,
                    &c->rms_partial, &c->ph_res, &c->scratch, &c->stage, &c->ad_ph, &c->ad_K, &c->ad_w,
                    &c->ad_coh, &c->ad_grid, &c->ad_win, &c->ad_filt, &c->ad_gfilt, &c->ad_gph, &c->ad_gK,
                    &c->ad_gf, &c->ad_part};
  for (DevBuf* b : bufs) b->release();
  drop_loop_graph(c);
  for (cudaEvent_t e : c->evpool) cudaEventDestroy(e);
  if (c->ad_ev) cudaEventDestroy(c->ad_ev);
  c->stage_bp.release();
  if (c->ev_ph) cudaEventDestroy(c->ev_ph);
  if (c->ev_bp) cudaEventDestroy(c->ev_bp);
  if (c->cst) cudaStreamDestroy(c->cst);
  c->bt.release();
  if (c->h_active) cudaFreeHost(c->h_active);
  if (c->h_stats) cudaFreeHost(c->h_stats);
  if (c->st) cudaStreamDestroy(c->st);
  delete c;
}

int ps2_load_patch(ps2_ctx* c, const ps2_patch_desc* d) {
  if (!c || !d) return set_err(PS2_ERR_INVALID_ARG, "ps2_load_patch: NULL argument");
  if (d->n_ps <= 0 || d->n_ifg <= 0) return set_err(PS2_ERR_INVALID_ARG, "n_ps and n_ifg must be positive");
  if (d->n_ifg > 256) return set_err(PS2_ERR_UNSUPPORTED, "n_ifg %lld > 256 is not supported", (long long)d->n_ifg);
  if (d->n_ps > INT32_MAX - 1) return set_err(PS2_ERR_UNSUPPORTED, "n_ps too large");
  if (!d->ph_nm || !d->bperp || !d->grid_lin || !d->weight0 || !d->low_pass || !d->nr)
    return set_err(PS2_ERR_INVALID_ARG, "ps2_load_patch: a required array is NULL");
  if (d->n_i <= 0 || d->n_j <= 0) return set_err(PS2_ERR_INVALID_ARG, "grid size must be positive");
  if (d->n_win_ex != 32) return set_err(PS2_ERR_UNSUPPORTED, "CLAP FFT size %lld unsupported (32)", (long long)d->n_win_ex);
  if (d->precision != PS2_PRECISION_FP32 && d->precision != PS2_PRECISION_FP64)
    return set_err(PS2_ERR_INVALID_ARG, "unknown precision %d", d->precision);
  if (!d->psquare && !d->amp) return set_err(PS2_ERR_INVALID_ARG, "SNR weighting needs amp");
  if (d->low_coh_thresh < 0 || d->low_coh_thresh > PS2_COH_BINS)
    return set_err(PS2_ERR_INVALID_ARG, "low_coh_thresh %lld outside 0..100", (long long)d->low_coh_thresh);
  if (!(d->n_trial_wraps >= 0.0) || d->n_trial_wraps > 1.0e4)
    return set_err(PS2_ERR_INVALID_ARG, "n_trial_wraps %g out of range", d->n_trial_wraps);
  CK(cudaSetDevice(c->device));
  int n_inc, nwi, nwj;
  int rc = clap_geometry(d->n_i, d->n_j, d->clap_window, &n_inc, &nwi, &nwj);
  if (rc) return rc;
  c->loaded = false;
  drop_loop_graph(c);
  c->graph_failed = false;
  c->fp64 = d->precision == PS2_PRECISION_FP64;
  c->N = d->n_ps;
  c->M = static_cast<int>(d->n_ifg);
  c->Mp = (c->M + 3) & ~3;
  c->n_i = static_cast<int>(d->n_i);
  c->n_j = static_cast<int>(d->n_j);
  c->G = d->n_i * d->n_j;
  c->n_win = static_cast<int>(d->clap_window);
  c->n_inc = n_inc;
  c->nwi = nwi;
  c->nwj = nwj;
  c->nchunk = (c->M + 31) / 32;
  c->n_half = static_cast<int>(std::ceil(8.0 * d->n_trial_wraps));
  c->bp_row_inv = d->bperp_row_invariant ? 1 : 0;
  c->psquare = d->psquare ? 1 : 0;
  c->low_coh_thresh = static_cast<int>(d->low_coh_thresh);
  c->alpha = d->clap_alpha;
  c->beta = d->clap_beta;
  c->alpha_is_one = std::fabs(d->clap_alpha - 1.0) <= 2.220446049250313e-16 ? 1 : 0;
  c->conv = d->gamma_change_convergence;
  c->max_iter = d->gamma_max_iterations;
  c->nr_max_nz_ix = d->nr_max_nz_ix;
  const bool dev = d->pointers_on_device != 0;
  const int64_t N = c->N, M = c->M, G = c->G;

  // The phase rows (and per-row bperp) start up the copy stream first, so the
  // transfer overlaps the host's cell sort; the gathers below wait for them.
  // Every return from here on waits for these copies (the caller's buffers are
  // not kept past the call).
  if (!c->cst) CK(cudaStreamCreateWithFlags(&c->cst, cudaStreamNonBlocking));
  if (!c->ev_ph) CK(cudaEventCreateWithFlags(&c->ev_ph, cudaEventDisableTiming));
  if (!c->ev_bp) CK(cudaEventCreateWithFlags(&c->ev_bp, cudaEventDisableTiming));
  CK(cudaStreamSynchronize(c->st));
  struct CopyJoin {
    cudaStream_t s;
    ~CopyJoin() { cudaStreamSynchronize(s); }
  } join{c->cst};
  const cudaMemcpyKind kind = dev ? cudaMemcpyDeviceToDevice : cudaMemcpyHostToDevice;
  CK(c->stage.alloc(sizeof(float) * 2 * N * M));
  CK(cudaMemcpyAsync(c->stage.p, d->ph_nm, sizeof(float) * 2 * N * M, kind, c->cst));
  CK(cudaEventRecord(c->ev_ph, c->cst));
  if (!c->bp_row_inv) {
    CK(c->stage_bp.alloc(sizeof(float) * N * M));
    CK(cudaMemcpyAsync(c->stage_bp.p, d->bperp, sizeof(float) * N * M, kind, c->cst));
    CK(cudaEventRecord(c->ev_bp, c->cst));
  }

  // stable counting sort of rows by cell (host)
  std::vector<int64_t> gl(N);
  if (dev)
    CK(cudaMemcpy(gl.data(), d->grid_lin, sizeof(int64_t) * N, cudaMemcpyDeviceToHost));
  else
    std::memcpy(gl.data(), d->grid_lin, sizeof(int64_t) * N);
  std::vector<int32_t> start(G + 1, 0), perm(N), cell_of(N);
  for (int64_t r = 0; r < N; ++r) {
    if (gl[r] < 0 || gl[r] >= G)
      return set_err(PS2_ERR_INVALID_ARG, "grid_lin[%lld] = %lld outside the %lldx%lld grid", (long long)r,
                     (long long)gl[r], (long long)c->n_i, (long long)c->n_j);
    start[gl[r] + 1] += 1;
  }
  for (int64_t g = 0; g < G; ++g) start[g + 1] += start[g];
  c->h_sorted_pos.resize(static_cast<size_t>(N));
  c->h_cell.resize(static_cast<size_t>(N));
  c->gmax_i = 0;
  c->gmax_j = 0;
  {
    std::vector<int32_t> fillp(start.begin(), start.end() - 1);
    for (int64_t r = 0; r < N; ++r) {
      const int32_t s = fillp[gl[r]]++;
      perm[s] = static_cast<int32_t>(r);
      cell_of[s] = static_cast<int32_t>(gl[r]);
      c->h_sorted_pos[r] = s;
      c->h_cell[r] = static_cast<int32_t>(gl[r]);
    }
  }
  // largest 1-based grid row and column holding a PS (from the occupied cells)
  for (int64_t g = 0; g < G; ++g) {
    if (start[g + 1] == start[g]) continue;
    c->gmax_i = std::max<int64_t>(c->gmax_i, g / c->n_j + 1);
    c->gmax_j = std::max<int64_t>(c->gmax_j, g % c->n_j + 1);
  }

  const size_t R = rsz(c), Cz = csz(c);
  CK(c->perm.alloc(sizeof(int32_t) * N));
  CK(cudaMemcpyAsync(c->perm.p, perm.data(), sizeof(int32_t) * N, cudaMemcpyHostToDevice, c->st));
  CK(c->cell_start.alloc(sizeof(int32_t) * (G + 1)));
  CK(cudaMemcpyAsync(c->cell_start.p, start.data(), sizeof(int32_t) * (G + 1), cudaMemcpyHostToDevice, c->st));
  CK(c->cell_of.alloc(sizeof(int32_t) * N));
  CK(cudaMemcpyAsync(c->cell_of.p, cell_of.data(), sizeof(int32_t) * N, cudaMemcpyHostToDevice, c->st));
  // row data, gathered into cell order on the device
  CK(c->ph_nm.alloc(sizeof(float) * 2 * N * M));
  CK(cudaStreamWaitEvent(c->st, c->ev_ph, 0));
  CK(launch_gather_rows(c->stage.p, c->ph_nm.p, c->perm.as<int32_t>(), N, sizeof(float) * 2 * M, c->st));
  if (c->bp_row_inv) {
    rc = copy_in(c, c->bp, d->bperp, sizeof(float) * M, dev);
    if (rc) return rc;
  } else {
    CK(c->bp.alloc(sizeof(float) * N * M));
    CK(cudaStreamWaitEvent(c->st, c->ev_bp, 0));
    CK(launch_gather_rows(c->stage_bp.p, c->bp.p, c->perm.as<int32_t>(), N, sizeof(float) * M, c->st));
  }
  if (!c->psquare) {
    rc = copy_in(c, c->stage, d->amp, sizeof(float) * N * M, dev);
    if (rc) return rc;
    CK(c->amp.alloc(sizeof(float) * N * M));
    CK(launch_gather_rows(c->stage.p, c->amp.p, c->perm.as<int32_t>(), N, sizeof(float) * M, c->st));
    CK(c->ph_res.alloc(R * N * M));
  } else {
    c->amp.release();
    c->ph_res.release();
  }
  rc = copy_in(c, c->w0, d->weight0, sizeof(double) * N, dev);
  if (rc) return rc;
  rc = copy_in(c, c->low_pass, d->low_pass, sizeof(double) * 32 * 32, dev);
  if (rc) return rc;
  rc = copy_in(c, c->nr0, d->nr, sizeof(double) * PS2_COH_BINS, dev);
  if (rc) return rc;
  // loop state and work buffers
  CK(c->K[0].alloc(R * N));
  CK(c->K[1].alloc(R * N));
  CK(c->w.alloc(R * N));
  CK(c->coh.alloc(R * N));
  CK(c->C.alloc(R * N));
  CK(c->nopt.alloc(N));
  CK(c->grid.alloc(Cz * G * c->Mp));
  CK(c->filt.alloc(Cz * G * c->Mp));
  const int64_t W = static_cast<int64_t>(nwi) * nwj;
  // CLAP's window stack (two-pass form) and window-block partial sums (fused
  // form, complex FP64): the launch shapes choose the form
  CK(c->win.alloc(Cz * std::max<int64_t>(W, 1) * c->n_win * c->n_win * c->Mp));
  CK(c->wpart.alloc(sizeof(double) * 2 * clap_part_elems(nwi, nwj, c->n_win, c->Mp)));
  if (W == 0) CK(cudaMemsetAsync(c->filt.p, 0, Cz * G * c->Mp, c->st));
  std::vector<double> ws = window_weight_scaled(c->n_win, 32);
  CK(c->wscaled.alloc(sizeof(double) * ws.size()));
  CK(cudaMemcpyAsync(c->wscaled.p, ws.data(), sizeof(double) * ws.size(), cudaMemcpyHostToDevice, c->st));
  CK(c->taps.alloc(sizeof(double) * 79));
  CK(cudaMemcpyAsync(c->taps.p, kStage2Interp10Taps, sizeof(double) * 79, cudaMemcpyHostToDevice, c->st));
  CK(c->lut.alloc(sizeof(double) * 1001));
  CK(cudaMemsetAsync(c->lut.p, 0, sizeof(double) * 1001, c->st));
  CK(c->nr_scaled.alloc(sizeof(double) * PS2_COH_BINS));
  CK(c->state.alloc(sizeof(double) * 4));
  CK(c->stats.alloc(sizeof(double) * 8));
  CK(c->hist.alloc(sizeof(int32_t) * PS2_COH_BINS));
  CK(c->n_invalid.alloc(sizeof(int32_t)));
  c->topo_blocks = topofit_grid_blocks(c->sm_count, c->fp64);
  {
    TuneShape ts;
    if (!tune_lookup(tune_key(c->M, c->N, c->fp64), &ts)) ts = TuneShape{};
    c->topo_lanes = ts.lanes;
    c->clap_nw = ts.clap_nw;
    c->clap_bps = ts.clap_bps;
    c->bin_bps = ts.bin_bps;
    c->clap_fused = ts.clap_fused;
  }
  CK(cudaMemsetAsync(c->filt.p, 0, Cz * G * c->Mp, c->st));
  CK(c->rms_partial.alloc(sizeof(double) * c->topo_blocks));
  rc = reset_state(c);
  if (rc) return rc;
  c->loaded = true;
  return PS2_OK;
}

int ps2_step(ps2_ctx* c, ps2_iter_stats* stats) {
  if (!c || !c->loaded) return set_err(PS2_ERR_NOT_LOADED, "no patch loaded");
  CK(cudaSetDevice(c->device));
  int rc = ensure_events(c, 5);
  if (rc) return rc;
  c->launches = 0;
  rc = run_one_iteration(c, false, c->evpool.data());
  if (rc) return rc;
  CK(cudaMemcpyAsync(c->h_stats, c->stats.p, 8 * sizeof(double), cudaMemcpyDeviceToHost, c->st));
  CK(cudaStreamSynchronize(c->st));
  float ms;
  c->last_ms = 0.0;
  for (int i = 0; i < 4; ++i) {
    CK(cudaEventElapsedTime(&ms, c->evpool[i], c->evpool[i + 1]));
    c->kernel_ms[i] = ms;
    c->last_ms += ms;
  }
  fill_stats(c->h_stats, &c->last);
  if (stats) *stats = c->last;
  return PS2_OK;
}

int ps2_reset(ps2_ctx* c) {
  if (!c || !c->loaded) return set_err(PS2_ERR_NOT_LOADED, "no patch loaded");
  CK(cudaSetDevice(c->device));
  return reset_state(c);
}

int ps2_iterate(ps2_ctx* c, int64_t n_iter, ps2_iter_stats* stats) {
  if (!c || !c->loaded) return set_err(PS2_ERR_NOT_LOADED, "no patch loaded");
  if (n_iter <= 0) return set_err(PS2_ERR_INVALID_ARG, "n_iter must be positive");
  CK(cudaSetDevice(c->device));
  int rc = ensure_events(c, static_cast<size_t>(5 * n_iter + 2));
  if (rc) return rc;
  std::vector<double> hs(static_cast<size_t>(8 * n_iter));
  c->launches = 0;
  cudaEvent_t span0 = c->evpool[5 * n_iter], span1 = c->evpool[5 * n_iter + 1];
  CK(cudaEventRecord(span0, c->st));
  for (int64_t k = 0; k < n_iter; ++k) {
    rc = run_one_iteration(c, true, &c->evpool[5 * k]);
    if (rc) return rc;
    CK(cudaMemcpyAsync(&c->h_stats[0], c->stats.p, 8 * sizeof(double), cudaMemcpyDeviceToHost, c->st));
    if (stats) {
      CK(cudaStreamSynchronize(c->st));
      std::memcpy(&hs[8 * k], c->h_stats, 8 * sizeof(double));
    }
  }
  CK(cudaEventRecord(span1, c->st));
  CK(cudaStreamSynchronize(c->st));
  if (!stats) std::memcpy(&hs[8 * (n_iter - 1)], c->h_stats, 8 * sizeof(double));
  for (int i = 0; i < 4; ++i) c->kernel_ms[i] = 0.0;
  float span_ms = 0.f;
  CK(cudaEventElapsedTime(&span_ms, span0, span1));
  c->last_ms = span_ms;
  for (int64_t k = 0; k < n_iter; ++k) {
    float ms;
    for (int i = 0; i < 4; ++i) {
      CK(cudaEventElapsedTime(&ms, c->evpool[5 * k + i], c->evpool[5 * k + i + 1]));
      c->kernel_ms[i] += ms;
    }
    if (stats) fill_stats(&hs[8 * k], &stats[k]);
  }
  fill_stats(&hs[8 * (n_iter - 1)], &c->last);
  return PS2_OK;
}

int ps2_run_to_convergence(ps2_ctx* c, ps2_iter_stats* last) {
  if (!c || !c->loaded) return set_err(PS2_ERR_NOT_LOADED, "no patch loaded");
  CK(cudaSetDevice(c->device));
  const int64_t cap = std::max<int64_t>(c->max_iter, 1) + 1;
  int rc = ensure_events(c, 7);
  if (rc) return rc;
  c->launches = 0;
  c->last_ms = 0.0;
  c->last_run_graph = false;
  for (int i = 0; i < 4; ++i) c->kernel_ms[i] = 0.0;
  const char* ng = getenv("PS2_NO_GRAPH");
  const bool no_graph = ng != nullptr && ng[0] != '\0' && ng[0] != '0';
  for (int64_t k = 0; k < cap; ++k) {
    if (c->iters_done > 0 && !no_graph && !c->graph_failed && !c->loop_exec) {
      if (build_loop_graph(c, &c->graph_body_launches)) {
        // capture refused (driver too old, ...): individual launches from here on
        drop_loop_graph(c);
        cudaGetLastError();
        c->graph_failed = true;
      }
    }
    if (c->iters_done > 0 && !no_graph && c->loop_exec) {
      // iterations 2.. as one graph launch
      const int64_t before = c->last.i_loop;
      CK(cudaEventRecord(c->evpool[5], c->st));
      CK(cudaGraphLaunch(c->loop_exec, c->st));
      CK(cudaEventRecord(c->evpool[6], c->st));
      CK(cudaMemcpyAsync(c->h_stats, c->stats.p, 8 * sizeof(double), cudaMemcpyDeviceToHost, c->st));
      CK(cudaStreamSynchronize(c->st));
      float ms;
      CK(cudaEventElapsedTime(&ms, c->evpool[5], c->evpool[6]));
      c->last_ms += ms;
      fill_stats(c->h_stats, &c->last);
      const int64_t ran = c->last.i_loop - before;
      c->iters_done += ran;
      c->launches += ran * c->graph_body_launches;
      c->last_run_graph = true;
      break;
    }
    rc = run_one_iteration(c, false, c->evpool.data());
    if (rc) return rc;
    CK(cudaMemcpyAsync(c->h_stats, c->stats.p, 8 * sizeof(double), cudaMemcpyDeviceToHost, c->st));
    CK(cudaStreamSynchronize(c->st));
    float ms;
    for (int i = 0; i < 4; ++i) {
      CK(cudaEventElapsedTime(&ms, c->evpool[i], c->evpool[i + 1]));
      c->kernel_ms[i] += ms;
    }
    CK(cudaEventElapsedTime(&ms, c->evpool[0], c->evpool[4]));
    c->last_ms += ms;
    fill_stats(c->h_stats, &c->last);
    if (c->last.stop) break;
  }
  if (last) *last = c->last;
  return PS2_OK;
}

int ps2_export_state(ps2_ctx* c, void* buf, int64_t* bytes) {
  if (!c || !c->loaded) return set_err(PS2_ERR_NOT_LOADED, "no patch loaded");
  if (!bytes) return set_err(PS2_ERR_INVALID_ARG, "ps2_export_state: bytes is NULL");
  const size_t need = state_bytes(c);
  if (!buf) {
    *bytes = static_cast<int64_t>(need);
    return PS2_OK;
  }
  if (*bytes < static_cast<int64_t>(need))
    return set_err(PS2_ERR_INVALID_ARG, "ps2_export_state: buffer of %lld bytes, %zu needed", (long long)*bytes, need);
  CK(cudaSetDevice(c->device));
  StateHeader h{};
  std::memcpy(h.magic, "PS2LOOP", 8);
  h.version = kStateVersion;
  h.fp64 = c->fp64 ? 1 : 0;
  h.psquare = c->psquare;
  h.N = c->N;
  h.M = c->M;
  h.G = c->G;
  h.iters_done = c->iters_done;
  h.last = c->last;
  unsigned char* out = static_cast<unsigned char*>(buf);
  std::memcpy(out, &h, sizeof(h));
  size_t off = sizeof(h);
  for (const auto& p : state_parts(c)) {
    CK(cudaMemcpyAsync(out + off, p.buf->p, p.bytes, cudaMemcpyDeviceToHost, c->st));
    off += p.bytes;
  }
  CK(cudaStreamSynchronize(c->st));
  *bytes = static_cast<int64_t>(need);
  return PS2_OK;
}

int ps2_import_state(ps2_ctx* c, const void* buf, int64_t bytes) {
  if (!c || !c->loaded) return set_err(PS2_ERR_NOT_LOADED, "no patch loaded");
  if (!buf || bytes < static_cast<int64_t>(sizeof(StateHeader)))
    return set_err(PS2_ERR_INVALID_ARG, "ps2_import_state: no state");
  StateHeader h;
  std::memcpy(&h, buf, sizeof(h));
  if (std::memcmp(h.magic, "PS2LOOP", 8) != 0 || h.version != kStateVersion)
    return set_err(PS2_ERR_INVALID_ARG, "ps2_import_state: not a loop state of this library version");
  if (h.fp64 != (c->fp64 ? 1 : 0) || h.psquare != c->psquare || h.N != c->N || h.M != c->M || h.G != c->G)
    return set_err(PS2_ERR_INVALID_ARG,
                   "ps2_import_state: the state is of a %lld x %lld patch (%lld cells, %s, %s weighting); the "
                   "loaded patch is %lld x %lld (%lld cells, %s, %s weighting)",
                   (long long)h.N, (long long)h.M, (long long)h.G, h.fp64 ? "FP64" : "FP32",
                   h.psquare ? "P-square" : "SNR", (long long)c->N, (long long)c->M, (long long)c->G,
                   c->fp64 ? "FP64" : "FP32", c->psquare ? "P-square" : "SNR");
  if (bytes < static_cast<int64_t>(state_bytes(c)))
    return set_err(PS2_ERR_INVALID_ARG, "ps2_import_state: state truncated (%lld of %zu bytes)", (long long)bytes,
                   state_bytes(c));
  CK(cudaSetDevice(c->device));
  const unsigned char* in = static_cast<const unsigned char*>(buf);
  size_t off = sizeof(h);
  for (const auto& p : state_parts(c)) {
    CK(cudaMemcpyAsync(p.buf->p, in + off, p.bytes, cudaMemcpyHostToDevice, c->st));
    off += p.bytes;
  }
  CK(cudaStreamSynchronize(c->st));
  c->iters_done = h.iters_done;
  c->last = h.last;
  return PS2_OK;
}

int ps2_autotune(ps2_ctx* c, int32_t* chosen_lanes, double* ms_per_candidate) {
  if (!c || !c->loaded) return set_err(PS2_ERR_NOT_LOADED, "no patch loaded");
  CK(cudaSetDevice(c->device));
  int rc = ensure_events(c, 2);
  if (rc) return rc;
  auto timed = [&](auto&& launch, double* ms_out) -> int {
    CK(launch());  // warm-up
    CK(cudaEventRecord(c->evpool[0], c->st));
    CK(launch());
    CK(cudaEventRecord(c->evpool[1], c->st));
    CK(cudaStreamSynchronize(c->st));
    float ms;
    CK(cudaEventElapsedTime(&ms, c->evpool[0], c->evpool[1]));
    *ms_out = ms;
    return PS2_OK;
  };
  TuneShape best;
  // topofit lanes per PS (FP32; the plain FP64 kernel has a single shape),
  // on scratch outputs so the loop state is untouched
  if (!c->fp64) {
    const int cands[4] = {4, 8, 16, 32};
    DevBuf kk, cc, hh;
    CK(kk.alloc(rsz(c) * c->N));
    CK(cc.alloc(rsz(c) * c->N));
    CK(hh.alloc(rsz(c) * c->N));
    double best_ms = 1e300;
    for (int i = 0; i < 4; ++i) {
      TopoArgs t = topo_args(c, kk.p, cc.p, hh.p);
      t.nopt = nullptr;
      t.accumulate_stats = 0;
      t.lanes = cands[i];
      double ms = 0;
      rc = timed([&] { return launch_topofit(t, false, c->topo_blocks, c->st); }, &ms);
      if (rc) return rc;
      if (ms_per_candidate) ms_per_candidate[i] = ms;
      if (ms < best_ms) {
        best_ms = ms;
        best.lanes = cands[i];
      }
    }
  } else if (chosen_lanes) {
    *chosen_lanes = 0;
  }
  // CLAP form, warps per block and resident blocks per SM, each timed with its
  // second pass (overlap-add or combine) into the filtered grid the loop
  // rewrites every iteration
  {
    const int nws[2] = {8, 4}, bpss[2] = {0, 1};
    double best_ms = 1e300;
    for (int f = 0; f < 2; ++f)
      for (int a = 0; a < (c->fp64 ? 1 : 2); ++a)
        for (int b = 0; b < 2; ++b) {
          ClapArgs ca = clap_args_loop(c, c->grid.p, f);
          ca.nw_block = c->fp64 ? 0 : nws[a];
          ca.blocks_per_sm = bpss[b];
          OverlapArgs ov = overlap_args_loop(c, c->filt.p, f);
          ov.normalize = c->fp64 ? 0 : 1;
          double ms = 0;
          rc = timed(
              [&] {
                const cudaError_t e = launch_clap(ca, c->fp64, c->twf, c->twd, c->sm_count, c->st);
                return e != cudaSuccess ? e : launch_overlap(ov, c->fp64, c->st);
              },
              &ms);
          if (rc) return rc;
          if (ms < best_ms) {
            best_ms = ms;
            best.clap_nw = ca.nw_block;
            best.clap_bps = bpss[b];
            best.clap_fused = f;
          }
        }
  }
  // binning resident blocks per SM, mode 0 into a scratch grid
  {
    DevBuf g2;
    CK(g2.alloc(csz(c) * c->G * c->Mp));
    const int bpss[3] = {0, 3, 2};
    double best_ms = 1e300;
    for (int b = 0; b < 3; ++b) {
      BinArgs ba = bin_args(c, 0, c->K[0].p);
      ba.grid = g2.p;
      ba.blocks_per_sm = bpss[b];
      double ms = 0;
      rc = timed([&] { return launch_bin(ba, c->fp64, c->sm_count, c->st); }, &ms);
      if (rc) return rc;
      if (ms < best_ms) {
        best_ms = ms;
        best.bin_bps = bpss[b];
      }
    }
  }
  c->topo_lanes = best.lanes;
  c->clap_nw = best.clap_nw;
  c->clap_bps = best.clap_bps;
  c->bin_bps = best.bin_bps;
  c->clap_fused = best.clap_fused;
  drop_loop_graph(c);  // the captured loop holds the previous shapes
  tune_store(tune_key(c->M, c->N, c->fp64), best);
  if (chosen_lanes && !c->fp64) *chosen_lanes = best.lanes;
  return PS2_OK;
}

int ps2_launch_shapes(ps2_ctx* c, int32_t* get, const int32_t* set) {
  if (!c || !c->loaded) return set_err(PS2_ERR_NOT_LOADED, "no patch loaded");
  if (get) {
    get[0] = c->topo_lanes;
    get[1] = c->clap_nw;
    get[2] = c->clap_bps;
    get[3] = c->bin_bps;
    get[4] = c->clap_fused;
  }
  if (set) {
    if (!(set[0] == 0 || set[0] == 4 || set[0] == 8 || set[0] == 16 || set[0] == 32) ||
        !(set[1] == 0 || set[1] == 4 || set[1] == 8) || set[2] < 0 || set[3] < 0 || (set[4] != 0 && set[4] != 1))
      return set_err(PS2_ERR_INVALID_ARG,
                     "ps2_launch_shapes: lanes 0/4/8/16/32, CLAP warps 0/4/8, blocks per SM >= 0, CLAP form 0/1");
    if (c->fp64 && set[1] == 8) return set_err(PS2_ERR_UNSUPPORTED, "ps2_launch_shapes: FP64 CLAP runs 4 warps");
    c->topo_lanes = set[0];
    c->clap_nw = set[1];
    c->clap_bps = set[2];
    c->bin_bps = set[3];
    c->clap_fused = set[4];
    drop_loop_graph(c);
  }
  return PS2_OK;
}

int ps2_last_timing(const ps2_ctx* c, double* total_ms, double* per_kernel_ms) {
  if (!c) return set_err(PS2_ERR_INVALID_ARG, "NULL context");
  if (total_ms) *total_ms = c->last_ms;
  if (per_kernel_ms)
    for (int i = 0; i < 4; ++i) per_kernel_ms[i] = c->kernel_ms[i];
  return PS2_OK;
}

int64_t ps2_last_launch_count(const ps2_ctx* c) { return c ? c->launches : -1; }

int ps2_download(ps2_ctx* c, ps2_outputs* o) {
  if (!c || !c->loaded) return set_err(PS2_ERR_NOT_LOADED, "no patch loaded");
  if (!o) return set_err(PS2_ERR_INVALID_ARG, "NULL outputs");
  CK(cudaSetDevice(c->device));
  const int64_t N = c->N, M = c->M, G = c->G;
  const size_t R = rsz(c), Cz = csz(c);
  const int32_t* perm = c->perm.as<int32_t>();
  const bool fp64 = c->fp64;
  // per-PS vectors: scattered to the caller's order and widened to f64 on the
  // device, one slice of the scratch each, then copied straight into the
  // caller's arrays (one synchronisation for all of them)
  {
    double* dsts[5] = {o->K_ps, o->C_ps, o->coh_ps, o->coh_ps_save, o->N_opt};
    const void* srcs[5] = {c->K[0].p, c->C.p, c->coh.p, c->coh.p, c->nopt.p};
    CK(c->scratch.alloc(sizeof(double) * 5 * N));
    double* sc = c->scratch.as<double>();
    for (int k = 0; k < 5; ++k) {
      if (!dsts[k]) continue;
      if (fp64 && k < 4)
        CK(launch_scatter_rows(srcs[k], sc + k * N, perm, N, sizeof(double), c->st));
      else
        CK(launch_scatter_widen(srcs[k], k == 4, sc + k * N, perm, N, c->st));
      CK(cudaMemcpyAsync(dsts[k], sc + k * N, sizeof(double) * N, cudaMemcpyDeviceToHost, c->st));
    }
    CK(cudaStreamSynchronize(c->st));
  }
  // residual phase and normalised patch phase: recomputed from the final
  // state by the same topofit code (deterministic, bit-identical values)
  const bool want_res = fp64 ? (o->ph_res_f64 || o->ph_res) : (o->ph_res != nullptr);
  const bool want_patch = fp64 ? (o->ph_patch_f64 || o->ph_patch) : (o->ph_patch != nullptr);
  if (c->iters_done > 0 && (want_res || want_patch)) {
    DevBuf kk, cc, hh, res, pat;
    CK(kk.alloc(R * N));
    CK(cc.alloc(R * N));
    CK(hh.alloc(R * N));
    CK(res.alloc(R * N * M));
    CK(pat.alloc(Cz * N * M));
    TopoArgs t = topo_args(c, kk.p, cc.p, hh.p);
    t.nopt = nullptr;
    t.accumulate_stats = 0;
    t.ph_res = res.p;
    t.ph_patch = pat.p;
    CK(launch_topofit(t, fp64, c->topo_blocks, c->st));
    DevBuf out;
    if (want_res) {
      CK(out.alloc(R * N * M));
      CK(launch_scatter_rows(res.p, out.p, perm, N, R * M, c->st));
      if (fp64) {
        if (o->ph_res_f64) CK(cudaMemcpyAsync(o->ph_res_f64, out.p, R * N * M, cudaMemcpyDeviceToHost, c->st));
        CK(cudaStreamSynchronize(c->st));
        if (o->ph_res) {
          std::vector<double> t2(N * M);
          CK(cudaMemcpy(t2.data(), out.p, R * N * M, cudaMemcpyDeviceToHost));
          for (int64_t i = 0; i < N * M; ++i) o->ph_res[i] = static_cast<float>(t2[i]);
        }
      } else {
        CK(cudaMemcpyAsync(o->ph_res, out.p, R * N * M, cudaMemcpyDeviceToHost, c->st));
      }
    }
    if (want_patch) {
      CK(out.alloc(Cz * N * M));
      CK(launch_scatter_rows(pat.p, out.p, perm, N, Cz * M, c->st));
      if (fp64) {
        if (o->ph_patch_f64) CK(cudaMemcpyAsync(o->ph_patch_f64, out.p, Cz * N * M, cudaMemcpyDeviceToHost, c->st));
        CK(cudaStreamSynchronize(c->st));
        if (o->ph_patch) {
          std::vector<double> t2(2 * N * M);
          CK(cudaMemcpy(t2.data(), out.p, Cz * N * M, cudaMemcpyDeviceToHost));
          for (int64_t i = 0; i < 2 * N * M; ++i) o->ph_patch[i] = static_cast<float>(t2[i]);
        }
      } else {
        CK(cudaMemcpyAsync(o->ph_patch, out.p, Cz * N * M, cudaMemcpyDeviceToHost, c->st));
      }
    }
    CK(cudaStreamSynchronize(c->st));
  }
  const bool want_w = fp64 ? (o->ph_weight_f64 || o->ph_weight) : (o->ph_weight != nullptr);
  if (want_w && c->iters_done > 0) {
    DevBuf out;
    CK(out.alloc(Cz * N * M));
    BinArgs a = bin_args(c, 0, c->K[1].p);
    CK(launch_ph_weight(a, N, fp64, perm, out.p, c->st));
    CK(cudaStreamSynchronize(c->st));
    if (fp64) {
      if (o->ph_weight_f64) CK(cudaMemcpy(o->ph_weight_f64, out.p, Cz * N * M, cudaMemcpyDeviceToHost));
      if (o->ph_weight) {
        std::vector<double> t2(2 * N * M);
        CK(cudaMemcpy(t2.data(), out.p, Cz * N * M, cudaMemcpyDeviceToHost));
        for (int64_t i = 0; i < 2 * N * M; ++i) o->ph_weight[i] = static_cast<float>(t2[i]);
      }
    } else {
      CK(cudaMemcpy(o->ph_weight, out.p, Cz * N * M, cudaMemcpyDeviceToHost));
    }
  }
  const bool want_g = fp64 ? (o->ph_grid_f64 || o->ph_grid) : (o->ph_grid != nullptr);
  if (want_g) {
    DevBuf out;
    CK(out.alloc(Cz * G * M));
    CK(launch_unpad_grid(c->grid.p, out.p, G, c->M, c->Mp, static_cast<int>(Cz), c->st));
    CK(cudaStreamSynchronize(c->st));
    if (fp64) {
      if (o->ph_grid_f64) CK(cudaMemcpy(o->ph_grid_f64, out.p, Cz * G * M, cudaMemcpyDeviceToHost));
      if (o->ph_grid) {
        std::vector<double> t2(2 * G * M);
        CK(cudaMemcpy(t2.data(), out.p, Cz * G * M, cudaMemcpyDeviceToHost));
        for (int64_t i = 0; i < 2 * G * M; ++i) o->ph_grid[i] = static_cast<float>(t2[i]);
      }
    } else {
      CK(cudaMemcpy(o->ph_grid, out.p, Cz * G * M, cudaMemcpyDeviceToHost));
    }
  }
  if (o->Nr) CK(cudaMemcpy(o->Nr, c->nr_scaled.p, sizeof(double) * PS2_COH_BINS, cudaMemcpyDeviceToHost));
  if (o->gamma_change_save || o->i_loop) {
    double st[4];
    CK(cudaMemcpy(st, c->state.p, sizeof(st), cudaMemcpyDeviceToHost));
    if (o->gamma_change_save) *o->gamma_change_save = st[0];
    if (o->i_loop) *o->i_loop = c->last.i_loop;
  }
  return PS2_OK;
}

// ------------------------------------------------------ stateless kernels --
namespace {
struct Scoped {
  cudaStream_t st = nullptr;
  int sm = 148;
  ~Scoped() {
    if (st) cudaStreamDestroy(st);
  }
};
int scoped_init(Scoped& s) {
  int dev;
  CK(cudaGetDevice(&dev));
  cudaDeviceProp p;
  CK(cudaGetDeviceProperties(&p, dev));
  s.sm = p.multiProcessorCount;
  CK(cudaStreamCreateWithFlags(&s.st, cudaStreamNonBlocking));
  return PS2_OK;
}
}  // namespace

int ps2_grid_accumulate(const float* ph_weight, const int64_t* grid_lin, int64_t n_ps, int64_t n_ifg, int64_t n_i,
                        int64_t n_j, float* out) {
  if (!ph_weight || !grid_lin || !out || n_ps < 0 || n_ifg <= 0 || n_i <= 0 || n_j <= 0)
    return set_err(PS2_ERR_INVALID_ARG, "ps2_grid_accumulate: invalid arguments");
  Scoped sc;
  int rc = scoped_init(sc);
  if (rc) return rc;
  const int64_t G = n_i * n_j, M = n_ifg;
  const int Mp = static_cast<int>((M + 3) & ~int64_t(3));
  // rows outside the grid are skipped (accumulate_grid, native_stage2.rs:733-735)
  std::vector<int32_t> start(G + 1, 0), perm;
  perm.reserve(n_ps);
  for (int64_t r = 0; r < n_ps; ++r)
    if (grid_lin[r] >= 0 && grid_lin[r] < G) start[grid_lin[r] + 1] += 1;
  for (int64_t g = 0; g < G; ++g) start[g + 1] += start[g];
  const int64_t nv = start[G];
  perm.resize(nv);
  {
    std::vector<int32_t> fp(start.begin(), start.end() - 1);
    for (int64_t r = 0; r < n_ps; ++r)
      if (grid_lin[r] >= 0 && grid_lin[r] < G) perm[fp[grid_lin[r]]++] = static_cast<int32_t>(r);
  }
  DevBuf src, sorted, dperm, dstart, grid, outb;
  CK(src.alloc(sizeof(float) * 2 * std::max<int64_t>(n_ps, 1) * M));
  if (n_ps) CK(cudaMemcpyAsync(src.p, ph_weight, sizeof(float) * 2 * n_ps * M, cudaMemcpyHostToDevice, sc.st));
  CK(dperm.alloc(sizeof(int32_t) * std::max<int64_t>(nv, 1)));
  if (nv) CK(cudaMemcpyAsync(dperm.p, perm.data(), sizeof(int32_t) * nv, cudaMemcpyHostToDevice, sc.st));
  CK(sorted.alloc(sizeof(float) * 2 * std::max<int64_t>(nv, 1) * M));
  CK(launch_gather_rows(src.p, sorted.p, dperm.as<int32_t>(), nv, sizeof(float) * 2 * M, sc.st));
  CK(dstart.alloc(sizeof(int32_t) * (G + 1)));
  CK(cudaMemcpyAsync(dstart.p, start.data(), sizeof(int32_t) * (G + 1), cudaMemcpyHostToDevice, sc.st));
  CK(grid.alloc(sizeof(float) * 2 * G * Mp));
  BinArgs a{};
  a.ph_nm = sorted.p;
  a.cell_start = dstart.as<int32_t>();
  a.G = G;
  a.M = static_cast<int>(M);
  a.Mp = Mp;
  a.nchunk = static_cast<int>((M + 31) / 32);
  a.mode = 3;
  a.grid = grid.p;
  CK(launch_bin(a, false, sc.sm, sc.st));
  CK(outb.alloc(sizeof(float) * 2 * G * M));
  CK(launch_unpad_grid(grid.p, outb.p, G, static_cast<int>(M), Mp, 8, sc.st));
  CK(cudaMemcpyAsync(out, outb.p, sizeof(float) * 2 * G * M, cudaMemcpyDeviceToHost, sc.st));
  CK(cudaStreamSynchronize(sc.st));
  return PS2_OK;
}

int ps2_topofit(const float* cpxphase, const float* bperp, int32_t row_inv, double n_trial_wraps, int64_t n,
                int64_t m, double* K, double* C, double* coh, float* residual) {
  if (!cpxphase || !bperp || !K || !C || !coh || n < 0 || m <= 0)
    return set_err(PS2_ERR_INVALID_ARG, "ps2_topofit: invalid arguments");
  if (m > 256) return set_err(PS2_ERR_UNSUPPORTED, "m %lld > 256 is not supported", (long long)m);
  if (!(n_trial_wraps >= 0.0) || n_trial_wraps > 1.0e4)
    return set_err(PS2_ERR_INVALID_ARG, "n_trial_wraps %g out of range", n_trial_wraps);
  if (n == 0) return PS2_OK;
  Scoped sc;
  int rc = scoped_init(sc);
  if (rc) return rc;
  DevBuf dc, db, dk, dcc, dh, dr;
  CK(dc.alloc(sizeof(float) * 2 * n * m));
  CK(cudaMemcpyAsync(dc.p, cpxphase, sizeof(float) * 2 * n * m, cudaMemcpyHostToDevice, sc.st));
  const int64_t nb = row_inv ? m : n * m;
  CK(db.alloc(sizeof(float) * nb));
  CK(cudaMemcpyAsync(db.p, bperp, sizeof(float) * nb, cudaMemcpyHostToDevice, sc.st));
  CK(dk.alloc(sizeof(float) * n));
  CK(dcc.alloc(sizeof(float) * n));
  CK(dh.alloc(sizeof(float) * n));
  if (residual) CK(dr.alloc(sizeof(float) * 2 * n * m));
  TopoArgs t{};
  t.cpx = dc.p;
  t.bp = db.as<float>();
  t.bp_row_inv = row_inv ? 1 : 0;
  t.N = n;
  t.M = static_cast<int>(m);
  t.Mp = static_cast<int>(m);
  t.n_half = static_cast<int>(std::ceil(8.0 * n_trial_wraps));
  t.zero_mode = 1;
  t.K_out = dk.p;
  t.C_out = dcc.p;
  t.coh_io = dh.p;
  t.residual = residual ? dr.p : nullptr;
  t.accumulate_stats = 0;
  CK(launch_topofit(t, false, topofit_grid_blocks(sc.sm, false), sc.st));
  std::vector<float> hk(n), hc(n), hh(n);
  CK(cudaMemcpyAsync(hk.data(), dk.p, sizeof(float) * n, cudaMemcpyDeviceToHost, sc.st));
  CK(cudaMemcpyAsync(hc.data(), dcc.p, sizeof(float) * n, cudaMemcpyDeviceToHost, sc.st));
  CK(cudaMemcpyAsync(hh.data(), dh.p, sizeof(float) * n, cudaMemcpyDeviceToHost, sc.st));
  if (residual) CK(cudaMemcpyAsync(residual, dr.p, sizeof(float) * 2 * n * m, cudaMemcpyDeviceToHost, sc.st));
  CK(cudaStreamSynchronize(sc.st));
  for (int64_t i = 0; i < n; ++i) {
    K[i] = hk[i];
    C[i] = hc[i];
    coh[i] = hh[i];
  }
  return PS2_OK;
}

int ps2_topofit_near_max(const void* cpxphase, const void* bperp, int32_t row_inv, int32_t precision,
                         double n_trial_wraps, int64_t n, int64_t m, double near_max_tol, double* K, double* C,
                         double* coh, float* residual) {
  if (!cpxphase || !bperp || !K || !C || !coh || n < 0 || m <= 0 || !(near_max_tol >= 0.0))
    return set_err(PS2_ERR_INVALID_ARG, "ps2_topofit_near_max: invalid arguments");
  if (precision != PS2_PRECISION_FP32 && precision != PS2_PRECISION_FP64)
    return set_err(PS2_ERR_INVALID_ARG, "ps2_topofit_near_max: precision %d", precision);
  if (m > 4096) return set_err(PS2_ERR_UNSUPPORTED, "m %lld > 4096 is not supported", (long long)m);
  if (!(n_trial_wraps >= 0.0) || n_trial_wraps > 512.0)
    return set_err(PS2_ERR_INVALID_ARG, "n_trial_wraps %g out of range [0, 512]", n_trial_wraps);
  if (n == 0) return PS2_OK;
  const bool fp64 = precision == PS2_PRECISION_FP64;
  const int n_half = static_cast<int>(std::ceil(8.0 * n_trial_wraps));
  const size_t smem = topofit_near_max_smem(fp64, static_cast<int>(m), n_half);
  int dev = 0, smem_max = 0;
  CK(cudaGetDevice(&dev));
  CK(cudaDeviceGetAttribute(&smem_max, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev));
  if (smem > static_cast<size_t>(smem_max))
    return set_err(PS2_ERR_UNSUPPORTED, "ps2_topofit_near_max: %lld columns x %d trials need %zu bytes of shared "
                   "memory per row (device limit %d)", (long long)m, 2 * n_half + 1, smem, smem_max);
  Scoped sc;
  int rc = scoped_init(sc);
  if (rc) return rc;
  const size_t rs = fp64 ? sizeof(double) : sizeof(float);
  DevBuf dc, db, dk, dcc, dh, dr;
  CK(dc.alloc(2 * rs * n * m));
  CK(cudaMemcpyAsync(dc.p, cpxphase, 2 * rs * n * m, cudaMemcpyHostToDevice, sc.st));
  const int64_t nb = row_inv ? m : n * m;
  CK(db.alloc(rs * nb));
  CK(cudaMemcpyAsync(db.p, bperp, rs * nb, cudaMemcpyHostToDevice, sc.st));
  CK(dk.alloc(sizeof(double) * n));
  CK(dcc.alloc(sizeof(double) * n));
  CK(dh.alloc(sizeof(double) * n));
  if (residual) CK(dr.alloc(sizeof(float) * 2 * n * m));
  NearMaxArgs a{};
  a.cpx = dc.p;
  a.bp = db.p;
  a.bp_row_inv = row_inv ? 1 : 0;
  a.n = n;
  a.M = static_cast<int>(m);
  a.n_half = n_half;
  a.tol = near_max_tol;
  a.K = dk.as<double>();
  a.C = dcc.as<double>();
  a.coh = dh.as<double>();
  a.residual = residual ? dr.as<float2>() : nullptr;
  CK(launch_topofit_near_max(a, fp64, sc.sm, sc.st));
  CK(cudaMemcpyAsync(K, dk.p, sizeof(double) * n, cudaMemcpyDeviceToHost, sc.st));
  CK(cudaMemcpyAsync(C, dcc.p, sizeof(double) * n, cudaMemcpyDeviceToHost, sc.st));
  CK(cudaMemcpyAsync(coh, dh.p, sizeof(double) * n, cudaMemcpyDeviceToHost, sc.st));
  if (residual) CK(cudaMemcpyAsync(residual, dr.p, sizeof(float) * 2 * n * m, cudaMemcpyDeviceToHost, sc.st));
  CK(cudaStreamSynchronize(sc.st));
  return PS2_OK;
}

int ps2_histogram_with_centers(const double* values, int64_t n, const double* centers, int64_t n_centers,
                               double* out) {
  if ((!values && n > 0) || n < 0 || n_centers < 0 || (!centers && n_centers > 0) || (!out && n_centers > 0))
    return set_err(PS2_ERR_INVALID_ARG, "ps2_histogram_with_centers: invalid arguments");
  if (n_centers == 0) return PS2_OK;
  if (n_centers > (1 << 24)) return set_err(PS2_ERR_UNSUPPORTED, "ps2_histogram_with_centers: too many centres");
  const int nc = static_cast<int>(n_centers);
  if (nc == 1) {  // every finite value in the one bin
    int64_t k = 0;
    for (int64_t i = 0; i < n; ++i) k += std::isfinite(values[i]) ? 1 : 0;
    out[0] = static_cast<double>(k);
    return PS2_OK;
  }
  // equal spacing test and the ceil rule's constants, as the reference computes them
  double amax = 0.0;
  for (int i = 0; i < nc; ++i) amax = std::max(amax, std::fabs(centers[i]));
  const double d0 = centers[1] - centers[0];
  bool equal = true;  // all |diff - diff[0]| <= eps * max(1, max |centre|)
  for (int i = 0; i + 1 < nc; ++i)
    if (!(std::fabs((centers[i + 1] - centers[i]) - d0) <= 2.220446049250313e-16 * std::max(1.0, amax))) equal = false;
  const double d = nc < 3 ? 1.0 : (centers[nc - 1] - centers[0]) / static_cast<double>(nc - 1);
  const double cutoff0 = (centers[0] + centers[1]) / 2.0;
  std::vector<double> mids(nc - 1);
  for (int i = 0; i + 1 < nc; ++i) mids[i] = (centers[i] + centers[i + 1]) / 2.0;
  if (n == 0) {
    for (int i = 0; i < nc; ++i) out[i] = 0.0;
    return PS2_OK;
  }
  Scoped sc;
  int rc = scoped_init(sc);
  if (rc) return rc;
  DevBuf dv, dm, dcnt;
  CK(dv.alloc(sizeof(double) * n));
  CK(cudaMemcpyAsync(dv.p, values, sizeof(double) * n, cudaMemcpyHostToDevice, sc.st));
  CK(dm.alloc(sizeof(double) * (nc - 1)));
  CK(cudaMemcpyAsync(dm.p, mids.data(), sizeof(double) * (nc - 1), cudaMemcpyHostToDevice, sc.st));
  CK(dcnt.alloc(sizeof(unsigned long long) * nc));
  CK(cudaMemsetAsync(dcnt.p, 0, sizeof(unsigned long long) * nc, sc.st));
  CK(launch_hist_centers(dv.as<double>(), n, dm.as<double>(), nc, equal ? 1 : 0, d, cutoff0,
                         dcnt.as<unsigned long long>(), sc.sm, sc.st));
  std::vector<unsigned long long> cnt(nc);
  CK(cudaMemcpyAsync(cnt.data(), dcnt.p, sizeof(unsigned long long) * nc, cudaMemcpyDeviceToHost, sc.st));
  CK(cudaStreamSynchronize(sc.st));
  for (int i = 0; i < nc; ++i) out[i] = static_cast<double>(cnt[i]);
  return PS2_OK;
}

int ps2_clap_filter_grid(const float* ph_grid, int64_t n_i, int64_t n_j, int64_t m, int64_t clap_window, double alpha,
                         double beta, const double* low_pass, int64_t n_win_ex, float* out) {
  if (!ph_grid || !out || !low_pass || n_i <= 0 || n_j <= 0 || m <= 0)
    return set_err(PS2_ERR_INVALID_ARG, "ps2_clap_filter_grid: invalid arguments");
  if (n_win_ex != 32) return set_err(PS2_ERR_UNSUPPORTED, "CLAP FFT size %lld unsupported (32)", (long long)n_win_ex);
  int n_inc, nwi, nwj;
  int rc = clap_geometry(n_i, n_j, clap_window, &n_inc, &nwi, &nwj);
  if (rc) return rc;
  Scoped sc;
  rc = scoped_init(sc);
  if (rc) return rc;
  const int64_t G = n_i * n_j;
  const int Mp = static_cast<int>((m + 3) & ~int64_t(3));
  DevBuf raw, grid, win, filt, lp, wsd, outb;
  CK(raw.alloc(sizeof(float) * 2 * G * m));
  CK(cudaMemcpyAsync(raw.p, ph_grid, sizeof(float) * 2 * G * m, cudaMemcpyHostToDevice, sc.st));
  CK(grid.alloc(sizeof(float) * 2 * G * Mp));
  CK(launch_pad_grid(raw.p, grid.p, G, static_cast<int>(m), Mp, 8, sc.st));
  CK(filt.alloc(sizeof(float) * 2 * G * Mp));
  const int64_t W = static_cast<int64_t>(nwi) * nwj;
  CK(win.alloc(sizeof(float) * 2 * std::max<int64_t>(W, 1) * clap_window * clap_window * Mp));
  CK(lp.alloc(sizeof(double) * 1024));
  CK(cudaMemcpyAsync(lp.p, low_pass, sizeof(double) * 1024, cudaMemcpyHostToDevice, sc.st));
  std::vector<double> ws = window_weight_scaled(static_cast<int>(clap_window), 32);
  CK(wsd.alloc(sizeof(double) * ws.size()));
  CK(cudaMemcpyAsync(wsd.p, ws.data(), sizeof(double) * ws.size(), cudaMemcpyHostToDevice, sc.st));
  ClapArgs a{};
  a.grid = grid.p;
  a.n_i = static_cast<int>(n_i);
  a.n_j = static_cast<int>(n_j);
  a.M = static_cast<int>(m);
  a.Mp = Mp;
  a.n_win = static_cast<int>(clap_window);
  a.nwi = nwi;
  a.nwj = nwj;
  a.alpha = alpha;
  a.beta = beta;
  a.alpha_is_one = std::fabs(alpha - 1.0) <= 2.220446049250313e-16 ? 1 : 0;
  a.low_pass = lp.as<double>();
  a.wscaled = wsd.as<double>();
  gauss7(a.g7, nullptr);
  a.win_out = win.p;
  Twiddles32f tf;
  Twiddles32d td;
  twiddles(&tf, &td);
  if (W > 0) {
    CK(launch_clap(a, false, tf, td, sc.sm, sc.st));
    OverlapArgs o{};
    o.win_out = win.p;
    o.filt = filt.p;
    o.n_i = a.n_i;
    o.n_j = a.n_j;
    o.M = a.M;
    o.Mp = Mp;
    o.n_win = a.n_win;
    o.n_inc = n_inc;
    o.nwi = nwi;
    o.nwj = nwj;
    CK(launch_overlap(o, false, sc.st));
  } else {
    CK(cudaMemsetAsync(filt.p, 0, sizeof(float) * 2 * G * Mp, sc.st));
  }
  CK(outb.alloc(sizeof(float) * 2 * G * m));
  CK(launch_unpad_grid(filt.p, outb.p, G, static_cast<int>(m), Mp, 8, sc.st));
  CK(cudaMemcpyAsync(out, outb.p, sizeof(float) * 2 * G * m, cudaMemcpyDeviceToHost, sc.st));
  CK(cudaStreamSynchronize(sc.st));
  return PS2_OK;
}

int ps2_random_coherence_histogram(const double* bperp_nm, int64_t n_ifg, double n_trial_wraps, int64_t n_rand,
                                   int32_t small_baseline, const int64_t* ifgday_ix, int64_t n_image, double* nr_out,
                                   double* nr_max_nz_ix) {
  if (!bperp_nm || !nr_out || !nr_max_nz_ix || n_ifg <= 0 || n_ifg > 256 || n_rand <= 0)
    return set_err(PS2_ERR_INVALID_ARG, "ps2_random_coherence_histogram: invalid arguments");
  if (!(n_trial_wraps >= 0.0) || n_trial_wraps > 1.0e4)
    return set_err(PS2_ERR_INVALID_ARG, "n_trial_wraps %g out of range", n_trial_wraps);
  std::vector<int64_t> ia(n_ifg, 0), ib(n_ifg, 0);
  int64_t cols = n_ifg;
  if (small_baseline) {
    if (!ifgday_ix || n_image <= 0) return set_err(PS2_ERR_INVALID_ARG, "small baselines need ifgday_ix and n_image");
    for (int64_t k = 0; k < n_ifg; ++k) {
      ia[k] = ifgday_ix[2 * k] - 1;
      ib[k] = ifgday_ix[2 * k + 1] - 1;
      if (ia[k] < 0 || ib[k] < 0 || ia[k] >= n_image || ib[k] >= n_image)
        return set_err(PS2_ERR_INVALID_ARG, "ps1.ifgday_ix must contain positive one-based image ids");
    }
    cols = n_image;
  }
  // random phases, column-major [cols][n_rand] (MATLAB draws the whole matrix first)
  std::vector<double> rnd(static_cast<size_t>(n_rand) * cols);
  {
    V5Uniform rng(2005);
    const double two_pi = 2.0 * M_PI;
    for (auto& v : rnd) v = rng.next() * two_pi;
  }
  Scoped sc;
  int rc = scoped_init(sc);
  if (rc) return rc;
  DevBuf dr, db, dia, dib, dh;
  CK(dr.alloc(sizeof(double) * rnd.size()));
  CK(cudaMemcpyAsync(dr.p, rnd.data(), sizeof(double) * rnd.size(), cudaMemcpyHostToDevice, sc.st));
  CK(db.alloc(sizeof(double) * n_ifg));
  CK(cudaMemcpyAsync(db.p, bperp_nm, sizeof(double) * n_ifg, cudaMemcpyHostToDevice, sc.st));
  CK(dia.alloc(sizeof(int64_t) * n_ifg));
  CK(dib.alloc(sizeof(int64_t) * n_ifg));
  CK(cudaMemcpyAsync(dia.p, ia.data(), sizeof(int64_t) * n_ifg, cudaMemcpyHostToDevice, sc.st));
  CK(cudaMemcpyAsync(dib.p, ib.data(), sizeof(int64_t) * n_ifg, cudaMemcpyHostToDevice, sc.st));
  CK(dh.alloc(sizeof(int32_t) * PS2_COH_BINS));
  CK(cudaMemsetAsync(dh.p, 0, sizeof(int32_t) * PS2_COH_BINS, sc.st));
  double cutoff0, dbin;
  coh_bin_rule(&cutoff0, &dbin);
  const int n_half = static_cast<int>(std::ceil(8.0 * n_trial_wraps));
  DevBuf dE;
  CK(dE.alloc(sizeof(double2) * n_ifg * (2 * n_half + 1)));
  CK(launch_random_hist(dr.as<double>(), n_rand, db.as<double>(), static_cast<int>(n_ifg), dia.as<int64_t>(),
                        dib.as<int64_t>(), small_baseline ? 1 : 0, n_half, cutoff0, dbin, dE.as<double2>(),
                        dh.as<int32_t>(), sc.sm, sc.st));
  int32_t h[PS2_COH_BINS];
  CK(cudaMemcpyAsync(h, dh.p, sizeof(h), cudaMemcpyDeviceToHost, sc.st));
  CK(cudaStreamSynchronize(sc.st));
  double mx = 1.0;
  for (int i = 0; i < PS2_COH_BINS; ++i) nr_out[i] = static_cast<double>(h[i]);
  for (int i = PS2_COH_BINS - 1; i >= 0; --i)
    if (nr_out[i] > 0.0) {
      mx = static_cast<double>(i + 1);
      break;
    }
  *nr_max_nz_ix = mx;
  return PS2_OK;
}


// ------------------------------------------- CLAP without device allocation --
// Scratch for ps2_clap_filter_grid_noalloc: a fixed 32 MiB array in the module
// (every GPU that loads the library holds it until the process exits). Host
// code never uses the symbol itself as an address: ps2_clap_noalloc_scratch()
// resolves the device address once per device with cudaGetSymbolAddress.
namespace {
constexpr size_t kNoAllocScratchBytes = size_t(32) << 20;
__device__ __align__(256) unsigned char g_noalloc_scratch[kNoAllocScratchBytes];

std::mutex g_noalloc_mu;
void* g_noalloc_ptr[128] = {nullptr};

// The low-pass filter and the scaled pyramid weights reach the scratch array
// as a kernel argument (copied when the launch is queued), so the call queues
// no copy from host memory whose lifetime ends with the call.
struct NoAllocTables {
  double low_pass[1024];
  double ws[1024];
  int n_ws;
};

__global__ void k_noalloc_tables(const NoAllocTables t, double* __restrict__ lp, double* __restrict__ ws) {
  for (int i = threadIdx.x; i < 1024; i += blockDim.x) lp[i] = t.low_pass[i];
  for (int i = threadIdx.x; i < t.n_ws; i += blockDim.x) ws[i] = t.ws[i];
}

int noalloc_scratch(void** out) {
  int dev = 0;
  CK(cudaGetDevice(&dev));
  if (dev < 0 || dev >= 128) return set_err(PS2_ERR_UNSUPPORTED, "device ordinal %d unsupported", dev);
  std::lock_guard<std::mutex> g(g_noalloc_mu);
  if (!g_noalloc_ptr[dev]) {
    void* p = nullptr;
    CK(cudaGetSymbolAddress(&p, g_noalloc_scratch));
    g_noalloc_ptr[dev] = p;
  }
  *out = g_noalloc_ptr[dev];
  return PS2_OK;
}
}  // namespace

int ps2_clap_filter_grid_noalloc(const float* d_ph_grid, int64_t n_i, int64_t n_j, int64_t m, int64_t clap_window,
                                 double alpha, double beta, const double* low_pass, int64_t n_win_ex, float* d_out,
                                 void* stream) {
  if (!d_ph_grid || !d_out || !low_pass || n_i <= 0 || n_j <= 0 || m <= 0)
    return set_err(PS2_ERR_INVALID_ARG, "ps2_clap_filter_grid_noalloc: invalid arguments");
  if (n_win_ex != 32) return set_err(PS2_ERR_UNSUPPORTED, "CLAP FFT size %lld unsupported (32)", (long long)n_win_ex);
  int n_inc, nwi, nwj;
  int rc = clap_geometry(n_i, n_j, clap_window, &n_inc, &nwi, &nwj);
  if (rc) return rc;
  const int64_t G = n_i * n_j;
  const int Mp = static_cast<int>((m + 3) & ~int64_t(3));
  const int64_t W = static_cast<int64_t>(nwi) * nwj;
  const size_t cz = 2 * sizeof(float);
  auto up = [](size_t b) { return (b + 255) & ~size_t(255); };
  const size_t b_grid = up(cz * G * Mp), b_filt = up(cz * G * Mp);
  const size_t b_win = up(cz * static_cast<size_t>(W) * clap_window * clap_window * Mp);
  const size_t b_lp = up(sizeof(double) * 1024), b_ws = up(sizeof(double) * clap_window * clap_window);
  const size_t need = b_grid + b_filt + b_win + b_lp + b_ws;
  if (need > kNoAllocScratchBytes)
    return set_err(PS2_ERR_UNSUPPORTED,
                   "ps2_clap_filter_grid_noalloc: a %lldx%lld grid with %lld interferograms needs %zu bytes of "
                   "scratch, more than the fixed %zu; use ps2_clap_filter_grid",
                   (long long)n_i, (long long)n_j, (long long)m, need, kNoAllocScratchBytes);
  unsigned char* base = nullptr;
  rc = noalloc_scratch(reinterpret_cast<void**>(&base));
  if (rc) return rc;
  void* grid = base;
  void* filt = base + b_grid;
  void* win = base + b_grid + b_filt;
  double* lp = reinterpret_cast<double*>(base + b_grid + b_filt + b_win);
  double* wsd = reinterpret_cast<double*>(base + b_grid + b_filt + b_win + b_lp);
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  int dev = 0, sms = 148;
  CK(cudaGetDevice(&dev));
  CK(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
  std::vector<double> ws = window_weight_scaled(static_cast<int>(clap_window), 32);
  if (ws.size() > 1024) return set_err(PS2_ERR_UNSUPPORTED, "ps2_clap_filter_grid_noalloc: window too large");
  NoAllocTables tables;
  std::memcpy(tables.low_pass, low_pass, sizeof(double) * 1024);
  std::memcpy(tables.ws, ws.data(), sizeof(double) * ws.size());
  tables.n_ws = static_cast<int>(ws.size());
  k_noalloc_tables<<<1, 256, 0, st>>>(tables, lp, wsd);
  CK(cudaGetLastError());
  // the padded copy rewrites every element, so nothing stale survives from an earlier call
  CK(launch_pad_grid(d_ph_grid, grid, G, static_cast<int>(m), Mp, 8, st));
  if (W > 0) {
    ClapArgs a{};
    a.grid = grid;
    a.n_i = static_cast<int>(n_i);
    a.n_j = static_cast<int>(n_j);
    a.M = static_cast<int>(m);
    a.Mp = Mp;
    a.n_win = static_cast<int>(clap_window);
    a.nwi = nwi;
    a.nwj = nwj;
    a.alpha = alpha;
    a.beta = beta;
    a.alpha_is_one = std::fabs(alpha - 1.0) <= 2.220446049250313e-16 ? 1 : 0;
    a.low_pass = lp;
    a.wscaled = wsd;
    gauss7(a.g7, nullptr);
    a.win_out = win;
    Twiddles32f tf;
    Twiddles32d td;
    twiddles(&tf, &td);
    CK(launch_clap(a, false, tf, td, sms, st));
    OverlapArgs o{};
    o.win_out = win;
    o.filt = filt;
    o.n_i = a.n_i;
    o.n_j = a.n_j;
    o.M = a.M;
    o.Mp = Mp;
    o.n_win = a.n_win;
    o.n_inc = n_inc;
    o.nwi = nwi;
    o.nwj = nwj;
    CK(launch_overlap(o, false, st));
  } else {
    CK(cudaMemsetAsync(filt, 0, cz * G * Mp, st));
  }
  CK(launch_unpad_grid(filt, d_out, G, static_cast<int>(m), Mp, 8, st));
  return PS2_OK;
}

}  // extern "C"

// ------------------------------------------------ differentiable coherence --
namespace {

int coh_check(ps2_ctx* c, const void* a, const void* b, const void* d, double alpha, double beta, const char* who) {
  if (!c) return set_err(PS2_ERR_INVALID_ARG, "%s: NULL context", who);
  if (!c->loaded) return set_err(PS2_ERR_NOT_LOADED, "%s: no patch loaded", who);
  if (!a || !b || !d) return set_err(PS2_ERR_INVALID_ARG, "%s: a required device array is NULL", who);
  if (!(alpha > 0.0) || !(beta >= 0.0) || !std::isfinite(alpha) || !std::isfinite(beta))
    return set_err(PS2_ERR_INVALID_ARG, "%s: need alpha > 0 and beta >= 0 (got %g, %g)", who, alpha, beta);
  return PS2_OK;
}

// gathers the caller's rows into cell order (widened to the context's
// precision) and recomputes grid -> CLAP -> filt
int coh_prologue(ps2_ctx* c, const float* d_ph, const float* d_K, const float* d_w, double alpha, double beta,
                 cudaStream_t st, ClapArgs* ca_out) {
  CK(cudaSetDevice(c->device));
  // the patch upload and any loop work run on the context's stream: order after them
  if (!c->ad_ev) CK(cudaEventCreateWithFlags(&c->ad_ev, cudaEventDisableTiming));
  CK(cudaEventRecord(c->ad_ev, c->st));
  CK(cudaStreamWaitEvent(st, c->ad_ev, 0));
  const bool fp64 = c->fp64;
  const size_t R = rsz(c), Cz = csz(c);
  const int64_t N = c->N, M = c->M, G = c->G;
  const int64_t W = std::max<int64_t>(static_cast<int64_t>(c->nwi) * c->nwj, 1);
  CK(c->ad_ph.alloc(sizeof(float) * 2 * N * M));
  CK(c->ad_K.alloc(R * N));
  CK(c->ad_w.alloc(R * N));
  CK(c->ad_coh.alloc(sizeof(float) * N));
  CK(c->ad_grid.alloc(Cz * G * c->Mp));
  CK(c->ad_filt.alloc(Cz * G * c->Mp));
  CK(c->ad_win.alloc(Cz * W * c->n_win * c->n_win * c->Mp));
  const int32_t* perm = c->perm.as<int32_t>();
  CK(launch_gather_rows(d_ph, c->ad_ph.p, perm, N, sizeof(float) * 2 * M, st));
  if (fp64) {
    CK(launch_gather_widen(d_K, c->ad_K.as<double>(), perm, N, st));
    CK(launch_gather_widen(d_w, c->ad_w.as<double>(), perm, N, st));
  } else {
    CK(launch_gather_rows(d_K, c->ad_K.p, perm, N, sizeof(float), st));
    CK(launch_gather_rows(d_w, c->ad_w.p, perm, N, sizeof(float), st));
  }
  BinArgs b = bin_args(c, 0, c->ad_K.p);
  b.ph_nm = c->ad_ph.p;
  b.w = c->ad_w.p;
  b.grid = c->ad_grid.p;
  CK(launch_bin(b, fp64, c->sm_count, st));
  ClapArgs ca = clap_args(c, c->ad_grid.p, c->ad_win.p);
  ca.alpha = alpha;
  ca.beta = beta;
  ca.alpha_is_one = alpha == 1.0 ? 1 : 0;
  if (c->nwi > 0 && c->nwj > 0) {
    CK(launch_clap(ca, fp64, c->twf, c->twd, c->sm_count, st));
    CK(launch_overlap(overlap_args(c, c->ad_win.p, c->ad_filt.p), fp64, st));
  } else {
    CK(cudaMemsetAsync(c->ad_filt.p, 0, Cz * G * c->Mp, st));
  }
  *ca_out = ca;
  c->launches = (c->nwi > 0 && c->nwj > 0) ? 6 : 4;
  return PS2_OK;
}

CohArgs coh_args(ps2_ctx* c) {
  CohArgs a{};
  a.filt = c->ad_filt.p;
  a.ph = c->ad_ph.as<float2>();
  a.K = c->ad_K.p;
  a.w = c->ad_w.p;
  a.bp = c->bp.as<float>();
  a.bp_row_inv = c->bp_row_inv;
  a.cell_of = c->cell_of.as<int32_t>();
  a.N = c->N;
  a.M = c->M;
  a.Mp = c->Mp;
  return a;
}

}  // namespace

extern "C" {

int ps2_coherence_forward(ps2_ctx* c, const float* d_ph, const float* d_K, const float* d_w, double alpha,
                          double beta, float* d_coh, void* stream) {
  int rc = coh_check(c, d_ph, d_K, d_w, alpha, beta, "ps2_coherence_forward");
  if (rc) return rc;
  if (!d_coh) return set_err(PS2_ERR_INVALID_ARG, "ps2_coherence_forward: d_coh is NULL");
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  ClapArgs ca;
  rc = coh_prologue(c, d_ph, d_K, d_w, alpha, beta, st, &ca);
  if (rc) return rc;
  CohArgs a = coh_args(c);
  a.coh = c->ad_coh.as<float>();
  CK(launch_coh(a, 0, c->fp64, c->sm_count, st));
  CK(launch_scatter_rows(c->ad_coh.p, d_coh, c->perm.as<int32_t>(), c->N, sizeof(float), st));
  c->launches += 2;
  return PS2_OK;
}

int ps2_coherence_backward(ps2_ctx* c, const float* d_ph, const float* d_K, const float* d_w, double alpha,
                           double beta, const float* d_gcoh, float* d_gph, float* d_gK, double* d_galpha_beta,
                           void* stream) {
  int rc = coh_check(c, d_ph, d_K, d_w, alpha, beta, "ps2_coherence_backward");
  if (rc) return rc;
  if (!d_gcoh || !d_gph || !d_gK || !d_galpha_beta)
    return set_err(PS2_ERR_INVALID_ARG, "ps2_coherence_backward: a gradient array is NULL");
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  ClapArgs ca;
  rc = coh_prologue(c, d_ph, d_K, d_w, alpha, beta, st, &ca);
  if (rc) return rc;
  const bool fp64 = c->fp64;
  const size_t R = rsz(c), Cz = csz(c);
  const int64_t N = c->N, M = c->M, G = c->G;
  int& cap = fp64 ? c->ad_blocks64 : c->ad_blocks;
  if (cap == 0) {
    cap = clap_bwd_max_blocks(c->sm_count, fp64);
    if (cap <= 0) return set_err(PS2_ERR_CUDA, "ps2_coherence_backward: occupancy query failed");
  }
  CK(c->ad_gfilt.alloc(Cz * G * c->Mp));
  CK(c->ad_gph.alloc(Cz * N * M));
  CK(c->ad_gf.alloc(Cz * N * M));
  CK(c->ad_gK.alloc(R * N));
  CK(c->ad_part.alloc(sizeof(double) * 2 * cap));
  const int32_t* perm = c->perm.as<int32_t>();
  // the incoming gradient is in the caller's row order
  CK(launch_gather_rows(d_gcoh, c->ad_coh.p, perm, N, sizeof(float), st));
  CohArgs a = coh_args(c);
  a.gcoh = c->ad_coh.as<float>();
  a.gph = c->ad_gph.p;
  a.gK = c->ad_gK.p;
  a.gf = c->ad_gf.p;
  CK(launch_coh(a, 1, fp64, c->sm_count, st));
  // sum of d L / d filt over each cell's PS = d L / d (CLAP output)
  CK(launch_cell_sum(a, c->cell_start.as<int32_t>(), G, c->ad_gfilt.p, fp64, c->sm_count, st));
  int launched = 0;
  if (c->nwi > 0 && c->nwj > 0) {
    ClapBwdArgs cb{};
    cb.f = ca;
    cb.gfilt = c->ad_gfilt.p;
    cb.wgrad = c->ad_win.p;
    cb.ab_partial = c->ad_part.as<double>();
    launched = cap;
    CK(launch_clap_bwd(cb, fp64, c->twf, c->twd, &launched, st));
    // window-input gradients back onto the grid: the overlap gather is the
    // adjoint of the window extraction
    CK(launch_overlap(overlap_args(c, c->ad_win.p, c->ad_filt.p), fp64, st));
  } else {
    CK(cudaMemsetAsync(c->ad_filt.p, 0, Cz * G * c->Mp, st));
  }
  CK(launch_reduce_ab(c->ad_part.as<double>(), launched, d_galpha_beta, st));
  a.ggrid = c->ad_filt.p;
  CK(launch_coh(a, 2, fp64, c->sm_count, st));
  if (fp64) {
    CK(launch_scatter_narrow(c->ad_gph.as<double>(), d_gph, perm, N, 2 * M, st));
    CK(launch_scatter_narrow(c->ad_gK.as<double>(), d_gK, perm, N, 1, st));
  } else {
    CK(launch_scatter_rows(c->ad_gph.p, d_gph, perm, N, sizeof(float) * 2 * M, st));
    CK(launch_scatter_rows(c->ad_gK.p, d_gK, perm, N, sizeof(float), st));
  }
  c->launches += 7 + (launched > 0 ? 2 : 0);
  return PS2_OK;
}

}  // extern "C"

// ============================================================ batch runner ==
namespace {

// device image of a batch, laid out in one allocation
struct BatchPlan {
  std::vector<PatchDev> patch;
  std::vector<int64_t> bin_prefix, clap_prefix, ov_prefix;
  std::vector<int32_t> units[4];  // (patch, virtual block) pairs per lane class 4, 8, 16, 32
  size_t smem_max[4] = {0, 0, 0, 0};
};

int lane_class(int L) { return L == 4 ? 0 : L == 8 ? 1 : L == 16 ? 2 : 3; }

size_t align256(size_t v) { return (v + 255) & ~size_t(255); }

}  // namespace

extern "C" {

int ps2_batch_run(ps2_ctx* const* ctxs, int64_t n, ps2_iter_stats* last) {
  if (!ctxs || n <= 0) return set_err(PS2_ERR_INVALID_ARG, "ps2_batch_run: need at least one context");
  if (n > INT32_MAX / 2) return set_err(PS2_ERR_INVALID_ARG, "ps2_batch_run: too many patches");
  ps2_ctx* c0 = ctxs[0];
  for (int64_t p = 0; p < n; ++p) {
    ps2_ctx* c = ctxs[p];
    if (!c || !c->loaded) return set_err(PS2_ERR_NOT_LOADED, "ps2_batch_run: context %lld has no patch", (long long)p);
    if (c->fp64) return set_err(PS2_ERR_UNSUPPORTED, "ps2_batch_run: context %lld is FP64 (batches are FP32)", (long long)p);
    if (!c->psquare)
      return set_err(PS2_ERR_UNSUPPORTED, "ps2_batch_run: context %lld uses SNR weighting (batches are P-square)",
                     (long long)p);
    if (c->device != c0->device)
      return set_err(PS2_ERR_INVALID_ARG, "ps2_batch_run: context %lld is on device %d, not %d", (long long)p,
                     c->device, c0->device);
    for (int64_t q = 0; q < p; ++q)
      if (ctxs[q] == c) return set_err(PS2_ERR_INVALID_ARG, "ps2_batch_run: context %lld appears twice", (long long)p);
  }
  CK(cudaSetDevice(c0->device));
  cudaStream_t st = c0->st;
  int rc = ensure_events(c0, 2);
  if (rc) return rc;
  // start after every patch's own queued work (its upload)
  for (int64_t p = 1; p < n; ++p) {
    rc = ensure_events(ctxs[p], 1);
    if (rc) return rc;
    CK(cudaEventRecord(ctxs[p]->evpool[0], ctxs[p]->st));
    CK(cudaStreamWaitEvent(st, ctxs[p]->evpool[0], 0));
  }
  BatchPlan plan;
  plan.patch.resize(static_cast<size_t>(n));
  plan.bin_prefix.assign(1, 0);
  plan.clap_prefix.assign(1, 0);
  plan.ov_prefix.assign(1, 0);
  int64_t cap_iter = 1;
  for (int64_t p = 0; p < n; ++p) {
    ps2_ctx* c = ctxs[p];
    PatchDev& d = plan.patch[p];
    d.bin = bin_args(c, 0, c->K[0].p);
    d.clap = clap_args_loop(c, c->grid.p, c->clap_fused);
    d.ov = overlap_args_loop(c, c->filt.p, c->clap_fused);
    d.ov.normalize = 1;
    d.topo = topo_args(c, c->K[0].p, c->C.p, c->coh.p);
    d.fin = finalize_args(c, false);
    d.K1 = c->K[1].as<float>();
    d.psquare = c->psquare;
    int L = 0, mpad = 0, nvb = 0;
    CK(topofit_geometry(d.topo, c->topo_blocks, &L, &mpad, &nvb));
    d.mpad = mpad;
    d.nvb = nvb;
    d.lanes = L;
    const int cls = lane_class(L);
    plan.smem_max[cls] = std::max(plan.smem_max[cls], topofit_smem_bytes(L, mpad, d.topo.n_half));
    for (int vb = 0; vb < nvb; ++vb) {
      plan.units[cls].push_back(static_cast<int32_t>(p));
      plan.units[cls].push_back(vb);
    }
    plan.bin_prefix.push_back(plan.bin_prefix.back() + c->G * c->nchunk);
    const int64_t clap_units = c->clap_fused ? static_cast<int64_t>(clap_block_count(c->nwi)) * clap_block_count(c->nwj)
                                             : static_cast<int64_t>(c->nwi) * c->nwj;
    plan.clap_prefix.push_back(plan.clap_prefix.back() + clap_units * (c->Mp / 4));
    plan.ov_prefix.push_back(plan.ov_prefix.back() + c->G * c->Mp);
    cap_iter = std::max<int64_t>(cap_iter, std::max<int64_t>(c->max_iter, 1) + 1);
  }
  // one device allocation: patches | active | n_active | prefixes | unit lists
  const size_t o_patch = 0;
  const size_t o_active = align256(o_patch + sizeof(PatchDev) * n);
  const size_t o_nact = align256(o_active + sizeof(int) * n);
  const size_t o_pref = align256(o_nact + sizeof(int));
  const size_t o_units = align256(o_pref + sizeof(int64_t) * 3 * (n + 1));
  size_t o_cls[4], end = o_units;
  for (int k = 0; k < 4; ++k) {
    o_cls[k] = end;
    end = align256(end + sizeof(int32_t) * plan.units[k].size());
  }
  std::vector<unsigned char> img(end, 0);
  std::memcpy(img.data() + o_patch, plan.patch.data(), sizeof(PatchDev) * n);
  for (int64_t p = 0; p < n; ++p) reinterpret_cast<int*>(img.data() + o_active)[p] = 1;
  *reinterpret_cast<int*>(img.data() + o_nact) = static_cast<int>(n);
  int64_t* pref = reinterpret_cast<int64_t*>(img.data() + o_pref);
  std::memcpy(pref, plan.bin_prefix.data(), sizeof(int64_t) * (n + 1));
  std::memcpy(pref + (n + 1), plan.clap_prefix.data(), sizeof(int64_t) * (n + 1));
  std::memcpy(pref + 2 * (n + 1), plan.ov_prefix.data(), sizeof(int64_t) * (n + 1));
  for (int k = 0; k < 4; ++k)
    if (!plan.units[k].empty())
      std::memcpy(img.data() + o_cls[k], plan.units[k].data(), sizeof(int32_t) * plan.units[k].size());
  CK(c0->bt.alloc(end));
  CK(cudaMemcpyAsync(c0->bt.p, img.data(), end, cudaMemcpyHostToDevice, st));
  if (!c0->h_active) CK(cudaMallocHost(reinterpret_cast<void**>(&c0->h_active), sizeof(int)));
  unsigned char* base = static_cast<unsigned char*>(c0->bt.p);
  BatchArgs b{};
  b.patch = reinterpret_cast<const PatchDev*>(base + o_patch);
  b.P = static_cast<int>(n);
  b.active = reinterpret_cast<int*>(base + o_active);
  b.n_active = reinterpret_cast<int*>(base + o_nact);
  b.bin_prefix = reinterpret_cast<const int64_t*>(base + o_pref);
  b.clap_prefix = b.bin_prefix + (n + 1);
  b.ov_prefix = b.bin_prefix + 2 * (n + 1);
  std::vector<int64_t> before(static_cast<size_t>(n));
  for (int64_t p = 0; p < n; ++p) before[p] = ctxs[p]->last.i_loop;
  const int lanes_of[4] = {4, 8, 16, 32};
  int per_iter = 5;  // reset, bin, clap, overlap, finalize + one topofit per lane class
  for (int cls = 0; cls < 4; ++cls) per_iter += plan.units[cls].empty() ? 0 : 1;
  auto enqueue = [&]() -> int {
    CK(launch_batch_reset(b, st));
    CK(launch_batch_bin(b, plan.bin_prefix.back(), c0->sm_count, st));
    CK(launch_batch_clap(b, plan.clap_prefix.back(), c0->twf, c0->sm_count, st));
    CK(launch_batch_overlap(b, plan.ov_prefix.back(), c0->sm_count, st));
    for (int cls = 0; cls < 4; ++cls) {
      if (plan.units[cls].empty()) continue;
      CK(launch_batch_topofit(b, lanes_of[cls], reinterpret_cast<const int32_t*>(base + o_cls[cls]),
                              static_cast<int>(plan.units[cls].size() / 2), plan.smem_max[cls], c0->sm_count, st));
    }
    CK(launch_batch_finalize(b, st));
    return PS2_OK;
  };
  // The loop as one graph launch: a WHILE conditional node whose body is one
  // batched iteration followed by k_batch_continue (continue while any patch
  // iterates). Eager launches with a host check per iteration if capture is
  // refused or PS2_NO_GRAPH is set.
  const char* ng = getenv("PS2_NO_GRAPH");
  bool use_graph = !(ng != nullptr && ng[0] != '\0' && ng[0] != '0');
  cudaGraph_t graph = nullptr;
  cudaGraphExec_t exec = nullptr;
  if (use_graph) {
    bool ok = cudaGraphCreate(&graph, 0) == cudaSuccess;
    cudaGraphConditionalHandle h{};
    cudaGraphNodeParams gp{};
    if (ok) ok = cudaGraphConditionalHandleCreate(&h, graph, 1, cudaGraphCondAssignDefault) == cudaSuccess;
    if (ok) {
      gp.type = cudaGraphNodeTypeConditional;
      gp.conditional.handle = h;
      gp.conditional.type = cudaGraphCondTypeWhile;
      gp.conditional.size = 1;
      cudaGraphNode_t node;
      ok = cudaGraphAddNode(&node, graph, nullptr, 0, &gp) == cudaSuccess;
    }
    if (ok) {
      ok = cudaStreamBeginCaptureToGraph(st, gp.conditional.phGraph_out[0], nullptr, nullptr, 0,
                                         cudaStreamCaptureModeThreadLocal) == cudaSuccess;
      if (ok) {
        const int rc_e = enqueue();
        const bool ok_c = rc_e == PS2_OK && launch_batch_continue(h, b.n_active, st) == cudaSuccess;
        cudaGraph_t captured = nullptr;
        const bool ok_end = cudaStreamEndCapture(st, &captured) == cudaSuccess;
        ok = ok_c && ok_end;
      }
    }
    if (ok) ok = cudaGraphInstantiate(&exec, graph, 0) == cudaSuccess;
    if (!ok) {
      if (exec) cudaGraphExecDestroy(exec);
      if (graph) cudaGraphDestroy(graph);
      exec = nullptr;
      graph = nullptr;
      cudaGetLastError();
      use_graph = false;
    }
  }
  CK(cudaEventRecord(c0->evpool[0], st));
  if (use_graph) {
    const cudaError_t e1 = cudaGraphLaunch(exec, st);
    const cudaError_t e2 = cudaStreamSynchronize(st);
    cudaGraphExecDestroy(exec);
    cudaGraphDestroy(graph);
    CK(e1);
    CK(e2);
  } else {
    for (int64_t k = 0; k < cap_iter; ++k) {
      rc = enqueue();
      if (rc) return rc;
      CK(cudaMemcpyAsync(c0->h_active, b.n_active, sizeof(int), cudaMemcpyDeviceToHost, st));
      CK(cudaStreamSynchronize(st));
      if (*c0->h_active == 0) break;
    }
  }
  CK(cudaEventRecord(c0->evpool[1], st));
  CK(cudaStreamSynchronize(st));
  float ms = 0.f;
  CK(cudaEventElapsedTime(&ms, c0->evpool[0], c0->evpool[1]));
  int64_t iterations = 0;
  for (int64_t p = 0; p < n; ++p) {
    ps2_ctx* c = ctxs[p];
    CK(cudaMemcpy(c->h_stats, c->stats.p, 8 * sizeof(double), cudaMemcpyDeviceToHost));
    fill_stats(c->h_stats, &c->last);
    iterations = std::max<int64_t>(iterations, c->last.i_loop - before[p]);
  }
  const int64_t launched = iterations * (per_iter + (use_graph ? 1 : 0));
  for (int64_t p = 0; p < n; ++p) {
    ps2_ctx* c = ctxs[p];
    c->iters_done += c->last.i_loop - before[p];
    c->launches = launched;
    c->last_ms = ms;
    c->last_run_graph = use_graph;
    for (int i = 0; i < 4; ++i) c->kernel_ms[i] = 0.0;
    if (last) last[p] = c->last;
  }
  return PS2_OK;
}

}  // extern "C"

// ======================================================= stage-3 re-estimate ==
namespace {

// One patch per distinct PS cell (ported.py:4496-4516): jobs[4 k..4 k+3] =
// patch origin row, col (0-based; -1 when the 32-cell patch does not fit) and
// the PS cell inside the patch; job_of[r] = the job of selected row r.
template <typename CellOf>
int s3_plan_jobs(int64_t n, int64_t n_i, int64_t n_j, int64_t nw, CellOf cell_of, std::vector<int32_t>* job_of,
                 std::vector<int32_t>* jobs, const char* who) {
  const int64_t half = nw / 2;
  std::vector<int32_t> cell_job(static_cast<size_t>(n_i * n_j), -1);
  job_of->assign(static_cast<size_t>(n), 0);
  jobs->clear();
  for (int64_t r = 0; r < n; ++r) {
    int64_t pi = 0, pj = 0;
    cell_of(r, &pi, &pj);
    if (pi < 1 || pi > n_i || pj < 1 || pj > n_j)
      return set_err(PS2_ERR_INVALID_ARG, "%s: grid_ij of row %lld = (%lld, %lld) outside 1..%lld x 1..%lld", who,
                     (long long)r, (long long)pi, (long long)pj, (long long)n_i, (long long)n_j);
    int32_t& j = cell_job[(pi - 1) * n_j + (pj - 1)];
    if (j < 0) {
      j = static_cast<int32_t>(jobs->size() / 4);
      int64_t i_min = std::max<int64_t>(pi - half, 1), i_max = i_min + nw - 1;
      if (i_max > n_i) i_min = i_min - i_max + n_i;
      int64_t j_min = std::max<int64_t>(pj - half, 1), j_max = j_min + nw - 1;
      if (j_max > n_j) j_min = j_min - j_max + n_j;
      const bool ok = i_min >= 1 && j_min >= 1;
      jobs->push_back(ok ? static_cast<int32_t>(i_min - 1) : -1);
      jobs->push_back(ok ? static_cast<int32_t>(j_min - 1) : -1);
      jobs->push_back(static_cast<int32_t>(pi - i_min));
      jobs->push_back(static_cast<int32_t>(pj - j_min));
    }
    (*job_of)[r] = j;
  }
  return PS2_OK;
}

}  // namespace

extern "C" {

int ps3_reestimate(const ps3_reestimate_desc* d, ps3_reestimate_out* o, int device) {
  if (!d || !o) return set_err(PS2_ERR_INVALID_ARG, "ps3_reestimate: NULL argument");
  if (d->n_sel < 0 || d->n_ifg <= 0 || d->n_ifg > 4096)
    return set_err(PS2_ERR_INVALID_ARG, "ps3_reestimate: n_sel %lld / n_ifg %lld out of range", (long long)d->n_sel,
                   (long long)d->n_ifg);
  if (d->clap_win != 32) return set_err(PS2_ERR_UNSUPPORTED, "ps3_reestimate: clap_win %lld unsupported (32)", (long long)d->clap_win);
  if (d->n_fit <= 0 || d->n_fit > d->n_ifg || d->n_fit > 1024)
    return set_err(PS2_ERR_INVALID_ARG, "ps3_reestimate: n_fit %lld out of range", (long long)d->n_fit);
  if (!(d->n_trial_wraps >= 0.0) || d->n_trial_wraps > 512.0)
    return set_err(PS2_ERR_INVALID_ARG, "ps3_reestimate: n_trial_wraps %g out of range", d->n_trial_wraps);
  if (d->slc_osf < 1) return set_err(PS2_ERR_INVALID_ARG, "ps3_reestimate: slc_osf must be >= 1");
  if (d->n_i > d->grid_rows || d->n_j > d->grid_cols || d->n_i < 1 || d->n_j < 1)
    return set_err(PS2_ERR_UNSUPPORTED,
                   "ps3_reestimate: cell range %lldx%lld outside the %lldx%lld ph_grid (the reference would filter a "
                   "truncated patch)", (long long)d->n_i, (long long)d->n_j, (long long)d->grid_rows,
                   (long long)d->grid_cols);
  if (d->n_sel > 0 && (!d->ph || !d->bperp || !d->grid_ij || !d->ph_grid || !d->fit_ifg || !d->low_pass))
    return set_err(PS2_ERR_INVALID_ARG, "ps3_reestimate: a required array is NULL");
  if (d->n_sel > 0 && (!o->ph_patch2 || !o->K_ps2 || !o->C_ps2 || !o->coh_ps2 || !o->ph_res2))
    return set_err(PS2_ERR_INVALID_ARG, "ps3_reestimate: an output array is NULL");
  for (int64_t k = 0; k < d->n_fit; ++k)
    if (d->fit_ifg[k] < 0 || d->fit_ifg[k] >= d->n_ifg)
      return set_err(PS2_ERR_INVALID_ARG, "ps3_reestimate: fit_ifg[%lld] = %lld outside 0..%lld", (long long)k,
                     (long long)d->fit_ifg[k], (long long)d->n_ifg - 1);
  if (d->n_sel == 0) return PS2_OK;
  CK(cudaSetDevice(device));
  const int64_t M = d->n_ifg, n = d->n_sel, n_i = d->n_i, n_j = d->n_j;
  std::vector<int32_t> job_of, jobs;
  int rc = s3_plan_jobs(n, n_i, n_j, d->clap_win, [&](int64_t r, int64_t* pi, int64_t* pj) {
    *pi = d->grid_ij[2 * r];
    *pj = d->grid_ij[2 * r + 1];
  }, &job_of, &jobs, "ps3_reestimate");
  if (rc) return rc;
  const int64_t n_jobs = static_cast<int64_t>(jobs.size() / 4);
  std::vector<int32_t> fit(d->fit_ifg, d->fit_ifg + d->n_fit);
  cudaDeviceProp prop;
  CK(cudaGetDeviceProperties(&prop, device));
  cudaStream_t st;
  CK(cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking));
  struct StreamGuard {
    cudaStream_t s;
    ~StreamGuard() { cudaStreamDestroy(s); }
  } guard{st};
  DevBuf grid, ph, bp, djobs, djob_of, jout, dfit, lp, pp2, K2, C2, coh2, res2;
  const size_t gbytes = sizeof(float2) * d->grid_rows * d->grid_cols * M;
  CK(grid.alloc(gbytes));
  CK(cudaMemcpyAsync(grid.p, d->ph_grid, gbytes, cudaMemcpyHostToDevice, st));
  CK(ph.alloc(sizeof(float2) * n * M));
  CK(cudaMemcpyAsync(ph.p, d->ph, sizeof(float2) * n * M, cudaMemcpyHostToDevice, st));
  CK(bp.alloc(sizeof(float) * n * M));
  CK(cudaMemcpyAsync(bp.p, d->bperp, sizeof(float) * n * M, cudaMemcpyHostToDevice, st));
  CK(djobs.alloc(sizeof(int32_t) * jobs.size()));
  CK(cudaMemcpyAsync(djobs.p, jobs.data(), sizeof(int32_t) * jobs.size(), cudaMemcpyHostToDevice, st));
  CK(djob_of.alloc(sizeof(int32_t) * n));
  CK(cudaMemcpyAsync(djob_of.p, job_of.data(), sizeof(int32_t) * n, cudaMemcpyHostToDevice, st));
  CK(dfit.alloc(sizeof(int32_t) * fit.size()));
  CK(cudaMemcpyAsync(dfit.p, fit.data(), sizeof(int32_t) * fit.size(), cudaMemcpyHostToDevice, st));
  CK(lp.alloc(sizeof(double) * 1024));
  CK(cudaMemcpyAsync(lp.p, d->low_pass, sizeof(double) * 1024, cudaMemcpyHostToDevice, st));
  CK(jout.alloc(sizeof(float2) * n_jobs * M));
  CK(pp2.alloc(sizeof(float2) * n * M));
  CK(res2.alloc(sizeof(float) * n * M));
  CK(K2.alloc(sizeof(double) * n));
  CK(C2.alloc(sizeof(double) * n));
  CK(coh2.alloc(sizeof(double) * n));
  Twiddles32f tf;
  Twiddles32d td;
  twiddles(&tf, &td);
  S3ClapArgs ca{};
  ca.grid = grid.as<float2>();
  ca.grid_cols = static_cast<int>(d->grid_cols);
  ca.M = static_cast<int>(M);
  ca.grid_stride = static_cast<int>(M);
  ca.jobs = djobs.as<int32_t>();
  ca.n_jobs = n_jobs;
  ca.ngroups = static_cast<int>((M + 3) / 4);
  ca.slc_rad = static_cast<int>(d->slc_osf - 1);
  ca.alpha = d->clap_alpha;
  ca.beta = d->clap_beta;
  ca.alpha_is_one = d->clap_alpha == 1.0 ? 1 : 0;
  ca.low_pass = lp.as<double>();
  gauss7(ca.g7, nullptr);
  ca.job_out = jout.as<float2>();
  CK(launch_s3_clap(ca, tf, prop.multiProcessorCount, st));
  S3FitArgs fa{};
  fa.ph = ph.as<float2>();
  fa.bp = bp.as<float>();
  fa.job_of = djob_of.as<int32_t>();
  fa.job_out = jout.as<float2>();
  fa.fit = dfit.as<int32_t>();
  fa.n_fit = static_cast<int>(d->n_fit);
  fa.M = static_cast<int>(M);
  fa.n_half = static_cast<int>(std::ceil(8.0 * d->n_trial_wraps));
  fa.n_sel = n;
  const int T = 2 * fa.n_half + 1;
  fa.warp_smem = (static_cast<size_t>(d->n_fit) * 16 + static_cast<size_t>(T) * 4 + 15) & ~size_t(15);
  if (4 * fa.warp_smem > 200 * 1024)
    return set_err(PS2_ERR_UNSUPPORTED, "ps3_reestimate: %lld fit interferograms x %d trials exceed shared memory",
                   (long long)d->n_fit, T);
  fa.ph_patch2 = pp2.as<float2>();
  fa.K2 = K2.as<double>();
  fa.C2 = C2.as<double>();
  fa.coh2 = coh2.as<double>();
  fa.ph_res2 = res2.as<float>();
  CK(launch_s3_fit(fa, prop.multiProcessorCount, st));
  CK(cudaMemcpyAsync(o->ph_patch2, pp2.p, sizeof(float2) * n * M, cudaMemcpyDeviceToHost, st));
  CK(cudaMemcpyAsync(o->ph_res2, res2.p, sizeof(float) * n * M, cudaMemcpyDeviceToHost, st));
  CK(cudaMemcpyAsync(o->K_ps2, K2.p, sizeof(double) * n, cudaMemcpyDeviceToHost, st));
  CK(cudaMemcpyAsync(o->C_ps2, C2.p, sizeof(double) * n, cudaMemcpyDeviceToHost, st));
  CK(cudaMemcpyAsync(o->coh_ps2, coh2.p, sizeof(double) * n, cudaMemcpyDeviceToHost, st));
  CK(cudaStreamSynchronize(st));
  return PS2_OK;
}


int ps2_stage3_reestimate(ps2_ctx* c, const int64_t* sel, int64_t n_sel, const int64_t* fit_ifg, int64_t n_fit,
                          int64_t slc_osf, ps3_reestimate_out* o, int outputs_on_device) {
  if (!c || !c->loaded) return set_err(PS2_ERR_NOT_LOADED, "ps2_stage3_reestimate: no patch loaded");
  if (c->fp64) return set_err(PS2_ERR_UNSUPPORTED, "ps2_stage3_reestimate: the context is FP64 (stage 3 is FP32)");
  if (!o || (n_sel > 0 && (!sel || !fit_ifg)))
    return set_err(PS2_ERR_INVALID_ARG, "ps2_stage3_reestimate: NULL argument");
  if (n_sel < 0) return set_err(PS2_ERR_INVALID_ARG, "ps2_stage3_reestimate: n_sel < 0");
  if (n_fit <= 0 || n_fit > c->M || n_fit > 1024)
    return set_err(PS2_ERR_INVALID_ARG, "ps2_stage3_reestimate: n_fit %lld out of range", (long long)n_fit);
  if (slc_osf < 1) return set_err(PS2_ERR_INVALID_ARG, "ps2_stage3_reestimate: slc_osf must be >= 1");
  if (c->iters_done <= 0) return set_err(PS2_ERR_INVALID_ARG, "ps2_stage3_reestimate: stage 2 has not run");
  if (n_sel > 0 && (!o->ph_patch2 || !o->K_ps2 || !o->C_ps2 || !o->coh_ps2 || !o->ph_res2))
    return set_err(PS2_ERR_INVALID_ARG, "ps2_stage3_reestimate: an output array is NULL");
  for (int64_t k = 0; k < n_fit; ++k)
    if (fit_ifg[k] < 0 || fit_ifg[k] >= c->M)
      return set_err(PS2_ERR_INVALID_ARG, "ps2_stage3_reestimate: fit_ifg[%lld] = %lld outside 0..%d", (long long)k,
                     (long long)fit_ifg[k], c->M - 1);
  for (int64_t r = 0; r < n_sel; ++r)
    if (sel[r] < 0 || sel[r] >= c->N)
      return set_err(PS2_ERR_INVALID_ARG, "ps2_stage3_reestimate: sel[%lld] = %lld outside 0..%lld", (long long)r,
                     (long long)sel[r], (long long)c->N - 1);
  if (n_sel == 0) return PS2_OK;
  CK(cudaSetDevice(c->device));
  const int64_t M = c->M, n = n_sel;
  std::vector<int32_t> job_of, jobs, rows(static_cast<size_t>(n));
  const int64_t nj_grid = c->n_j;
  int rc = s3_plan_jobs(n, c->gmax_i, c->gmax_j, 32, [&](int64_t r, int64_t* pi, int64_t* pj) {
    const int64_t g = c->h_cell[sel[r]];
    *pi = g / nj_grid + 1;
    *pj = g % nj_grid + 1;
  }, &job_of, &jobs, "ps2_stage3_reestimate");
  if (rc) return rc;
  for (int64_t r = 0; r < n; ++r) rows[r] = c->h_sorted_pos[sel[r]];
  const int64_t n_jobs = static_cast<int64_t>(jobs.size() / 4);
  std::vector<int32_t> fit(fit_ifg, fit_ifg + n_fit);
  const int n_half = c->n_half;  // the stage-2 trial count (pm1.n_trial_wraps)
  const size_t warp_smem = (static_cast<size_t>(n_fit) * 16 + static_cast<size_t>(2 * n_half + 1) * 4 + 15) & ~size_t(15);
  if (4 * warp_smem > 200 * 1024)
    return set_err(PS2_ERR_UNSUPPORTED, "ps2_stage3_reestimate: %lld fit interferograms x %d trials exceed shared memory",
                   (long long)n_fit, 2 * n_half + 1);
  cudaStream_t st = c->st;
  DevBuf djobs, djob_of, drow, dfit, jout, pp2, K2, C2, coh2, res2;
  CK(djobs.alloc(sizeof(int32_t) * jobs.size()));
  CK(cudaMemcpyAsync(djobs.p, jobs.data(), sizeof(int32_t) * jobs.size(), cudaMemcpyHostToDevice, st));
  CK(djob_of.alloc(sizeof(int32_t) * n));
  CK(cudaMemcpyAsync(djob_of.p, job_of.data(), sizeof(int32_t) * n, cudaMemcpyHostToDevice, st));
  CK(drow.alloc(sizeof(int32_t) * n));
  CK(cudaMemcpyAsync(drow.p, rows.data(), sizeof(int32_t) * n, cudaMemcpyHostToDevice, st));
  CK(dfit.alloc(sizeof(int32_t) * fit.size()));
  CK(cudaMemcpyAsync(dfit.p, fit.data(), sizeof(int32_t) * fit.size(), cudaMemcpyHostToDevice, st));
  CK(jout.alloc(sizeof(float2) * n_jobs * M));
  float2* o_pp = reinterpret_cast<float2*>(o->ph_patch2);
  float* o_res = o->ph_res2;
  double *o_K = o->K_ps2, *o_C = o->C_ps2, *o_coh = o->coh_ps2;
  if (!outputs_on_device) {
    CK(pp2.alloc(sizeof(float2) * n * M));
    CK(res2.alloc(sizeof(float) * n * M));
    CK(K2.alloc(sizeof(double) * n));
    CK(C2.alloc(sizeof(double) * n));
    CK(coh2.alloc(sizeof(double) * n));
    o_pp = pp2.as<float2>();
    o_res = res2.as<float>();
    o_K = K2.as<double>();
    o_C = C2.as<double>();
    o_coh = coh2.as<double>();
  }
  S3ClapArgs ca{};
  ca.grid = c->grid.as<float2>();  // the last iteration's binned grid (pm1.ph_grid)
  ca.grid_cols = c->n_j;
  ca.M = static_cast<int>(M);
  ca.grid_stride = c->Mp;
  ca.jobs = djobs.as<int32_t>();
  ca.n_jobs = n_jobs;
  ca.ngroups = static_cast<int>((M + 3) / 4);
  ca.slc_rad = static_cast<int>(slc_osf - 1);
  ca.alpha = c->alpha;
  ca.beta = c->beta;
  ca.alpha_is_one = c->alpha == 1.0 ? 1 : 0;
  ca.low_pass = c->low_pass.as<double>();
  gauss7(ca.g7, nullptr);
  ca.job_out = jout.as<float2>();
  CK(launch_s3_clap(ca, c->twf, c->sm_count, st));
  S3FitArgs fa{};
  fa.ph = c->ph_nm.as<float2>();
  fa.bp = c->bp.as<float>();
  fa.row = drow.as<int32_t>();
  fa.bp_row_inv = c->bp_row_inv;
  fa.job_of = djob_of.as<int32_t>();
  fa.job_out = jout.as<float2>();
  fa.fit = dfit.as<int32_t>();
  fa.n_fit = static_cast<int>(n_fit);
  fa.M = static_cast<int>(M);
  fa.n_half = n_half;
  fa.n_sel = n;
  fa.warp_smem = warp_smem;
  fa.ph_patch2 = o_pp;
  fa.K2 = o_K;
  fa.C2 = o_C;
  fa.coh2 = o_coh;
  fa.ph_res2 = o_res;
  CK(launch_s3_fit(fa, c->sm_count, st));
  if (!outputs_on_device) {
    CK(cudaMemcpyAsync(o->ph_patch2, pp2.p, sizeof(float2) * n * M, cudaMemcpyDeviceToHost, st));
    CK(cudaMemcpyAsync(o->ph_res2, res2.p, sizeof(float) * n * M, cudaMemcpyDeviceToHost, st));
    CK(cudaMemcpyAsync(o->K_ps2, K2.p, sizeof(double) * n, cudaMemcpyDeviceToHost, st));
    CK(cudaMemcpyAsync(o->C_ps2, C2.p, sizeof(double) * n, cudaMemcpyDeviceToHost, st));
    CK(cudaMemcpyAsync(o->coh_ps2, coh2.p, sizeof(double) * n, cudaMemcpyDeviceToHost, st));
  }
  CK(cudaStreamSynchronize(st));
  c->launches = 2;
  return PS2_OK;
}


// ------------------------------------------------ one patch over several GPUs
// A patch whose rows are split by contiguous cell ranges: each rank's context
// holds its rows and the full grid. One iteration is
//   ps2_shard_bin      -> sum the ranks' grids (disjoint cells)
//   ps2_shard_filter   (CLAP windows over the rank's rows of cells, overlap-add
//                       of its cells)
//   ps2_shard_fit      -> sum the ranks' statistics
//   ps2_shard_finalize (the same finalize on every rank)
// which is enqueue_iteration with the two exchanges cut in.

int ps2_shard_bin(ps2_ctx* c, void* d_grid) {
  if (!c || !c->loaded) return set_err(PS2_ERR_NOT_LOADED, "ps2_shard_bin: no patch loaded");
  if (!d_grid) return set_err(PS2_ERR_INVALID_ARG, "ps2_shard_bin: NULL grid");
  CK(cudaSetDevice(c->device));
  const bool fp64 = c->fp64, later = c->iters_done > 0;
  if (!c->psquare && later) {
    TopoArgs t = topo_args(c, nullptr, nullptr, nullptr);
    t.ph_res = c->ph_res.p;
    CK(launch_snr_weight(t, c->amp.as<float>(), c->w.p, fp64, c->sm_count, c->st));
  }
  CK(cudaMemsetAsync(c->hist.p, 0, sizeof(int32_t) * PS2_COH_BINS, c->st));
  CK(cudaMemsetAsync(c->n_invalid.p, 0, sizeof(int32_t), c->st));
  CK(cudaMemsetAsync(c->rms_partial.p, 0, sizeof(double) * c->topo_blocks, c->st));
  if (later && c->psquare) CK(launch_psquare_weights(bin_args(c, 1, c->K[0].p), c->N, fp64, c->sm_count, c->st));
  CK(launch_bin(bin_args(c, 0, c->K[0].p), fp64, c->sm_count, c->st));
  CK(cudaMemcpyAsync(d_grid, c->grid.p, csz(c) * c->G * c->Mp, cudaMemcpyDeviceToDevice, c->st));
  CK(cudaStreamSynchronize(c->st));
  return PS2_OK;
}

int ps2_shard_filter(ps2_ctx* c, const void* d_grid, int64_t cell_lo, int64_t cell_hi) {
  if (!c || !c->loaded) return set_err(PS2_ERR_NOT_LOADED, "ps2_shard_filter: no patch loaded");
  if (!d_grid) return set_err(PS2_ERR_INVALID_ARG, "ps2_shard_filter: NULL grid");
  if (cell_lo < 0 || cell_hi > c->G || cell_lo > cell_hi)
    return set_err(PS2_ERR_INVALID_ARG, "ps2_shard_filter: cells [%lld, %lld) outside 0..%lld", (long long)cell_lo,
                   (long long)cell_hi, (long long)c->G);
  CK(cudaSetDevice(c->device));
  const bool fp64 = c->fp64;
  CK(cudaMemcpyAsync(c->grid.p, d_grid, csz(c) * c->G * c->Mp, cudaMemcpyDeviceToDevice, c->st));
  if (cell_hi > cell_lo && static_cast<int64_t>(c->nwi) * c->nwj > 0) {
    // windows whose rows of cells meet rows cell_lo / n_j .. (cell_hi - 1) / n_j
    // (clap_windows, native_stage2.rs:957-995: window ix1 covers rows
    // min(ix1 * n_inc, n_i - n_win) .. + n_win - 1)
    const int64_t r_lo = cell_lo / c->n_j, r_hi = (cell_hi - 1) / c->n_j;
    int64_t ix_lo = -1, ix_hi = -1;
    for (int64_t ix = 0; ix < c->nwi; ++ix) {
      const int64_t i1 = std::min<int64_t>(ix * c->n_inc, c->n_i - c->n_win);
      if (i1 <= r_hi && i1 + c->n_win - 1 >= r_lo) {
        if (ix_lo < 0) ix_lo = ix;
        ix_hi = ix;
      }
    }
    if (ix_lo >= 0) {
      ClapArgs ca = clap_args_loop(c, c->grid.p, c->clap_fused);
      if (c->clap_fused) {
        // whole window blocks: every block holding one of those windows, so each
        // partial the combine reads is the one a whole-patch pass computes
        const int64_t nbj = clap_block_count(c->nwj), b_lo = ix_lo / 4, b_hi = ix_hi / 4;
        ca.w_lo = b_lo * nbj;
        ca.w_n = (b_hi - b_lo + 1) * nbj;
      } else {
        ca.w_lo = ix_lo * c->nwj;
        ca.w_n = (ix_hi - ix_lo + 1) * c->nwj;
      }
      CK(launch_clap(ca, fp64, c->twf, c->twd, c->sm_count, c->st));
    }
  }
  if (cell_hi > cell_lo) {
    OverlapArgs ov = overlap_args_loop(c, c->filt.p, c->clap_fused);
    ov.normalize = fp64 ? 0 : 1;
    ov.cell_lo = cell_lo;
    ov.cell_n = cell_hi - cell_lo;
    CK(launch_overlap(ov, fp64, c->st));
  }
  CK(cudaStreamSynchronize(c->st));
  return PS2_OK;
}

int ps2_shard_fit(ps2_ctx* c, double* stats) {
  if (!c || !c->loaded) return set_err(PS2_ERR_NOT_LOADED, "ps2_shard_fit: no patch loaded");
  if (!stats) return set_err(PS2_ERR_INVALID_ARG, "ps2_shard_fit: NULL statistics");
  CK(cudaSetDevice(c->device));
  CK(cudaMemcpyAsync(c->K[1].p, c->K[0].p, rsz(c) * c->N, cudaMemcpyDeviceToDevice, c->st));
  TopoArgs t = topo_args(c, c->K[0].p, c->C.p, c->coh.p);
  if (!c->psquare) t.ph_res = c->ph_res.p;
  CK(launch_topofit(t, c->fp64, c->topo_blocks, c->st));
  std::vector<int32_t> hist(PS2_COH_BINS);
  std::vector<double> part(static_cast<size_t>(c->topo_blocks));
  int32_t inv = 0;
  CK(cudaMemcpyAsync(hist.data(), c->hist.p, sizeof(int32_t) * PS2_COH_BINS, cudaMemcpyDeviceToHost, c->st));
  CK(cudaMemcpyAsync(part.data(), c->rms_partial.p, sizeof(double) * part.size(), cudaMemcpyDeviceToHost, c->st));
  CK(cudaMemcpyAsync(&inv, c->n_invalid.p, sizeof(int32_t), cudaMemcpyDeviceToHost, c->st));
  CK(cudaStreamSynchronize(c->st));
  double sum = 0.0;
  for (const double v : part) sum += v;
  for (int i = 0; i < PS2_COH_BINS; ++i) stats[i] = static_cast<double>(hist[i]);
  stats[PS2_COH_BINS] = sum;
  stats[PS2_COH_BINS + 1] = static_cast<double>(inv);
  return PS2_OK;
}

int ps2_shard_finalize(ps2_ctx* c, const double* stats, int64_t n_total, ps2_iter_stats* out) {
  if (!c || !c->loaded) return set_err(PS2_ERR_NOT_LOADED, "ps2_shard_finalize: no patch loaded");
  if (!stats) return set_err(PS2_ERR_INVALID_ARG, "ps2_shard_finalize: NULL statistics");
  if (n_total < c->N) return set_err(PS2_ERR_INVALID_ARG, "ps2_shard_finalize: n_total %lld < this shard's %lld rows",
                                     (long long)n_total, (long long)c->N);
  CK(cudaSetDevice(c->device));
  std::vector<int32_t> hist(PS2_COH_BINS);
  for (int i = 0; i < PS2_COH_BINS; ++i) {
    const double v = stats[i];
    if (!(v >= 0.0) || v > 2147483647.0)
      return set_err(PS2_ERR_INVALID_ARG, "ps2_shard_finalize: histogram bin %d = %g", i, v);
    hist[i] = static_cast<int32_t>(v);
  }
  const int32_t inv = static_cast<int32_t>(stats[PS2_COH_BINS + 1]);
  const double sum = stats[PS2_COH_BINS];
  CK(cudaMemcpyAsync(c->hist.p, hist.data(), sizeof(int32_t) * PS2_COH_BINS, cudaMemcpyHostToDevice, c->st));
  CK(cudaMemsetAsync(c->rms_partial.p, 0, sizeof(double) * c->topo_blocks, c->st));
  CK(cudaMemcpyAsync(c->rms_partial.p, &sum, sizeof(double), cudaMemcpyHostToDevice, c->st));
  CK(cudaMemcpyAsync(c->n_invalid.p, &inv, sizeof(int32_t), cudaMemcpyHostToDevice, c->st));
  FinalizeArgs f = finalize_args(c, false);
  f.N = n_total;
  CK(launch_finalize(f, c->st));
  CK(cudaMemcpyAsync(c->h_stats, c->stats.p, 8 * sizeof(double), cudaMemcpyDeviceToHost, c->st));
  CK(cudaStreamSynchronize(c->st));
  fill_stats(c->h_stats, &c->last);
  c->iters_done += 1;
  if (out) *out = c->last;
  return PS2_OK;
}


// ------------------------------------------------ host-side preparation ------
// prepare_stage2_inputs (native_stage2.rs:447-467, 563-612) in one threaded pass
// per array: the same float32 hypotf, zero guard and IEEE divisions as the
// numpy statement of it, element for element.
}  // extern "C"

namespace {
// Host threads this process may run on: its CPU affinity set (a job on a
// shared host is usually pinned to fewer cores than the machine has).
int usable_cores() {
  cpu_set_t set;
  CPU_ZERO(&set);
  if (sched_getaffinity(0, sizeof(set), &set) == 0) {
    const int n = CPU_COUNT(&set);
    if (n > 0) return n;
  }
  const int hc = static_cast<int>(std::thread::hardware_concurrency());
  return hc > 0 ? hc : 1;
}

// Splits rows [0, n) into contiguous ranges, one per thread (threads <= 0:
// the usable cores), capped at the row count. The last range runs on the
// calling thread, and so does any range whose thread cannot be started, so no
// exception crosses the C ABI.
template <typename F>
void for_rows(int64_t n, int threads, F&& body) {
  int nt = threads > 0 ? threads : usable_cores();
  if (nt < 1) nt = 1;
  if (static_cast<int64_t>(nt) > n) nt = static_cast<int>(std::max<int64_t>(n, 1));
  std::vector<std::thread> pool;
  std::vector<std::pair<int64_t, int64_t>> left;
  const int64_t per = (n + nt - 1) / nt;
  for (int t = 0; t < nt; ++t) {
    const int64_t a = t * per, b = std::min<int64_t>(n, a + per);
    if (a >= b) break;
    if (t + 1 == nt) {
      left.emplace_back(a, b);
      continue;
    }
    try {
      pool.emplace_back([&body, a, b] { body(a, b); });
    } catch (const std::system_error&) {
      left.emplace_back(a, b);
    }
  }
  for (const auto& r : left) body(r.first, r.second);
  for (auto& th : pool) th.join();
}
}  // namespace

extern "C" {

int ps2_prepare_phase(const float* ph, int64_t n_ps, int64_t n_full, const int64_t* cols, int64_t m, float* ph_nm,
                      float* amp, int threads) {
  if (!ph || !cols || !ph_nm || !amp || n_ps < 0 || n_full <= 0 || m <= 0 || m > n_full)
    return set_err(PS2_ERR_INVALID_ARG, "ps2_prepare_phase: invalid arguments");
  for (int64_t k = 0; k < m; ++k)
    if (cols[k] < 0 || cols[k] >= n_full)
      return set_err(PS2_ERR_INVALID_ARG, "ps2_prepare_phase: cols[%lld] = %lld outside 0..%lld", (long long)k,
                     (long long)cols[k], (long long)n_full - 1);
  for_rows(n_ps, threads, [&](int64_t a, int64_t b) {
    for (int64_t r = a; r < b; ++r) {
      const float* src = ph + 2 * r * n_full;
      float* dst = ph_nm + 2 * r * m;
      float* am = amp + r * m;
      for (int64_t k = 0; k < m; ++k) {
        const float re = src[2 * cols[k]], im = src[2 * cols[k] + 1];
        const float mag = std::hypot(re, im);
        const float safe = mag == 0.0f ? 1.0f : mag;  // a zero magnitude keeps the zero (:452-467)
        dst[2 * k] = re / safe;
        dst[2 * k + 1] = im / safe;
        am[k] = safe;
      }
    }
  });
  return PS2_OK;
}

int ps2_prepare_bperp(const double* bmat, int64_t n_ps, int64_t width, const int64_t* cols, int64_t m, float* out,
                      int32_t* row_invariant, int threads) {
  if (!bmat || !out || !row_invariant || n_ps <= 0 || width <= 0 || m <= 0 || (!cols && width != m))
    return set_err(PS2_ERR_INVALID_ARG, "ps2_prepare_bperp: invalid arguments");
  if (cols)
    for (int64_t k = 0; k < m; ++k)
      if (cols[k] < 0 || cols[k] >= width)
        return set_err(PS2_ERR_INVALID_ARG, "ps2_prepare_bperp: cols[%lld] = %lld outside 0..%lld", (long long)k,
                       (long long)cols[k], (long long)width - 1);
  std::vector<double> row0(static_cast<size_t>(m));
  for (int64_t k = 0; k < m; ++k) row0[k] = bmat[cols ? cols[k] : k];
  std::mutex mu;
  bool same = true;
  for_rows(n_ps, threads, [&](int64_t a, int64_t b) {
    bool local = true;
    for (int64_t r = a; r < b; ++r) {
      const double* src = bmat + r * width;
      float* dst = out + r * m;
      for (int64_t k = 0; k < m; ++k) {
        const double v = src[cols ? cols[k] : k];
        local = local && (v == row0[k]);  // NaN makes the rows differ, as in numpy
        dst[k] = static_cast<float>(v);
      }
    }
    if (!local) {
      std::lock_guard<std::mutex> g(mu);
      same = false;
    }
  });
  *row_invariant = same ? 1 : 0;
  return PS2_OK;
}

}  // extern "C"
