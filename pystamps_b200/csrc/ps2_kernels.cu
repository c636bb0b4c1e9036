// Stage-2 gamma-estimation kernels for B200 (sm_100a).
//
// One iteration of the reference loop (crates/pystamps-core/src/native_stage2.rs:261-406)
// is five launches on one stream:
//   k_bin       fill_phase_weight + accumulate_grid (:629-657, :722-740), fused,
//               as a sort-by-cell sequential segmented reduction (no float atomics)
//   k_clap      clap_filter_one_ifg per (window, ifg) (:823-916): 32x32 FFT in
//               registers + shared memory, |H| smoothing, median, filter, IFFT
//   k_overlap   the pyramid-weighted overlap-add (:904-915) as a gather in the
//               reference's window order (deterministic)
//   k_topofit   extract_patch_phase + fit_stage2_rows + topofit_row + refine_candidate
//               (:1186-1303): one warp per PS, trial sweep by phasor recurrence
//   k_finalize  rms_difference, stop rule, P-square weighting table (:307-381, :1538-1783)
#include <math.h>
#include <stdint.h>

#include <algorithm>
#include <cstdlib>
#include <mutex>

#include "ps2_device.cuh"
#include "ps2_kernels.cuh"
#include "atan_poly.h"
#include "sincos_poly.h"
#include "trial_interp_taps.h"

namespace ps2 {

cudaError_t kernel_attributes_once(size_t dynamic_smem);

template <typename R>
struct CT;
template <>
struct CT<float> {
  using C = float2;
  using Tw = Twiddles32f;
  using U = uint32_t;
};
template <>
struct CT<double> {
  using C = double2;
  using Tw = Twiddles32d;
  using U = unsigned long long;
};

// sin and cos of an FP32 phase (the phase ramps of binning and of the row
// refinements): Cody and Waite's reduction by pi/2 ("Software Manual for the
// Elementary Functions", 1980) with pi/2 split in three FP32 parts, each
// removed by one FMA, then minimax polynomials on [-pi/4, pi/4]
// (sincos_poly.h, fitted by make_sincos_poly.py) and the quadrant's swap and
// signs. Largest absolute error 9.2e-8 for |x| <= 5000, the FP32 rounding of a
// unit phasor; about 20 instructions. sin(+-0) = +-0; NaN and inf give NaN.
__device__ __forceinline__ void sincos_cw(float x, float* s, float* c) {
  const float k = rintf(x * kTwoOverPi);
  float r = fmaf(-k, kHalfPi1, x);
  r = fmaf(-k, kHalfPi2, r);
  r = fmaf(-k, kHalfPi3, r);
  const float u = r * r;
  float sv = fmaf(r * u, fmaf(fmaf(kSinS3, u, kSinS2), u, kSinS1), r);
  const float cv = fmaf(u * u, fmaf(fmaf(kCosQ3, u, kCosQ2), u, kCosQ1), fmaf(-0.5f, u, 1.f));
  if (x == 0.f) sv = x;
  const int q = __float2int_rn(k);
  const float s1 = (q & 1) ? cv : sv, c1 = (q & 1) ? sv : cv;
  *s = (q & 2) ? -s1 : s1;
  *c = ((q + 1) & 2) ? -c1 : c1;
}
__device__ __forceinline__ void sincos_r(float x, float* s, float* c) { sincos_cw(x, s, c); }

// atan2(y, x) in FP32 for the topofit refinement's residual angles: t =
// min(|x|, |y|) / max(|x|, |y|) in [0, 1], atan t by a minimax polynomial in
// t^2 (atan_poly.h, fitted by make_atan_poly.py, 4.9e-8), then the octant's
// reflections and the sign of y. Largest absolute error 3.1e-7 (near +-pi,
// where an FP32 ulp is 2.4e-7); atan2(+-0, +0) = +-0, atan2(+-0, x < 0) = +-pi.
__device__ __forceinline__ float atan2_poly(float y, float x) {
  const float ax = fabsf(x), ay = fabsf(y);
  const float mn = fminf(ax, ay), mx = fmaxf(ax, ay);
  const float t = mx > 0.f ? __fdiv_rn(mn, mx) : 0.f;
  const float u = t * t;
  float p = fmaf(kAtanA7, u, kAtanA6);
  p = fmaf(p, u, kAtanA5);
  p = fmaf(p, u, kAtanA4);
  p = fmaf(p, u, kAtanA3);
  p = fmaf(p, u, kAtanA2);
  p = fmaf(p, u, kAtanA1);
  float r = fmaf(t * u, p, t);
  if (ay > ax) r = kHalfPiF - r;
  if (x < 0.f) r = kPiF - r;
  return copysignf(r, y);
}
__device__ __forceinline__ void sincos_r(double x, double* s, double* c) { sincos(x, s, c); }
__device__ __forceinline__ float mul_rn(float a, float b) { return __fmul_rn(a, b); }
__device__ __forceinline__ double mul_rn(double a, double b) { return __dmul_rn(a, b); }
__device__ __forceinline__ float add_rn(float a, float b) { return __fadd_rn(a, b); }
__device__ __forceinline__ double add_rn(double a, double b) { return __dadd_rn(a, b); }
__device__ __forceinline__ float hypot_r(float a, float b) { return hypotf(a, b); }
__device__ __forceinline__ double hypot_r(double a, double b) { return hypot(a, b); }
__device__ __forceinline__ float atan2_r(float y, float x) { return atan2f(y, x); }
__device__ __forceinline__ double atan2_r(double y, double x) { return atan2(y, x); }
__device__ __forceinline__ float2 mk(float a, float b) { return make_float2(a, b); }
__device__ __forceinline__ double2 mk(double a, double b) { return make_double2(a, b); }

// ============================================================= binning ====
template <typename R, int MODE>
__device__ __forceinline__ R bin_weight(const BinArgs& a, const R* __restrict__ W, const R* __restrict__ coh,
                                        const int s) {
  if (MODE == 3) return R(1);
  if (MODE != 1) return W[s];
  // psquare_weighting lookup (native_stage2.rs:1674-1682)
  const double v = __dmul_rn(static_cast<double>(coh[s]), 1000.0);
  double r = v >= 0.0 ? floor(__dadd_rn(v, 0.5)) : ceil(__dsub_rn(v, 0.5));
  r = fmin(fmax(r, 0.0), static_cast<double>(a.lut_len - 1));
  const int ix = isnan(r) ? 0 : static_cast<int>(r);
  const double t = 1.0 - a.lut[ix];
  return static_cast<R>(t * t);
}

// One warp-task of the binning: cell `task / nchunk`, interferograms
// 32 * (task % nchunk) + lane.
template <typename R, int MODE, bool ROWINV>
__device__ __forceinline__ void bin_task_t(const BinArgs& a, const int64_t task, const int lane) {
  using C = typename CT<R>::C;
  const float2* __restrict__ ph = static_cast<const float2*>(a.ph_nm);
  const R* __restrict__ K = static_cast<const R*>(a.K);
  R* __restrict__ W = static_cast<R*>(a.w);
  const R* __restrict__ coh = static_cast<const R*>(a.coh);
  C* __restrict__ grid = static_cast<C*>(a.grid);
  const float* __restrict__ bp = a.bp;
  const int64_t M = a.M;
  {
    const int64_t cell = task / a.nchunk;
    const int chunk = static_cast<int>(task - cell * a.nchunk);
    const int c = chunk * 32 + lane;
    const bool active = c < a.M;
    const bool write_w = MODE == 1 && chunk == 0 && lane == 0;
    const int s0 = a.cell_start[cell], s1 = a.cell_start[cell + 1];
    R ax = R(0), ay = R(0);
    // rows are taken eight at a time with every load issued before the
    // arithmetic; the sum itself stays sequential in row order
    for (int sb = s0; sb < s1; sb += 8) {
      R wv[8], kv[8], bv[8];
      float2 v[8];
#pragma unroll
      for (int i = 0; i < 8; ++i) {
        const int s = sb + i;
        wv[i] = R(0);
        kv[i] = R(0);
        bv[i] = R(0);
        v[i] = make_float2(0.f, 0.f);
        if (s < s1) {
          wv[i] = bin_weight<R, MODE>(a, W, coh, s);
          if (MODE != 3) kv[i] = K[s];
          if (active) {
            v[i] = ph[static_cast<int64_t>(s) * M + c];
            if (MODE != 3)
              bv[i] = ROWINV ? static_cast<R>(bp[c]) : static_cast<R>(bp[static_cast<int64_t>(s) * M + c]);
          }
        }
      }
#pragma unroll
      for (int i = 0; i < 8; ++i) {
        const int s = sb + i;
        if (s >= s1) break;
        if (write_w) W[s] = wv[i];
        if (!active) continue;
        if (MODE == 3) {
          // accumulate_grid alone: ph_nm holds ph_weight, no ramp and no weight
          ax = add_rn(ax, static_cast<R>(v[i].x));
          ay = add_rn(ay, static_cast<R>(v[i].y));
        } else {
          const R phs = -(bv[i] * kv[i]);
          R sn, cs;
          sincos_r(phs, &sn, &cs);
          const C r = cmul_rn(mk(static_cast<R>(v[i].x), static_cast<R>(v[i].y)), mk(cs, sn));
          ax = add_rn(ax, mul_rn(r.x, wv[i]));
          ay = add_rn(ay, mul_rn(r.y, wv[i]));
        }
      }
    }
    if (c < a.Mp) grid[cell * a.Mp + c] = active ? mk(ax, ay) : mk(R(0), R(0));
  }
}

// The P-square weights of every row from its previous coherence and the table
// of the last update (psquare_weighting's lookup, native_stage2.rs:1674-1682),
// the same function bin_weight applies in mode 1, as one elementwise pass ahead
// of binning: the binning warps then read w (mode 0) instead of each lane of
// each interferogram chunk repeating the lookup and its dependent table load.
template <typename R>
__global__ void __launch_bounds__(256) k_psquare_weights(BinArgs a, int64_t N) {
  const R* __restrict__ coh = static_cast<const R*>(a.coh);
  R* __restrict__ W = static_cast<R*>(a.w);
  const int64_t stride = static_cast<int64_t>(gridDim.x) * blockDim.x;
  for (int64_t s = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x; s < N; s += stride)
    W[s] = bin_weight<R, 1>(a, W, coh, static_cast<int>(s));
}

cudaError_t launch_psquare_weights(const BinArgs& a, int64_t N, bool fp64, int sm_count, cudaStream_t st) {
  if (N <= 0) return cudaSuccess;
  const int64_t blocks = std::min<int64_t>((N + 255) / 256, static_cast<int64_t>(sm_count) * 16);
  if (fp64)
    k_psquare_weights<double><<<static_cast<unsigned>(blocks), 256, 0, st>>>(a, N);
  else
    k_psquare_weights<float><<<static_cast<unsigned>(blocks), 256, 0, st>>>(a, N);
  return cudaGetLastError();
}

// The weighting mode and the row invariance of bperp are compile-time in the
// task body (no per-element branches on them).
template <typename R>
__device__ __forceinline__ void bin_task(const BinArgs& a, const int64_t task, const int lane) {
  if (a.mode == 3)
    bin_task_t<R, 3, false>(a, task, lane);
  else if (a.mode == 1)
    a.bp_row_inv ? bin_task_t<R, 1, true>(a, task, lane) : bin_task_t<R, 1, false>(a, task, lane);
  else
    a.bp_row_inv ? bin_task_t<R, 0, true>(a, task, lane) : bin_task_t<R, 0, false>(a, task, lane);
}

// FP32: held to 64 registers so four blocks of eight warps reside per SM
// (three at its natural 76): more rows in flight against the HBM latency
// (0.281 -> 0.256 ms at 500,000 PS x 150 ifg, the same bits).
template <typename R>
__global__ void __launch_bounds__(256, sizeof(R) == 4 ? 4 : 1) k_bin(BinArgs a) {
  const int lane = threadIdx.x & 31;
  const int64_t gw = (static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x) >> 5;
  const int64_t nw = (static_cast<int64_t>(gridDim.x) * blockDim.x) >> 5;
  const int64_t ntask = a.G * a.nchunk;
  for (int64_t task = gw; task < ntask; task += nw) bin_task<R>(a, task, lane);
}

cudaError_t launch_bin(const BinArgs& a, bool fp64, int sm_count, cudaStream_t st) {
  const int64_t warps = a.G * a.nchunk;
  int64_t blocks = (warps + 7) / 8;
  // 16 blocks per SM (registers allow about three resident), or the launch shape's cap
  const int64_t cap = static_cast<int64_t>(sm_count) * (a.blocks_per_sm > 0 ? a.blocks_per_sm : 16);
  if (blocks > cap) blocks = cap;
  if (blocks < 1) blocks = 1;
  if (fp64)
    k_bin<double><<<static_cast<unsigned>(blocks), 256, 0, st>>>(a);
  else
    k_bin<float><<<static_cast<unsigned>(blocks), 256, 0, st>>>(a);
  return cudaGetLastError();
}

// ====================================================================== FFT
// Radix-2 decimation-in-time FFT of 32 points held in registers (textbook
// Cooley-Tukey). Forward uses e^{-2 pi i k/32}; inverse the conjugate and no
// scaling (the 1/1024 is folded into the overlap-add weight, like rustfft's
// unnormalised inverse followed by inv_scale in the reference).
template <typename R, bool INV>
__device__ __forceinline__ void fft32(typename CT<R>::C (&x)[32], const typename CT<R>::Tw& tw) {
  using C = typename CT<R>::C;
#pragma unroll
  for (int i = 0; i < 32; ++i) {
    const int r = ((i & 1) << 4) | ((i & 2) << 2) | (i & 4) | ((i & 8) >> 2) | ((i & 16) >> 4);
    if (r > i) {
      C t = x[i];
      x[i] = x[r];
      x[r] = t;
    }
  }
#pragma unroll
  for (int half = 1; half < 32; half <<= 1) {
    const int step = 16 / half;
#pragma unroll
    for (int s = 0; s < 32; s += 2 * half) {
#pragma unroll
      for (int k = 0; k < half; ++k) {
        const int ti = k * step;
        const C u = x[s + k];
        const C v = x[s + k + half];
        C t;
        if (ti == 0) {
          t = v;
        } else if (ti == 8) {
          t = INV ? mk(-v.y, v.x) : mk(v.y, -v.x);
        } else {
          C w = tw.w[ti];
          if (INV) w.y = -w.y;
          t = cmul(v, w);
        }
        x[s + k] = mk(u.x + t.x, u.y + t.y);
        x[s + k + half] = mk(u.x - t.x, u.y - t.y);
      }
    }
  }
}

// ================================================================== CLAP ==
// One warp's 32x32 working set (33-column rows avoid bank conflicts along
// columns). PAD staggers consecutive tiles: 8 floats for 4 tiles per block, 4
// for 8, so the block's interleaved loads (all tiles' ifgs of one cell at once)
// hit distinct banks.
template <typename R, int PAD>
struct ClapTileT {
  R re[32][33];
  R im[32][33];
  R hs[32][33];
  R pad[PAD];
};
template <typename R>
using ClapTile = ClapTileT<R, 8>;

// Row stride of the pyramid-weight table in shared memory: lane l reads row l,
// so rows 33 words apart put the 32 lanes on 32 different banks.
constexpr int kWtStride = 33;

// warps per CLAP block and the matching tile stagger
template <int NW>
struct ClapShape;
template <>
struct ClapShape<4> {
  static constexpr int kPad = 8;
};
template <>
struct ClapShape<8> {
  static constexpr int kPad = 4;
};

__device__ __forceinline__ uint32_t to_bits(float v) { return __float_as_uint(v); }
__device__ __forceinline__ unsigned long long to_bits(double v) {
  return static_cast<unsigned long long>(__double_as_longlong(v));
}
__device__ __forceinline__ float from_bits(uint32_t u) { return __uint_as_float(u); }
__device__ __forceinline__ double from_bits(unsigned long long u) {
  return __longlong_as_double(static_cast<long long>(u));
}
__device__ __forceinline__ uint32_t warp_min_u(uint32_t v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v = min(v, __shfl_xor_sync(kFull, v, o));
  return v;
}
__device__ __forceinline__ uint32_t warp_max_u(uint32_t v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v = max(v, __shfl_xor_sync(kFull, v, o));
  return v;
}
__device__ __forceinline__ unsigned long long warp_min_u(unsigned long long v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v = min(v, __shfl_xor_sync(kFull, v, o));
  return v;
}
__device__ __forceinline__ unsigned long long warp_max_u(unsigned long long v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v = max(v, __shfl_xor_sync(kFull, v, o));
  return v;
}

// Median of the 1,024 non-negative values held 32 per lane (median(),
// native_stage2.rs:1173-1184: mean of the 512th and 513th smallest), exact.
// Bisection on the IEEE bit pattern (which orders non-negative floats like
// their values) narrows a bracket [lo, hi] holding the 512th smallest until it
// holds at most 32 of the values; those are copied to `scratch` (32 slots of
// the warp's shared memory) and ranked among themselves. v0, v1 = the 512th
// and 513th smallest.
template <typename R>
__device__ __forceinline__ void warp_median_pair(const R (&o)[32], R* scratch, R& v0, R& v1) {
  using U = typename CT<R>::U;
  const int lane = threadIdx.x & 31;
  U lo = to_bits(o[0]), hi = lo;
#pragma unroll
  for (int i = 1; i < 32; ++i) {
    const U u = to_bits(o[i]);
    lo = min(lo, u);
    hi = max(hi, u);
  }
  lo = warp_min_u(lo);
  hi = warp_max_u(hi);
  int cnt_lo = 0, cnt_hi = 1024;  // values below lo, values up to hi
  while (lo < hi && cnt_hi - cnt_lo > 32) {
    const U mid = lo + ((hi - lo) >> 1);
    unsigned cnt = 0;
#pragma unroll
    for (int i = 0; i < 32; ++i) cnt += (to_bits(o[i]) <= mid) ? 1u : 0u;
    cnt = __reduce_add_sync(kFull, cnt);
    if (cnt >= 512u) {
      hi = mid;
      cnt_hi = static_cast<int>(cnt);
    } else {
      lo = mid + 1;
      cnt_lo = static_cast<int>(cnt);
    }
  }
  const int r0 = 511 - cnt_lo;  // rank of the 512th smallest inside the bracket
  if (lo == hi) {
    v0 = from_bits(lo);
    if (cnt_hi >= 513) {
      v1 = v0;
    } else {
      U nxt = ~U(0);
#pragma unroll
      for (int i = 0; i < 32; ++i) {
        const U u = to_bits(o[i]);
        if (u > hi) nxt = min(nxt, u);
      }
      v1 = from_bits(warp_min_u(nxt));
    }
    return;
  }
  // copy the bracket's values to scratch (exclusive prefix over lanes)
  int mine = 0;
#pragma unroll
  for (int i = 0; i < 32; ++i) {
    const U u = to_bits(o[i]);
    mine += (u >= lo && u <= hi) ? 1 : 0;
  }
  int incl = mine;
#pragma unroll
  for (int d = 1; d < 32; d <<= 1) {
    const int t = __shfl_up_sync(kFull, incl, d);
    if (lane >= d) incl += t;
  }
  int off = incl - mine;
  __syncwarp();
#pragma unroll
  for (int i = 0; i < 32; ++i) {
    const U u = to_bits(o[i]);
    if (u >= lo && u <= hi) scratch[off++] = o[i];
  }
  __syncwarp();
  const int nb = cnt_hi - cnt_lo;
  const R x = lane < nb ? scratch[lane] : R(0);
  int rank = 0;
  for (int j = 0; j < nb; ++j) {
    const R y = scratch[j];
    rank += (y < x || (y == x && j < lane)) ? 1 : 0;
  }
  const unsigned m0 = __ballot_sync(kFull, lane < nb && rank == r0);
  v0 = __shfl_sync(kFull, x, __ffs(m0) - 1);
  if (r0 + 1 < nb) {
    const unsigned m1 = __ballot_sync(kFull, lane < nb && rank == r0 + 1);
    v1 = __shfl_sync(kFull, x, __ffs(m1) - 1);
  } else {
    U nxt = ~U(0);
#pragma unroll
    for (int i = 0; i < 32; ++i) {
      const U u = to_bits(o[i]);
      if (u > hi) nxt = min(nxt, u);
    }
    v1 = from_bits(warp_min_u(nxt));
  }
  __syncwarp();
}

template <typename R>
__device__ __forceinline__ R warp_median1024(const R (&o)[32], R* scratch) {
  R v0, v1;
  warp_median_pair<R>(o, scratch, v0, v1);
  return (v0 + v1) * R(0.5);
}

template <typename R>
__device__ __forceinline__ R warp_median1024_pair(const R (&o)[32], R* scratch, R& v0_out, R& v1_out) {
  warp_median_pair<R>(o, scratch, v0_out, v1_out);
  return (v0_out + v1_out) * R(0.5);
}

// One 32-point FFT per lane over a row (rows = true, lane = row) or a column
// (lane = column) of the tile, in place. The direction is a template parameter
// (every shared-memory access then has one address form); not inlined: the
// window code calls it four times and two copies keep the kernel inside the
// instruction cache.
// tw holds e^{-2 pi i k/32} (forward) or its conjugate (inverse), k < 16.
template <typename R, bool rows, int NZ = 32>
__device__ __noinline__ void fft_pass_t(R (*re)[33], R (*im)[33], const typename CT<R>::C* tw, const int lane) {
  using C = typename CT<R>::C;
  C x[32];
  // entries NZ..31 of the row / column are zero (the window's padding) and are
  // not read
#pragma unroll
  for (int k = 0; k < 32; ++k)
    x[k] = k >= NZ ? mk(R(0), R(0)) : (rows ? mk(re[lane][k], im[lane][k]) : mk(re[k][lane], im[k][lane]));
#pragma unroll
  for (int i = 0; i < 32; ++i) {
    const int r = ((i & 1) << 4) | ((i & 2) << 2) | (i & 4) | ((i & 8) >> 2) | ((i & 16) >> 4);
    if (r > i) {
      C t = x[i];
      x[i] = x[r];
      x[r] = t;
    }
  }
#pragma unroll
  for (int half = 1; half < 32; half <<= 1) {
    const int step = 16 / half;
#pragma unroll
    for (int s = 0; s < 32; s += 2 * half) {
#pragma unroll
      for (int k = 0; k < half; ++k) {
        const int ti = k * step;
        const C u = x[s + k];
        const C v = x[s + k + half];
        const C t = ti == 0 ? v : cmul(v, tw[ti]);
        x[s + k] = mk(u.x + t.x, u.y + t.y);
        x[s + k + half] = mk(u.x - t.x, u.y - t.y);
      }
    }
  }
#pragma unroll
  for (int k = 0; k < 32; ++k) {
    if (rows) {
      re[lane][k] = x[k].x;
      im[lane][k] = x[k].y;
    } else {
      re[k][lane] = x[k].x;
      im[k][lane] = x[k].y;
    }
  }
}

template <typename R>
__device__ __forceinline__ void fft_pass(R (*re)[33], R (*im)[33], const typename CT<R>::C* tw, const int lane,
                                         const bool rows) {
  if (rows)
    fft_pass_t<R, true>(re, im, tw, lane);
  else
    fft_pass_t<R, false>(re, im, tw, lane);
}

// One window of one interferogram, computed by one warp in its tile.
// On entry the tile holds the 24x24 window zero-padded to 32x32; on exit rows
// and columns < n_win hold the filtered values times the pyramid weight / 1024.
template <typename R, int NWIN, typename Tile>
__device__ __forceinline__ void clap_window_warp(Tile& T, const int lane, const ClapArgs& a,
                                                 const typename CT<R>::C* twf, const typename CT<R>::C* twi,
                                                 const R* lp, const R* wt, const R (&g7)[7], const int rs,
                                                 const int cs) {
  // forward FFT along rows (rows >= n_win are zero and stay zero), then columns
  if constexpr (NWIN > 0) {
    // a compile-time window: the padding is zero by construction, never stored
    if (lane < NWIN) fft_pass_t<R, true, NWIN>(T.re, T.im, twf, lane);
    __syncwarp();
    fft_pass_t<R, false, NWIN>(T.re, T.im, twf, lane);
  } else {
    if (lane < a.n_win) fft_pass<R>(T.re, T.im, twf, lane, true);
    __syncwarp();
    fft_pass<R>(T.re, T.im, twf, lane, false);
  }
#pragma unroll
  for (int k = 0; k < 32; ++k) {
    const R xr = T.re[k][lane], xi = T.im[k][lane];
    T.hs[k][lane] = sqrt(xr * xr + xi * xi);
  }
  __syncwarp();
  // 7x7 separable Gaussian 'same' convolution of fftshift(|H|), then
  // ifftshift (native_stage2.rs:1097-1166). In unshifted coordinates this is a
  // circular convolution cut at the Nyquist seam: neighbour k+d is used iff
  // 0 <= ((k+16) mod 32) + d < 32.
  R t[32];
  const int sj = (lane + 16) & 31;
  // this lane's taps: zero where the neighbour lies across the seam (adding
  // x * 0 leaves the sum unchanged, so this equals skipping the tap)
  R gl7[7];
#pragma unroll
  for (int d = -3; d <= 3; ++d) gl7[d + 3] = (sj + d >= 0 && sj + d < 32) ? g7[d + 3] : R(0);
#pragma unroll
  for (int k = 0; k < 32; ++k) {
    R acc = R(0);
#pragma unroll
    for (int d = -3; d <= 3; ++d) acc += T.hs[k][(lane + d) & 31] * gl7[d + 3];
    t[k] = acc;
  }
  R o[32];
#pragma unroll
  for (int k = 0; k < 32; ++k) {
    const int sk = (k + 16) & 31;
    R acc = R(0);
#pragma unroll
    for (int d = -3; d <= 3; ++d) {
      if (sk + d >= 0 && sk + d < 32) acc += t[(k + d) & 31] * g7[d + 3];
    }
    o[k] = acc;
  }
  const R med = warp_median1024<R>(o, &T.hs[0][0]);
  // H <- max((H/med)^alpha - 1, 0); spectrum *= H*beta + low_pass
  const R beta = static_cast<R>(a.beta);
  const R alpha = static_cast<R>(a.alpha);
  const R inv_med = med != R(0) ? R(1) / med : R(1);
#pragma unroll
  for (int k = 0; k < 32; ++k) {
    R v = o[k] * inv_med;
    v = a.alpha_is_one ? v - R(1) : pow(v, alpha) - R(1);
    if (v < R(0)) v = R(0);
    const R gk = v * beta + lp[k * 32 + lane];
    T.re[k][lane] *= gk;
    T.im[k][lane] *= gk;
  }
  // inverse FFT along columns, then rows; keep the n_win x n_win corner, weighted
  fft_pass<R>(T.re, T.im, twi, lane, false);
  __syncwarp();
  const int nwv = NWIN > 0 ? NWIN : a.n_win;
  if (lane < nwv) {
    fft_pass<R>(T.re, T.im, twi, lane, true);
    const bool row_zero = lane < rs;
    for (int l = 0; l < nwv; ++l) {
      const R wv = (row_zero || l < cs) ? R(0) : wt[(lane - rs) * kWtStride + (l - cs)];
      T.re[lane][l] *= wv;
      T.im[lane][l] *= wv;
    }
  }
  __syncwarp();
}

// Per-patch constants of the CLAP blocks: the low-pass filter and the
// pyramid weights (the twiddles and smoothing taps are the same for every patch).
template <typename R>
__device__ __forceinline__ void clap_consts(const ClapArgs& a, R* lp, R* wt) {
  const int nw2 = a.n_win * a.n_win;
  for (int i = threadIdx.x; i < 1024; i += blockDim.x) lp[i] = static_cast<R>(a.low_pass[i]);
  for (int i = threadIdx.x; i < nw2; i += blockDim.x)
    wt[(i / a.n_win) * kWtStride + i % a.n_win] = static_cast<R>(a.wscaled[i]);
}

// Window loads and stores of a CLAP block: NW interferograms of one window,
// pixel (li, lj) of interferogram NW*g + q in tiles[q]. FP32 moves two
// interferograms (16 bytes) per access; each thread issues U accesses before
// it touches shared memory. Pixel -> (row, column) uses pix * inv_nw >> 16
// (inv_nw = ceil(65536 / nw)), exact for pix < 1024 and nw <= 32.
template <typename R>
struct ClapIo;
template <>
struct ClapIo<float> {
  static constexpr int kPer = 2;  // interferograms per access
  static constexpr int kU = 8;    // accesses in flight per thread
};
template <>
struct ClapIo<double> {
  static constexpr int kPer = 1;
  static constexpr int kU = 4;
};

// Interferograms c and c + 1 (columns >= M read as zero; only columns < M
// are dereferenced).
__device__ __forceinline__ void clap_fetch(const float2* p, const int c, const int M, float (&v)[4]) {
  if (c + 1 < M) {
    const float4 q = *reinterpret_cast<const float4*>(p);
    v[0] = q.x;
    v[1] = q.y;
    v[2] = q.z;
    v[3] = q.w;
  } else {
    const float2 q = c < M ? *p : make_float2(0.f, 0.f);
    v[0] = q.x;
    v[1] = q.y;
    v[2] = 0.f;
    v[3] = 0.f;
  }
}
__device__ __forceinline__ void clap_fetch(const double2* p, const int c, const int M, double (&v)[2]) {
  const double2 q = c < M ? *p : make_double2(0.0, 0.0);
  v[0] = q.x;
  v[1] = q.y;
}

template <typename R, int NW, typename Tile>
__device__ __forceinline__ void clap_load_tiles(const ClapArgs& a, Tile* tiles, const typename CT<R>::C* grid,
                                                const int i1, const int j1, const int g, const int nw, const int nw2,
                                                const uint32_t inv_nw, const int tid) {
  constexpr int NT = 32 * NW, PER = ClapIo<R>::kPer, U = ClapIo<R>::kU, NQ = NW / PER;
  const int n_items = nw2 * NQ;
  for (int b0 = 0; b0 < n_items; b0 += NT * U) {
    R v[U][2 * PER];
#pragma unroll
    for (int u = 0; u < U; ++u) {
      const int idx = b0 + u * NT + tid;
#pragma unroll
      for (int e = 0; e < 2 * PER; ++e) v[u][e] = R(0);
      if (idx < n_items) {
        const int pix = idx / NQ, q0 = (idx % NQ) * PER;
        const int li = static_cast<int>((static_cast<uint32_t>(pix) * inv_nw) >> 16), lj = pix - li * nw;
        const int c = NW * g + q0;
        clap_fetch(grid + (static_cast<int64_t>(i1 + li) * a.n_j + (j1 + lj)) * a.Mp + c, c, a.M, v[u]);
      }
    }
#pragma unroll
    for (int u = 0; u < U; ++u) {
      const int idx = b0 + u * NT + tid;
      if (idx < n_items) {
        const int pix = idx / NQ, q0 = (idx % NQ) * PER;
        const int li = static_cast<int>((static_cast<uint32_t>(pix) * inv_nw) >> 16), lj = pix - li * nw;
#pragma unroll
        for (int e = 0; e < PER; ++e) {
          R x = v[u][2 * e], y = v[u][2 * e + 1];
          if (isnan(x) || isnan(y)) x = y = R(0);  // NaN -> 0 (clap_filter_one_ifg)
          tiles[q0 + e].re[li][lj] = x;
          tiles[q0 + e].im[li][lj] = y;
        }
      }
    }
  }
}

template <typename R, int NW, typename Tile>
__device__ __forceinline__ void clap_store_tiles(const ClapArgs& a, const Tile* tiles, typename CT<R>::C* out,
                                                 const int64_t wi, const int g, const int nw, const int nw2,
                                                 const uint32_t inv_nw, const int tid) {
  constexpr int NT = 32 * NW, PER = ClapIo<R>::kPer, NQ = NW / PER;
  const int n_items = nw2 * NQ;
  for (int idx = tid; idx < n_items; idx += NT) {
    const int pix = idx / NQ, q0 = (idx % NQ) * PER;
    const int li = static_cast<int>((static_cast<uint32_t>(pix) * inv_nw) >> 16), lj = pix - li * nw;
    const int c = NW * g + q0;
    if (c >= a.Mp) continue;
    typename CT<R>::C* dst = out + (wi * nw2 + pix) * a.Mp + c;
    if constexpr (PER == 2) {
      // Mp is a multiple of 4 and c even: c + 1 < Mp, 16-byte aligned
      *reinterpret_cast<float4*>(dst) = make_float4(tiles[q0].re[li][lj], tiles[q0].im[li][lj],
                                                    tiles[q0 + 1].re[li][lj], tiles[q0 + 1].im[li][lj]);
    } else {
      *dst = mk(tiles[q0].re[li][lj], tiles[q0].im[li][lj]);
    }
  }
}

// Interferogram groups of a CLAP unit (window or window block): a task is
// (unit, group), group g holding interferograms NW * g .. NW * g + NW - 1.
template <typename R, int NW>
__device__ __forceinline__ int clap_groups(const ClapArgs& a) {
  return (a.Mp + NW - 1) / NW;
}

// Window (ix1, ix2) of interferograms NW * g + warp through the block's
// tiles: clap_windows' corner (native_stage2.rs:957-995) returned in i1, j1;
// on exit the tiles hold the weighted filtered window (rows, columns < nw).
template <typename R, int NW, int NWIN = 0>
__device__ __forceinline__ void clap_compute_window(const ClapArgs& a, const int ix1, const int ix2, const int g,
                                                    ClapTileT<R, ClapShape<NW>::kPad>* tiles,
                                                    const typename CT<R>::C* twf, const typename CT<R>::C* twi,
                                                    const R* lp, const R* wt, const R (&g7)[7], int& i1, int& j1) {
  using C = typename CT<R>::C;
  constexpr int NT = 32 * NW;
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const int nw = NWIN > 0 ? NWIN : a.n_win, nw2 = nw * nw;
  const int n_inc = nw / 4 > 1 ? nw / 4 : 1;
  const C* __restrict__ grid = static_cast<const C*>(a.grid);
  auto& T = tiles[warp];
  i1 = ix1 * n_inc;
  int rs = 0;
  if (i1 + nw > a.n_i) {
    rs = i1 + nw - a.n_i;
    i1 = a.n_i - nw;
  }
  j1 = ix2 * n_inc;
  int cs = 0;
  if (j1 + nw > a.n_j) {
    cs = j1 + nw - a.n_j;
    j1 = a.n_j - nw;
  }
  __syncthreads();
  // zero the padding of the tiles (none for a 32-pixel window)
  if (NWIN == 0 && nw < 32) {
    for (int idx = tid; idx < NW * 32 * 32; idx += NT) {
      const int q = idx >> 10, e = idx & 1023, r = e >> 5, cc = e & 31;
      if (r >= nw || cc >= nw) {
        tiles[q].re[r][cc] = R(0);
        tiles[q].im[r][cc] = R(0);
      }
    }
  }
  const uint32_t inv_nw = (65536u + static_cast<uint32_t>(nw) - 1u) / static_cast<uint32_t>(nw);
  clap_load_tiles<R, NW>(a, tiles, grid, i1, j1, g, nw, nw2, inv_nw, tid);
  __syncthreads();
  if (NW * g + warp < a.M) clap_window_warp<R, NWIN>(T, lane, a, twf, twi, lp, wt, g7, rs, cs);
  __syncthreads();
}

// One block-task of the window-stack form: window a.w_lo + task / ngroups; the
// weighted window goes to win_out for the overlap-add pass.
template <typename R, int NW, int NWIN = 0>
__device__ __forceinline__ void clap_task(const ClapArgs& a, const int64_t task,
                                          ClapTileT<R, ClapShape<NW>::kPad>* tiles, const typename CT<R>::C* twf,
                                          const typename CT<R>::C* twi, const R* lp, const R* wt, const R (&g7)[7]) {
  const int ngroups = clap_groups<R, NW>(a);
  const int nw = NWIN > 0 ? NWIN : a.n_win, nw2 = nw * nw;
  const int64_t wi = a.w_lo + task / ngroups;
  const int g = static_cast<int>(task - (wi - a.w_lo) * ngroups);
  const int ix1 = static_cast<int>(wi / a.nwj), ix2 = static_cast<int>(wi - static_cast<int64_t>(ix1) * a.nwj);
  int i1, j1;
  clap_compute_window<R, NW, NWIN>(a, ix1, ix2, g, tiles, twf, twi, lp, wt, g7, i1, j1);
  const uint32_t inv_nw = (65536u + static_cast<uint32_t>(nw) - 1u) / static_cast<uint32_t>(nw);
  clap_store_tiles<R, NW>(a, tiles, static_cast<typename CT<R>::C*>(a.win_out), wi, g, nw, nw2, inv_nw,
                          threadIdx.x);
}

// ---- overlap-add fused into the window pass (window blocks) -------------------
// The windows are taken in blocks of 4 x 4 (window rows 4 bi .. 4 bi + 3,
// columns 4 bj .. 4 bj + 3). A block's windows cover a box of at most
// clap_box(n_win) = 3 n_inc + n_win cells a side from the corner of its first
// window; one block-task runs the block's windows in order (ix1, then ix2) for
// NW interferograms and adds each weighted window into the block's FP64
// partial sum of the box (part: [block][box row][box column][Mp] of complex
// FP64; the first window of the block that covers a cell stores instead of
// adding), so a cell's partial is the reference's ordered sum
// (native_stage2.rs:1166-1184) over the block's windows. The combine pass
// adds a cell's block partials (2 x 2 at most for 24-cell windows) in block
// order and rounds once. The window stack of the two-pass form (1.1 GB for a
// 256 x 256 x 150 grid) is never written; the partials are 2.7x the grid and a
// block's box stays in L2 while its windows run.
constexpr int kClapBlockWin = 4;
__host__ __device__ inline int clap_box(int n_win) {
  const int n_inc = n_win / 4 > 1 ? n_win / 4 : 1;
  return (kClapBlockWin - 1) * n_inc + n_win;
}
__host__ __device__ inline int clap_block_rows(int nw_axis) { return (nw_axis + kClapBlockWin - 1) / kClapBlockWin; }

// Add (or store, for a cell no earlier window of the block covered) the
// weighted window in the tiles to the block partial. Box corner (r0, c0); pi1 /
// pj1 the corner row / column of the block's previous window row / column
// (rows < pi1 + nw were covered already), or a value that marks none. One item
// per (pixel, interferogram): NW consecutive threads write one cell's NW
// interferograms, 16 * NW contiguous bytes; each thread issues the partial
// loads of kAccBatch items before any add, so their L2 round trips overlap.
constexpr int kAccBatch = 6;
template <typename R, int NW, typename Tile>
__device__ __forceinline__ void clap_accum_tiles(const ClapArgs& a, const Tile* tiles, double2* __restrict__ part,
                                                 const int64_t blk, const int box, const int i1, const int j1,
                                                 const int r0, const int c0, const int pi1, const int pj1,
                                                 const int g, const int nw, const int nw2, const uint32_t inv_nw,
                                                 const int tid) {
  constexpr int NT = 32 * NW;
  const int n_items = nw2 * NW;
  for (int b0 = tid; b0 < n_items; b0 += NT * kAccBatch) {
    double2 old[kAccBatch];
    int64_t off[kAccBatch];
    int li[kAccBatch], lj[kAccBatch], qq[kAccBatch];
    bool live[kAccBatch], first[kAccBatch];
#pragma unroll
    for (int u = 0; u < kAccBatch; ++u) {
      const int idx = b0 + u * NT;
      const int pix = idx / NW, q = idx - (idx / NW) * NW;
      const int c = NW * g + q;
      live[u] = idx < n_items && c < a.M;
      li[u] = static_cast<int>((static_cast<uint32_t>(pix) * inv_nw) >> 16);
      lj[u] = pix - li[u] * nw;
      qq[u] = q;
      const int ai = i1 + li[u], aj = j1 + lj[u];
      first[u] = ai >= pi1 + nw && aj >= pj1 + nw;
      off[u] = ((blk * box + (ai - r0)) * box + (aj - c0)) * a.Mp + c;
      old[u] = make_double2(0.0, 0.0);
      if (live[u] && !first[u]) old[u] = part[off[u]];
    }
#pragma unroll
    for (int u = 0; u < kAccBatch; ++u) {
      if (!live[u]) continue;
      const double vx = static_cast<double>(tiles[qq[u]].re[li[u]][lj[u]]);
      const double vy = static_cast<double>(tiles[qq[u]].im[li[u]][lj[u]]);
      part[off[u]] = first[u] ? make_double2(vx, vy) : make_double2(__dadd_rn(old[u].x, vx), __dadd_rn(old[u].y, vy));
    }
  }
}

// One block-task of the fused form: window block a.w_lo + task / ngroups.
template <typename R, int NW, int NWIN = 0>
__device__ __forceinline__ void clap_block_task(const ClapArgs& a, const int64_t task,
                                                ClapTileT<R, ClapShape<NW>::kPad>* tiles,
                                                const typename CT<R>::C* twf, const typename CT<R>::C* twi,
                                                const R* lp, const R* wt, const R (&g7)[7]) {
  const int ngroups = clap_groups<R, NW>(a);
  const int nw = NWIN > 0 ? NWIN : a.n_win, nw2 = nw * nw;
  const int n_inc = nw / 4 > 1 ? nw / 4 : 1;
  const int box = clap_box(nw);
  const int nbj = clap_block_rows(a.nwj);
  const int64_t blk = a.w_lo + task / ngroups;
  const int g = static_cast<int>(task - (blk - a.w_lo) * ngroups);
  const int bi = static_cast<int>(blk / nbj), bj = static_cast<int>(blk - static_cast<int64_t>(bi) * nbj);
  const int ixa = kClapBlockWin * bi, ixb = min(ixa + kClapBlockWin, a.nwi);
  const int jxa = kClapBlockWin * bj, jxb = min(jxa + kClapBlockWin, a.nwj);
  const int r0 = min(ixa * n_inc, a.n_i - nw), c0 = min(jxa * n_inc, a.n_j - nw);
  const uint32_t inv_nw = (65536u + static_cast<uint32_t>(nw) - 1u) / static_cast<uint32_t>(nw);
  double2* part = static_cast<double2*>(a.part);
  constexpr int kNone = -(1 << 20);
  for (int ix1 = ixa; ix1 < ixb; ++ix1) {
    const int pi1 = ix1 > ixa ? min((ix1 - 1) * n_inc, a.n_i - nw) : kNone;
    for (int ix2 = jxa; ix2 < jxb; ++ix2) {
      const int pj1 = ix2 > jxa ? min((ix2 - 1) * n_inc, a.n_j - nw) : kNone;
      int i1, j1;
      clap_compute_window<R, NW, NWIN>(a, ix1, ix2, g, tiles, twf, twi, lp, wt, g7, i1, j1);
      clap_accum_tiles<R, NW>(a, tiles, part, blk, box, i1, j1, r0, c0, pi1, pj1, g, nw, nw2, inv_nw,
                              threadIdx.x);
    }
  }
}

// shared-memory carve-up of a CLAP block: NW tiles, low-pass, weights, twiddles
template <typename R, int NW>
struct ClapSmem {
  ClapTileT<R, ClapShape<NW>::kPad>* tiles;
  R* lp;
  R* wt;
  typename CT<R>::C* twf;
  typename CT<R>::C* twi;
};

template <typename R, int NW>
__device__ __forceinline__ ClapSmem<R, NW> clap_smem(unsigned char* raw, const typename CT<R>::Tw& tw) {
  ClapSmem<R, NW> m;
  m.tiles = reinterpret_cast<ClapTileT<R, ClapShape<NW>::kPad>*>(raw);
  m.lp = reinterpret_cast<R*>(m.tiles + NW);
  m.wt = m.lp + 1024;
  m.twf = reinterpret_cast<typename CT<R>::C*>(m.wt + 32 * kWtStride);
  m.twi = m.twf + 16;
  if (threadIdx.x < 16) {
    m.twf[threadIdx.x] = tw.w[threadIdx.x];
    m.twi[threadIdx.x] = mk(tw.w[threadIdx.x].x, -tw.w[threadIdx.x].y);
  }
  return m;
}

// FUSED: window blocks into the partials (the loop's form); otherwise windows
// into the window stack. FP32 blocks are held to the registers that let as
// many of them reside as their shared memory does (two of eight warps, three
// of four).
template <typename R, int NW, int NWIN, bool FUSED>
__global__ void __launch_bounds__(32 * NW, sizeof(R) == 4 ? (NW == 8 ? 2 : 3) : 1)
    k_clap(ClapArgs a, typename CT<R>::Tw tw) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  const ClapSmem<R, NW> m = clap_smem<R, NW>(smem_raw, tw);
  clap_consts<R>(a, m.lp, m.wt);
  R g7[7];
#pragma unroll
  for (int i = 0; i < 7; ++i) g7[i] = static_cast<R>(a.g7[i]);
  // units: window blocks (fused) or windows (window stack)
  const int64_t nunit = a.w_n > 0 ? a.w_n
                        : FUSED ? static_cast<int64_t>(clap_block_rows(a.nwi)) * clap_block_rows(a.nwj)
                                : static_cast<int64_t>(a.nwi) * a.nwj;
  const int64_t ntask = nunit * clap_groups<R, NW>(a);
  for (int64_t task = blockIdx.x; task < ntask; task += gridDim.x) {
    if constexpr (FUSED)
      clap_block_task<R, NW, NWIN>(a, task, m.tiles, m.twf, m.twi, m.lp, m.wt, g7);
    else
      clap_task<R, NW, NWIN>(a, task, m.tiles, m.twf, m.twi, m.lp, m.wt, g7);
  }
}

template <typename R, int NW>
static size_t clap_smem_bytes() {
  return NW * sizeof(ClapTileT<R, ClapShape<NW>::kPad>) + (1024 + 32 * kWtStride) * sizeof(R) + 32 * 2 * sizeof(R);
}

template <typename R, int NW, int NWIN>
static cudaError_t launch_clap_nwin(const ClapArgs& a, const typename CT<R>::Tw& tw, int sm_count, cudaStream_t st) {
  if (a.nwi <= 0 || a.nwj <= 0) return cudaSuccess;
  const int64_t nunit = a.w_n > 0 ? a.w_n
                        : a.part ? static_cast<int64_t>(clap_block_rows(a.nwi)) * clap_block_rows(a.nwj)
                                 : static_cast<int64_t>(a.nwi) * a.nwj;
  const int64_t ntask = nunit * ((a.Mp + NW - 1) / NW);
  if (ntask <= 0) return cudaSuccess;
  const size_t sm = clap_smem_bytes<R, NW>();
  cudaError_t e = kernel_attributes_once(sm);
  if (e != cudaSuccess) return e;
  int per_sm = 0;
  if (a.part)
    e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_clap<R, NW, NWIN, true>, 32 * NW, sm);
  else
    e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_clap<R, NW, NWIN, false>, 32 * NW, sm);
  if (e != cudaSuccess) return e;
  if (a.blocks_per_sm > 0 && a.blocks_per_sm < per_sm) per_sm = a.blocks_per_sm;
  const int64_t blocks = std::min<int64_t>(ntask, static_cast<int64_t>(sm_count) * (per_sm > 0 ? per_sm : 1));
  if (a.part)
    k_clap<R, NW, NWIN, true><<<static_cast<unsigned>(blocks), 32 * NW, sm, st>>>(a, tw);
  else
    k_clap<R, NW, NWIN, false><<<static_cast<unsigned>(blocks), 32 * NW, sm, st>>>(a, tw);
  return cudaGetLastError();
}

// the 24-pixel window (clap_win 32 x 0.75) as a compile-time shape, others at run time
template <typename R, int NW>
static cudaError_t launch_clap_nw(const ClapArgs& a, const typename CT<R>::Tw& tw, int sm_count, cudaStream_t st) {
  return a.n_win == 24 ? launch_clap_nwin<R, NW, 24>(a, tw, sm_count, st) : launch_clap_nwin<R, NW, 0>(a, tw, sm_count, st);
}

// FP32: 8 warps per block by default (16 resident warps per SM, shared memory
// bound), 4 when the launch shape asks for it; FP64: 4 (its tiles are twice the
// size). Every window's arithmetic is the same whatever the shape.
cudaError_t launch_clap(const ClapArgs& a, bool fp64, const Twiddles32f& tf, const Twiddles32d& td, int sm_count,
                        cudaStream_t st) {
  if (fp64) return launch_clap_nw<double, 4>(a, td, sm_count, st);
  return a.nw_block == 4 ? launch_clap_nw<float, 4>(a, tf, sm_count, st) : launch_clap_nw<float, 8>(a, tf, sm_count, st);
}

// Overlap-add as a gather: cell (i, j) sums the windows that cover it, in the
// reference's raster window order, in f64 (the reference accumulates in f64).
template <typename R>
__device__ __forceinline__ void overlap_elem(const OverlapArgs& a, const int64_t idx) {
  using C = typename CT<R>::C;
  const C* __restrict__ win = static_cast<const C*>(a.win_out);
  C* __restrict__ filt = static_cast<C*>(a.filt);
  const int nw = a.n_win, nw2 = nw * nw;
  {
    const int64_t cell = idx / a.Mp;
    const int c = static_cast<int>(idx - cell * a.Mp);
    const int i = static_cast<int>(cell / a.n_j), j = static_cast<int>(cell - static_cast<int64_t>(i) * a.n_j);
    double sx = 0.0, sy = 0.0;
    if (c < a.M && a.nwi > 0 && a.nwj > 0) {
      const int a1 = max(0, i / a.n_inc - 4), b1 = min(a.nwi - 1, i / a.n_inc + 1);
      const int a2 = max(0, j / a.n_inc - 4), b2 = min(a.nwj - 1, j / a.n_inc + 1);
      // the (at most 6) candidate windows along j, their offsets and validity
      int lj6[6];
      bool okj[6];
#pragma unroll
      for (int w = 0; w < 6; ++w) {
        const int ix2 = a2 + w;
        const int lj = j - min(ix2 * a.n_inc, a.n_j - nw);
        okj[w] = ix2 <= b2 && lj >= 0 && lj < nw;
        lj6[w] = lj;
      }
      for (int ix1 = a1; ix1 <= b1; ++ix1) {
        const int i1 = min(ix1 * a.n_inc, a.n_i - nw);
        const int li = i - i1;
        if (li < 0 || li >= nw) continue;
        // one row of covering windows: every load issued before the ordered sum
        C v[6];
#pragma unroll
        for (int w = 0; w < 6; ++w)
          v[w] = okj[w] ? win[((static_cast<int64_t>(ix1) * a.nwj + a2 + w) * nw2 + li * nw + lj6[w]) * a.Mp + c]
                        : mk(R(0), R(0));
#pragma unroll
        for (int w = 0; w < 6; ++w)
          if (okj[w]) {
            sx += static_cast<double>(v[w].x);
            sy += static_cast<double>(v[w].y);
          }
      }
    }
    C f = mk(static_cast<R>(sx), static_cast<R>(sy));
    if constexpr (sizeof(R) == 4) {
      if (a.normalize) {
        // normalize_complex_unit_magnitude (:1186-1205) once per cell instead of
        // once per PS of the cell in the topofit; the same expression, the same bits
        const float mag = hypotf(f.x, f.y);
        if (mag != 0.f) f = make_float2(f.x / mag, f.y / mag);
      }
    }
    filt[idx] = f;
  }
}

// Fused form: the cell's block partials (those whose boxes hold the cell: 2 x 2
// at most for 24-cell windows) added in block order in FP64, then rounded and
// normalised as overlap_elem does.
template <typename R>
__device__ __forceinline__ void combine_elem(const OverlapArgs& a, const int64_t idx) {
  using C = typename CT<R>::C;
  const double2* __restrict__ part = static_cast<const double2*>(a.part);
  C* __restrict__ filt = static_cast<C*>(a.filt);
  const int nw = a.n_win, box = clap_box(nw);
  const int64_t cell = idx / a.Mp;
  const int c = static_cast<int>(idx - cell * a.Mp);
  const int i = static_cast<int>(cell / a.n_j), j = static_cast<int>(cell - static_cast<int64_t>(i) * a.n_j);
  double sx = 0.0, sy = 0.0;
  if (c < a.M && a.nwi > 0 && a.nwj > 0) {
    const int nbi = clap_block_rows(a.nwi), nbj = clap_block_rows(a.nwj);
    // blocks whose boxes [corner of the first window, corner of the last + nw)
    // hold (i, j), in block order: the box corners do not decrease along an
    // axis, and no box that holds i starts before block (i - nw) / (4 n_inc) - 1
    const int bj_lo = max(0, (j - nw) / (kClapBlockWin * a.n_inc) - 1);
    for (int bi = max(0, (i - nw) / (kClapBlockWin * a.n_inc) - 1); bi < nbi; ++bi) {
      const int r0 = min(kClapBlockWin * bi * a.n_inc, a.n_i - nw);
      if (r0 > i) break;
      const int r1 = min((min(kClapBlockWin * bi + kClapBlockWin, a.nwi) - 1) * a.n_inc, a.n_i - nw) + nw;
      if (i >= r1) continue;
      for (int bj = bj_lo; bj < nbj; ++bj) {
        const int c0 = min(kClapBlockWin * bj * a.n_inc, a.n_j - nw);
        if (c0 > j) break;
        const int c1 = min((min(kClapBlockWin * bj + kClapBlockWin, a.nwj) - 1) * a.n_inc, a.n_j - nw) + nw;
        if (j >= c1) continue;
        const int64_t blk = static_cast<int64_t>(bi) * nbj + bj;
        const double2 p = part[((blk * box + (i - r0)) * box + (j - c0)) * a.Mp + c];
        sx = __dadd_rn(sx, p.x);
        sy = __dadd_rn(sy, p.y);
      }
    }
  }
  C f = mk(static_cast<R>(sx), static_cast<R>(sy));
  if constexpr (sizeof(R) == 4) {
    if (a.normalize) {
      const float mag = hypotf(f.x, f.y);
      if (mag != 0.f) f = make_float2(f.x / mag, f.y / mag);
    }
  }
  filt[idx] = f;
}

template <typename R>
__global__ void __launch_bounds__(256) k_overlap(OverlapArgs a) {
  const int64_t cells = a.cell_n > 0 ? a.cell_n : static_cast<int64_t>(a.n_i) * a.n_j;
  const int64_t total = cells * a.Mp, base = a.cell_lo * a.Mp;
  for (int64_t idx = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x; idx < total;
       idx += static_cast<int64_t>(gridDim.x) * blockDim.x) {
    if (a.part)
      combine_elem<R>(a, base + idx);
    else
      overlap_elem<R>(a, base + idx);
  }
}

cudaError_t launch_overlap(const OverlapArgs& a, bool fp64, cudaStream_t st) {
  const int64_t cells = a.cell_n > 0 ? a.cell_n : static_cast<int64_t>(a.n_i) * a.n_j;
  const int64_t total = cells * a.Mp;
  int64_t blocks = (total + 255) / 256;
  if (blocks > 148 * 32) blocks = 148 * 32;
  if (blocks < 1) blocks = 1;
  if (fp64)
    k_overlap<double><<<static_cast<unsigned>(blocks), 256, 0, st>>>(a);
  else
    k_overlap<float><<<static_cast<unsigned>(blocks), 256, 0, st>>>(a);
  return cudaGetLastError();
}

// =============================================================== topofit ==
// One group of L lanes per PS (L = 4, 8, 16 or 32, chosen from the number of
// interferograms so a lane owns about 5-10 columns); a warp holds 32/L PS.
// Column data (psdph z_c, the per-step rotation, bp_c) live in shared memory.
// The trial sweep finds the first argmax over the trials of |S_m|,
//   S_m = sum_c z_c e^{-j theta_c m},  theta_c = bp_c / range * pi/4,
// 16 magnitudes |m| at a time with the trial pairs +-m sharing one phasor
// chain, two trials per packed FP32x2 value, the chain started exactly in the
// middle of the block and run both ways by the three-term recurrence; the group
// then reduces its partial sums with a transposing butterfly. For n_half in
// 41 .. 87 it is sampled (sampled_sweep): the centred sum is evaluated at every
// 4th trial and interpolated between; otherwise every magnitude is swept
// (sweep_trial_pairs).

constexpr float kQuarterPiF = 3.14159265358979323846f / 4.0f;  // Rust std::f32::consts::PI / 4.0

// e^{-j x} for the re-anchoring points, |x| < ~1e3: Cody-Waite argument
// reduction by 2 pi with a two-constant split of 2 pi (Cody & Waite, "Software
// Manual for the Elementary Functions", 1980) to |r| <= pi, then the hardware
// sin/cos approximations (absolute error ~4e-7 on that range; a reduction to
// pi/4 with a quadrant rotation buys no accuracy there and costs a conversion
// and four selects per call).
__device__ __forceinline__ float2 cis_neg_anchor(float x) {
  const float k = rintf(x * 0.159154943091895335769f);
  float r = fmaf(-k, 6.28318548202514648438f, x);
  r = fmaf(-k, -1.74845553146951715e-7f, r);
  return make_float2(__cosf(r), -__sinf(r));
}

template <int L>
__device__ __forceinline__ float group_sum(float v) {
#pragma unroll
  for (int o = L / 2; o > 0; o >>= 1) v += __shfl_xor_sync(kFull, v, o);
  return v;
}
template <int L>
__device__ __forceinline__ double group_sum(double v) {
#pragma unroll
  for (int o = L / 2; o > 0; o >>= 1) v += __shfl_xor_sync(kFull, v, o);
  return v;
}
template <int L>
__device__ __forceinline__ float group_min(float v) {
#pragma unroll
  for (int o = L / 2; o > 0; o >>= 1) v = fminf(v, __shfl_xor_sync(kFull, v, o));
  return v;
}
template <int L>
__device__ __forceinline__ float group_max(float v) {
#pragma unroll
  for (int o = L / 2; o > 0; o >>= 1) v = fmaxf(v, __shfl_xor_sync(kFull, v, o));
  return v;
}

// Sum over the L lanes of a group of each of the W slots of v. Halving steps
// (lanes whose offset bit is set keep the upper half) while more than one slot
// remains, plain xor reductions after that. Returns the number of slots the
// lane holds (max(W/L, 1)) in v[0..]; they are slots base .. base+count-1.
template <int W, int L>
__device__ __forceinline__ int group_transpose_reduce(float2 (&v)[W], const int gl, int& base) {
  int cnt = W;
  base = 0;
#pragma unroll
  for (int o = L / 2; o >= 1; o >>= 1) {
    if (cnt > 1) {
      const int h = cnt / 2;
      const bool upper = (gl & o) != 0;
#pragma unroll
      for (int i = 0; i < W / 2; ++i) {
        if (i < h) {
          const float2 lo = v[i], hi = v[i + h];
          float2 send = upper ? lo : hi;
          const float2 keep = upper ? hi : lo;
          send.x = __shfl_xor_sync(kFull, send.x, o);
          send.y = __shfl_xor_sync(kFull, send.y, o);
          v[i] = make_float2(keep.x + send.x, keep.y + send.y);
        }
      }
      if (upper) base += h;
      cnt = h;
    } else {
      v[0].x += __shfl_xor_sync(kFull, v[0].x, o);
      v[0].y += __shfl_xor_sync(kFull, v[0].y, o);
    }
  }
  return cnt;
}

// Per-PS column store: z (psdph), e^{-j theta} (the per-trial rotation, theta =
// bp/range*pi/4 as the reference rounds it) and bp. Anchor angles are formed as
// bp * ((pi/4)/range) * m.
struct ColumnSmem {
  float *zx, *zy, *rx, *ry, *bp;
};

// Trials +m and -m from one rotation chain, two columns per packed FP32x2
// instruction (the form of the last, odd magnitude of a sweep; the blocks of
// 2-16 magnitudes pack two trials instead, sweep_trial_pairs). For a column z = (x, y) and w = e^{-j m theta}:
//   z w       = (x w.x - y w.y, x w.y + y w.x)               trial +m
//   z conj(w) = (x w.x + y w.y, y w.x - x w.y) = z e^{+j m theta}   trial -m
// so the four sums  sum x w.x, sum x w.y, sum y w.y, sum y w.x  give both
// trials. A lane holds its columns in pairs (c0, c1) = (gl + L k, gl + L (k+1)):
// Wx = (w0.x, w1.x), Wy = (w0.y, w1.y) and the accumulators are FP32x2 pairs
// (one column of the pair in each half), added together once per block. One
// |m| step is then 4 packed instructions for the rotation
//   Wx <- Wx Rx - Wy Ry,  Wy <- Wx Ry + Wy Rx      (R = e^{-j theta})
// and 4 for the sums, i.e. 1 instruction per (trial, column). w is re-anchored
// exactly (cis_neg_anchor of theta * m) at the first |m| of every block, so a
// chain is at most W - 1 rotations long.
struct PackedCols {
  float2 x, y, rx, ry, nry, wx, wy;
};

__device__ __forceinline__ PackedCols load_packed_cols(const ColumnSmem& cs, const int c0, const int c1,
                                                       const float qr, const int m0) {
  PackedCols p;
  p.x = make_float2(cs.zx[c0], cs.zx[c1]);
  p.y = make_float2(cs.zy[c0], cs.zy[c1]);
  p.rx = make_float2(cs.rx[c0], cs.rx[c1]);
  p.ry = make_float2(cs.ry[c0], cs.ry[c1]);
  p.nry = make_float2(-p.ry.x, -p.ry.y);
  const float2 w0 = cis_neg_anchor(cs.bp[c0] * qr * static_cast<float>(m0));
  const float2 w1 = cis_neg_anchor(cs.bp[c1] * qr * static_cast<float>(m0));
  p.wx = make_float2(w0.x, w1.x);
  p.wy = make_float2(w0.y, w1.y);
  return p;
}

template <int W>
__device__ __forceinline__ void accumulate_packed(float2 (&Axx)[W], float2 (&Axy)[W], float2 (&Ayy)[W],
                                                  float2 (&Ayx)[W], PackedCols& p, const int k) {
  Axx[k] = __ffma2_rn(p.x, p.wx, Axx[k]);
  Axy[k] = __ffma2_rn(p.x, p.wy, Axy[k]);
  Ayy[k] = __ffma2_rn(p.y, p.wy, Ayy[k]);
  Ayx[k] = __ffma2_rn(p.y, p.wx, Ayx[k]);
  if (k + 1 < W) {
    const float2 t = __fmul2_rn(p.wy, p.nry);
    const float2 u = __fmul2_rn(p.wy, p.rx);
    const float2 wx = p.wx;
    p.wx = __ffma2_rn(wx, p.rx, t);
    p.wy = __ffma2_rn(wx, p.ry, u);
  }
}

// One block of W trial pairs |m| = m0 .. m0+W-1 (m0 >= 1): trial indices
// n_half + m and n_half - m. ncl (columns per lane) is even. The running best
// keeps the first maximum in trial order (argmax_first_f32, :1526-1536)
// although the trials arrive out of order.
template <int W, int L>
__device__ __forceinline__ void sweep_pairs(const ColumnSmem& cs, const float qr, const int ncl, const int gl,
                                            const int m0, const int n_half, float& best_sq, int& best_t) {
  float2 Axx[W], Axy[W], Ayy[W], Ayx[W];
#pragma unroll
  for (int k = 0; k < W; ++k) {
    Axx[k] = make_float2(0.f, 0.f);
    Axy[k] = make_float2(0.f, 0.f);
    Ayy[k] = make_float2(0.f, 0.f);
    Ayx[k] = make_float2(0.f, 0.f);
  }
  int k = 0;
  for (; k + 3 < ncl; k += 4) {
    PackedCols p0 = load_packed_cols(cs, gl + L * k, gl + L * (k + 1), qr, m0);
    PackedCols p1 = load_packed_cols(cs, gl + L * (k + 2), gl + L * (k + 3), qr, m0);
#pragma unroll
    for (int j = 0; j < W; ++j) {
      accumulate_packed<W>(Axx, Axy, Ayy, Ayx, p0, j);
      accumulate_packed<W>(Axx, Axy, Ayy, Ayx, p1, j);
    }
  }
  if (k < ncl) {
    PackedCols p0 = load_packed_cols(cs, gl + L * k, gl + L * (k + 1), qr, m0);
#pragma unroll
    for (int j = 0; j < W; ++j) accumulate_packed<W>(Axx, Axy, Ayy, Ayx, p0, j);
  }
  float2 S[2 * W];
#pragma unroll
  for (int j = 0; j < W; ++j) {
    const float xx = Axx[j].x + Axx[j].y, xy = Axy[j].x + Axy[j].y;
    const float yy = Ayy[j].x + Ayy[j].y, yx = Ayx[j].x + Ayx[j].y;
    S[j] = make_float2(xx - yy, xy + yx);
    S[W + j] = make_float2(xx + yy, yx - xy);
  }
  int base;
  const int cnt = group_transpose_reduce<2 * W, L>(S, gl, base);
#pragma unroll
  for (int j = 0; j < (2 * W / L > 1 ? 2 * W / L : 1); ++j) {
    if (j < cnt) {
      const int idx = base + j;
      const int t = idx < W ? n_half + m0 + idx : n_half - (m0 + idx - W);
      const float sq = S[j].x * S[j].x + S[j].y * S[j].y;
      if (sq > best_sq || (sq == best_sq && t < best_t)) {
        best_sq = sq;
        best_t = t;
      }
    }
  }
}

// One block of W trial magnitudes |m| = m0 .. m0+W-1 (W even, m0 >= 1) with
// two TRIALS per packed FP32x2 value: slot i of each accumulator holds
// (|m| = m0+2i, m0+2i+1), so W trial pairs cost 2W accumulator registers and
// one exact anchor per column covers all W magnitudes. Per column, with
// A = H/2 - 1 the middle slot: w(m0+2A) = e^{-j (m0+2A) theta} exactly,
// w(m0+2A+1) = w(m0+2A) e^{-j theta}, the next pair by one complex multiply with
// e^{-2j theta}, and every other pair, up and down from there, by the
// three-term recurrence of cos and sin (Chebyshev):
//   w(m+2) = 2 cos(2 theta) w(m) - w(m-2),   w(m-2) = 2 cos(2 theta) w(m) - w(m+2),
// one packed FMA per component instead of a complex multiply. It is carried as
// u_i = s_i w(m0+2i) with the sign pattern s_{A+j} = +,+,-,-,+,+,... (j mod 4)
// so that each step is a plain FMA (C = 2 cos 2theta):
//   u_{i+1} = ((i-A) odd ? -C : C) u_i + u_{i-1},  u_{i-1} = u_{i+1} - ((i-A) odd ? -C : C) u_i;
// the slot's sums then carry the factor s_i, which |S|^2 does not see.
// An error e in the two starting pairs grows to at most (k+1) e after k steps
// (|U_k(cos phi)| = |sin (k+1) phi / sin phi| <= k+1); starting in the middle
// keeps k <= H/2, so the phasor error stays near 2e-6 for H = 8 (1.4e-6 for a
// chain of complex multiplies), against 5.5e-6 for a chain started at slot 0.
// The four sums P = sum x w.x, Q = sum x w.y, R = sum y w.x, U = sum y w.y give
// S(+m) = (P - U, Q + R) and S(-m) = (P + U, R - Q) for both trials of a slot
// (up to the common sign s_i). Each lane sums its columns in column order; the
// group joins its lanes with the transposing reduction.
template <int W, int L>
__device__ __forceinline__ void sweep_trial_pairs(const ColumnSmem& cs, const float qr, const int ncl, const int gl,
                                                  const int m0, const int n_half, float& best_sq, int& best_t) {
  constexpr int H = W / 2;
  float2 P[H], Q[H], R[H], U[H];
#pragma unroll
  for (int i = 0; i < H; ++i) {
    P[i] = make_float2(0.f, 0.f);
    Q[i] = make_float2(0.f, 0.f);
    R[i] = make_float2(0.f, 0.f);
    U[i] = make_float2(0.f, 0.f);
  }
#pragma unroll 2
  for (int k = 0; k < ncl; ++k) {
    const int c = gl + L * k;
    const float x = cs.zx[c], y = cs.zy[c], rx = cs.rx[c], ry = cs.ry[c];
    // the chain starts at slot A (the middle of the block) and runs both ways
    constexpr int A = H > 1 ? H / 2 - 1 : 0;
    const float2 a0 = cis_neg_anchor(cs.bp[c] * qr * static_cast<float>(m0 + 2 * A));
    const float a1x = fmaf(a0.x, rx, -a0.y * ry), a1y = fmaf(a0.x, ry, a0.y * rx);
    const float r2x = fmaf(rx, rx, -ry * ry), r2y = 2.f * rx * ry;
    const float2 X = make_float2(x, x), Y = make_float2(y, y);
    const float2 Cp = make_float2(2.f * r2x, 2.f * r2x), Cn = make_float2(-2.f * r2x, -2.f * r2x);
    // u_A = (w(m0+2A), w(m0+2A+1)), u_{A+1} = u_A e^{-2j theta}
    const float2 UAx = make_float2(a0.x, a1x), UAy = make_float2(a0.y, a1y);
    P[A] = __ffma2_rn(X, UAx, P[A]);
    Q[A] = __ffma2_rn(X, UAy, Q[A]);
    R[A] = __ffma2_rn(Y, UAx, R[A]);
    U[A] = __ffma2_rn(Y, UAy, U[A]);
    if (H > 1) {
      const float2 UBx = make_float2(fmaf(a0.x, r2x, -a0.y * r2y), fmaf(a1x, r2x, -a1y * r2y));
      const float2 UBy = make_float2(fmaf(a0.x, r2y, a0.y * r2x), fmaf(a1x, r2y, a1y * r2x));
      // forward: u_{i+1} = (i - A odd ? -C : C) u_i + u_{i-1}
      float2 Vx = UAx, Vy = UAy, Wx = UBx, Wy = UBy;
#pragma unroll
      for (int i = A + 1; i < H; ++i) {
        P[i] = __ffma2_rn(X, Wx, P[i]);
        Q[i] = __ffma2_rn(X, Wy, Q[i]);
        R[i] = __ffma2_rn(Y, Wx, R[i]);
        U[i] = __ffma2_rn(Y, Wy, U[i]);
        if (i + 1 < H) {
          const float2 nx = __ffma2_rn(((i - A) & 1) ? Cn : Cp, Wx, Vx);
          const float2 ny = __ffma2_rn(((i - A) & 1) ? Cn : Cp, Wy, Vy);
          Vx = Wx;
          Vy = Wy;
          Wx = nx;
          Wy = ny;
        }
      }
      // backward: u_{i-1} = u_{i+1} - (i - A odd ? -C : C) u_i
      Vx = UBx;
      Vy = UBy;
      Wx = UAx;
      Wy = UAy;
#pragma unroll
      for (int i = A; i > 0; --i) {
        const float2 nx = __ffma2_rn(((A - i) & 1) ? Cp : Cn, Wx, Vx);
        const float2 ny = __ffma2_rn(((A - i) & 1) ? Cp : Cn, Wy, Vy);
        Vx = Wx;
        Vy = Wy;
        Wx = nx;
        Wy = ny;
        P[i - 1] = __ffma2_rn(X, Wx, P[i - 1]);
        Q[i - 1] = __ffma2_rn(X, Wy, Q[i - 1]);
        R[i - 1] = __ffma2_rn(Y, Wx, R[i - 1]);
        U[i - 1] = __ffma2_rn(Y, Wy, U[i - 1]);
      }
    }
  }
  // slots 0..W-1: trials +m0..+m0+W-1; W..2W-1: trials -m0..-(m0+W-1)
  float2 S[2 * W];
#pragma unroll
  for (int i = 0; i < H; ++i) {
    S[2 * i] = make_float2(P[i].x - U[i].x, Q[i].x + R[i].x);
    S[2 * i + 1] = make_float2(P[i].y - U[i].y, Q[i].y + R[i].y);
    S[W + 2 * i] = make_float2(P[i].x + U[i].x, R[i].x - Q[i].x);
    S[W + 2 * i + 1] = make_float2(P[i].y + U[i].y, R[i].y - Q[i].y);
  }
  int base;
  const int cnt = group_transpose_reduce<2 * W, L>(S, gl, base);
#pragma unroll
  for (int j = 0; j < (2 * W / L > 1 ? 2 * W / L : 1); ++j) {
    if (j < cnt) {
      const int idx = base + j;
      const int t = idx < W ? n_half + m0 + idx : n_half - (m0 + idx - W);
      const float sq = S[j].x * S[j].x + S[j].y * S[j].y;
      if (sq > best_sq || (sq == best_sq && t < best_t)) {
        best_sq = sq;
        best_t = t;
      }
    }
  }
}

// ---- sampled trial sweep ---------------------------------------------------
// Only the argmax of |S_m|^2 over the trials leaves the sweep (the refinement
// recomputes K and the coherence exactly), and |S_m| = |T(m)| for the trial sum
// centred on the middle of the PS's bperp range,
//   T(m) = sum_c z_c e^{-j phi_c m},  phi_c = (bp_c - mid) (pi/4) / range,
// whose phases span exactly [-pi/8, pi/8]: T is band-limited to a quarter of
// the trial rate. It is evaluated exactly (same recurrences as the full sweep)
// at every 4th trial, m = 4k for |k| <= 16 NB, and between the samples by
// 20-tap fractional-delay filters (trial_interp_taps.h: error at most 6.8e-8 of
// sum |z_c|, below the FP32 rounding of the sums), so the sweep costs 16 NB + ~8
// magnitude steps instead of n_half. The samples stay in registers until the
// sweep ends (the column store's rotation slots, which the sample region
// overlays, are read until then).
constexpr int kMaxSampleBlocks = 2;

// Number of 16-magnitude sample blocks for n_half, or 0 where the full sweep
// is the cheaper (n_half <= 16 NB + 8) or the samples would exceed three blocks.
__host__ __device__ inline int trial_sample_blocks(int n_half) {
  const int ks = n_half / kTrialStride + (kInterpTapLo + kInterpTaps);  // floor(n/4) + 11 > the top tap
  const int nb = (ks + 15) / 16;
  if (nb < 2 || nb > kMaxSampleBlocks || 16 * nb + 8 >= n_half) return 0;
  return nb;
}

// Samples the filters read: T(4k) for k in [-kn, kp], kn = ceil(n/4) - tap_lo,
// kp = floor(n/4) + the top tap; kept at samp[kn + k].
__host__ __device__ inline int trial_samples_below(int n_half) { return (n_half + 3) / 4 - kInterpTapLo; }
__host__ __device__ inline int trial_samples_count(int n_half) {
  return trial_samples_below(n_half) + n_half / 4 + (kInterpTapLo + kInterpTaps - 1) + 1;
}

// Per-PS slot of the column store in floats: z (2), rotation (2) and bp
// columns, with the sample array over the rotation columns when it fits there
// and after bp otherwise; padded so the groups of a warp start in different
// banks.
__host__ __device__ inline int topofit_sample_offset(int mpad, int n_half) {
  const int nb = trial_sample_blocks(n_half);
  return (nb == 0 || trial_samples_count(n_half) <= mpad) ? 2 * mpad : 5 * mpad;
}
__host__ __device__ inline int topofit_stride(int L, int mpad, int n_half) {
  const int nb = trial_sample_blocks(n_half);
  int need = 5 * mpad;
  if (nb > 0) {
    const int top = topofit_sample_offset(mpad, n_half) + 2 * trial_samples_count(n_half);
    need = top > need ? top : need;
  }
  return ((need + 31) / 32) * 32 + (L % 32);
}

// One block of 16 sample magnitudes |k| = k0 .. k0+15 (the body of
// sweep_trial_pairs<16> with the centred phase per sample a_c = (bp_c - mid) qa
// and rotation e^{-j a_c} in the column store). Returns the lane's 32/L
// group-summed slots (slot idx < 16: T(4 (k0+idx)); else T(-4 (k0+idx-16))),
// the first of them at slot `base`.
template <int L>
__device__ __forceinline__ void sweep_sample_block(const ColumnSmem& cs, const float qa, const float mid,
                                                   const int ncl, const int gl, const int k0,
                                                   float2 (&out)[32 / L], int& base) {
  constexpr int H = 8;
  float2 P[H], Q[H], R[H], U[H];
#pragma unroll
  for (int i = 0; i < H; ++i) {
    P[i] = make_float2(0.f, 0.f);
    Q[i] = make_float2(0.f, 0.f);
    R[i] = make_float2(0.f, 0.f);
    U[i] = make_float2(0.f, 0.f);
  }
#pragma unroll 3
  for (int k = 0; k < ncl; ++k) {
    const int c = gl + L * k;
    const float x = cs.zx[c], y = cs.zy[c], rx = cs.rx[c], ry = cs.ry[c];
    constexpr int A = H / 2 - 1;
    const float2 a0 = cis_neg_anchor((cs.bp[c] - mid) * qa * static_cast<float>(k0 + 2 * A));
    const float a1x = fmaf(a0.x, rx, -a0.y * ry), a1y = fmaf(a0.x, ry, a0.y * rx);
    const float r2x = fmaf(rx, rx, -ry * ry), r2y = 2.f * rx * ry;
    const float2 X = make_float2(x, x), Y = make_float2(y, y);
    const float2 Cp = make_float2(2.f * r2x, 2.f * r2x), Cn = make_float2(-2.f * r2x, -2.f * r2x);
    const float2 UAx = make_float2(a0.x, a1x), UAy = make_float2(a0.y, a1y);
    const float2 UBx = make_float2(fmaf(a0.x, r2x, -a0.y * r2y), fmaf(a1x, r2x, -a1y * r2y));
    const float2 UBy = make_float2(fmaf(a0.x, r2y, a0.y * r2x), fmaf(a1x, r2y, a1y * r2x));
    P[A] = __ffma2_rn(X, UAx, P[A]);
    Q[A] = __ffma2_rn(X, UAy, Q[A]);
    R[A] = __ffma2_rn(Y, UAx, R[A]);
    U[A] = __ffma2_rn(Y, UAy, U[A]);
    float2 Vx = UAx, Vy = UAy, Wx = UBx, Wy = UBy;
#pragma unroll
    for (int i = A + 1; i < H; ++i) {
      P[i] = __ffma2_rn(X, Wx, P[i]);
      Q[i] = __ffma2_rn(X, Wy, Q[i]);
      R[i] = __ffma2_rn(Y, Wx, R[i]);
      U[i] = __ffma2_rn(Y, Wy, U[i]);
      if (i + 1 < H) {
        const float2 nx = __ffma2_rn(((i - A) & 1) ? Cn : Cp, Wx, Vx);
        const float2 ny = __ffma2_rn(((i - A) & 1) ? Cn : Cp, Wy, Vy);
        Vx = Wx;
        Vy = Wy;
        Wx = nx;
        Wy = ny;
      }
    }
    Vx = UBx;
    Vy = UBy;
    Wx = UAx;
    Wy = UAy;
#pragma unroll
    for (int i = A; i > 0; --i) {
      const float2 nx = __ffma2_rn(((A - i) & 1) ? Cp : Cn, Wx, Vx);
      const float2 ny = __ffma2_rn(((A - i) & 1) ? Cp : Cn, Wy, Vy);
      Vx = Wx;
      Vy = Wy;
      Wx = nx;
      Wy = ny;
      P[i - 1] = __ffma2_rn(X, Wx, P[i - 1]);
      Q[i - 1] = __ffma2_rn(X, Wy, Q[i - 1]);
      R[i - 1] = __ffma2_rn(Y, Wx, R[i - 1]);
      U[i - 1] = __ffma2_rn(Y, Wy, U[i - 1]);
    }
  }
  // the chain's sign s_i is common to a slot's four sums: T itself carries it,
  // so undo it here (s_{A+j} = -1 for j mod 4 in {2, 3}; A = 3)
  float2 S[32];
#pragma unroll
  for (int i = 0; i < H; ++i) {
    const float s = (((i - 3) & 3) >= 2) ? -1.f : 1.f;
    S[2 * i] = make_float2(s * (P[i].x - U[i].x), s * (Q[i].x + R[i].x));
    S[2 * i + 1] = make_float2(s * (P[i].y - U[i].y), s * (Q[i].y + R[i].y));
    S[16 + 2 * i] = make_float2(s * (P[i].x + U[i].x), s * (R[i].x - Q[i].x));
    S[16 + 2 * i + 1] = make_float2(s * (P[i].y + U[i].y), s * (R[i].y - Q[i].y));
  }
  group_transpose_reduce<32, L>(S, gl, base);
#pragma unroll
  for (int j = 0; j < 32 / L; ++j) out[j] = S[j];
}

// Sampled sweep of a group: NB sample blocks, the samples the filters read
// written to `samp` (T(4k) at samp[kn + k]), then every trial t = n_half + m evaluated (exact
// at m = 4k, interpolated between) and the first maximum of |T|^2 kept in
// trial order. Lanes take chunks of 3 sample periods (12 trials) in turn and
// hold the 22 samples a chunk's filters read in registers.
template <int L, int NB>
__device__ __forceinline__ void sampled_sweep(const ColumnSmem& cs, float2* samp, const float qa, const float mid,
                                              const int ncl, const int gl, const int n_half, const float2 s0,
                                              float& best_sq, int& best_t) {
  constexpr int NO = 32 / L;
  const int kn = trial_samples_below(n_half), kp = trial_samples_count(n_half) - 1 - kn;
  float2 held[NB][NO];
  int bases[NB];
#pragma unroll
  for (int b = 0; b < NB; ++b) sweep_sample_block<L>(cs, qa, mid, ncl, gl, 1 + 16 * b, held[b], bases[b]);
  __syncwarp();  // every lane of the warp is done with the rotation columns
#pragma unroll
  for (int b = 0; b < NB; ++b) {
#pragma unroll
    for (int j = 0; j < NO; ++j) {
      const int idx = bases[b] + j;
      const int k = idx < 16 ? 1 + 16 * b + idx : -(1 + 16 * b + idx - 16);
      if (k >= -kn && k <= kp) samp[kn + k] = held[b][j];
    }
  }
  if (gl == 0) samp[kn] = s0;
  __syncwarp();
  constexpr int CP = 3, NWIN = CP + kInterpTaps - 1;
  const int klo = -((n_half + 3) / 4), khi = n_half / 4;  // floor(-n/4), floor(n/4)
  const int nch = (khi - klo + CP) / CP;
  best_sq = -1.f;
  best_t = 0x7fffffff;
  for (int ch = gl; ch < nch; ch += L) {
    const int kb = klo + ch * CP;
    float2 win[NWIN];  // T(4 (kb + kInterpTapLo + i))
#pragma unroll
    for (int i = 0; i < NWIN; ++i) {
      const int k = kb + kInterpTapLo + i;
      win[i] = (k >= -kn && k <= kp) ? samp[kn + k] : make_float2(0.f, 0.f);
    }
#pragma unroll
    for (int pp = 0; pp < CP; ++pp) {
      const int k = kb + pp;
#pragma unroll
      for (int r = 0; r < 4; ++r) {
        const int m = 4 * k + r;
        float2 v;
        if (r == 0) {
          v = win[pp - kInterpTapLo];
        } else {
          v = make_float2(0.f, 0.f);
#pragma unroll
          for (int i = 0; i < kInterpTaps; ++i) {
            const float h = kInterpTaps_c[r - 1][i];
            v = __ffma2_rn(make_float2(h, h), win[pp + i], v);
          }
        }
        const float sq = v.x * v.x + v.y * v.y;
        const int t = n_half + m;
        if (m >= -n_half && m <= n_half && (sq > best_sq || (sq == best_sq && t < best_t))) {
          best_sq = sq;
          best_t = t;
        }
      }
    }
  }
}

// L2 prefetch of the rows a warp reads on its next pass (the PS group s0n ..
// s0n+G-1): the phase rows and, unless bperp is row invariant, the bperp rows,
// one 128-byte line per lane per instruction, all inside the arrays.
template <int G, bool ROWINV>
__device__ __forceinline__ void prefetch_rows(const void* ph, const float* bp, const int64_t s0n, const int64_t N,
                                              const int64_t M, const int lane) {
  if (s0n >= N) return;
  const int64_t s1 = s0n + G < N ? s0n + G : N;
  const char* p0 = static_cast<const char*>(ph) + s0n * M * 8;
  const int64_t nb = (s1 - s0n) * M * 8;
  for (int64_t o = static_cast<int64_t>(lane) * 128; o < nb; o += 32 * 128)
    asm volatile("prefetch.global.L2 [%0];" ::"l"(p0 + o));
  if (!ROWINV) {
    const char* b0 = reinterpret_cast<const char*>(bp + s0n * M);
    const int64_t nbb = (s1 - s0n) * M * 4;
    for (int64_t o = static_cast<int64_t>(lane) * 128; o < nbb; o += 32 * 128)
      asm volatile("prefetch.global.L2 [%0];" ::"l"(b0 + o));
  }
}

constexpr int kTopoLoadCols = 8;  // columns whose loads a lane issues together in the prologue

// The work of block `vb` of a launch of `nvb` blocks over one patch: PS
// groups s0 = (vb * 4 + warp) * G + k * nvb * 4 * G. The batched kernel runs
// the same virtual blocks, so a patch's per-block rms partials, and with them
// its stop decisions, are the same as when it runs alone.
template <int L, bool LOOP, bool ROWINV>
__device__ __forceinline__ void topofit_vblock_t(const TopoArgs& a, const int mpad, const int vb, const int nvb,
                                                 unsigned char* smem_raw, int* sh_hist, double* sh_rms, int* sh_inv) {
  constexpr int G = 32 / L;
  const int tid = threadIdx.x, lane = tid & 31, wib = tid >> 5;
  const int g = lane / L, gl = lane % L;
  __syncthreads();
  for (int i = tid; i < kCohBins; i += blockDim.x) sh_hist[i] = 0;
  __syncthreads();
  // per-PS slot stride = L (mod 32) floats so the groups of a warp hit different banks
  const int stride = topofit_stride(L, mpad, a.n_half);
  float* base_ptr = reinterpret_cast<float*>(smem_raw) + static_cast<int64_t>(wib * G + g) * stride;
  ColumnSmem cs{base_ptr, base_ptr + mpad, base_ptr + 2 * mpad, base_ptr + 3 * mpad, base_ptr + 4 * mpad};
  const int nb = trial_sample_blocks(a.n_half);
  float2* samp = reinterpret_cast<float2*>(base_ptr + topofit_sample_offset(mpad, a.n_half));
  const float2* __restrict__ ph_nm = static_cast<const float2*>(a.ph_nm);
  const float2* __restrict__ filt = static_cast<const float2*>(a.filt);
  const float2* __restrict__ cpx = static_cast<const float2*>(a.cpx);
  float* __restrict__ K_out = static_cast<float*>(a.K_out);
  float* __restrict__ C_out = static_cast<float*>(a.C_out);
  float* __restrict__ coh_io = static_cast<float*>(a.coh_io);
  float2* __restrict__ resid = static_cast<float2*>(a.residual);
  float* __restrict__ ph_res = static_cast<float*>(a.ph_res);
  float2* __restrict__ ph_patch = static_cast<float2*>(a.ph_patch);
  const int64_t M = a.M;
  const int ncl = mpad / L;
  const unsigned gmask = (L == 32) ? kFull : (((1u << L) - 1u) << (g * L));
  double rms_acc = 0.0;
  int inv_acc = 0;
  const int64_t step = static_cast<int64_t>(nvb) * 4 * G;
  // the cell of this lane's next PS is loaded one pass ahead, so the
  // filtered-grid gather of a pass does not wait on it
  const int64_t s_first = (static_cast<int64_t>(vb) * 4 + wib) * G + g;
  int64_t cell_next = (LOOP && s_first < a.N) ? a.cell_of[s_first] : 0;
  for (int64_t s0 = (static_cast<int64_t>(vb) * 4 + wib) * G; s0 < a.N; s0 += step) {
    const int64_t s = s0 + g;
    const bool active = s < a.N;
    const int64_t cell = cell_next;
    if (LOOP) cell_next = s + step < a.N ? a.cell_of[s + step] : 0;
    prefetch_rows<G, ROWINV>(LOOP ? static_cast<const void*>(ph_nm) : static_cast<const void*>(cpx), a.bp, s0 + step,
                             a.N, M, lane);
    bool zero = false, nonzero = false;
    float mn = __int_as_float(0x7f800000), mx = -mn;
    // kTopoLoadCols columns per round with their global loads issued first
    constexpr int PR = kTopoLoadCols;
    for (int k0c = 0; k0c < ncl; k0c += PR) {
      float2 fv[PR], pv[PR];
      float bv[PR];
#pragma unroll
      for (int i = 0; i < PR; ++i) {
        const int c = gl + L * (k0c + i);
        fv[i] = make_float2(0.f, 0.f);
        pv[i] = make_float2(0.f, 0.f);
        bv[i] = 0.f;
        if (active && k0c + i < ncl && c < a.M) {
          if (!LOOP) {
            pv[i] = cpx[s * M + c];
          } else {
            fv[i] = filt[cell * a.Mp + c];
            pv[i] = ph_nm[s * M + c];
          }
          bv[i] = ROWINV ? a.bp[c] : a.bp[s * M + c];
        }
      }
#pragma unroll
      for (int i = 0; i < PR; ++i) {
        const int c = gl + L * (k0c + i);
        if (k0c + i >= ncl) break;
        float2 v = make_float2(0.f, 0.f);
        if (active && c < a.M) {
          if (!LOOP) {
            v = pv[i];
          } else {
            // extract_patch_phase + normalize_complex_unit_magnitude (:1186-1205)
            float2 f = fv[i];
            if (!a.filt_unit) {
              const float mag = hypotf(f.x, f.y);
              if (mag != 0.f) f = make_float2(f.x / mag, f.y / mag);
            }
            if (ph_patch) ph_patch[s * M + c] = f;
            v = cmul_rn(conjf2(f), pv[i]);  // psdph (:687-689)
          }
          if (v.x == 0.f && v.y == 0.f) {
            zero = true;
          } else {
            nonzero = true;
            mn = fminf(mn, bv[i]);
            mx = fmaxf(mx, bv[i]);
          }
        }
        cs.zx[c] = v.x;
        cs.zy[c] = v.y;
        cs.bp[c] = bv[i];
      }
    }
    const bool any_zero = (__ballot_sync(kFull, zero) & gmask) != 0u;
    const bool any_nonzero = (__ballot_sync(kFull, nonzero) & gmask) != 0u;
    const bool invalid = !active || (a.zero_mode == 0 ? any_zero : !any_nonzero);
    mn = group_min<L>(mn);
    mx = group_max<L>(mx);
    float range = mx - mn;
    if (!(range != 0.f) || invalid) range = 1.f;
    // sampled sweep: rotation e^{-j a_c} per sample step, a_c = (bp_c - mid) qa;
    // full sweep: e^{-j theta_c} per trial, theta_c = bp_c / range * pi/4
    const float mid = (nb > 0 && !invalid && mx >= mn) ? 0.5f * (mn + mx) : 0.f;
    const float qa = (kQuarterPiF / range) * static_cast<float>(kTrialStride);
    for (int k = 0; k < ncl; ++k) {
      const int c = gl + L * k;
      const float t = nb > 0 ? (cs.bp[c] - mid) * qa : (cs.bp[c] / range) * kQuarterPiF;
      float sn, cn;
      sincos_cw(t, &sn, &cn);
      cs.rx[c] = cn;
      cs.ry[c] = -sn;
    }
    const float qr = kQuarterPiF / range;
    __syncwarp();
    // trial sweep over m = -n .. n (all groups run it; invalid ones discard it):
    // m = 0 is the plain column sum, then the pairs +-m
    float best_sq, s0x = 0.f, s0y = 0.f;
    for (int k = 0; k < ncl; ++k) {
      const int c = gl + L * k;
      s0x += cs.zx[c];
      s0y += cs.zy[c];
    }
    s0x = group_sum<L>(s0x);
    s0y = group_sum<L>(s0y);
    best_sq = s0x * s0x + s0y * s0y;
    int best_t = a.n_half;
    if (nb == 2) {
      sampled_sweep<L, 2>(cs, samp, qa, mid, ncl, gl, a.n_half, make_float2(s0x, s0y), best_sq, best_t);
    } else {
      int m0 = 1;
      for (; a.n_half - m0 + 1 >= 16; m0 += 16)
        sweep_trial_pairs<16, L>(cs, qr, ncl, gl, m0, a.n_half, best_sq, best_t);
      if (a.n_half - m0 + 1 >= 8) {
        sweep_trial_pairs<8, L>(cs, qr, ncl, gl, m0, a.n_half, best_sq, best_t);
        m0 += 8;
      }
      if (a.n_half - m0 + 1 >= 4) {
        sweep_trial_pairs<4, L>(cs, qr, ncl, gl, m0, a.n_half, best_sq, best_t);
        m0 += 4;
      }
      if (a.n_half - m0 + 1 >= 2) {
        sweep_trial_pairs<2, L>(cs, qr, ncl, gl, m0, a.n_half, best_sq, best_t);
        m0 += 2;
      }
      if (a.n_half - m0 + 1 >= 1) sweep_pairs<1, L>(cs, qr, ncl, gl, m0, a.n_half, best_sq, best_t);
    }
    // first maximum over the group (argmax_first_f32, :1526-1536)
#pragma unroll
    for (int o = L / 2; o > 0; o >>= 1) {
      const float osq = __shfl_xor_sync(kFull, best_sq, o);
      const int ot = __shfl_xor_sync(kFull, best_t, o);
      if (osq > best_sq || (osq == best_sq && ot < best_t)) {
        best_sq = osq;
        best_t = ot;
      }
    }
    if (best_t == 0x7fffffff) best_t = a.n_half;  // no finite |T|^2: the m = 0 trial, as the full sweep keeps
    __syncwarp();  // the sample array overlays the rotation slots written next
    // refine_candidate (:1259-1303) with FP64 normal-equation sums; the
    // rotation slots of the column store now hold z e^{-j k0 bp}
    const float k0 = kQuarterPiF / range * static_cast<float>(best_t - a.n_half);
    float ox = 0.f, oy = 0.f;
    for (int k = 0; k < ncl; ++k) {
      const int c = gl + L * k;
      const float2 r = cmul_rn(make_float2(cs.zx[c], cs.zy[c]), cis_neg_anchor(k0 * cs.bp[c]));
      cs.rx[c] = r.x;
      cs.ry[c] = r.y;
      ox += r.x;
      oy += r.y;
    }
    ox = group_sum<L>(ox);
    oy = group_sum<L>(oy);
    const float2 oc = make_float2(ox, -oy);
    double mopt = 0.0, dl = 0.0;
    float den_w = 0.f;  // sum |z|: |residual| = |z| (a rotation), the refined coherence's denominator
    for (int k = 0; k < ncl; ++k) {
      const int c = gl + L * k;
      // in the loop |z| is that of a product of two unit (or zero) phasors, with
      // no overflow or underflow to guard against: sqrt(x^2 + y^2) is within an
      // ulp of hypotf at a third of its cost; standalone rows take any magnitude
      const float wf = LOOP ? sqrtf(fmaf(cs.zx[c], cs.zx[c], cs.zy[c] * cs.zy[c])) : hypotf(cs.zx[c], cs.zy[c]);
      den_w += wf;
      const double wgt = static_cast<double>(wf);
      const double wb = __dmul_rn(wgt, static_cast<double>(cs.bp[c]));
      dl = __dadd_rn(dl, __dmul_rn(wb, wb));
      const float2 q = cmul_rn(make_float2(cs.rx[c], cs.ry[c]), oc);
      mopt = __dadd_rn(mopt, __dmul_rn(wb, __dmul_rn(wgt, static_cast<double>(atan2_poly(q.y, q.x)))));
    }
    mopt = group_sum<L>(mopt);
    dl = group_sum<L>(dl);
    if (dl == 0.0) dl = 1.0;
    const float K1 = static_cast<float>(static_cast<double>(k0) + mopt / dl);
    float mx2 = 0.f, my2 = 0.f, den2 = den_w;
    for (int k = 0; k < ncl; ++k) {
      const int c = gl + L * k;
      const float2 r = cmul_rn(make_float2(cs.zx[c], cs.zy[c]), cis_neg_anchor(K1 * cs.bp[c]));
      mx2 += r.x;
      my2 += r.y;
      if (active && c < a.M) {
        if (resid) resid[s * M + c] = invalid ? make_float2(0.f, 0.f) : r;
        if (ph_res) ph_res[s * M + c] = invalid ? 0.f : atan2f(r.y, r.x);
      }
    }
    mx2 = group_sum<L>(mx2);
    my2 = group_sum<L>(my2);
    den2 = group_sum<L>(den2);
    if (den2 == 0.f) den2 = 1.f;
    __syncwarp();
    if (gl == 0 && active) {
      float Kv, Cv, cohv;
      if (invalid) {
        // fit_stage2_rows invalid row (:676-697) / topofit_row empty row (:1216-1222)
        Kv = __int_as_float(0x7fffffff);
        Cv = a.zero_mode == 0 ? 0.f : Kv;
        cohv = a.zero_mode == 0 ? 0.f : Kv;
        inv_acc += 1;
      } else {
        Kv = K1;
        Cv = atan2f(my2, mx2);
        cohv = hypotf(mx2, my2) / den2;
      }
      if (a.accumulate_stats) {
        const double d = static_cast<double>(cohv) - static_cast<double>(coh_io[s]);
        rms_acc += d * d;
        const int b = coh_bin(static_cast<double>(cohv), a.cutoff0, a.dbin);
        if (b >= 0) atomicAdd(&sh_hist[b], 1);
      }
      K_out[s] = Kv;
      C_out[s] = Cv;
      coh_io[s] = cohv;
      if (a.nopt) a.nopt[s] = invalid ? 0 : 1;
    }
  }
  if (!a.accumulate_stats) return;
  rms_acc = warp_sum(rms_acc);
  inv_acc = warp_sum(inv_acc);
  if (lane == 0) {
    sh_rms[wib] = rms_acc;
    sh_inv[wib] = inv_acc;
  }
  __syncthreads();
  if (tid == 0) {
    a.rms_partial[vb] = sh_rms[0] + sh_rms[1] + sh_rms[2] + sh_rms[3];
    const int iv = sh_inv[0] + sh_inv[1] + sh_inv[2] + sh_inv[3];
    if (iv) atomicAdd(a.n_invalid, iv);
  }
  for (int i = tid; i < kCohBins; i += blockDim.x)
    if (sh_hist[i]) atomicAdd(&a.hist[i], sh_hist[i]);
}

// The input form (loop: ph_nm + filtered grid; standalone: psdph rows) and the
// row invariance of bperp are compile-time in the body.
template <int L>
__device__ __forceinline__ void topofit_vblock(const TopoArgs& a, const int mpad, const int vb, const int nvb,
                                               unsigned char* smem_raw, int* sh_hist, double* sh_rms, int* sh_inv) {
  if (a.cpx)
    a.bp_row_inv ? topofit_vblock_t<L, false, true>(a, mpad, vb, nvb, smem_raw, sh_hist, sh_rms, sh_inv)
                 : topofit_vblock_t<L, false, false>(a, mpad, vb, nvb, smem_raw, sh_hist, sh_rms, sh_inv);
  else
    a.bp_row_inv ? topofit_vblock_t<L, true, true>(a, mpad, vb, nvb, smem_raw, sh_hist, sh_rms, sh_inv)
                 : topofit_vblock_t<L, true, false>(a, mpad, vb, nvb, smem_raw, sh_hist, sh_rms, sh_inv);
}

template <int L>
__global__ void __launch_bounds__(128, 4) k_topofit_f32(TopoArgs a, int mpad) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  __shared__ int sh_hist[kCohBins];
  __shared__ double sh_rms[4];
  __shared__ int sh_inv[4];
  topofit_vblock<L>(a, mpad, blockIdx.x, gridDim.x, smem_raw, sh_hist, sh_rms, sh_inv);
}

// Plain FP64 topofit: direct sincos for every (trial, column), lanes over
// trials for the sweep and over columns for the refinement. This is the
// comparison path; it shares only the data layout with the FP32 kernel.
__global__ void __launch_bounds__(256) k_topofit_f64(TopoArgs a) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  const int tid = threadIdx.x, lane = tid & 31, wib = tid >> 5;
  double2* zs = reinterpret_cast<double2*>(smem_raw) + static_cast<int64_t>(wib) * a.M;
  double* ths = reinterpret_cast<double*>(reinterpret_cast<double2*>(smem_raw) + 8 * a.M) + static_cast<int64_t>(wib) * a.M;
  __shared__ int sh_hist[kCohBins];
  __shared__ double sh_rms[8];
  __shared__ int sh_inv[8];
  for (int i = tid; i < kCohBins; i += blockDim.x) sh_hist[i] = 0;
  __syncthreads();
  const float2* __restrict__ ph_nm = static_cast<const float2*>(a.ph_nm);
  const double2* __restrict__ filt = static_cast<const double2*>(a.filt);
  double* K_out = static_cast<double*>(a.K_out);
  double* C_out = static_cast<double*>(a.C_out);
  double* coh_io = static_cast<double*>(a.coh_io);
  double2* resid = static_cast<double2*>(a.residual);
  double* ph_res = static_cast<double*>(a.ph_res);
  double2* ph_patch = static_cast<double2*>(a.ph_patch);
  const int64_t M = a.M;
  const int T = 2 * a.n_half + 1;
  const double qpi = 3.14159265358979323846 / 4.0;
  double rms_acc = 0.0;
  int inv_acc = 0;
  const int64_t gw = (static_cast<int64_t>(blockIdx.x) * blockDim.x + tid) >> 5;
  const int64_t nwarps = (static_cast<int64_t>(gridDim.x) * blockDim.x) >> 5;
  for (int64_t s = gw; s < a.N; s += nwarps) {
    const int64_t cell = a.cell_of[s];
    bool zero = false;
    double mn = INFINITY, mx = -INFINITY;
    for (int c = lane; c < a.M; c += 32) {
      double2 f = filt[cell * a.Mp + c];
      const double mag = hypot(f.x, f.y);
      if (mag != 0.0) f = make_double2(f.x / mag, f.y / mag);
      if (ph_patch) ph_patch[s * M + c] = f;
      const float2 p = ph_nm[s * M + c];
      const double2 v = cmul_rn(conjd2(f), make_double2(p.x, p.y));
      zs[c] = v;
      if (v.x == 0.0 && v.y == 0.0) zero = true;
      const double b = a.bp_row_inv ? static_cast<double>(a.bp[c]) : static_cast<double>(a.bp[s * M + c]);
      ths[c] = b;
      mn = fmin(mn, b);
      mx = fmax(mx, b);
    }
    const bool invalid = __any_sync(kFull, zero);
    double Kv, Cv, cohv;
    if (invalid) {
      Kv = __longlong_as_double(0x7ff8000000000000LL);
      Cv = 0.0;
      cohv = 0.0;
      for (int c = lane; c < a.M; c += 32) {
        if (resid) resid[s * M + c] = make_double2(0.0, 0.0);
        if (ph_res) ph_res[s * M + c] = 0.0;
      }
      inv_acc += 1;
    } else {
      mn = warp_min(mn);
      mx = warp_max(mx);
      double range = mx - mn;
      if (range == 0.0) range = 1.0;
      __syncwarp();
      for (int c = lane; c < a.M; c += 32) ths[c] = (ths[c] / range) * qpi;  // keeps bp in registers below
      __syncwarp();
      double best = -1.0;
      int bt = 0;
      for (int t = lane; t < T; t += 32) {
        const double m = static_cast<double>(t - a.n_half);
        double sx = 0.0, sy = 0.0;
        for (int c = 0; c < a.M; ++c) {
          double sn, cs;
          sincos(ths[c] * m, &sn, &cs);
          const double2 zz = zs[c];
          sx += zz.x * cs + zz.y * sn;
          sy += zz.y * cs - zz.x * sn;
        }
        const double sq = sx * sx + sy * sy;
        if (sq > best) {
          best = sq;
          bt = t;
        }
      }
#pragma unroll
      for (int o = 16; o > 0; o >>= 1) {
        const double ob = __shfl_xor_sync(kFull, best, o);
        const int ot = __shfl_xor_sync(kFull, bt, o);
        if (ob > best || (ob == best && ot < bt)) {
          best = ob;
          bt = ot;
        }
      }
      const double k0 = qpi / range * static_cast<double>(bt - a.n_half);
      double ox = 0.0, oy = 0.0;
      for (int c = lane; c < a.M; c += 32) {
        const double b = a.bp_row_inv ? static_cast<double>(a.bp[c]) : static_cast<double>(a.bp[s * M + c]);
        double sn, cs;
        sincos(k0 * b, &sn, &cs);
        const double2 r = cmul_rn(zs[c], make_double2(cs, -sn));
        ox += r.x;
        oy += r.y;
      }
      ox = warp_sum(ox);
      oy = warp_sum(oy);
      double mopt = 0.0, dl = 0.0;
      for (int c = lane; c < a.M; c += 32) {
        const double b = a.bp_row_inv ? static_cast<double>(a.bp[c]) : static_cast<double>(a.bp[s * M + c]);
        double sn, cs;
        sincos(k0 * b, &sn, &cs);
        const double2 r = cmul_rn(zs[c], make_double2(cs, -sn));
        const double wgt = hypot(zs[c].x, zs[c].y);
        const double wb = wgt * b;
        dl += wb * wb;
        const double2 q = cmul_rn(r, make_double2(ox, -oy));
        mopt += wb * (wgt * atan2(q.y, q.x));
      }
      mopt = warp_sum(mopt);
      dl = warp_sum(dl);
      if (dl == 0.0) dl = 1.0;
      const double K1 = k0 + mopt / dl;
      double mx2 = 0.0, my2 = 0.0, den2 = 0.0;
      for (int c = lane; c < a.M; c += 32) {
        const double b = a.bp_row_inv ? static_cast<double>(a.bp[c]) : static_cast<double>(a.bp[s * M + c]);
        double sn, cs;
        sincos(K1 * b, &sn, &cs);
        const double2 r = cmul_rn(zs[c], make_double2(cs, -sn));
        mx2 += r.x;
        my2 += r.y;
        den2 += hypot(r.x, r.y);
        if (resid) resid[s * M + c] = r;
        if (ph_res) ph_res[s * M + c] = atan2(r.y, r.x);
      }
      mx2 = warp_sum(mx2);
      my2 = warp_sum(my2);
      den2 = warp_sum(den2);
      if (den2 == 0.0) den2 = 1.0;
      Kv = K1;
      Cv = atan2(my2, mx2);
      cohv = hypot(mx2, my2) / den2;
    }
    __syncwarp();
    if (lane == 0) {
      if (a.accumulate_stats) {
        const double d = cohv - coh_io[s];
        rms_acc += d * d;
        const int b = coh_bin(cohv, a.cutoff0, a.dbin);
        if (b >= 0) atomicAdd(&sh_hist[b], 1);
      }
      K_out[s] = Kv;
      C_out[s] = Cv;
      coh_io[s] = cohv;
      if (a.nopt) a.nopt[s] = invalid ? 0 : 1;
    }
  }
  if (!a.accumulate_stats) return;
  if (lane == 0) {
    sh_rms[wib] = rms_acc;
    sh_inv[wib] = inv_acc;
  }
  __syncthreads();
  if (tid == 0) {
    double t = 0.0;
    int iv = 0;
    for (int w = 0; w < static_cast<int>(blockDim.x >> 5); ++w) {
      t += sh_rms[w];
      iv += sh_inv[w];
    }
    a.rms_partial[blockIdx.x] = t;
    if (iv) atomicAdd(a.n_invalid, iv);
  }
  for (int i = tid; i < kCohBins; i += blockDim.x)
    if (sh_hist[i]) atomicAdd(&a.hist[i], sh_hist[i]);
}

int topofit_grid_blocks(int sm_count, bool fp64) { return sm_count * 16; }

int topofit_lanes(int M) {
  static const int forced = [] {
    const char* e = getenv("PS2_TOPOFIT_LANES");
    return e ? atoi(e) : 0;
  }();
  if (forced == 4 || forced == 8 || forced == 16 || forced == 32) return forced;
  int L = 4;
  while (L < 32 && L * 24 < M) L *= 2;
  return L;
}

int clap_block_count(int nw_axis) { return clap_block_rows(nw_axis); }

int64_t clap_part_elems(int nwi, int nwj, int n_win, int Mp) {
  const int64_t box = clap_box(n_win);
  return std::max<int64_t>(static_cast<int64_t>(clap_block_rows(nwi)) * clap_block_rows(nwj), 1) * box * box * Mp;
}

size_t topofit_smem_bytes(int L, int mpad, int n_half) {
  return static_cast<size_t>(4 * (32 / L)) * topofit_stride(L, mpad, n_half) * sizeof(float);
}

// Columns per PS padded to a multiple of 2L (zero columns): each lane holds an
// even number of columns, the packed pairs of the trial sweep.
int topofit_mpad(int L, int M) { return ((M + 2 * L - 1) / (2 * L)) * (2 * L); }

template <int L>
static cudaError_t topofit_geometry_l(const TopoArgs& a, int grid_cap, size_t* smem, int* blocks_out) {
  const int mpad = topofit_mpad(L, a.M);
  const size_t sm = topofit_smem_bytes(L, mpad, a.n_half);
  cudaError_t e = kernel_attributes_once(sm);
  if (e != cudaSuccess) return e;
  int per_sm = 0;
  e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_topofit_f32<L>, 128, sm);
  if (e != cudaSuccess) return e;
  int dev = 0, sms = 148;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  const int64_t per_block = 4 * (32 / L);
  int64_t blocks = (a.N + per_block - 1) / per_block;
  const int64_t cap = std::min<int64_t>(grid_cap, static_cast<int64_t>(sms) * std::max(per_sm, 1));
  if (blocks > cap) blocks = cap;
  if (blocks < 1) blocks = 1;
  *smem = sm;
  *blocks_out = static_cast<int>(blocks);
  return cudaSuccess;
}

// Blocks of the FP32 topofit launch for this patch (the virtual blocks a batch
// reproduces); the lane count is a.lanes or the rule from M.
cudaError_t topofit_geometry(const TopoArgs& a, int grid_cap, int* L_out, int* mpad_out, int* blocks_out) {
  const int L = a.lanes ? a.lanes : topofit_lanes(a.M);
  size_t sm = 0;
  cudaError_t e;
  switch (L) {
    case 4: e = topofit_geometry_l<4>(a, grid_cap, &sm, blocks_out); break;
    case 8: e = topofit_geometry_l<8>(a, grid_cap, &sm, blocks_out); break;
    case 16: e = topofit_geometry_l<16>(a, grid_cap, &sm, blocks_out); break;
    case 32: e = topofit_geometry_l<32>(a, grid_cap, &sm, blocks_out); break;
    default: return cudaErrorInvalidValue;
  }
  *L_out = L;
  *mpad_out = topofit_mpad(L, a.M);
  return e;
}

template <int L>
static cudaError_t launch_topofit_l(const TopoArgs& a, int grid_cap, cudaStream_t st) {
  size_t sm = 0;
  int blocks = 0;
  cudaError_t e = topofit_geometry_l<L>(a, grid_cap, &sm, &blocks);
  if (e != cudaSuccess) return e;
  k_topofit_f32<L><<<static_cast<unsigned>(blocks), 128, sm, st>>>(a, topofit_mpad(L, a.M));
  return cudaGetLastError();
}

cudaError_t launch_topofit(const TopoArgs& a, bool fp64, int grid_blocks, cudaStream_t st) {
  if (a.N <= 0) return cudaSuccess;
  if (fp64) {
    int64_t need = (a.N + 7) / 8;
    const int blocks = static_cast<int>(std::min<int64_t>(need, grid_blocks));
    const size_t sm = static_cast<size_t>(8) * a.M * (sizeof(double2) + sizeof(double));
    cudaError_t e = kernel_attributes_once(sm);
    if (e != cudaSuccess) return e;
    k_topofit_f64<<<blocks, 256, sm, st>>>(a);
    return cudaGetLastError();
  }
  switch (a.lanes ? a.lanes : topofit_lanes(a.M)) {
    case 4: return launch_topofit_l<4>(a, grid_blocks, st);
    case 8: return launch_topofit_l<8>(a, grid_blocks, st);
    case 16: return launch_topofit_l<16>(a, grid_blocks, st);
    default: return launch_topofit_l<32>(a, grid_blocks, st);
  }
}

// ============================================================= finalize ===
// rms_difference + stop rule (:307-313, :2045-2057); when continuing, the
// P-square update (:364-381, :1642-1683) producing the prand_hi table that the
// next k_bin turns into weights. Sums use explicit _rn arithmetic and the
// reference's order so the table matches the reference given equal inputs.
__device__ __forceinline__ void finalize_body(const FinalizeArgs& a) {
  __shared__ double sh[256];
  __shared__ double na[kCohBins], prand[kCohBins], interp_in[kCohBins + 1];
  __shared__ double scale_s;
  __shared__ int go_on;
  const int tid = threadIdx.x;
  double s = 0.0;
  for (int i = tid; i < a.n_partial; i += 256) s += a.rms_partial[i];
  sh[tid] = s;
  if (tid < kCohBins) na[tid] = static_cast<double>(a.hist[tid]);
  __syncthreads();
  for (int w = 128; w > 0; w >>= 1) {
    if (tid < w) sh[tid] += sh[tid + w];
    __syncthreads();
  }
  if (tid == 0) {
    const double rms = sqrt(sh[0] / static_cast<double>(a.N > 0 ? a.N : 1));
    const double gcs = a.state[0];
    const double delta = rms - gcs;
    const int64_t i_loop = static_cast<int64_t>(a.state[1]);
    const int64_t cap = a.gamma_max_iterations > 1 ? a.gamma_max_iterations : 1;
    const bool stop = fabs(delta) < a.gamma_change_convergence || i_loop >= cap;
    a.state[0] = rms;
    a.state[1] = static_cast<double>(i_loop + 1);
    a.state[2] = rms;
    a.state[3] = delta;
    a.stats_out[0] = static_cast<double>(i_loop);
    a.stats_out[1] = rms;
    a.stats_out[2] = delta;
    a.stats_out[3] = stop ? 1.0 : 0.0;
    a.stats_out[4] = static_cast<double>(*a.n_invalid);
    go_on = ((!stop || a.force_continue) && a.psquare) ? 1 : 0;
    if (go_on) {
      // Nr rescaled so its low-coherence mass matches Na's (sequential sums)
      double den = 0.0;
      for (int i = 0; i < a.low_coh_thresh; ++i) den = __dadd_rn(den, a.nr_scaled[i]);
      double sc = 1.0;
      if (den > 0.0) {
        double num = 0.0;
        for (int i = 0; i < a.low_coh_thresh; ++i) num = __dadd_rn(num, na[i]);
        sc = num / den;
      }
      scale_s = sc;
      interp_in[0] = 1.0;
    }
  }
  __syncthreads();
  if (!go_on) return;
  if (tid < kCohBins) {
    const double nrv = __dmul_rn(a.nr_scaled[tid], scale_s);
    a.nr_scaled[tid] = nrv;
    const double d = na[tid] == 0.0 ? 1.0 : na[tid];
    double p = fmin(nrv / d, 1.0);
    if (tid < a.low_coh_thresh) p = 1.0;
    if (tid >= static_cast<int>(a.nr_max_nz_ix)) p = 0.0;
    prand[tid] = p;
  }
  __syncthreads();
  // lfilter(gausswin, [1]*7 ++ prand), shifted by 7, / sum(gausswin)
  if (tid < kCohBins) {
    const int ix = tid + 7;
    double acc = 0.0;
    for (int k = 0; k < 7; ++k) {
      const int j = ix - k;
      const double v = j < 7 ? 1.0 : prand[j - 7];
      acc = __dadd_rn(acc, __dmul_rn(a.g7w[k], v));
    }
    interp_in[1 + tid] = acc / a.g7sum;
  }
  __syncthreads();
  // matlab_interp(.., 10) with the 79-tap FIR, delay 39, tail trimmed to 1001
  for (int i = tid; i < 1001; i += 256) {
    const int n = i + 39;
    double acc = 0.0;
    for (int k = 0; k < 79; ++k) {
      const int p = n - k;
      if (p < 0) continue;
      const double v = (p % 10 == 0 && p / 10 < 101) ? interp_in[p / 10] : 0.0;
      acc = __dadd_rn(acc, __dmul_rn(a.taps79[k], v));
    }
    a.lut[i] = __dmul_rn(acc, 10.0);
  }
}

__global__ void __launch_bounds__(256) k_finalize(FinalizeArgs a) { finalize_body(a); }

// Body tail of the graph that runs the loop to convergence: keep looping while
// the finalize of this iteration did not raise the stop flag.
__global__ void k_loop_continue(cudaGraphConditionalHandle h, const double* stats) {
  if (threadIdx.x == 0) cudaGraphSetConditional(h, stats[3] == 0.0 ? 1u : 0u);
}

cudaError_t launch_loop_continue(cudaGraphConditionalHandle h, const double* stats, cudaStream_t st) {
  k_loop_continue<<<1, 32, 0, st>>>(h, stats);
  return cudaGetLastError();
}

cudaError_t launch_finalize(const FinalizeArgs& a, cudaStream_t st) {
  k_finalize<<<1, 256, 0, st>>>(a);
  return cudaGetLastError();
}

// ========================================================= SNR weighting ==
// snr_weighting (:1875-1897) from the residual phase written by the last
// topofit: w = g / sqrt(0.5 (mean amp^2 - g^2)), g = mean(amp cos(ph_res)).
template <typename R>
__global__ void __launch_bounds__(256) k_snr_weight(const R* ph_res, const float* amp, int64_t N, int M, R* w_out) {
  const int lane = threadIdx.x & 31;
  const int64_t gw = (static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x) >> 5;
  const int64_t nw = (static_cast<int64_t>(gridDim.x) * blockDim.x) >> 5;
  for (int64_t s = gw; s < N; s += nw) {
    double g = 0.0, a2 = 0.0;
    for (int c = lane; c < M; c += 32) {
      const double am = static_cast<double>(amp[s * M + c]);
      g += am * cos(static_cast<double>(ph_res[s * M + c]));
      a2 += am * am;
    }
    g = warp_sum(g);
    a2 = warp_sum(a2);
    if (lane == 0) {
      const double mm = static_cast<double>(M > 0 ? M : 1);
      g /= mm;
      a2 /= mm;
      const double sig = sqrt(0.5 * (a2 - g * g));
      w_out[s] = static_cast<R>(sig != 0.0 ? g / sig : 0.0);
    }
  }
}

cudaError_t launch_snr_weight(const TopoArgs& t, const float* amp, void* w_out, bool fp64, int sm_count,
                              cudaStream_t st) {
  const int blocks = sm_count * 8;
  if (fp64)
    k_snr_weight<double><<<blocks, 256, 0, st>>>(static_cast<const double*>(t.ph_res), amp, t.N, t.M,
                                                 static_cast<double*>(w_out));
  else
    k_snr_weight<float><<<blocks, 256, 0, st>>>(static_cast<const float*>(t.ph_res), amp, t.N, t.M,
                                                static_cast<float*>(w_out));
  return cudaGetLastError();
}

// ============================================== random-phase histogram ====
// random_coherence_histogram / topofit_phase_row_coh (:1310-1512) in FP64:
// one warp per random row, lanes over trials for the sweep (each lane sums its
// trial over the columns in the reference's order), lanes over columns for the
// refinement with the sums taken in column order by lane 0.
// The trial phasors e^{-j theta_c m} of every (column, trial), theta_c =
// (bp_c / range) * pi/4 (topofit_phase_row_coh, native_stage2.rs:1438-1470):
// the same for every random row, so they are evaluated once, [m][T].
__global__ void __launch_bounds__(256) k_trial_phasors(const double* __restrict__ bp, int m, int n_half,
                                                       double2* __restrict__ E) {
  const int T = 2 * n_half + 1;
  double mn = INFINITY, mx = -INFINITY;
  for (int c = 0; c < m; ++c) {
    mn = fmin(mn, bp[c]);
    mx = fmax(mx, bp[c]);
  }
  double range = mx - mn;
  if (range == 0.0) range = 1.0;
  const double qpi = 3.14159265358979323846 / 4.0;
  const int64_t total = static_cast<int64_t>(m) * T;
  for (int64_t idx = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x; idx < total;
       idx += static_cast<int64_t>(gridDim.x) * blockDim.x) {
    const int c = static_cast<int>(idx / T), t = static_cast<int>(idx - static_cast<int64_t>(c) * T);
    double sn, cs;
    sincos(__dmul_rn(__dmul_rn(bp[c] / range, qpi), static_cast<double>(t - n_half)), &sn, &cs);
    E[idx] = make_double2(cs, sn);
  }
}

__global__ void __launch_bounds__(256) k_random_hist(const double* __restrict__ rnd, int64_t n_rand,
                                                     const double* __restrict__ bp, int m,
                                                     const int64_t* __restrict__ ia, const int64_t* __restrict__ ib,
                                                     int small_baseline, int n_half, double cutoff0, double dbin,
                                                     const double2* __restrict__ E, int32_t* hist) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  const int tid = threadIdx.x, lane = tid & 31, wib = tid >> 5;
  double* ph = reinterpret_cast<double*>(smem_raw) + static_cast<int64_t>(wib) * 3 * m;
  double* t1 = ph + m;
  double* t2 = t1 + m;
  __shared__ int sh_hist[kCohBins];
  for (int i = tid; i < kCohBins; i += blockDim.x) sh_hist[i] = 0;
  __syncthreads();
  const int T = 2 * n_half + 1;
  double mn = INFINITY, mx = -INFINITY;
  for (int c = 0; c < m; ++c) {
    mn = fmin(mn, bp[c]);
    mx = fmax(mx, bp[c]);
  }
  double range = mx - mn;
  if (range == 0.0) range = 1.0;
  const double qpi = 3.14159265358979323846 / 4.0;
  const int64_t gw = (static_cast<int64_t>(blockIdx.x) * blockDim.x + tid) >> 5;
  const int64_t nw = (static_cast<int64_t>(gridDim.x) * blockDim.x) >> 5;
  for (int64_t row = gw; row < n_rand; row += nw) {
    __syncwarp();
    for (int c = lane; c < m; c += 32)
      ph[c] = small_baseline ? rnd[row + ib[c] * n_rand] - rnd[row + ia[c] * n_rand] : rnd[row + c * n_rand];
    // e^{j ph_c} once per row; the trial sum of e^{j (ph_c - theta_c m)} is then
    // e^{j ph_c} e^{-j theta_c m} from the phasor table: 4 FP64 operations per
    // (trial, column) instead of a sincos (the terms differ from sincos of the
    // rounded angle in the last bit; the sums keep the column order)
    for (int c = lane; c < m; c += 32) {
      double sn, cs;
      sincos(ph[c], &sn, &cs);
      t1[c] = cs;
      t2[c] = sn;
    }
    __syncwarp();
    double best = -1.0;
    int bt = 0;
    for (int t = lane; t < T; t += 32) {
      double sre = 0.0, sim = 0.0;
      for (int c = 0; c < m; ++c) {
        const double2 e = E[static_cast<int64_t>(c) * T + t];
        const double cp = t1[c], sp = t2[c];
        sre = __dadd_rn(sre, __fma_rn(cp, e.x, __dmul_rn(sp, e.y)));
        sim = __dadd_rn(sim, __fma_rn(sp, e.x, -__dmul_rn(cp, e.y)));
      }
      const double v = hypot(sre, sim) / static_cast<double>(m);
      if (v > best) {
        best = v;
        bt = t;
      }
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
      const double ob = __shfl_xor_sync(kFull, best, o);
      const int ot = __shfl_xor_sync(kFull, bt, o);
      if (ob > best || (ob == best && ot < bt)) {
        best = ob;
        bt = ot;
      }
    }
    const double k0 = qpi / range * static_cast<double>(bt - n_half);
    for (int c = lane; c < m; c += 32) {
      double sn, cs;
      sincos(__dsub_rn(ph[c], __dmul_rn(k0, bp[c])), &sn, &cs);
      t1[c] = cs;
      t2[c] = sn;
    }
    __syncwarp();
    double ore = 0.0, oim = 0.0;
    for (int c = 0; c < m; ++c) {
      ore = __dadd_rn(ore, t1[c]);
      oim = __dadd_rn(oim, t2[c]);
    }
    __syncwarp();
    for (int c = lane; c < m; c += 32) {
      const double cs = t1[c], sn = t2[c];
      const double pre = __dsub_rn(__dmul_rn(cs, ore), __dmul_rn(sn, -oim));
      const double pim = __dadd_rn(__dmul_rn(cs, -oim), __dmul_rn(sn, ore));
      t1[c] = __dmul_rn(bp[c], atan2(pim, pre));
      t2[c] = __dmul_rn(bp[c], bp[c]);
    }
    __syncwarp();
    double mopt = 0.0, den = 0.0;
    for (int c = 0; c < m; ++c) {
      den = __dadd_rn(den, t2[c]);
      mopt = __dadd_rn(mopt, t1[c]);
    }
    if (den == 0.0) den = 1.0;
    const double k = k0 + mopt / den;
    __syncwarp();
    for (int c = lane; c < m; c += 32) {
      double sn, cs;
      sincos(__dsub_rn(ph[c], __dmul_rn(k, bp[c])), &sn, &cs);
      t1[c] = cs;
      t2[c] = sn;
    }
    __syncwarp();
    if (lane == 0) {
      double sre = 0.0, sim = 0.0;
      for (int c = 0; c < m; ++c) {
        sre = __dadd_rn(sre, t1[c]);
        sim = __dadd_rn(sim, t2[c]);
      }
      const double coh = hypot(sre, sim) / static_cast<double>(m > 1 ? m : 1);
      const int b = coh_bin(coh, cutoff0, dbin);
      if (b >= 0) atomicAdd(&sh_hist[b], 1);
    }
  }
  __syncthreads();
  for (int i = tid; i < kCohBins; i += blockDim.x)
    if (sh_hist[i]) atomicAdd(&hist[i], sh_hist[i]);
}

cudaError_t launch_random_hist(const double* rnd, int64_t n_rand, const double* bp, int m, const int64_t* ia,
                               const int64_t* ib, int small_baseline, int n_half, double cutoff0, double dbin,
                               double2* phasors, int32_t* hist, int sm_count, cudaStream_t st) {
  const size_t sm = static_cast<size_t>(8) * 3 * m * sizeof(double);
  cudaError_t e = kernel_attributes_once(sm);
  if (e != cudaSuccess) return e;
  const int64_t n_ph = static_cast<int64_t>(m) * (2 * n_half + 1);
  k_trial_phasors<<<static_cast<unsigned>(std::min<int64_t>((n_ph + 255) / 256, static_cast<int64_t>(sm_count) * 8)),
                    256, 0, st>>>(bp, m, n_half, phasors);
  int64_t blocks = (n_rand + 7) / 8;
  if (blocks > static_cast<int64_t>(sm_count) * 8) blocks = static_cast<int64_t>(sm_count) * 8;
  if (blocks < 1) blocks = 1;
  k_random_hist<<<static_cast<unsigned>(blocks), 256, sm, st>>>(rnd, n_rand, bp, m, ia, ib, small_baseline, n_half,
                                                                cutoff0, dbin, phasors, hist);
  return cudaGetLastError();
}


// ============================================================== stage 3 ===
// Stage-3 re-estimate (pystamps/pipeline/ported.py:4489-4550): for every grid
// cell holding a selected PS, the 32x32 patch of the stage-2 grid around it with
// the PS's own cell zeroed is CLAP-filtered (_clap_filt_patch, :992-1009) and
// the filtered value at that cell is kept; then each selected PS is re-fitted
// (_ps_topofit_single, :2355-2431) against it.

// One warp: the 32x32 patch in its tile -> the filtered value at (bi, bj),
// times 1024. The inverse FFT is evaluated at that one point:
// y = sum_{k1,k2} Y[k1][k2] e^{+2 pi i (k1 bi + k2 bj) / 32}.
__device__ __forceinline__ float2 s3_patch_point(ClapTile<float>& T, const int lane, const S3ClapArgs& a,
                                                 const float2* twf, const float2* wp, const float* lp,
                                                 const float (&g7)[7], const int bi, const int bj) {
  fft_pass<float>(T.re, T.im, twf, lane, true);
  __syncwarp();
  fft_pass<float>(T.re, T.im, twf, lane, false);
#pragma unroll
  for (int k = 0; k < 32; ++k) {
    const float xr = T.re[k][lane], xi = T.im[k][lane];
    T.hs[k][lane] = sqrtf(xr * xr + xi * xi);
  }
  __syncwarp();
  // 7x7 Gaussian 'same' smoothing of fftshift(|X|), then ifftshift, in
  // unshifted coordinates (the seam at the Nyquist row / column)
  float t[32];
  const int sj = (lane + 16) & 31;
#pragma unroll
  for (int k = 0; k < 32; ++k) {
    float acc = 0.f;
#pragma unroll
    for (int d = -3; d <= 3; ++d)
      if (sj + d >= 0 && sj + d < 32) acc += T.hs[k][(lane + d) & 31] * g7[d + 3];
    t[k] = acc;
  }
  float o[32];
#pragma unroll
  for (int k = 0; k < 32; ++k) {
    const int sk = (k + 16) & 31;
    float acc = 0.f;
#pragma unroll
    for (int d = -3; d <= 3; ++d)
      if (sk + d >= 0 && sk + d < 32) acc += t[(k + d) & 31] * g7[d + 3];
    o[k] = acc;
  }
  const float med = warp_median1024<float>(o, &T.hs[0][0]);
  const float beta = static_cast<float>(a.beta), alpha = static_cast<float>(a.alpha);
  const float inv_med = med != 0.f ? 1.f / med : 1.f;
  float2 acc = make_float2(0.f, 0.f);
#pragma unroll
  for (int k = 0; k < 32; ++k) {
    float v = o[k] * inv_med;
    v = a.alpha_is_one ? v - 1.f : powf(v, alpha) - 1.f;
    if (v < 0.f) v = 0.f;
    const float gk = v * beta + lp[k * 32 + lane];
    const float2 y = make_float2(T.re[k][lane] * gk, T.im[k][lane] * gk);
    const float2 w = wp[(k * bi) & 31];
    acc.x += y.x * w.x - y.y * w.y;
    acc.y += y.x * w.y + y.y * w.x;
  }
  const float2 w = wp[(lane * bj) & 31];
  float2 r = make_float2(acc.x * w.x - acc.y * w.y, acc.x * w.y + acc.y * w.x);
  r.x = warp_sum(r.x);
  r.y = warp_sum(r.y);
  return r;
}

__global__ void __launch_bounds__(128) k_s3_clap(S3ClapArgs a, Twiddles32f tw) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  ClapTile<float>* tiles = reinterpret_cast<ClapTile<float>*>(smem_raw);
  float* lp = reinterpret_cast<float*>(tiles + 4);
  float2* twf = reinterpret_cast<float2*>(lp + 1024);
  float2* wp = twf + 16;  // e^{+2 pi i k / 32}, k < 32
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  for (int i = tid; i < 1024; i += 128) lp[i] = static_cast<float>(a.low_pass[i]);
  if (tid < 16) {
    twf[tid] = tw.w[tid];
    wp[tid] = make_float2(tw.w[tid].x, -tw.w[tid].y);
    wp[tid + 16] = make_float2(-tw.w[tid].x, tw.w[tid].y);
  }
  float g7[7];
#pragma unroll
  for (int i = 0; i < 7; ++i) g7[i] = static_cast<float>(a.g7[i]);
  const int M = a.M;
  const int64_t ntask = a.n_jobs * a.ngroups;
  for (int64_t task = blockIdx.x; task < ntask; task += gridDim.x) {
    const int64_t job = task / a.ngroups;
    const int g = static_cast<int>(task - job * a.ngroups);
    const int i0 = a.jobs[4 * job], j0 = a.jobs[4 * job + 1], bi = a.jobs[4 * job + 2], bj = a.jobs[4 * job + 3];
    const int c_warp = 4 * g + warp;
    if (i0 < 0) {
      // the 32-cell patch does not fit: the reference sets ph_patch2 to 0
      if (lane == 0 && c_warp < M) a.job_out[job * M + c_warp] = make_float2(0.f, 0.f);
      continue;
    }
    __syncthreads();
    for (int idx = tid; idx < 4 * 1024; idx += 128) {
      const int pix = idx >> 2, q = idx & 3;
      const int li = pix >> 5, lj = pix & 31;
      const int c = 4 * g + q;
      float2 v = make_float2(0.f, 0.f);
      if (c < M) {
        v = a.grid[(static_cast<int64_t>(i0 + li) * a.grid_cols + (j0 + lj)) * a.grid_stride + c];
        if (isnan(v.x) || isnan(v.y)) v = make_float2(0.f, 0.f);
        const bool own = li == bi && lj == bj;
        const bool osf = c == 0 && abs(li - bi) <= a.slc_rad && abs(lj - bj) <= a.slc_rad;
        if (own || osf) v = make_float2(0.f, 0.f);
      }
      tiles[q].re[li][lj] = v.x;
      tiles[q].im[li][lj] = v.y;
    }
    __syncthreads();
    if (c_warp < M) {
      const float2 r = s3_patch_point(tiles[warp], lane, a, twf, wp, lp, g7, bi, bj);
      if (lane == 0) a.job_out[job * M + c_warp] = make_float2(r.x * (1.f / 1024.f), r.y * (1.f / 1024.f));
    }
  }
}

size_t s3_clap_smem() { return 4 * sizeof(ClapTile<float>) + 1024 * sizeof(float) + 48 * sizeof(float2); }

cudaError_t launch_s3_clap(const S3ClapArgs& a, const Twiddles32f& tf, int sm_count, cudaStream_t st) {
  const int64_t ntask = a.n_jobs * a.ngroups;
  if (ntask <= 0) return cudaSuccess;
  const size_t sm = s3_clap_smem();
  cudaError_t e = kernel_attributes_once(sm);
  if (e != cudaSuccess) return e;
  int per_sm = 0;
  e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_s3_clap, 128, sm);
  if (e != cudaSuccess) return e;
  const int64_t blocks = std::min<int64_t>(ntask, static_cast<int64_t>(sm_count) * std::max(per_sm, 1));
  k_s3_clap<<<static_cast<unsigned>(blocks), 128, sm, st>>>(a, tf);
  return cudaGetLastError();
}

// np.exp(-1j * x) in complex64: (cos x, -sin x)
__device__ __forceinline__ float2 s3_cis_neg(float x) {
  float s, c;
  sincosf(x, &s, &c);
  return make_float2(c, -s);
}

struct S3Fit {
  float K, C, coh;
};

// _ps_topofit_refine_candidate (ported.py:2473-2508), float32, lanes over columns
__device__ S3Fit s3_refine(const float2* cpx, const float* bp, int n, double den_lin, double coarse_k0, int lane) {
  float K0 = static_cast<float>(coarse_k0);
  float ox = 0.f, oy = 0.f;
  for (int k = lane; k < n; k += 32) {
    const float2 r = cmul_rn(cpx[k], s3_cis_neg(__fmul_rn(K0, bp[k])));
    ox += r.x;
    oy += r.y;
  }
  ox = warp_sum(ox);
  oy = warp_sum(oy);
  float mo = 0.f;
  for (int k = lane; k < n; k += 32) {
    const float2 r = cmul_rn(cpx[k], s3_cis_neg(__fmul_rn(K0, bp[k])));
    const float2 q = cmul_rn(r, make_float2(ox, -oy));
    const float wgt = hypotf(cpx[k].x, cpx[k].y);
    mo += __fmul_rn(__fmul_rn(wgt, bp[k]), __fmul_rn(wgt, atan2f(q.y, q.x)));
  }
  mo = warp_sum(mo);
  K0 = __fadd_rn(K0, __fdiv_rn(mo, static_cast<float>(den_lin)));
  float mx = 0.f, my = 0.f, den = 0.f;
  for (int k = lane; k < n; k += 32) {
    const float2 r = cmul_rn(cpx[k], s3_cis_neg(__fmul_rn(K0, bp[k])));
    mx += r.x;
    my += r.y;
    den += hypotf(r.x, r.y);
  }
  mx = warp_sum(mx);
  my = warp_sum(my);
  den = warp_sum(den);
  if (den == 0.f) den = 1.f;
  return {K0, atan2f(my, mx), hypotf(mx, my) / den};
}

// One warp per selected PS: psdph against the re-estimated patch phase, the
// reference's invalid-row rule, then _ps_topofit_single with the near-max
// candidate rule (tolerance 2e-4), refinement of every candidate and the
// reference's choice among them.
__global__ void __launch_bounds__(128) k_s3_fit(S3FitArgs a) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  const int lane = threadIdx.x & 31, wib = threadIdx.x >> 5;
  const int T = 2 * a.n_half + 1;
  const int nf = a.n_fit, M = a.M;
  unsigned char* base = smem_raw + static_cast<size_t>(wib) * a.warp_smem;
  float2* cpx = reinterpret_cast<float2*>(base);
  float* bp = reinterpret_cast<float*>(cpx + nf);
  float* tp = bp + nf;
  float* ct = tp + nf;
  const int64_t gw = static_cast<int64_t>(blockIdx.x) * 4 + wib;
  const int64_t nw = static_cast<int64_t>(gridDim.x) * 4;
  for (int64_t r = gw; r < a.n_sel; r += nw) {
    const int job = a.job_of[r];
    const int64_t row = a.row ? static_cast<int64_t>(a.row[r]) : r;  // row of ph / bp
    bool zero = false;
    for (int c = lane; c < M; c += 32) {
      const float2 pp = a.job_out[static_cast<int64_t>(job) * M + c];
      a.ph_patch2[r * M + c] = pp;
      a.ph_res2[r * M + c] = 0.f;
      const float2 h = a.ph[row * M + c];
      // psdph = ph * conj(ph_patch2) in f64 (exact products of f32 values)
      const double re = static_cast<double>(h.x) * pp.x + static_cast<double>(h.y) * pp.y;
      const double im = static_cast<double>(h.y) * pp.x - static_cast<double>(h.x) * pp.y;
      if (re == 0.0 && im == 0.0) zero = true;
    }
    if (__any_sync(0xffffffffu, zero)) {
      if (lane == 0) {
        a.K2[r] = __longlong_as_double(0x7ff8000000000000LL);
        a.coh2[r] = __longlong_as_double(0x7ff8000000000000LL);
        a.C2[r] = 0.0;
      }
      continue;
    }
    float mn = __int_as_float(0x7f800000), mx = -mn;
    for (int k = lane; k < nf; k += 32) {
      const int c = a.fit[k];
      const float2 pp = a.job_out[static_cast<int64_t>(job) * M + c];
      const float2 h = a.ph[row * M + c];
      const double re = static_cast<double>(h.x) * pp.x + static_cast<double>(h.y) * pp.y;
      const double im = static_cast<double>(h.y) * pp.x - static_cast<double>(h.x) * pp.y;
      const double mg = hypot(re, im);
      cpx[k] = make_float2(static_cast<float>(re / mg), static_cast<float>(im / mg));
      bp[k] = a.bp_row_inv ? a.bp[c] : a.bp[row * M + c];
      mn = fminf(mn, bp[k]);
      mx = fmaxf(mx, bp[k]);
    }
    mn = -warp_max(-mn);
    mx = warp_max(mx);
    double range = static_cast<double>(__fsub_rn(mx, mn));
    if (range == 0.0) range = 1.0;
    const float rf = static_cast<float>(range), qp = 0.785398163397448309615f;
    float den = 0.f, dl = 0.f;
    for (int k = lane; k < nf; k += 32) {
      tp[k] = __fmul_rn(__fdiv_rn(bp[k], rf), qp);
      const float ab = hypotf(cpx[k].x, cpx[k].y);
      const float wb = __fmul_rn(ab, bp[k]);
      den += ab;
      dl += __fmul_rn(wb, wb);
    }
    double denom = static_cast<double>(warp_sum(den));
    double den_lin = static_cast<double>(warp_sum(dl));
    if (denom == 0.0) denom = 1.0;
    if (den_lin == 0.0) den_lin = 1.0;
    __syncwarp();
    // coherence of every trial, columns summed in order (the reference adds
    // the rows of its (columns, trials) product one after another)
    float cmax = -1.f;
    for (int t = lane; t < T; t += 32) {
      const float tm = static_cast<float>(t - a.n_half);
      float sx = 0.f, sy = 0.f;
      for (int k = 0; k < nf; ++k) {
        const float2 p = cmul_rn(s3_cis_neg(__fmul_rn(tp[k], tm)), cpx[k]);
        sx = __fadd_rn(sx, p.x);
        sy = __fadd_rn(sy, p.y);
      }
      ct[t] = __fdiv_rn(hypotf(sx, sy), static_cast<float>(denom));
      cmax = fmaxf(cmax, ct[t]);
    }
    cmax = warp_max(cmax);
    __syncwarp();
    // candidates in trial order: local maxima within 2e-4 of the maximum
    int n_cand = 0, first = -1, last = -1, coarse_best = -1, refined_best = -1;
    S3Fit best_fit{0.f, 0.f, -1.f};
    float coarse_best_v = -1.f;
    for (int t0 = 0; t0 < T; t0 += 32) {
      const int t = t0 + lane;
      bool cand = false;
      if (t < T) {
        const float v = ct[t];
        bool lm;
        if (T == 1) lm = true;
        else if (t == 0) lm = v >= ct[1];
        else if (t == T - 1) lm = v >= ct[T - 2];
        else lm = v >= ct[t - 1] && v >= ct[t + 1];
        cand = lm && static_cast<double>(v) >= static_cast<double>(cmax) - 2.0e-4;
      }
      unsigned bal = __ballot_sync(0xffffffffu, cand);
      while (bal) {
        const int tt = t0 + __ffs(bal) - 1;
        bal &= bal - 1;
        if (first < 0) first = tt;
        last = tt;
        ++n_cand;
        if (ct[tt] > coarse_best_v) {
          coarse_best_v = ct[tt];
          coarse_best = tt;
        }
        const S3Fit f = s3_refine(cpx, bp, nf, den_lin, (3.14159265358979323846 / 4.0) / range * (tt - a.n_half), lane);
        if (static_cast<double>(f.coh) > static_cast<double>(best_fit.coh)) {
          best_fit = f;
          refined_best = tt;
        }
      }
    }
    int pick = refined_best;
    if (n_cand == 2 && first == 0 && last == T - 1) pick = coarse_best;
    if (pick < 0) pick = coarse_best >= 0 ? coarse_best : 0;  // refined coherences all NaN
    S3Fit f = best_fit;
    if (pick != refined_best)
      f = s3_refine(cpx, bp, nf, den_lin, (3.14159265358979323846 / 4.0) / range * (pick - a.n_half), lane);
    for (int k = lane; k < nf; k += 32) {
      const float2 res = cmul_rn(cpx[k], s3_cis_neg(__fmul_rn(f.K, bp[k])));
      a.ph_res2[r * M + a.fit[k]] = atan2f(res.y, res.x);
    }
    if (lane == 0) {
      a.K2[r] = static_cast<double>(f.K);
      a.C2[r] = static_cast<double>(f.C);
      a.coh2[r] = static_cast<double>(f.coh);
    }
    __syncwarp();
  }
}

cudaError_t launch_s3_fit(const S3FitArgs& a, int sm_count, cudaStream_t st) {
  if (a.n_sel <= 0) return cudaSuccess;
  const size_t sm = 4 * a.warp_smem;
  cudaError_t e = kernel_attributes_once(sm);
  if (e != cudaSuccess) return e;
  int per_sm = 0;
  e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_s3_fit, 128, sm);
  if (e != cudaSuccess) return e;
  const int64_t blocks =
      std::min<int64_t>((a.n_sel + 3) / 4, static_cast<int64_t>(sm_count) * std::max(per_sm, 1));
  k_s3_fit<<<static_cast<unsigned>(blocks), 128, sm, st>>>(a);
  return cudaGetLastError();
}

// ================================================= registry topofit =======
// The registry's topofit (pystamps/kernels/accelerated.py:316-380 ->
// ported._ps_topofit_single, pystamps/pipeline/ported.py:2355-2431; the PyO3
// twin src/lib.rs:525-586 uses the same rule with tolerance 5e-3): per row,
// the non-zero columns only (zero columns take no part; an all-zero row gives
// NaN), trial coherences with columns summed in order, the near-max candidate
// set (local maxima within `tol` of the maximum), every candidate refined
// (_ps_topofit_refine_candidate, :2480-2513) and the reference's choice among
// them (_ps_topofit_select_candidate, :2451-2477). R is the row's real type:
// float for complex64 rows (the reference's single-precision path), double for
// complex128 rows. One warp per row.
template <typename R>
struct NearFit {
  R K, C, coh;
};

template <typename R>
__device__ __forceinline__ typename CT<R>::C cis_neg_r(R x) {
  R s, c;
  sincos_r(x, &s, &c);
  return mk(c, -s);
}

template <typename R>
__device__ NearFit<R> near_refine(const typename CT<R>::C* cv, const R* bv, int nf, R den_lin, double coarse_k0,
                                  int lane) {
  using C = typename CT<R>::C;
  R K0 = static_cast<R>(coarse_k0);
  R ox = 0, oy = 0;
  for (int k = lane; k < nf; k += 32) {
    const C r = cmul_rn(cv[k], cis_neg_r<R>(mul_rn(K0, bv[k])));
    ox = add_rn(ox, r.x);
    oy = add_rn(oy, r.y);
  }
  ox = warp_sum(ox);
  oy = warp_sum(oy);
  R mo = 0;
  for (int k = lane; k < nf; k += 32) {
    const C r = cmul_rn(cv[k], cis_neg_r<R>(mul_rn(K0, bv[k])));
    const C q = cmul_rn(r, mk(ox, -oy));
    const R wgt = hypot_r(cv[k].x, cv[k].y);
    mo = add_rn(mo, mul_rn(mul_rn(wgt, bv[k]), mul_rn(wgt, atan2_r(q.y, q.x))));
  }
  mo = warp_sum(mo);
  K0 = add_rn(K0, mo / den_lin);
  R mx = 0, my = 0, den = 0;
  for (int k = lane; k < nf; k += 32) {
    const C r = cmul_rn(cv[k], cis_neg_r<R>(mul_rn(K0, bv[k])));
    mx = add_rn(mx, r.x);
    my = add_rn(my, r.y);
    den = add_rn(den, hypot_r(r.x, r.y));
  }
  mx = warp_sum(mx);
  my = warp_sum(my);
  den = warp_sum(den);
  if (den == R(0)) den = R(1);
  return {K0, atan2_r(my, mx), hypot_r(mx, my) / den};
}

template <typename R>
__global__ void __launch_bounds__(32) k_topofit_near_max(NearMaxArgs a) {
  using C = typename CT<R>::C;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  const int lane = threadIdx.x;
  const int M = a.M, T = 2 * a.n_half + 1;
  C* cv = reinterpret_cast<C*>(smem_raw);  // valid columns, compacted in column order
  R* bv = reinterpret_cast<R*>(cv + M);
  R* tp = bv + M;
  R* ct = tp + M;
  int* col = reinterpret_cast<int*>(ct + T);
  const C* cpx = static_cast<const C*>(a.cpx);
  const R* bp = static_cast<const R*>(a.bp);
  const double nanv = __longlong_as_double(0x7ff8000000000000LL);
  for (int64_t r = blockIdx.x; r < a.n; r += gridDim.x) {
    int nf = 0;
    for (int c0 = 0; c0 < M; c0 += 32) {
      const int c = c0 + lane;
      C v = mk(R(0), R(0));
      R b = 0;
      bool valid = false;
      if (c < M) {
        v = cpx[r * M + c];
        b = a.bp_row_inv ? bp[c] : bp[r * M + c];
        valid = !(v.x == R(0) && v.y == R(0));  // complex != 0 (NaN parts count as non-zero)
        if (a.residual) a.residual[r * M + c] = make_float2(0.f, 0.f);
      }
      const unsigned bal = __ballot_sync(kFull, valid);
      if (valid) {
        const int k = nf + __popc(bal & ((1u << lane) - 1u));
        cv[k] = v;
        bv[k] = b;
        col[k] = c;
      }
      nf += __popc(bal);
    }
    __syncwarp();
    if (nf == 0) {
      if (lane == 0) a.K[r] = a.C[r] = a.coh[r] = nanv;
      continue;
    }
    R mn = bv[0], mx = bv[0];
    for (int k = lane; k < nf; k += 32) {
      mn = mn < bv[k] ? mn : bv[k];
      mx = mx > bv[k] ? mx : bv[k];
    }
    mn = warp_min(mn);
    mx = warp_max(mx);
    double range = static_cast<double>(add_rn(mx, -mn));
    if (range == 0.0) range = 1.0;
    const R range_r = static_cast<R>(range), qp = static_cast<R>(3.14159265358979323846 / 4.0);
    R den = 0, dl = 0;
    for (int k = lane; k < nf; k += 32) {
      tp[k] = mul_rn(bv[k] / range_r, qp);
      const R ab = hypot_r(cv[k].x, cv[k].y);
      const R wb = mul_rn(ab, bv[k]);
      den = add_rn(den, ab);
      dl = add_rn(dl, mul_rn(wb, wb));
    }
    R denom = warp_sum(den), den_lin = warp_sum(dl);
    if (denom == R(0)) denom = R(1);
    if (den_lin == R(0)) den_lin = R(1);
    __syncwarp();
    // coherence of every trial, columns summed in order
    R cmax = -1;
    for (int t = lane; t < T; t += 32) {
      const R tm = static_cast<R>(t - a.n_half);
      R sx = 0, sy = 0;
      for (int k = 0; k < nf; ++k) {
        const C p = cmul_rn(cis_neg_r<R>(mul_rn(tp[k], tm)), cv[k]);
        sx = add_rn(sx, p.x);
        sy = add_rn(sy, p.y);
      }
      ct[t] = hypot_r(sx, sy) / denom;
      cmax = cmax > ct[t] ? cmax : ct[t];
    }
    cmax = warp_max(cmax);
    __syncwarp();
    int n_cand = 0, first = -1, last = -1, coarse_best = -1, refined_best = -1;
    NearFit<R> best_fit{0, 0, -1};
    R coarse_best_v = -1;
    for (int t0 = 0; t0 < T; t0 += 32) {
      const int t = t0 + lane;
      bool cand = false;
      if (t < T) {
        const R v = ct[t];
        bool lm;
        if (T == 1) lm = true;
        else if (t == 0) lm = v >= ct[1];
        else if (t == T - 1) lm = v >= ct[T - 2];
        else lm = v >= ct[t - 1] && v >= ct[t + 1];
        cand = lm && static_cast<double>(v) >= static_cast<double>(cmax) - a.tol;
      }
      unsigned bal = __ballot_sync(kFull, cand);
      while (bal) {
        const int tt = t0 + __ffs(bal) - 1;
        bal &= bal - 1;
        if (first < 0) first = tt;
        last = tt;
        ++n_cand;
        if (ct[tt] > coarse_best_v) {
          coarse_best_v = ct[tt];
          coarse_best = tt;
        }
        const NearFit<R> f =
            near_refine<R>(cv, bv, nf, den_lin, (3.14159265358979323846 / 4.0) / range * (tt - a.n_half), lane);
        if (static_cast<double>(f.coh) > static_cast<double>(best_fit.coh)) {
          best_fit = f;
          refined_best = tt;
        }
      }
    }
    if (n_cand == 0) {  // no local maximum within tol (NaN coherences): np.argmax (a NaN wins)
      for (int t = 0; t < T; ++t) {
        if (isnan(ct[t])) {
          coarse_best = t;
          break;
        }
        if (ct[t] > coarse_best_v) {
          coarse_best_v = ct[t];
          coarse_best = t;
        }
      }
      if (coarse_best < 0) coarse_best = 0;
    }
    int pick = refined_best;
    if (n_cand <= 1 || (n_cand == 2 && first == 0 && last == T - 1)) pick = coarse_best;
    if (pick < 0) pick = coarse_best >= 0 ? coarse_best : 0;
    NearFit<R> f = best_fit;
    if (pick != refined_best)
      f = near_refine<R>(cv, bv, nf, den_lin, (3.14159265358979323846 / 4.0) / range * (pick - a.n_half), lane);
    if (a.residual)
      for (int k = lane; k < nf; k += 32) {
        const C res = cmul_rn(cv[k], cis_neg_r<R>(mul_rn(f.K, bv[k])));
        a.residual[r * M + col[k]] = make_float2(static_cast<float>(res.x), static_cast<float>(res.y));
      }
    if (lane == 0) {
      a.K[r] = static_cast<double>(f.K);
      a.C[r] = static_cast<double>(f.C);
      a.coh[r] = static_cast<double>(f.coh);
    }
    __syncwarp();
  }
}

size_t topofit_near_max_smem(bool fp64, int M, int n_half) {
  const size_t rs = fp64 ? sizeof(double) : sizeof(float);
  return static_cast<size_t>(M) * (2 * rs + rs + rs + sizeof(int)) + static_cast<size_t>(2 * n_half + 1) * rs + 16;
}

cudaError_t launch_topofit_near_max(const NearMaxArgs& a, bool fp64, int sm_count, cudaStream_t st) {
  if (a.n <= 0) return cudaSuccess;
  const size_t sm = topofit_near_max_smem(fp64, a.M, a.n_half);
  cudaError_t e = kernel_attributes_once(sm);
  if (e != cudaSuccess) return e;
  const int64_t blocks = std::min<int64_t>(a.n, static_cast<int64_t>(sm_count) * 32);
  if (fp64)
    k_topofit_near_max<double><<<static_cast<unsigned>(blocks), 32, sm, st>>>(a);
  else
    k_topofit_near_max<float><<<static_cast<unsigned>(blocks), 32, sm, st>>>(a);
  return cudaGetLastError();
}

// ================================================ histogram with centers ==
// The registry's stage2_histogram (pystamps/kernels/accelerated.py:235-265):
// equally spaced centres use the ceil rule 1 + max(0, min(nc-1,
// ceil((v - cutoff0) / d))); otherwise the bin is searchsorted(mids, v,
// 'left') clipped to [0, nc-1]. Non-finite values are skipped. Integer
// atomics: the counts do not depend on the order.
__global__ void __launch_bounds__(256) k_hist_centers(const double* __restrict__ v, int64_t n,
                                                      const double* __restrict__ mids, int nc, int equal, double d,
                                                      double cutoff0, unsigned long long* __restrict__ counts) {
  const int64_t stride = static_cast<int64_t>(gridDim.x) * blockDim.x;
  for (int64_t i = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x; i < n; i += stride) {
    const double s = v[i];
    if (!isfinite(s)) continue;
    int b;
    if (equal) {
      const double q = ceil((s - cutoff0) / d);
      b = static_cast<int>(fmax(0.0, fmin(static_cast<double>(nc - 1), q)));
    } else {
      int lo = 0, hi = nc - 1;  // first of the nc-1 mids that is >= s
      while (lo < hi) {
        const int mid = (lo + hi) >> 1;
        if (mids[mid] < s) lo = mid + 1;
        else hi = mid;
      }
      b = lo;
    }
    atomicAdd(&counts[b], 1ull);
  }
}

cudaError_t launch_hist_centers(const double* v, int64_t n, const double* mids, int nc, int equal, double d,
                                double cutoff0, unsigned long long* counts, int sm_count, cudaStream_t st) {
  if (n <= 0) return cudaSuccess;
  const int64_t blocks = std::min<int64_t>((n + 255) / 256, static_cast<int64_t>(sm_count) * 8);
  k_hist_centers<<<static_cast<unsigned>(blocks), 256, 0, st>>>(v, n, mids, nc, equal, d, cutoff0, counts);
  return cudaGetLastError();
}

// ============================================================== batches ===
// Many patches, each iteration one launch per step over every active patch.
// Work units are numbered patch after patch (prefix tables); a unit finds its
// patch by binary search. Each unit runs the single-patch code on its patch's
// arguments, so a patch's results do not depend on what it is batched with.

__device__ __forceinline__ int find_patch(const int64_t* __restrict__ prefix, int P, int64_t u) {
  int lo = 0, hi = P - 1;
  while (lo < hi) {
    const int mid = (lo + hi + 1) >> 1;
    if (prefix[mid] <= u)
      lo = mid;
    else
      hi = mid - 1;
  }
  return lo;
}

// per-iteration reset of the active patches: histogram, invalid count, rms
// partials, and K[1] <- K[0] (the K this iteration bins with)
__global__ void __launch_bounds__(256) k_batch_reset(BatchArgs b) {
  const int p = blockIdx.x;
  if (p >= b.P || !b.active[p]) return;
  const PatchDev& d = b.patch[p];
  for (int i = threadIdx.x; i < kCohBins; i += blockDim.x) d.topo.hist[i] = 0;
  if (threadIdx.x == 0) *d.topo.n_invalid = 0;
  for (int i = threadIdx.x; i < d.fin.n_partial; i += blockDim.x) d.topo.rms_partial[i] = 0.0;
  const float* __restrict__ k0 = static_cast<const float*>(d.bin.K);
  float* __restrict__ k1 = d.K1;
  for (int64_t i = threadIdx.x; i < d.topo.N; i += blockDim.x) k1[i] = k0[i];
}

__global__ void __launch_bounds__(256) k_batch_bin(BatchArgs b) {
  const int lane = threadIdx.x & 31;
  const int64_t gw = (static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x) >> 5;
  const int64_t nw = (static_cast<int64_t>(gridDim.x) * blockDim.x) >> 5;
  const int64_t total = b.bin_prefix[b.P];
  for (int64_t u = gw; u < total; u += nw) {
    const int p = find_patch(b.bin_prefix, b.P, u);
    if (!b.active[p]) continue;
    const PatchDev& d = b.patch[p];
    BinArgs a = d.bin;
    // iteration 1 bins with the initial weights, later ones with the P-square table
    a.mode = (d.psquare && d.fin.state[1] > 1.0) ? 1 : 0;
    bin_task<float>(a, u - b.bin_prefix[p], lane);
  }
}

__global__ void __launch_bounds__(128) k_batch_clap(BatchArgs b, Twiddles32f tw) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  const ClapSmem<float, 4> m = clap_smem<float, 4>(smem_raw, tw);
  float g7[7];
  int cur = -1;
  const int64_t total = b.clap_prefix[b.P];
  for (int64_t u = blockIdx.x; u < total; u += gridDim.x) {
    const int p = find_patch(b.clap_prefix, b.P, u);
    if (!b.active[p]) continue;
    const ClapArgs& a = b.patch[p].clap;
    if (p != cur) {
      // the previous task's readers of lp / wt passed its last barrier
      clap_consts<float>(a, m.lp, m.wt);
#pragma unroll
      for (int i = 0; i < 7; ++i) g7[i] = static_cast<float>(a.g7[i]);
      cur = p;
    }
    if (a.part)
      clap_block_task<float, 4>(a, u - b.clap_prefix[p], m.tiles, m.twf, m.twi, m.lp, m.wt, g7);
    else
      clap_task<float, 4>(a, u - b.clap_prefix[p], m.tiles, m.twf, m.twi, m.lp, m.wt, g7);
  }
}

__global__ void __launch_bounds__(256) k_batch_overlap(BatchArgs b) {
  const int64_t total = b.ov_prefix[b.P];
  for (int64_t u = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x; u < total;
       u += static_cast<int64_t>(gridDim.x) * blockDim.x) {
    const int p = find_patch(b.ov_prefix, b.P, u);
    if (!b.active[p]) continue;
    if (b.patch[p].ov.part)
      combine_elem<float>(b.patch[p].ov, u - b.ov_prefix[p]);
    else
      overlap_elem<float>(b.patch[p].ov, u - b.ov_prefix[p]);
  }
}

template <int L>
__global__ void __launch_bounds__(128, 4) k_batch_topofit(BatchArgs b, const int32_t* __restrict__ units, int n_units) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  __shared__ int sh_hist[kCohBins];
  __shared__ double sh_rms[4];
  __shared__ int sh_inv[4];
  for (int u = blockIdx.x; u < n_units; u += gridDim.x) {
    const int p = units[2 * u], vb = units[2 * u + 1];
    if (!b.active[p]) continue;
    const PatchDev& d = b.patch[p];
    // batches hold loaded contexts: always the loop form
    if (d.topo.bp_row_inv)
      topofit_vblock_t<L, true, true>(d.topo, d.mpad, vb, d.nvb, smem_raw, sh_hist, sh_rms, sh_inv);
    else
      topofit_vblock_t<L, true, false>(d.topo, d.mpad, vb, d.nvb, smem_raw, sh_hist, sh_rms, sh_inv);
  }
}

__global__ void __launch_bounds__(256) k_batch_finalize(BatchArgs b) {
  const int p = blockIdx.x;
  if (p >= b.P || !b.active[p]) return;
  const FinalizeArgs& f = b.patch[p].fin;
  finalize_body(f);
  __syncthreads();
  if (threadIdx.x == 0 && f.stats_out[3] != 0.0 && !f.force_continue) {
    b.active[p] = 0;
    atomicSub(b.n_active, 1);
  }
}

__global__ void k_batch_continue(cudaGraphConditionalHandle h, const int* n_active) {
  if (threadIdx.x == 0) cudaGraphSetConditional(h, *n_active > 0 ? 1u : 0u);
}

cudaError_t launch_batch_reset(const BatchArgs& b, cudaStream_t st) {
  k_batch_reset<<<b.P, 256, 0, st>>>(b);
  return cudaGetLastError();
}

cudaError_t launch_batch_bin(const BatchArgs& b, int64_t total, int sm_count, cudaStream_t st) {
  const int64_t blocks = std::max<int64_t>(1, std::min<int64_t>((total + 7) / 8, static_cast<int64_t>(sm_count) * 16));
  k_batch_bin<<<static_cast<unsigned>(blocks), 256, 0, st>>>(b);
  return cudaGetLastError();
}

cudaError_t launch_batch_clap(const BatchArgs& b, int64_t total, const Twiddles32f& tf, int sm_count,
                              cudaStream_t st) {
  if (total <= 0) return cudaSuccess;
  const size_t sm = clap_smem_bytes<float, 4>();
  cudaError_t e = kernel_attributes_once(sm);
  if (e != cudaSuccess) return e;
  int per_sm = 0;
  e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_batch_clap, 128, sm);
  if (e != cudaSuccess) return e;
  const int64_t blocks = std::min<int64_t>(total, static_cast<int64_t>(sm_count) * std::max(per_sm, 1));
  k_batch_clap<<<static_cast<unsigned>(blocks), 128, sm, st>>>(b, tf);
  return cudaGetLastError();
}

cudaError_t launch_batch_overlap(const BatchArgs& b, int64_t total, int sm_count, cudaStream_t st) {
  const int64_t blocks = std::max<int64_t>(1, std::min<int64_t>((total + 255) / 256, static_cast<int64_t>(sm_count) * 32));
  k_batch_overlap<<<static_cast<unsigned>(blocks), 256, 0, st>>>(b);
  return cudaGetLastError();
}

template <int L>
static cudaError_t batch_topofit_l(const BatchArgs& b, const int32_t* units, int n_units, size_t sm, int sm_count,
                                   cudaStream_t st) {
  cudaError_t e = kernel_attributes_once(sm);
  if (e != cudaSuccess) return e;
  int per_sm = 0;
  e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_batch_topofit<L>, 128, sm);
  if (e != cudaSuccess) return e;
  const int64_t blocks = std::min<int64_t>(n_units, static_cast<int64_t>(sm_count) * std::max(per_sm, 1));
  k_batch_topofit<L><<<static_cast<unsigned>(blocks), 128, sm, st>>>(b, units, n_units);
  return cudaGetLastError();
}

cudaError_t launch_batch_topofit(const BatchArgs& b, int L, const int32_t* units, int n_units, size_t smem,
                                 int sm_count, cudaStream_t st) {
  if (n_units <= 0) return cudaSuccess;
  switch (L) {
    case 4: return batch_topofit_l<4>(b, units, n_units, smem, sm_count, st);
    case 8: return batch_topofit_l<8>(b, units, n_units, smem, sm_count, st);
    case 16: return batch_topofit_l<16>(b, units, n_units, smem, sm_count, st);
    case 32: return batch_topofit_l<32>(b, units, n_units, smem, sm_count, st);
    default: return cudaErrorInvalidValue;
  }
}

cudaError_t launch_batch_finalize(const BatchArgs& b, cudaStream_t st) {
  k_batch_finalize<<<b.P, 256, 0, st>>>(b);
  return cudaGetLastError();
}

cudaError_t launch_batch_continue(cudaGraphConditionalHandle h, const int* n_active, cudaStream_t st) {
  k_batch_continue<<<1, 32, 0, st>>>(h, n_active);
  return cudaGetLastError();
}

// ============================================================== adjoints ==
// Differentiable stage-2 coherence with K given (no trial search):
//   grid  = bin(ph e^{-j K bp} w)              (k_bin, mode 0)
//   filt  = CLAP(grid; alpha, beta)            (k_clap + k_overlap)
//   p     = filt[cell] / |filt[cell]|          (resample + normalise)
//   gamma = |sum_c conj(p_c) ph_c e^{-j K bp_c}| / sum_c |conj(p_c) ph_c|
// Gradients use the complex convention g = dL/dRe + j dL/dIm. CLAP's window
// spectra are recomputed in the backward pass, not stored. R is the working
// precision (the context's): inputs arrive as float and are widened.

template <typename R>
__device__ __forceinline__ typename CT<R>::C unit_or_zero(const typename CT<R>::C f, R* mag) {
  const R m = hypot_r(f.x, f.y);
  *mag = m;
  return m != R(0) ? mk(f.x / m, f.y / m) : mk(R(0), R(0));
}

template <typename R>
__device__ __forceinline__ R row_bp(const CohArgs& a, int64_t s, int c) {
  return a.bp_row_inv ? static_cast<R>(a.bp[c]) : static_cast<R>(a.bp[s * a.M + c]);
}

template <typename R>
__device__ __forceinline__ typename CT<R>::C load_ph(const CohArgs& a, int64_t s, int c) {
  const float2 v = a.ph[s * a.M + c];
  return mk(static_cast<R>(v.x), static_cast<R>(v.y));
}

// S = sum_c conj(p_c) ph_c e^{-j K bp_c} and D = sum_c |conj(p_c) ph_c| of one PS (whole warp)
template <typename R>
__device__ __forceinline__ void coh_sums(const CohArgs& a, int64_t s, int lane, R* sx_o, R* sy_o, R* d_o) {
  using C = typename CT<R>::C;
  const C* __restrict__ filt = static_cast<const C*>(a.filt);
  const int64_t cell = a.cell_of[s];
  const R k = static_cast<const R*>(a.K)[s];
  R sx = R(0), sy = R(0), d = R(0);
  for (int c = lane; c < a.M; c += 32) {
    R mag;
    const C pp = unit_or_zero<R>(filt[cell * a.Mp + c], &mag);
    const C z = cmul(mk(pp.x, -pp.y), load_ph<R>(a, s, c));
    R sn, cs;
    sincos_r(k * row_bp<R>(a, s, c), &sn, &cs);
    const C r = cmul(z, mk(cs, -sn));
    sx += r.x;
    sy += r.y;
    d += hypot_r(z.x, z.y);
  }
  *sx_o = warp_sum(sx);
  *sy_o = warp_sum(sy);
  *d_o = warp_sum(d);
}

template <typename R>
__global__ void __launch_bounds__(256) k_coh_fwd(CohArgs a) {
  const int lane = threadIdx.x & 31;
  const int64_t gw = (static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x) >> 5;
  const int64_t nw = (static_cast<int64_t>(gridDim.x) * blockDim.x) >> 5;
  for (int64_t s = gw; s < a.N; s += nw) {
    R sx, sy, d;
    coh_sums<R>(a, s, lane, &sx, &sy, &d);
    if (lane == 0) a.coh[s] = static_cast<float>(hypot_r(sx, sy) / (d != R(0) ? d : R(1)));
  }
}

template <typename R>
__global__ void __launch_bounds__(256) k_coh_bwd(CohArgs a) {
  using C = typename CT<R>::C;
  const int lane = threadIdx.x & 31;
  const int64_t gw = (static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x) >> 5;
  const int64_t nw = (static_cast<int64_t>(gridDim.x) * blockDim.x) >> 5;
  const C* __restrict__ filt = static_cast<const C*>(a.filt);
  C* __restrict__ gph = static_cast<C*>(a.gph);
  C* __restrict__ gf_out = static_cast<C*>(a.gf);
  for (int64_t s = gw; s < a.N; s += nw) {
    R sx, sy, d;
    coh_sums<R>(a, s, lane, &sx, &sy, &d);
    const int64_t cell = a.cell_of[s];
    const R k = static_cast<const R*>(a.K)[s];
    const R dd = d != R(0) ? d : R(1);
    const R sm = hypot_r(sx, sy);
    const R g = static_cast<R>(a.gcoh[s]);
    const R gam = sm / dd;
    // d gamma / d S = S / (|S| D); d gamma / d |z_c| = -gamma / D
    const C gS = sm > R(0) ? mk(g * sx / (sm * dd), g * sy / (sm * dd)) : mk(R(0), R(0));
    const R gD = -g * gam / dd;
    R gk = R(0);
    for (int c = lane; c < a.M; c += 32) {
      R mag;
      const C pp = unit_or_zero<R>(filt[cell * a.Mp + c], &mag);
      const C h = load_ph<R>(a, s, c);
      const C z = cmul(mk(pp.x, -pp.y), h);
      const R b = row_bp<R>(a, s, c);
      R sn, cs;
      sincos_r(k * b, &sn, &cs);
      const C e = mk(cs, -sn);
      const C r = cmul(z, e);
      // r = z e:  g_z = conj(e) g_S (+ the denominator term);  dr/dK = -j bp r
      C gz = cmul(mk(e.x, -e.y), gS);
      const R zm = hypot_r(z.x, z.y);
      if (zm > R(0)) {
        gz.x += gD * z.x / zm;
        gz.y += gD * z.y / zm;
      }
      gk += gS.x * (b * r.y) + gS.y * (-b * r.x);
      // z = conj(p) h:  g_h = p g_z,  g_p = conj(g_z) h
      gph[s * a.M + c] = cmul(pp, gz);
      const C gp = cmul(mk(gz.x, -gz.y), h);
      // p = f / |f|:  g_f = (g_p - p Re(conj(p) g_p)) / |f|
      C gf = mk(R(0), R(0));
      if (mag > R(0)) {
        const R rp = pp.x * gp.x + pp.y * gp.y;
        gf = mk((gp.x - pp.x * rp) / mag, (gp.y - pp.y * rp) / mag);
      }
      gf_out[s * a.M + c] = gf;
    }
    gk = warp_sum(gk);
    if (lane == 0) static_cast<R*>(a.gK)[s] = gk;
  }
}

// bin backward: grid[cell, c] += a ph with a = e^{-j K bp} w
template <typename R>
__global__ void __launch_bounds__(256) k_bin_bwd(CohArgs a) {
  using C = typename CT<R>::C;
  const int lane = threadIdx.x & 31;
  const int64_t gw = (static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x) >> 5;
  const int64_t nw = (static_cast<int64_t>(gridDim.x) * blockDim.x) >> 5;
  const C* __restrict__ ggrid = static_cast<const C*>(a.ggrid);
  C* __restrict__ gph = static_cast<C*>(a.gph);
  for (int64_t s = gw; s < a.N; s += nw) {
    const int64_t cell = a.cell_of[s];
    const R k = static_cast<const R*>(a.K)[s], w = static_cast<const R*>(a.w)[s];
    R gk = R(0);
    for (int c = lane; c < a.M; c += 32) {
      const R b = row_bp<R>(a, s, c);
      R sn, cs;
      sincos_r(-(b * k), &sn, &cs);
      const C co = mk(cs * w, sn * w);
      const C gg = ggrid[cell * a.Mp + c];
      const C gh = cmul(mk(co.x, -co.y), gg);
      const C prev = gph[s * a.M + c];
      gph[s * a.M + c] = mk(prev.x + gh.x, prev.y + gh.y);
      const C v = cmul(co, load_ph<R>(a, s, c));  // d(a h)/dK = -j bp a h
      gk += gg.x * (b * v.y) + gg.y * (-b * v.x);
    }
    gk = warp_sum(gk);
    if (lane == 0) static_cast<R*>(a.gK)[s] += gk;
  }
}

// per-cell sum of complex rows [N, M] in cell order (rows of one cell are
// contiguous), sequential in row order: d L / d filt from d L / d p_c
template <typename R>
__global__ void __launch_bounds__(256) k_cell_sum(CohArgs a, const int32_t* __restrict__ cell_start, int64_t G,
                                                  int nchunk, void* out_v) {
  using C = typename CT<R>::C;
  const C* __restrict__ src = static_cast<const C*>(a.gf);
  C* __restrict__ out = static_cast<C*>(out_v);
  const int lane = threadIdx.x & 31;
  const int64_t gw = (static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x) >> 5;
  const int64_t nw = (static_cast<int64_t>(gridDim.x) * blockDim.x) >> 5;
  for (int64_t task = gw; task < G * nchunk; task += nw) {
    const int64_t cell = task / nchunk;
    const int c = static_cast<int>(task - cell * nchunk) * 32 + lane;
    R ax = R(0), ay = R(0);
    if (c < a.M) {
      for (int s = cell_start[cell]; s < cell_start[cell + 1]; ++s) {
        const C v = src[static_cast<int64_t>(s) * a.M + c];
        ax += v.x;
        ay += v.y;
      }
    }
    if (c < a.Mp) out[cell * a.Mp + c] = mk(ax, ay);
  }
}

template <typename R>
static cudaError_t coh_launch(const CohArgs& a, int which, int sm_count, cudaStream_t st) {
  int64_t blocks = (a.N + 7) / 8;
  if (blocks > static_cast<int64_t>(sm_count) * 16) blocks = static_cast<int64_t>(sm_count) * 16;
  if (blocks < 1) blocks = 1;
  if (which == 0)
    k_coh_fwd<R><<<static_cast<unsigned>(blocks), 256, 0, st>>>(a);
  else if (which == 1)
    k_coh_bwd<R><<<static_cast<unsigned>(blocks), 256, 0, st>>>(a);
  else
    k_bin_bwd<R><<<static_cast<unsigned>(blocks), 256, 0, st>>>(a);
  return cudaGetLastError();
}

cudaError_t launch_coh(const CohArgs& a, int which, bool fp64, int sm_count, cudaStream_t st) {
  return fp64 ? coh_launch<double>(a, which, sm_count, st) : coh_launch<float>(a, which, sm_count, st);
}

cudaError_t launch_cell_sum(const CohArgs& a, const int32_t* cell_start, int64_t G, void* out, bool fp64,
                            int sm_count, cudaStream_t st) {
  const int nchunk = (a.M + 31) / 32;
  int64_t blocks = (G * nchunk + 7) / 8;
  if (blocks > static_cast<int64_t>(sm_count) * 16) blocks = static_cast<int64_t>(sm_count) * 16;
  if (blocks < 1) blocks = 1;
  if (fp64)
    k_cell_sum<double><<<static_cast<unsigned>(blocks), 256, 0, st>>>(a, cell_start, G, nchunk, out);
  else
    k_cell_sum<float><<<static_cast<unsigned>(blocks), 256, 0, st>>>(a, cell_start, G, nchunk, out);
  return cudaGetLastError();
}

template <typename R>
struct ClapBwdTile {
  R re[32][33];
  R im[32][33];
  R hs[32][33];
  R gre[32][33];
  R gim[32][33];
  R pad[8];
};

template <typename R>
__global__ void __launch_bounds__(128) k_clap_bwd(ClapBwdArgs b, typename CT<R>::Tw tw) {
  using C = typename CT<R>::C;
  const ClapArgs& a = b.f;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  ClapBwdTile<R>* tiles = reinterpret_cast<ClapBwdTile<R>*>(smem_raw);
  R* lp = reinterpret_cast<R*>(tiles + 4);
  R* wt = lp + 1024;
  C* twf = reinterpret_cast<C*>(wt + 1024);
  C* twi = twf + 16;
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const int nw = a.n_win, nw2 = nw * nw;
  for (int i = tid; i < 1024; i += 128) lp[i] = static_cast<R>(a.low_pass[i]);
  for (int i = tid; i < nw2; i += 128) wt[i] = static_cast<R>(a.wscaled[i]);
  if (tid < 16) {
    twf[tid] = tw.w[tid];
    twi[tid] = mk(tw.w[tid].x, -tw.w[tid].y);
  }
  R g7[7];
#pragma unroll
  for (int i = 0; i < 7; ++i) g7[i] = static_cast<R>(a.g7[i]);
  const int n_inc = nw / 4 > 1 ? nw / 4 : 1;
  const int ngroups = a.Mp / 4;
  const int64_t ntask = static_cast<int64_t>(a.nwi) * a.nwj * ngroups;
  const C* __restrict__ grid = static_cast<const C*>(a.grid);
  const C* __restrict__ gfilt = static_cast<const C*>(b.gfilt);
  C* __restrict__ wgrad = static_cast<C*>(b.wgrad);
  ClapBwdTile<R>& T = tiles[warp];
  const R alpha = static_cast<R>(a.alpha), beta = static_cast<R>(a.beta);
  double ga_acc = 0.0, gb_acc = 0.0;
  for (int64_t task = blockIdx.x; task < ntask; task += gridDim.x) {
    const int64_t wi = task / ngroups;
    const int g = static_cast<int>(task - wi * ngroups);
    const int ix1 = static_cast<int>(wi / a.nwj), ix2 = static_cast<int>(wi - static_cast<int64_t>(ix1) * a.nwj);
    int i1 = ix1 * n_inc, rs = 0;
    if (i1 + nw > a.n_i) {
      rs = i1 + nw - a.n_i;
      i1 = a.n_i - nw;
    }
    int j1 = ix2 * n_inc, cs = 0;
    if (j1 + nw > a.n_j) {
      cs = j1 + nw - a.n_j;
      j1 = a.n_j - nw;
    }
    __syncthreads();
    for (int idx = tid; idx < 4 * 32 * 32; idx += 128) {
      const int q = idx >> 10, e = idx & 1023, r = e >> 5, cc = e & 31;
      if (r >= nw || cc >= nw) {
        tiles[q].re[r][cc] = R(0);
        tiles[q].im[r][cc] = R(0);
        tiles[q].gre[r][cc] = R(0);
        tiles[q].gim[r][cc] = R(0);
      }
    }
    for (int idx = tid; idx < nw2 * 4; idx += 128) {
      const int pix = idx >> 2, q = idx & 3;
      const int li = pix / nw, lj = pix - li * nw;
      const int c = 4 * g + q;
      C v = mk(R(0), R(0)), gy = mk(R(0), R(0));
      if (c < a.M) {
        const int64_t cell = static_cast<int64_t>(i1 + li) * a.n_j + (j1 + lj);
        v = grid[cell * a.Mp + c];
        if (isnan(v.x) || isnan(v.y)) v = mk(R(0), R(0));
        const R wv = (li < rs || lj < cs) ? R(0) : wt[(li - rs) * nw + (lj - cs)];
        const C go = gfilt[cell * a.Mp + c];
        gy = mk(go.x * wv, go.y * wv);  // out += w y  =>  g_y = w g_out
      }
      tiles[q].re[li][lj] = v.x;
      tiles[q].im[li][lj] = v.y;
      tiles[q].gre[li][lj] = gy.x;
      tiles[q].gim[li][lj] = gy.y;
    }
    __syncthreads();
    if (4 * g + warp < a.M) {
      // recompute the forward spectrum X = FFT2(x) and the smoothed magnitude
      if (lane < nw) fft_pass<R>(T.re, T.im, twf, lane, true);
      __syncwarp();
      fft_pass<R>(T.re, T.im, twf, lane, false);
#pragma unroll
      for (int k = 0; k < 32; ++k) {
        const R xr = T.re[k][lane], xi = T.im[k][lane];
        T.hs[k][lane] = sqrt(xr * xr + xi * xi);
      }
      __syncwarp();
      R t[32];
      const int sj = (lane + 16) & 31;
#pragma unroll
      for (int k = 0; k < 32; ++k) {
        R acc = R(0);
#pragma unroll
        for (int d = -3; d <= 3; ++d)
          if (sj + d >= 0 && sj + d < 32) acc += T.hs[k][(lane + d) & 31] * g7[d + 3];
        t[k] = acc;
      }
      R o[32];
#pragma unroll
      for (int k = 0; k < 32; ++k) {
        const int sk = (k + 16) & 31;
        R acc = R(0);
#pragma unroll
        for (int d = -3; d <= 3; ++d)
          if (sk + d >= 0 && sk + d < 32) acc += t[(k + d) & 31] * g7[d + 3];
        o[k] = acc;
      }
      R v0, v1;
      const R med = warp_median1024_pair<R>(o, &T.hs[0][0], v0, v1);
      // g_Y = FFT2(g_y) (adjoint of the unnormalised inverse FFT)
      if (lane < nw) fft_pass<R>(T.gre, T.gim, twf, lane, true);
      __syncwarp();
      fft_pass<R>(T.gre, T.gim, twf, lane, false);
      const R inv_med = med != R(0) ? R(1) / med : R(1);
      R gmed = R(0), ga = R(0), gb = R(0);
      // t becomes dL/d(smoothed |X|), starting with the direct term
#pragma unroll
      for (int k = 0; k < 32; ++k) {
        const R xr = T.re[k][lane], xi = T.im[k][lane];
        const R gyr = T.gre[k][lane], gyi = T.gim[k][lane];
        const R hn = o[k] * inv_med;
        const R pw = a.alpha_is_one ? hn : pow(hn, alpha);
        const bool act = pw - R(1) > R(0);
        const R G = (act ? pw - R(1) : R(0)) * beta + lp[k * 32 + lane];
        const R gG = xr * gyr + xi * gyi;
        R ghn = R(0);
        if (act) {
          ghn = gG * beta * (a.alpha_is_one ? R(1) : alpha * pow(hn, alpha - R(1)));
          gb += gG * (pw - R(1));
          ga += gG * beta * pw * log(hn);
        }
        if (med != R(0)) gmed += ghn * (-o[k] * inv_med * inv_med);
        t[k] = med != R(0) ? ghn * inv_med : ghn;
        T.gre[k][lane] = gyr * G;  // g_X from Y = X G
        T.gim[k][lane] = gyi * G;
      }
      gmed = warp_sum(gmed);
      ga = warp_sum(ga);
      gb = warp_sum(gb);
      if (med != R(0)) {
        // med = (v0 + v1) / 2 of the smoothed magnitudes; ties share evenly
        int c0 = 0, c1 = 0;
#pragma unroll
        for (int k = 0; k < 32; ++k) {
          c0 += o[k] == v0 ? 1 : 0;
          c1 += o[k] == v1 ? 1 : 0;
        }
        c0 = warp_sum(c0);
        c1 = warp_sum(c1);
        const R share0 = v0 == v1 ? gmed / static_cast<R>(c0) : R(0.5) * gmed / static_cast<R>(c0);
        const R share1 = v0 == v1 ? R(0) : R(0.5) * gmed / static_cast<R>(c1);
#pragma unroll
        for (int k = 0; k < 32; ++k) {
          if (o[k] == v0)
            t[k] += share0;
          else if (o[k] == v1)
            t[k] += share1;
        }
      }
      // adjoint of the separable smoothing: along k in registers, then across lanes
#pragma unroll
      for (int k = 0; k < 32; ++k) {
        const int sk = (k + 16) & 31;
        R acc = R(0);
#pragma unroll
        for (int d = -3; d <= 3; ++d)
          if (sk + d >= 0 && sk + d < 32) acc += t[(k + d) & 31] * g7[d + 3];
        o[k] = acc;
      }
      __syncwarp();
#pragma unroll
      for (int k = 0; k < 32; ++k) T.hs[k][lane] = o[k];
      __syncwarp();
#pragma unroll
      for (int k = 0; k < 32; ++k) {
        R acc = R(0);
#pragma unroll
        for (int d = -3; d <= 3; ++d)
          if (sj + d >= 0 && sj + d < 32) acc += T.hs[k][(lane + d) & 31] * g7[d + 3];
        // H = |X|:  g_X += g_H X / |X|
        const R xr = T.re[k][lane], xi = T.im[k][lane];
        const R xm = sqrt(xr * xr + xi * xi);
        if (xm > R(0)) {
          T.gre[k][lane] += acc * xr / xm;
          T.gim[k][lane] += acc * xi / xm;
        }
      }
      // g_x = IFFT2_unnormalised(g_X) (adjoint of the forward FFT)
      __syncwarp();
      fft_pass<R>(T.gre, T.gim, twi, lane, false);
      __syncwarp();
      if (lane < nw) fft_pass<R>(T.gre, T.gim, twi, lane, true);
      __syncwarp();
      if (lane == 0) {
        ga_acc += static_cast<double>(ga);
        gb_acc += static_cast<double>(gb);
      }
    }
    __syncthreads();
    for (int idx = tid; idx < nw2 * 4; idx += 128) {
      const int pix = idx >> 2, q = idx & 3;
      const int li = pix / nw, lj = pix - li * nw;
      const int c = 4 * g + q;
      C v = mk(tiles[q].gre[li][lj], tiles[q].gim[li][lj]);
      if (c < a.M) {
        const C x = grid[(static_cast<int64_t>(i1 + li) * a.n_j + (j1 + lj)) * a.Mp + c];
        if (isnan(x.x) || isnan(x.y)) v = mk(R(0), R(0));  // NaN inputs enter as constants
      } else {
        v = mk(R(0), R(0));
      }
      wgrad[(wi * nw2 + pix) * a.Mp + 4 * g + q] = v;
    }
  }
  __shared__ double sh_ab[8];
  if (lane == 0) {
    sh_ab[2 * warp] = ga_acc;
    sh_ab[2 * warp + 1] = gb_acc;
  }
  __syncthreads();
  if (tid == 0) {
    b.ab_partial[2 * blockIdx.x] = sh_ab[0] + sh_ab[2] + sh_ab[4] + sh_ab[6];
    b.ab_partial[2 * blockIdx.x + 1] = sh_ab[1] + sh_ab[3] + sh_ab[5] + sh_ab[7];
  }
}

// d L / d alpha and d L / d beta: the per-block partials summed in a fixed order
__global__ void __launch_bounds__(256) k_reduce_ab(const double* __restrict__ part, int n, double* __restrict__ out) {
  __shared__ double sh[2][256];
  const int t = threadIdx.x;
  double a = 0.0, b = 0.0;
  for (int i = t; i < n; i += 256) {
    a += part[2 * i];
    b += part[2 * i + 1];
  }
  sh[0][t] = a;
  sh[1][t] = b;
  __syncthreads();
  for (int h = 128; h > 0; h >>= 1) {
    if (t < h) {
      sh[0][t] += sh[0][t + h];
      sh[1][t] += sh[1][t + h];
    }
    __syncthreads();
  }
  if (t == 0) {
    out[0] = sh[0][0];
    out[1] = sh[1][0];
  }
}

cudaError_t launch_reduce_ab(const double* part, int n, double* out, cudaStream_t st) {
  k_reduce_ab<<<1, 256, 0, st>>>(part, n, out);
  return cudaGetLastError();
}

template <typename R>
static size_t clap_bwd_smem() {
  return 4 * sizeof(ClapBwdTile<R>) + 2048 * sizeof(R) + 32 * sizeof(typename CT<R>::C);
}

template <typename R>
static int clap_bwd_blocks(int sm_count) {
  const size_t sm = clap_bwd_smem<R>();
  if (kernel_attributes_once(sm) != cudaSuccess) return 0;
  int per_sm = 0;
  if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_clap_bwd<R>, 128, sm) != cudaSuccess) return 0;
  return sm_count * std::max(per_sm, 1);
}

// Resident blocks of k_clap_bwd on the whole device (the size of the
// alpha/beta partial array); 0 on error.
int clap_bwd_max_blocks(int sm_count, bool fp64) {
  return fp64 ? clap_bwd_blocks<double>(sm_count) : clap_bwd_blocks<float>(sm_count);
}

// Launches at most *blocks_out blocks (the partial array's capacity) and
// returns the number launched (0 when there are no windows).
cudaError_t launch_clap_bwd(const ClapBwdArgs& b, bool fp64, const Twiddles32f& tf, const Twiddles32d& td,
                            int* blocks_out, cudaStream_t st) {
  const int64_t ntask = static_cast<int64_t>(b.f.nwi) * b.f.nwj * (b.f.Mp / 4);
  const int64_t blocks = std::min<int64_t>(ntask, static_cast<int64_t>(*blocks_out));
  *blocks_out = static_cast<int>(std::max<int64_t>(blocks, 0));
  if (blocks <= 0) return cudaSuccess;
  if (fp64)
    k_clap_bwd<double><<<static_cast<unsigned>(blocks), 128, clap_bwd_smem<double>(), st>>>(b, td);
  else
    k_clap_bwd<float><<<static_cast<unsigned>(blocks), 128, clap_bwd_smem<float>(), st>>>(b, tf);
  return cudaGetLastError();
}

// dst[s] = double(src[perm[s]])
__global__ void k_gather_widen(const float* __restrict__ src, double* __restrict__ dst,
                               const int32_t* __restrict__ perm, int64_t n) {
  for (int64_t s = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x; s < n;
       s += static_cast<int64_t>(gridDim.x) * blockDim.x)
    dst[s] = static_cast<double>(src[perm[s]]);
}

// dst[perm[s] * words + k] = float(src[s * words + k])
__global__ void k_scatter_narrow(const double* __restrict__ src, float* __restrict__ dst,
                                 const int32_t* __restrict__ perm, int64_t n, int64_t words) {
  const int lane = threadIdx.x & 31;
  const int64_t gw = (static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x) >> 5;
  const int64_t nw = (static_cast<int64_t>(gridDim.x) * blockDim.x) >> 5;
  for (int64_t s = gw; s < n; s += nw) {
    const int64_t r = perm[s];
    for (int64_t k = lane; k < words; k += 32) dst[r * words + k] = static_cast<float>(src[s * words + k]);
  }
}

// dst[perm[s]] = double(src[s]): a per-PS vector back in the caller's row
// order, widened on the device (u8 flags as 0.0 / 1.0)
__device__ __forceinline__ double widen_elem(const float* p, int64_t s) { return static_cast<double>(p[s]); }
__device__ __forceinline__ double widen_elem(const uint8_t* p, int64_t s) { return p[s] ? 1.0 : 0.0; }
template <typename T>
__global__ void k_scatter_widen(const T* __restrict__ src, double* __restrict__ dst, const int32_t* __restrict__ perm,
                                int64_t n) {
  for (int64_t s = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x; s < n;
       s += static_cast<int64_t>(gridDim.x) * blockDim.x)
    dst[perm[s]] = widen_elem(src, s);
}

cudaError_t launch_scatter_widen(const void* src, bool flags, double* dst, const int32_t* perm, int64_t n,
                                 cudaStream_t st) {
  if (n <= 0) return cudaSuccess;
  const int64_t blocks = std::min<int64_t>((n + 255) / 256, 148 * 16);
  if (flags)
    k_scatter_widen<uint8_t><<<static_cast<unsigned>(blocks), 256, 0, st>>>(static_cast<const uint8_t*>(src), dst,
                                                                             perm, n);
  else
    k_scatter_widen<float><<<static_cast<unsigned>(blocks), 256, 0, st>>>(static_cast<const float*>(src), dst, perm,
                                                                           n);
  return cudaGetLastError();
}

cudaError_t launch_gather_widen(const float* src, double* dst, const int32_t* perm, int64_t n, cudaStream_t st) {
  if (n <= 0) return cudaSuccess;
  const int64_t blocks = std::min<int64_t>((n + 255) / 256, 148 * 16);
  k_gather_widen<<<static_cast<unsigned>(blocks), 256, 0, st>>>(src, dst, perm, n);
  return cudaGetLastError();
}

cudaError_t launch_scatter_narrow(const double* src, float* dst, const int32_t* perm, int64_t n, int64_t words,
                                  cudaStream_t st) {
  if (n <= 0) return cudaSuccess;
  const int64_t blocks = std::min<int64_t>((n + 7) / 8, 148 * 16);
  k_scatter_narrow<<<static_cast<unsigned>(blocks), 256, 0, st>>>(src, dst, perm, n, words);
  return cudaGetLastError();
}

// ============================================================== layout ====
// Row gathers/scatters in 4-byte words (row_bytes is a multiple of 4).
__global__ void k_gather_rows(const uint32_t* __restrict__ src, uint32_t* __restrict__ dst,
                              const int32_t* __restrict__ perm, int64_t n, int64_t words, int scatter) {
  const int lane = threadIdx.x & 31;
  const int64_t gw = (static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x) >> 5;
  const int64_t nw = (static_cast<int64_t>(gridDim.x) * blockDim.x) >> 5;
  for (int64_t s = gw; s < n; s += nw) {
    const int64_t r = perm[s];
    const uint32_t* a = scatter ? src + s * words : src + r * words;
    uint32_t* b = scatter ? dst + r * words : dst + s * words;
    for (int64_t k = lane; k < words; k += 32) b[k] = a[k];
  }
}

static cudaError_t gather_impl(const void* src, void* dst, const int32_t* perm, int64_t n, int64_t row_bytes,
                               int scatter, cudaStream_t st) {
  if (n <= 0) return cudaSuccess;
  if (row_bytes % 4) return cudaErrorInvalidValue;
  int64_t blocks = (n + 7) / 8;
  if (blocks > 148 * 16) blocks = 148 * 16;
  k_gather_rows<<<static_cast<unsigned>(blocks), 256, 0, st>>>(static_cast<const uint32_t*>(src),
                                                               static_cast<uint32_t*>(dst), perm, n, row_bytes / 4,
                                                               scatter);
  return cudaGetLastError();
}

cudaError_t launch_gather_rows(const void* src, void* dst, const int32_t* perm, int64_t n, int64_t row_bytes,
                               cudaStream_t st) {
  return gather_impl(src, dst, perm, n, row_bytes, 0, st);
}
cudaError_t launch_scatter_rows(const void* src, void* dst, const int32_t* perm, int64_t n, int64_t row_bytes,
                                cudaStream_t st) {
  return gather_impl(src, dst, perm, n, row_bytes, 1, st);
}

__global__ void k_repad(const uint8_t* __restrict__ src, uint8_t* __restrict__ dst, int64_t G, int M, int Mp, int eb,
                        int to_padded) {
  const int64_t total = G * static_cast<int64_t>(to_padded ? Mp : M) * eb;
  for (int64_t i = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x; i < total;
       i += static_cast<int64_t>(gridDim.x) * blockDim.x) {
    const int64_t e = i / eb, byte = i - e * eb;
    if (to_padded) {
      const int64_t g = e / Mp, c = e - g * Mp;
      dst[i] = c < M ? src[(g * M + c) * eb + byte] : 0;
    } else {
      const int64_t g = e / M, c = e - g * M;
      dst[i] = src[(g * Mp + c) * eb + byte];
    }
  }
}

cudaError_t launch_unpad_grid(const void* src, void* dst, int64_t G, int M, int Mp, int eb, cudaStream_t st) {
  k_repad<<<148 * 8, 256, 0, st>>>(static_cast<const uint8_t*>(src), static_cast<uint8_t*>(dst), G, M, Mp, eb, 0);
  return cudaGetLastError();
}
cudaError_t launch_pad_grid(const void* src, void* dst, int64_t G, int M, int Mp, int eb, cudaStream_t st) {
  k_repad<<<148 * 8, 256, 0, st>>>(static_cast<const uint8_t*>(src), static_cast<uint8_t*>(dst), G, M, Mp, eb, 1);
  return cudaGetLastError();
}

template <typename R>
__global__ void k_init_state(const double* __restrict__ w0, const int32_t* __restrict__ perm, int64_t N, R* K, R* w,
                             R* coh) {
  for (int64_t s = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x; s < N;
       s += static_cast<int64_t>(gridDim.x) * blockDim.x) {
    K[s] = R(0);
    w[s] = static_cast<R>(w0[perm[s]]);
    coh[s] = R(0);
  }
}

cudaError_t launch_init_state(const double* w0, const int32_t* perm, int64_t N, void* K, void* w, void* coh,
                              bool fp64, cudaStream_t st) {
  if (fp64)
    k_init_state<double><<<148 * 4, 256, 0, st>>>(w0, perm, N, static_cast<double*>(K), static_cast<double*>(w),
                                                  static_cast<double*>(coh));
  else
    k_init_state<float><<<148 * 4, 256, 0, st>>>(w0, perm, N, static_cast<float*>(K), static_cast<float*>(w),
                                                 static_cast<float*>(coh));
  return cudaGetLastError();
}

// ph_weight of the last iteration (fill_phase_weight with the K and w that
// iteration used), written in the caller's row order.
template <typename R>
__global__ void k_ph_weight(BinArgs a, const int32_t* __restrict__ perm, int64_t N,
                            typename CT<R>::C* __restrict__ out) {
  using C = typename CT<R>::C;
  const float2* ph = static_cast<const float2*>(a.ph_nm);
  const R* K = static_cast<const R*>(a.K);
  const R* W = static_cast<const R*>(a.w);
  const int64_t total = N * a.M;
  for (int64_t i = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x; i < total;
       i += static_cast<int64_t>(gridDim.x) * blockDim.x) {
    const int64_t s = i / a.M;
    const int c = static_cast<int>(i - s * a.M);
    const R b = a.bp_row_inv ? static_cast<R>(a.bp[c]) : static_cast<R>(a.bp[i]);
    const R phs = -(b * K[s]);
    R sn, cs;
    sincos_r(phs, &sn, &cs);
    const float2 v = ph[i];
    const C r = cmul_rn(mk(static_cast<R>(v.x), static_cast<R>(v.y)), mk(cs, sn));
    out[static_cast<int64_t>(perm[s]) * a.M + c] = mk(mul_rn(r.x, W[s]), mul_rn(r.y, W[s]));
  }
}

cudaError_t launch_ph_weight(const BinArgs& a, int64_t N, bool fp64, const int32_t* perm, void* out_orig,
                             cudaStream_t st) {
  if (fp64)
    k_ph_weight<double><<<148 * 8, 256, 0, st>>>(a, perm, N, static_cast<double2*>(out_orig));
  else
    k_ph_weight<float><<<148 * 8, 256, 0, st>>>(a, perm, N, static_cast<float2*>(out_orig));
  return cudaGetLastError();
}


// ====================================================== kernel attributes ==
// Every kernel that may take more than 48 KB of dynamic shared memory is opted
// in to the device's per-block maximum once per device and process, before its
// first launch; a launch then only checks its request against that limit.
// Kernel attributes are thereby never changed while another host thread
// captures, instantiates or launches a graph that holds the same kernel
// (contexts run concurrently from several threads).
namespace {
template <typename F>
cudaError_t opt_in_smem(F* f, int optin) {
  cudaFuncAttributes fa;
  cudaError_t e = cudaFuncGetAttributes(&fa, f);
  if (e != cudaSuccess) return e;
  return cudaFuncSetAttribute(f, cudaFuncAttributeMaxDynamicSharedMemorySize,
                              optin - static_cast<int>(fa.sharedSizeBytes));
}

constexpr int kMaxDevices = 64;
std::once_flag g_attr_once[kMaxDevices];
cudaError_t g_attr_result[kMaxDevices];
int g_attr_optin[kMaxDevices];
}  // namespace

cudaError_t kernel_attributes_once(size_t dynamic_smem) {
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return e;
  if (dev < 0 || dev >= kMaxDevices) return cudaErrorInvalidDevice;
  std::call_once(g_attr_once[dev], [dev] {
    int optin = 0;
    const cudaError_t r = cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev);
    const cudaError_t steps[] = {
        r,
        r == cudaSuccess ? opt_in_smem(k_clap<float, 8, 0, false>, optin) : r,
        r == cudaSuccess ? opt_in_smem(k_clap<double, 4, 0, false>, optin) : r,
        r == cudaSuccess ? opt_in_smem(k_clap<float, 8, 24, false>, optin) : r,
        r == cudaSuccess ? opt_in_smem(k_clap<float, 4, 0, false>, optin) : r,
        r == cudaSuccess ? opt_in_smem(k_clap<float, 4, 24, false>, optin) : r,
        r == cudaSuccess ? opt_in_smem(k_clap<double, 4, 24, false>, optin) : r,
        r == cudaSuccess ? opt_in_smem(k_clap<float, 8, 0, true>, optin) : r,
        r == cudaSuccess ? opt_in_smem(k_clap<double, 4, 0, true>, optin) : r,
        r == cudaSuccess ? opt_in_smem(k_clap<float, 8, 24, true>, optin) : r,
        r == cudaSuccess ? opt_in_smem(k_clap<float, 4, 0, true>, optin) : r,
        r == cudaSuccess ? opt_in_smem(k_clap<float, 4, 24, true>, optin) : r,
        r == cudaSuccess ? opt_in_smem(k_clap<double, 4, 24, true>, optin) : r,
        r == cudaSuccess ? opt_in_smem(k_topofit_f32<4>, optin) : r,
        r == cudaSuccess ? opt_in_smem(k_topofit_f32<8>, optin) : r,
        r == cudaSuccess ? opt_in_smem(k_topofit_f32<16>, optin) : r,
        r == cudaSuccess ? opt_in_smem(k_topofit_f32<32>, optin) : r,
        r == cudaSuccess ? opt_in_smem(k_topofit_f64, optin) : r,
        r == cudaSuccess ? opt_in_smem(k_random_hist, optin) : r,
        r == cudaSuccess ? opt_in_smem(k_s3_clap, optin) : r,
        r == cudaSuccess ? opt_in_smem(k_s3_fit, optin) : r,
        r == cudaSuccess ? opt_in_smem(k_topofit_near_max<float>, optin) : r,
        r == cudaSuccess ? opt_in_smem(k_topofit_near_max<double>, optin) : r,
        r == cudaSuccess ? opt_in_smem(k_batch_clap, optin) : r,
        r == cudaSuccess ? opt_in_smem(k_batch_topofit<4>, optin) : r,
        r == cudaSuccess ? opt_in_smem(k_batch_topofit<8>, optin) : r,
        r == cudaSuccess ? opt_in_smem(k_batch_topofit<16>, optin) : r,
        r == cudaSuccess ? opt_in_smem(k_batch_topofit<32>, optin) : r,
        r == cudaSuccess ? opt_in_smem(k_clap_bwd<float>, optin) : r,
        r == cudaSuccess ? opt_in_smem(k_clap_bwd<double>, optin) : r,
    };
    cudaError_t first = cudaSuccess;
    for (const cudaError_t x : steps)
      if (first == cudaSuccess && x != cudaSuccess) first = x;
    g_attr_result[dev] = first;
    g_attr_optin[dev] = optin;
  });
  if (g_attr_result[dev] != cudaSuccess) return g_attr_result[dev];
  return dynamic_smem <= static_cast<size_t>(g_attr_optin[dev]) ? cudaSuccess : cudaErrorInvalidValue;
}

}  // namespace ps2
