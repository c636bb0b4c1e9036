// ORACLE — test infrastructure only, never product code.
//
// CPU restatement of the pySTAMPS native Rust stage 2
// (crates/pystamps-core/src/native_stage2.rs), used by tests/, by
// __graft_entry__.smoke() and by bench.py's CPU-baseline leg as the checker.
// Nothing in pystamps_b200/ links or calls this file.
//
// Every routine cites the reference line range it restates. The arithmetic
// keeps the reference's precision mix: f32 phase ramps, f32 sincos, f32 complex
// sums, f64 CLAP, f64 K-refinement accumulators, f64 weighting.  Rust does not
// contract a*b+c into FMA, so this file is compiled with -ffp-contract=off, and
// Rust's f32::sin_cos / hypot / atan2 go to the platform libm, which is what
// sinf/cosf/hypotf/atan2f call here (glibc).
//
// Third-party arithmetic that is not in the reference tree:
//   * rustfft 6.4.1 (Cargo.lock) — a forward/inverse complex DFT. Restated here
//     as an iterative radix-2 decimation-in-time FFT in f64 (textbook
//     Cooley-Tukey); it agrees with rustfft to ~1e-16 relative, far below the
//     f32 cast that follows every CLAP output.
//   * num-complex 0.4.6: Complex * Complex = (ar*br - ai*bi, ar*bi + ai*br),
//     norm() = hypot(re, im), arg() = atan2(im, re).
//
// A second instantiation (Real = double) runs the same loop with every phase,
// sum and grid in f64: the "plain FP64" oracle used to state max|dgamma| and
// max|dK| of the FP32 GPU path.

#include <algorithm>
#include <atomic>
#include <chrono>
#include <cmath>
#include <complex>
#include <cstdint>
#include <cstring>
#include <functional>
#include <limits>
#include <mutex>
#include <thread>
#include <vector>

#include "interp10_taps.h"

namespace {

constexpr int kCohBins = 100;
constexpr double kCohBinStart = 0.005;
constexpr double kCohBinStep = 0.01;
constexpr uint32_t kRandomSeed = 2005;

// ---------------------------------------------------------------- threads ---
void parallel_for(int64_t n, int threads, const std::function<void(int64_t, int64_t)>& fn) {
  if (n <= 0) return;
  if (threads <= 0) {
    threads = static_cast<int>(std::thread::hardware_concurrency());
    if (threads <= 0) threads = 1;
  }
  if (threads == 1 || n < 2) {
    fn(0, n);
    return;
  }
  int64_t t = std::min<int64_t>(threads, n);
  // dynamic chunking (rayon-like work stealing granularity)
  int64_t chunk = std::max<int64_t>(1, n / (t * 8));
  std::atomic<int64_t> next(0);
  std::vector<std::thread> pool;
  pool.reserve(t);
  for (int64_t k = 0; k < t; ++k) {
    pool.emplace_back([&]() {
      for (;;) {
        int64_t b = next.fetch_add(chunk);
        if (b >= n) break;
        fn(b, std::min(n, b + chunk));
      }
    });
  }
  for (auto& th : pool) th.join();
}

// ------------------------------------------------------- complex helpers ---
template <typename R>
struct Cx {
  R re, im;
};
template <typename R>
inline Cx<R> cmul(Cx<R> a, Cx<R> b) {
  // num-complex Mul: (a.re*b.re - a.im*b.im, a.re*b.im + a.im*b.re)
  return {a.re * b.re - a.im * b.im, a.re * b.im + a.im * b.re};
}
template <typename R>
inline Cx<R> conj(Cx<R> a) { return {a.re, -a.im}; }
inline float norm(Cx<float> a) { return hypotf(a.re, a.im); }
inline double norm(Cx<double> a) { return hypot(a.re, a.im); }
inline float arg(Cx<float> a) { return atan2f(a.im, a.re); }
inline double arg(Cx<double> a) { return atan2(a.im, a.re); }
inline void sincos_r(float x, float* s, float* c) { *s = sinf(x); *c = cosf(x); }
inline void sincos_r(double x, double* s, double* c) { *s = sin(x); *c = cos(x); }

// ------------------------------------------------ MATLAB v5 uniform RNG ---
// native_stage2.rs:1785-1873
struct MatlabV5Rng {
  static constexpr double kUlp = 1.1102230246251565e-16;
  static constexpr uint64_t kMask52 = (uint64_t(1) << 52) - 1;
  int index = 0;
  double borrow = 0.0;
  uint32_t j;
  double state[32];

  static uint32_t randint32(uint32_t v) {
    v ^= v << 13;
    v ^= v >> 17;
    v ^= v << 5;
    return v;
  }
  explicit MatlabV5Rng(uint32_t seed) {
    j = seed == 0 ? (uint32_t(1) << 31) : seed;
    uint32_t jj = j;
    for (int k = 0; k < 32; ++k) {
      uint64_t x = 0;
      for (int b = 0; b < 53; ++b) {
        jj = randint32(jj);
        x = (x << 1) | ((jj >> 19) & 1u);
      }
      state[k] = static_cast<double>(x) * kUlp;
    }
  }
  static void frexp53(double v, uint64_t* mant, int* ex) {
    if (v == 0.0) { *mant = 0; *ex = 0; return; }
    uint64_t bits;
    std::memcpy(&bits, &v, 8);
    int eb = static_cast<int>((bits >> 52) & 0x7ff);
    uint64_t mb = bits & ((uint64_t(1) << 52) - 1);
    if (eb == 0) {
      int leading = 63 - __builtin_clzll(mb);
      *ex = leading - 1073;
      *mant = mb << (52 - leading);
    } else {
      *ex = eb - 1022;
      *mant = (uint64_t(1) << 52) | mb;
    }
  }
  double randbits(double v) {
    uint32_t jlo = j;
    uint32_t jhi = randint32(jlo);
    j = jhi;
    uint64_t mask = ((static_cast<uint64_t>(jhi) << 32) & kMask52) ^ static_cast<uint64_t>(jlo);
    uint64_t m;
    int e;
    frexp53(v, &m, &e);
    return std::ldexp(static_cast<double>(m ^ mask), e - 53);
  }
  double next() {
    double v = state[(index + 20) & 31] - state[(index + 5) & 31] - borrow;
    if (v < 0.0) {
      v += 1.0;
      borrow = kUlp;
    } else {
      borrow = 0.0;
    }
    state[index] = v;
    index = (index + 1) & 31;
    return randbits(v);
  }
};

// ------------------------------------------------------------ histogram ---
// native_stage2.rs:1581-1640 (equal-spacing Octave rule, else midpoint search)
bool centers_equal_spacing(const double* c, int64_t n) {
  if (n < 2) return true;
  double ref = c[1] - c[0];
  double maxc = 0.0;
  for (int64_t i = 0; i < n; ++i) maxc = std::max(maxc, std::fabs(c[i]));
  double tol = std::numeric_limits<double>::epsilon() * std::max(maxc, 1.0);
  for (int64_t i = 0; i + 1 < n; ++i)
    if (std::fabs((c[i + 1] - c[i]) - ref) > tol) return false;
  return true;
}

int64_t center_index(double v, const double* c, int64_t n, bool eq) {
  if (!std::isfinite(v) || n == 0) return -1;
  if (n == 1) return 0;
  if (eq) {
    double d = n < 3 ? 1.0 : (c[n - 1] - c[0]) / static_cast<double>(n - 1);
    if (d == 0.0) return 0;
    double cutoff0 = (c[0] + c[1]) / 2.0;
    double a = std::ceil((v - cutoff0) / d);
    a = std::min(std::max(a, 0.0), static_cast<double>(n - 1));
    return static_cast<int64_t>(a);
  }
  int64_t k = 0;
  for (int64_t i = 0; i + 1 < n; ++i) {
    double mid = (c[i] + c[i + 1]) / 2.0;
    if (mid < v) k = i + 1;
    else break;
  }
  return std::min<int64_t>(k, n - 1);
}

void hist_with_centers(const double* v, int64_t nv, const double* c, int64_t nc, double* out) {
  for (int64_t i = 0; i < nc; ++i) out[i] = 0.0;
  if (nc == 0) return;
  if (nc == 1) {
    double cnt = 0;
    for (int64_t i = 0; i < nv; ++i) if (std::isfinite(v[i])) cnt += 1.0;
    out[0] = cnt;
    return;
  }
  bool eq = centers_equal_spacing(c, nc);
  for (int64_t i = 0; i < nv; ++i) {
    int64_t ix = center_index(v[i], c, nc, eq);
    if (ix >= 0) out[ix] += 1.0;
  }
}

// --------------------------------------------------------- P-square LUT ---
// native_stage2.rs:1642-1783
std::vector<double> gausswin(int n, double alpha) {
  std::vector<double> w(n, 1.0);
  if (n <= 1 || alpha <= 0.0) return w;
  double sd = (n - 1.0) / (2.0 * alpha);
  for (int i = 0; i < n; ++i) {
    double x = i - (n - 1.0) / 2.0;
    w[i] = std::exp(-0.5 * (x / sd) * (x / sd));
  }
  return w;
}

std::vector<double> lfilter(const double* k, int nk, const std::vector<double>& v) {
  std::vector<double> out(v.size(), 0.0);
  for (size_t i = 0; i < v.size(); ++i) {
    double s = 0.0;
    for (int kk = 0; kk < nk; ++kk)
      if (static_cast<int64_t>(i) >= kk) s += k[kk] * v[i - kk];
    out[i] = s;
  }
  return out;
}

double round_half_away(double v) { return v >= 0.0 ? std::floor(v + 0.5) : std::ceil(v - 0.5); }

// prand_hi lookup table (1001 entries for 100 bins)
std::vector<double> psquare_lut(const double* nr, const double* na, int64_t nb, int64_t low_coh_thresh,
                                double nr_max_nz_ix) {
  std::vector<double> prand(nb);
  for (int64_t i = 0; i < nb; ++i) {
    double den = na[i] == 0.0 ? 1.0 : na[i];
    prand[i] = std::min(nr[i] / den, 1.0);
  }
  for (int64_t i = 0; i < std::min(low_coh_thresh, nb); ++i) prand[i] = 1.0;
  for (int64_t i = std::min<int64_t>(static_cast<int64_t>(nr_max_nz_ix), nb); i < nb; ++i) prand[i] = 0.0;
  std::vector<double> win = gausswin(7, 2.5);
  double wsum = 0.0;
  for (double x : win) wsum += x;
  std::vector<double> padded(7, 1.0);
  padded.insert(padded.end(), prand.begin(), prand.end());
  std::vector<double> filt = lfilter(win.data(), 7, padded);
  for (int64_t i = 0; i < nb; ++i) prand[i] = filt[i + 7] / wsum;
  std::vector<double> interp_in;
  interp_in.push_back(1.0);
  interp_in.insert(interp_in.end(), prand.begin(), prand.end());
  // interp_with_taps(values, 10, taps, 39), native_stage2.rs:1736-1748
  const int factor = 10, delay = 39;
  std::vector<double> expanded(interp_in.size() * factor + delay, 0.0);
  for (size_t i = 0; i < interp_in.size(); ++i) expanded[i * factor] = interp_in[i];
  std::vector<double> f2 = lfilter(kStage2Interp10Taps, 79, expanded);
  std::vector<double> hi;
  for (size_t i = 0; i < interp_in.size() * factor; ++i) hi.push_back(f2[i + delay] * factor);
  size_t keep = hi.size() >= 9 ? hi.size() - 9 : 0;
  hi.resize(keep);
  return hi;
}

void psquare_weighting(const double* nr, const double* na, int64_t nb, int64_t low_coh_thresh,
                       double nr_max_nz_ix, const double* coh, int64_t n, double* w) {
  std::vector<double> hi = psquare_lut(nr, na, nb, low_coh_thresh, nr_max_nz_ix);
  double top = hi.empty() ? 0.0 : static_cast<double>(hi.size() - 1);
  for (int64_t i = 0; i < n; ++i) {
    double ix = round_half_away(coh[i] * 1000.0);
    ix = std::min(std::max(ix, 0.0), top);  // NaN: Rust clamp keeps NaN -> as usize == 0
    size_t k = std::isnan(ix) ? 0 : static_cast<size_t>(ix);
    double p = hi[k];
    w[i] = (1.0 - p) * (1.0 - p);
  }
}

// ------------------------------------------------------------------ FFT ---
// In-place radix-2 DIT FFT of length n (power of two), f64. sign=-1 forward,
// +1 inverse (unnormalised, like rustfft).
struct Fft {
  int n;
  std::vector<int> rev;
  std::vector<std::complex<double>> tw;  // e^{-2 pi i k / n}
  explicit Fft(int n_) : n(n_), rev(n_), tw(n_ / 2) {
    int lg = 0;
    while ((1 << lg) < n) ++lg;
    for (int i = 0; i < n; ++i) {
      int r = 0;
      for (int b = 0; b < lg; ++b) if (i & (1 << b)) r |= 1 << (lg - 1 - b);
      rev[i] = r;
    }
    for (int k = 0; k < n / 2; ++k) {
      double a = -2.0 * M_PI * k / n;
      tw[k] = {std::cos(a), std::sin(a)};
    }
  }
  void run(std::complex<double>* x, int stride, bool inverse) const {
    std::vector<std::complex<double>> a(n);
    for (int i = 0; i < n; ++i) a[rev[i]] = x[i * stride];
    for (int len = 2; len <= n; len <<= 1) {
      int half = len / 2, step = n / len;
      for (int s = 0; s < n; s += len) {
        for (int k = 0; k < half; ++k) {
          std::complex<double> w = tw[k * step];
          if (inverse) w = std::conj(w);
          std::complex<double> u = a[s + k];
          std::complex<double> v = a[s + k + half] * w;
          a[s + k] = u + v;
          a[s + k + half] = u - v;
        }
      }
    }
    for (int i = 0; i < n; ++i) x[i * stride] = a[i];
  }
};

// ------------------------------------------------------------------ CLAP ---
struct ClapWindow {
  int64_t i1, j1, row_shift, col_shift;
};

// native_stage2.rs:957-995
std::vector<ClapWindow> clap_windows(int64_t n_i, int64_t n_j, int64_t n_win, int64_t n_inc, int64_t nwi,
                                     int64_t nwj) {
  std::vector<ClapWindow> w;
  for (int64_t ix1 = 0; ix1 < nwi; ++ix1) {
    int64_t i1 = ix1 * n_inc, i2 = i1 + n_win, rs = 0;
    if (i2 > n_i) { rs = i2 - n_i; i1 = n_i - n_win; }
    for (int64_t ix2 = 0; ix2 < nwj; ++ix2) {
      int64_t j1 = ix2 * n_inc, j2 = j1 + n_win, cs = 0;
      if (j2 > n_j) { cs = j2 - n_j; j1 = n_j - n_win; }
      w.push_back({i1, j1, rs, cs});
    }
  }
  return w;
}

// native_stage2.rs:1014-1037
std::vector<double> clap_window_weight(int64_t n_win) {
  int64_t h = n_win / 2;
  std::vector<double> out(n_win * n_win, 0.0);
  for (int64_t r = 0; r < h; ++r)
    for (int64_t c = 0; c < h; ++c) {
      double q = static_cast<double>(r) + static_cast<double>(c) + 1.0e-6;
      double qm = static_cast<double>(r) + static_cast<double>(h - 1 - c) + 1.0e-6;
      out[r * n_win + c] = q;
      out[r * n_win + h + c] = qm;
    }
  for (int64_t r = 0; r < h; ++r)
    for (int64_t c = 0; c < n_win; ++c) out[(h + r) * n_win + c] = out[(h - 1 - r) * n_win + c];
  return out;
}

// native_stage2.rs:1044-1053
std::vector<double> clap_kernel_1d() {
  double alpha = 2.5, sd = (7.0 - 1.0) / (2.0 * alpha);
  std::vector<double> g(7);
  for (int i = 0; i < 7; ++i) {
    double x = i - 3.0;
    g[i] = std::exp(-0.5 * (x / sd) * (x / sd));
  }
  return g;
}

// native_stage2.rs:823-922 for one ifg. Output written at stride `ostride`
// into `out` (cell-major [cell, ifg] layout) as f32 or f64.
template <typename OutR>
void clap_filter_one_ifg(const Cx<OutR>* grid, int64_t gstride, int64_t n_i, int64_t n_j, int64_t n_win,
                         int64_t n_ex, double alpha, bool alpha_is_one, double beta, const double* low_pass,
                         const std::vector<double>& kern, const std::vector<double>& wweight,
                         const std::vector<ClapWindow>& windows, Cx<OutR>* out, int64_t ostride) {
  std::vector<std::complex<double>> accum(n_i * n_j, {0.0, 0.0});
  std::vector<std::complex<double>> bit(n_ex * n_ex);
  std::vector<double> habs(n_ex * n_ex), hshift(n_ex * n_ex), tmp(n_ex * n_ex), hfilt(n_ex * n_ex),
      hmed(n_ex * n_ex);
  Fft fft(static_cast<int>(n_ex));
  double inv_scale = 1.0 / static_cast<double>(n_ex * n_ex);
  const int64_t rad = 3;
  for (const ClapWindow& w : windows) {
    std::fill(bit.begin(), bit.end(), std::complex<double>(0.0, 0.0));
    for (int64_t li = 0; li < n_win; ++li)
      for (int64_t lj = 0; lj < n_win; ++lj) {
        Cx<OutR> v = grid[((w.i1 + li) * n_j + (w.j1 + lj)) * gstride];
        bit[li * n_ex + lj] = (std::isnan(v.re) || std::isnan(v.im))
                                  ? std::complex<double>(0.0, 0.0)
                                  : std::complex<double>(static_cast<double>(v.re), static_cast<double>(v.im));
      }
    // fft2: rows then columns (native_stage2.rs:1055-1074)
    for (int64_t r = 0; r < n_ex; ++r) fft.run(&bit[r * n_ex], 1, false);
    for (int64_t c = 0; c < n_ex; ++c) fft.run(&bit[c], static_cast<int>(n_ex), false);
    for (int64_t k = 0; k < n_ex * n_ex; ++k) habs[k] = hypot(bit[k].real(), bit[k].imag());
    // fftshift (rows/2, cols/2)
    int64_t sh = n_ex / 2, ish = (n_ex + 1) / 2;
    for (int64_t r = 0; r < n_ex; ++r)
      for (int64_t c = 0; c < n_ex; ++c) hshift[r * n_ex + c] = habs[((r + sh) % n_ex) * n_ex + (c + sh) % n_ex];
    // separable 'same' convolution (native_stage2.rs:1122-1166)
    for (int64_t r = 0; r < n_ex; ++r)
      for (int64_t c = 0; c < n_ex; ++c) {
        double s = 0.0;
        for (int64_t kc = 0; kc < 7; ++kc) {
          int64_t sc = c + kc - rad;
          if (sc >= 0 && sc < n_ex) s += hshift[r * n_ex + sc] * kern[kc];
        }
        tmp[r * n_ex + c] = s;
      }
    for (int64_t r = 0; r < n_ex; ++r)
      for (int64_t c = 0; c < n_ex; ++c) {
        double s = 0.0;
        for (int64_t kr = 0; kr < 7; ++kr) {
          int64_t sr = r + kr - rad;
          if (sr >= 0 && sr < n_ex) s += tmp[sr * n_ex + c] * kern[kr];
        }
        hfilt[r * n_ex + c] = s;
      }
    // ifftshift
    for (int64_t r = 0; r < n_ex; ++r)
      for (int64_t c = 0; c < n_ex; ++c)
        hshift[r * n_ex + c] = hfilt[((r + ish) % n_ex) * n_ex + (c + ish) % n_ex];
    // median (native_stage2.rs:1168-1184)
    hmed = hshift;
    std::sort(hmed.begin(), hmed.end());
    size_t mid = hmed.size() / 2;
    double mean_h = hmed.size() % 2 == 0 ? (hmed[mid - 1] + hmed[mid]) / 2.0 : hmed[mid];
    for (int64_t k = 0; k < n_ex * n_ex; ++k) {
      double v = hshift[k];
      if (mean_h != 0.0) v /= mean_h;
      v = alpha_is_one ? v - 1.0 : std::pow(v, alpha) - 1.0;
      if (v < 0.0) v = 0.0;
      bit[k] *= v * beta + low_pass[k];
    }
    for (int64_t r = 0; r < n_ex; ++r) fft.run(&bit[r * n_ex], 1, true);
    for (int64_t c = 0; c < n_ex; ++c) fft.run(&bit[c], static_cast<int>(n_ex), true);
    for (int64_t li = 0; li < n_win; ++li)
      for (int64_t lj = 0; lj < n_win; ++lj) {
        double wgt = (li < w.row_shift || lj < w.col_shift)
                         ? 0.0
                         : wweight[(li - w.row_shift) * n_win + (lj - w.col_shift)];
        if (wgt == 0.0) continue;
        accum[(w.i1 + li) * n_j + (w.j1 + lj)] += bit[li * n_ex + lj] * (wgt * inv_scale);
      }
  }
  for (int64_t k = 0; k < n_i * n_j; ++k)
    out[k * ostride] = {static_cast<OutR>(accum[k].real()), static_cast<OutR>(accum[k].imag())};
}

// native_stage2.rs:742-808
template <typename R>
void clap_filter_grid_stack(const Cx<R>* grid, int64_t n_i, int64_t n_j, int64_t n_ifg, int64_t n_win,
                            double alpha, double beta, const double* low_pass, int64_t n_ex, Cx<R>* out,
                            int threads) {
  for (int64_t k = 0; k < n_i * n_j * n_ifg; ++k) out[k] = {R(0), R(0)};
  int64_t n_inc = std::max<int64_t>(n_win / 4, 1);
  int64_t nwi = static_cast<int64_t>(std::ceil(static_cast<double>(n_i) / n_inc)) - 3;
  int64_t nwj = static_cast<int64_t>(std::ceil(static_cast<double>(n_j) / n_inc)) - 3;
  if (nwi <= 0 || nwj <= 0) return;
  std::vector<double> kern = clap_kernel_1d();
  std::vector<double> ww = clap_window_weight(n_win);
  std::vector<ClapWindow> windows = clap_windows(n_i, n_j, n_win, n_inc, nwi, nwj);
  bool alpha_is_one = std::fabs(alpha - 1.0) <= std::numeric_limits<double>::epsilon();
  parallel_for(n_ifg, threads, [&](int64_t b, int64_t e) {
    for (int64_t ifg = b; ifg < e; ++ifg)
      clap_filter_one_ifg<R>(grid + ifg, n_ifg, n_i, n_j, n_win, n_ex, alpha, alpha_is_one, beta, low_pass, kern,
                             ww, windows, out + ifg, n_ifg);
  });
}

// --------------------------------------------------------------- topofit ---
template <typename R>
struct RowFit {
  double k, c, coh;
};

// refine_candidate, native_stage2.rs:1259-1303 (valid == every column here)
template <typename R>
RowFit<R> refine_candidate(const Cx<R>* z, const R* bp, int64_t m, double coarse_k0, Cx<R>* residual) {
  R k0 = static_cast<R>(coarse_k0);
  Cx<R> offset{R(0), R(0)};
  for (int64_t c = 0; c < m; ++c) {
    R ph = k0 * bp[c], sn, cs;
    sincos_r(ph, &sn, &cs);
    Cx<R> t = cmul(z[c], Cx<R>{cs, -sn});
    offset.re += t.re;
    offset.im += t.im;
  }
  Cx<R> oc = conj(offset);
  double mopt = 0.0, den = 0.0;
  for (int64_t c = 0; c < m; ++c) {
    double wgt = static_cast<double>(norm(z[c]));
    double wb = wgt * static_cast<double>(bp[c]);
    den += wb * wb;
    R ph = k0 * bp[c], sn, cs;
    sincos_r(ph, &sn, &cs);
    Cx<R> res = cmul(z[c], Cx<R>{cs, -sn});
    mopt += wb * (wgt * static_cast<double>(arg(cmul(res, oc))));
  }
  if (den == 0.0) den = 1.0;
  k0 = static_cast<R>(static_cast<double>(k0) + mopt / den);
  Cx<R> mean{R(0), R(0)};
  R denom = R(0);
  for (int64_t c = 0; c < m; ++c) {
    R ph = k0 * bp[c], sn, cs;
    sincos_r(ph, &sn, &cs);
    Cx<R> res = cmul(z[c], Cx<R>{cs, -sn});
    mean.re += res.re;
    mean.im += res.im;
    denom += norm(res);
    residual[c] = res;
  }
  if (denom == R(0)) denom = R(1);
  return {static_cast<double>(k0), static_cast<double>(arg(mean)), static_cast<double>(norm(mean) / denom)};
}

// topofit_row, native_stage2.rs:1207-1257, for a row with no zero element.
// Also returns the winning trial index and the best / runner-up coherence so
// the tests can classify near-ties.
template <typename R>
RowFit<R> topofit_row(const Cx<R>* z, const R* bp, int64_t m, const double* trials, int64_t nt,
                      Cx<R>* residual, int64_t* best_ix, double* best_coh, double* second_coh) {
  R denom = R(0);
  for (int64_t c = 0; c < m; ++c) denom += norm(z[c]);
  if (denom == R(0)) denom = R(1);
  R mn = std::numeric_limits<R>::infinity(), mx = -std::numeric_limits<R>::infinity();
  for (int64_t c = 0; c < m; ++c) {
    mn = std::min(mn, bp[c]);
    mx = std::max(mx, bp[c]);
  }
  R range = mx - mn;
  if (range == R(0)) range = R(1);
  const R quarter_pi = static_cast<R>(M_PI) / R(4);
  int64_t bi = 0;
  R bv = R(0), sv = -std::numeric_limits<R>::infinity();
  for (int64_t t = 0; t < nt; ++t) {
    Cx<R> s{R(0), R(0)};
    R tv = static_cast<R>(trials[t]);
    for (int64_t c = 0; c < m; ++c) {
      R ph = (bp[c] / range) * quarter_pi * tv, sn, cs;
      sincos_r(ph, &sn, &cs);
      Cx<R> p = cmul(z[c], Cx<R>{cs, -sn});
      s.re += p.re;
      s.im += p.im;
    }
    R coh = norm(s) / denom;
    if (t == 0) {
      bv = coh;
    } else if (coh > bv) {
      sv = std::max(sv, bv);
      bv = coh;
      bi = t;
    } else {
      sv = std::max(sv, coh);
    }
  }
  if (best_ix) *best_ix = bi;
  if (best_coh) *best_coh = static_cast<double>(bv);
  if (second_coh) *second_coh = static_cast<double>(sv);
  double k0 = static_cast<double>(quarter_pi / range * static_cast<R>(trials[bi]));
  return refine_candidate<R>(z, bp, m, k0, residual);
}

// fit_stage2_rows, native_stage2.rs:659-720. ph_patch / ph_nm are [N, M];
// bperp is [N, M] (row_inv == 0) or [M] (row_inv != 0).
template <typename R>
void fit_rows(const Cx<R>* ph_patch, const Cx<float>* ph_nm, const double* bperp, int row_inv,
              const double* trials, int64_t nt, int64_t n, int64_t m, double* K, double* C, double* coh,
              double* nopt, R* ph_res, int64_t* best_ix, double* best_coh, double* second_coh, int threads) {
  parallel_for(n, threads, [&](int64_t b, int64_t e) {
    std::vector<Cx<R>> z(m), resid(m);
    std::vector<R> bp(m);
    for (int64_t r = b; r < e; ++r) {
      K[r] = std::nan("");
      C[r] = 0.0;
      coh[r] = 0.0;
      nopt[r] = 0.0;
      if (best_ix) best_ix[r] = -1;
      if (best_coh) best_coh[r] = 0.0;
      if (second_coh) second_coh[r] = 0.0;
      for (int64_t c = 0; c < m; ++c) ph_res[r * m + c] = R(0);
      bool valid = true;
      for (int64_t c = 0; c < m; ++c) {
        Cx<R> nm{static_cast<R>(ph_nm[r * m + c].re), static_cast<R>(ph_nm[r * m + c].im)};
        Cx<R> v = cmul(conj(ph_patch[r * m + c]), nm);
        if (v.re == R(0) && v.im == R(0)) valid = false;
        z[c] = v;
      }
      if (!valid) continue;
      for (int64_t c = 0; c < m; ++c)
        bp[c] = static_cast<R>(row_inv ? bperp[c] : bperp[r * m + c]);
      RowFit<R> f = topofit_row<R>(z.data(), bp.data(), m, trials, nt, resid.data(), best_ix ? best_ix + r : nullptr,
                                   best_coh ? best_coh + r : nullptr, second_coh ? second_coh + r : nullptr);
      K[r] = f.k;
      C[r] = f.c;
      coh[r] = f.coh;
      nopt[r] = 1.0;
      for (int64_t c = 0; c < m; ++c) ph_res[r * m + c] = arg(resid[c]);
    }
  });
}

// ------------------------------------------- random-phase coherence (Nr) ---
// topofit_phase_row_coh + refine_phase_candidate_coh, native_stage2.rs:1438-1512
double topofit_phase_row_coh(int64_t m, const double* bp, const double* trials, int64_t nt,
                             const double* phase) {
  if (m == 0) return std::nan("");
  double mn = INFINITY, mx = -INFINITY;
  for (int64_t c = 0; c < m; ++c) { mn = std::fmin(mn, bp[c]); mx = std::fmax(mx, bp[c]); }
  double range = mx - mn;
  if (range == 0.0) range = 1.0;
  double denom = static_cast<double>(m);
  int64_t bi = 0;
  double bv = 0.0;
  for (int64_t t = 0; t < nt; ++t) {
    double sre = 0.0, sim = 0.0;
    for (int64_t c = 0; c < m; ++c) {
      double ph = phase[c] - (bp[c] / range) * (M_PI / 4.0) * trials[t];
      sre += std::cos(ph);
      sim += std::sin(ph);
    }
    double v = hypot(sre, sim) / denom;
    if (t == 0 || v > bv) {  // argmax_first, native_stage2.rs:1514-1524
      bv = v;
      bi = t;
    }
  }
  double k0 = (M_PI / 4.0) / range * trials[bi];
  double ore = 0.0, oim = 0.0;
  for (int64_t c = 0; c < m; ++c) {
    double ph = phase[c] - k0 * bp[c];
    ore += std::cos(ph);
    oim += std::sin(ph);
  }
  double mopt = 0.0, den = 0.0;
  for (int64_t c = 0; c < m; ++c) {
    den += bp[c] * bp[c];
    double ph = phase[c] - k0 * bp[c];
    double cs = std::cos(ph), sn = std::sin(ph);
    // (cs + i sn) * conj(offset)
    double pre = cs * ore - sn * (-oim);
    double pim = cs * (-oim) + sn * ore;
    mopt += bp[c] * atan2(pim, pre);
  }
  if (den == 0.0) den = 1.0;
  double k = k0 + mopt / den;
  double sre = 0.0, sim = 0.0;
  for (int64_t c = 0; c < m; ++c) {
    double ph = phase[c] - k * bp[c];
    sre += std::cos(ph);
    sim += std::sin(ph);
  }
  return hypot(sre, sim) / static_cast<double>(std::max<int64_t>(m, 1));
}

// random_coherence_histogram, native_stage2.rs:1310-1356 (+1405-1436)
void random_hist(const double* bperp_nm, int64_t m, const double* trials, int64_t nt, int64_t n_rand,
                 int small_baseline, const int64_t* image_a, const int64_t* image_b, int64_t n_image, double* nr,
                 double* nr_max_nz_ix, int threads, const double* rand_in) {
  std::vector<double> centers(kCohBins);
  for (int i = 0; i < kCohBins; ++i) centers[i] = kCohBinStart + kCohBinStep * i;
  int64_t cols = small_baseline ? n_image : m;
  std::vector<double> u;
  const double* rnd = rand_in;
  if (!rnd) {
    u.resize(n_rand * cols);
    MatlabV5Rng rng(kRandomSeed);
    for (auto& x : u) x = rng.next() * (2.0 * M_PI);
    rnd = u.data();
  }
  // Counts are integers held in f64, so the merge order of the per-chunk
  // histograms (rayon fold/reduce in the reference) does not change Nr.
  std::vector<double> total(kCohBins, 0.0);
  std::mutex mu;
  parallel_for(n_rand, threads, [&](int64_t b, int64_t e) {
    std::vector<double> ph(m);
    std::vector<double> local(kCohBins, 0.0);
    for (int64_t row = b; row < e; ++row) {
      for (int64_t c = 0; c < m; ++c)
        ph[c] = small_baseline ? rnd[row + image_b[c] * n_rand] - rnd[row + image_a[c] * n_rand]
                               : rnd[row + c * n_rand];
      double coh = topofit_phase_row_coh(m, bperp_nm, trials, nt, ph.data());
      int64_t ix = center_index(coh, centers.data(), kCohBins, true);
      if (ix >= 0) local[ix] += 1.0;
    }
    std::lock_guard<std::mutex> g(mu);
    for (int i = 0; i < kCohBins; ++i) total[i] += local[i];
  });
  for (int i = 0; i < kCohBins; ++i) nr[i] = total[i];
  double mx = 1.0;
  for (int i = kCohBins - 1; i >= 0; --i)
    if (nr[i] > 0.0) { mx = static_cast<double>(i + 1); break; }
  *nr_max_nz_ix = mx;
}

// ----------------------------------------------------------- grid index ---
// Rust's `f32 as i32`: truncation, saturating at the i32 range, NaN -> 0.
int32_t sat_i32(float v) {
  if (std::isnan(v)) return 0;
  if (v >= 2147483647.0f) return INT32_MAX;
  if (v <= -2147483648.0f) return INT32_MIN;
  return static_cast<int32_t>(v);
}

// stage2_grid_indices, native_stage2.rs:1971-2011 (f32::min / f32::max ignore
// NaN, as std::fmin / std::fmax do)
void grid_indices(const float* xy, int64_t n, double grid_size, float* gij) {
  float min_x = INFINITY, min_y = INFINITY;
  for (int64_t r = 0; r < n; ++r) {
    min_x = std::fmin(min_x, xy[r * 3 + 1]);
    min_y = std::fmin(min_y, xy[r * 3 + 2]);
  }
  float scale = static_cast<float>(grid_size), eps = 1.0e-6f;
  int32_t max_i = 1, max_j = 1;
  for (int64_t r = 0; r < n; ++r) {
    float fi = std::fmax(std::ceil((xy[r * 3 + 2] - min_y + eps) / scale), 1.0f);
    float fj = std::fmax(std::ceil((xy[r * 3 + 1] - min_x + eps) / scale), 1.0f);
    int32_t i = sat_i32(fi), j = sat_i32(fj);
    gij[r * 2] = static_cast<float>(i);
    gij[r * 2 + 1] = static_cast<float>(j);
    max_i = std::max(max_i, i);
    max_j = std::max(max_j, j);
  }
  if (max_i > 1 || max_j > 1)
    for (int64_t r = 0; r < n; ++r) {
      if (max_i > 1 && sat_i32(gij[r * 2]) == max_i) gij[r * 2] = static_cast<float>(max_i - 1);
      if (max_j > 1 && sat_i32(gij[r * 2 + 1]) == max_j) gij[r * 2 + 1] = static_cast<float>(max_j - 1);
    }
}

// build_low_pass, native_stage2.rs:2013-2043
double powi10(double x) {
  double x2 = x * x, x4 = x2 * x2, x8 = x4 * x4;
  return x2 * x8;
}
void build_low_pass(double clap_win, double lpw, double grid_size, double* out) {
  int64_t n = static_cast<int64_t>(std::max(std::round(clap_win), 1.0));
  double f0 = 1.0 / lpw;
  std::vector<double> butter(n);
  for (int64_t i = 0; i < n; ++i) {
    double fi = (static_cast<double>(i) - static_cast<double>(n) / 2.0) / (grid_size * static_cast<double>(n));
    butter[i] = 1.0 / (1.0 + powi10(fi / f0));
  }
  int64_t sh = n / 2;
  for (int64_t r = 0; r < n; ++r)
    for (int64_t c = 0; c < n; ++c) out[r * n + c] = butter[(r + sh) % n] * butter[(c + sh) % n];
}

}  // namespace

// ======================================================================
// C ABI (ctypes) — test infrastructure
// ======================================================================
extern "C" {

void orc_rng_uniform(uint32_t seed, int64_t n, double* out) {
  MatlabV5Rng rng(seed);
  for (int64_t i = 0; i < n; ++i) out[i] = rng.next();
}

void orc_grid_indices(const float* xy, int64_t n_ps, double grid_size, float* grid_ij) {
  grid_indices(xy, n_ps, grid_size, grid_ij);
}

void orc_build_low_pass(double clap_win, double lpw, double grid_size, double* out) {
  build_low_pass(clap_win, lpw, grid_size, out);
}

void orc_hist_with_centers(const double* v, int64_t n, const double* c, int64_t nc, double* out) {
  hist_with_centers(v, n, c, nc, out);
}

void orc_psquare_lut(const double* nr, const double* na, int64_t nb, int64_t low_coh_thresh, double nr_max_nz_ix,
                     double* lut, int64_t* lut_len) {
  std::vector<double> hi = psquare_lut(nr, na, nb, low_coh_thresh, nr_max_nz_ix);
  for (size_t i = 0; i < hi.size(); ++i) lut[i] = hi[i];
  *lut_len = static_cast<int64_t>(hi.size());
}

void orc_psquare_weighting(const double* nr, const double* na, int64_t nb, int64_t low_coh_thresh,
                           double nr_max_nz_ix, const double* coh, int64_t n, double* w) {
  psquare_weighting(nr, na, nb, low_coh_thresh, nr_max_nz_ix, coh, n, w);
}

void orc_random_hist(const double* bperp_nm, int64_t m, double n_trial_wraps, int64_t n_rand, int small_baseline,
                     const int64_t* image_a, const int64_t* image_b, int64_t n_image, double* nr,
                     double* nr_max_nz_ix, int threads) {
  int64_t tn = static_cast<int64_t>(std::ceil(8.0 * n_trial_wraps));
  std::vector<double> trials;
  for (int64_t v = -tn; v <= tn; ++v) trials.push_back(static_cast<double>(v));
  random_hist(bperp_nm, m, trials.data(), static_cast<int64_t>(trials.size()), n_rand, small_baseline, image_a,
              image_b, n_image, nr, nr_max_nz_ix, threads, nullptr);
}

// fill_phase_weight, native_stage2.rs:629-657 (f32 ramp)
void orc_fill_phase_weight(const float* ph_nm, const double* bperp, int row_inv, const double* k_ps,
                           const double* w, int64_t n, int64_t m, float* out, int threads) {
  const Cx<float>* src = reinterpret_cast<const Cx<float>*>(ph_nm);
  Cx<float>* dst = reinterpret_cast<Cx<float>*>(out);
  parallel_for(n, threads, [&](int64_t b, int64_t e) {
    for (int64_t r = b; r < e; ++r)
      for (int64_t c = 0; c < m; ++c) {
        double bp = row_inv ? bperp[c] : bperp[r * m + c];
        float ph = -(static_cast<float>(bp) * static_cast<float>(k_ps[r]));
        float sn = sinf(ph), cs = cosf(ph);
        Cx<float> v = cmul(src[r * m + c], Cx<float>{cs, sn});
        float wf = static_cast<float>(w[r]);
        dst[r * m + c] = {v.re * wf, v.im * wf};
      }
  });
}

// accumulate_grid, native_stage2.rs:722-740
void orc_accumulate_grid(const float* ph_weight, const int64_t* grid_lin, int64_t n, int64_t m, int64_t n_i,
                         int64_t n_j, float* out) {
  const Cx<float>* src = reinterpret_cast<const Cx<float>*>(ph_weight);
  Cx<float>* dst = reinterpret_cast<Cx<float>*>(out);
  int64_t cells = n_i * n_j;
  for (int64_t k = 0; k < cells * m; ++k) dst[k] = {0.0f, 0.0f};
  for (int64_t r = 0; r < n; ++r) {
    int64_t g = grid_lin[r];
    if (g < 0 || g >= cells) continue;
    for (int64_t c = 0; c < m; ++c) {
      dst[g * m + c].re += src[r * m + c].re;
      dst[g * m + c].im += src[r * m + c].im;
    }
  }
}

void orc_clap_filter_grid_stack(const float* grid, int64_t n_i, int64_t n_j, int64_t m, int64_t n_win,
                                double alpha, double beta, const double* low_pass, int64_t n_ex, float* out,
                                int threads) {
  clap_filter_grid_stack<float>(reinterpret_cast<const Cx<float>*>(grid), n_i, n_j, m, n_win, alpha, beta, low_pass,
                                n_ex, reinterpret_cast<Cx<float>*>(out), threads);
}

void orc_clap_filter_grid_stack_f64(const double* grid, int64_t n_i, int64_t n_j, int64_t m, int64_t n_win,
                                    double alpha, double beta, const double* low_pass, int64_t n_ex, double* out,
                                    int threads) {
  clap_filter_grid_stack<double>(reinterpret_cast<const Cx<double>*>(grid), n_i, n_j, m, n_win, alpha, beta,
                                 low_pass, n_ex, reinterpret_cast<Cx<double>*>(out), threads);
}

// extract_patch_phase + normalize, native_stage2.rs:1186-1205
void orc_extract_patch_phase(const float* ph_filt, const int64_t* grid_lin, int64_t n, int64_t m, float* out,
                             int threads) {
  const Cx<float>* src = reinterpret_cast<const Cx<float>*>(ph_filt);
  Cx<float>* dst = reinterpret_cast<Cx<float>*>(out);
  parallel_for(n, threads, [&](int64_t b, int64_t e) {
    for (int64_t r = b; r < e; ++r)
      for (int64_t c = 0; c < m; ++c) {
        Cx<float> v = src[grid_lin[r] * m + c];
        float mag = norm(v);
        if (mag != 0.0f) v = {v.re / mag, v.im / mag};
        dst[r * m + c] = v;
      }
  });
}

void orc_fit_rows(const float* ph_patch, const float* ph_nm, const double* bperp, int row_inv,
                  double n_trial_wraps, int64_t n, int64_t m, double* K, double* C, double* coh, double* nopt,
                  float* ph_res, int64_t* best_ix, double* best_coh, double* second_coh, int threads) {
  int64_t tn = static_cast<int64_t>(std::ceil(8.0 * n_trial_wraps));
  std::vector<double> trials;
  for (int64_t v = -tn; v <= tn; ++v) trials.push_back(static_cast<double>(v));
  fit_rows<float>(reinterpret_cast<const Cx<float>*>(ph_patch), reinterpret_cast<const Cx<float>*>(ph_nm), bperp,
                  row_inv, trials.data(), static_cast<int64_t>(trials.size()), n, m, K, C, coh, nopt, ph_res,
                  best_ix, best_coh, second_coh, threads);
}

}  // extern "C"


// Registry-level topofit (boundary of the Python kernel registry,
// src/lib.rs:1159-1247 / native_stage2.rs:1207-1257): per row, zero columns
// are skipped (topofit_row's valid filter); an all-zero row gives NaN K/C/coh.
template <typename R>
static void topofit_rows_valid(const Cx<R>* cpx, const double* bperp, int row_inv, double ntw, int64_t n, int64_t m,
                               double* K, double* C, double* coh, Cx<R>* residual, int64_t* best_ix, int threads) {
  int64_t tn = static_cast<int64_t>(std::ceil(8.0 * ntw));
  std::vector<double> trials;
  for (int64_t v = -tn; v <= tn; ++v) trials.push_back(static_cast<double>(v));
  const int64_t nt = static_cast<int64_t>(trials.size());
  parallel_for(n, threads, [&](int64_t b, int64_t e) {
    std::vector<Cx<R>> z, res;
    std::vector<R> bp;
    std::vector<int64_t> col;
    for (int64_t r = b; r < e; ++r) {
      z.clear(); bp.clear(); col.clear();
      for (int64_t c = 0; c < m; ++c) {
        Cx<R> v = cpx[r * m + c];
        residual[r * m + c] = {R(0), R(0)};
        if (v.re == R(0) && v.im == R(0)) continue;
        z.push_back(v);
        bp.push_back(static_cast<R>(row_inv ? bperp[c] : bperp[r * m + c]));
        col.push_back(c);
      }
      if (z.empty()) {
        K[r] = C[r] = coh[r] = std::nan("");
        if (best_ix) best_ix[r] = -1;
        continue;
      }
      res.assign(z.size(), {R(0), R(0)});
      RowFit<R> f = topofit_row<R>(z.data(), bp.data(), static_cast<int64_t>(z.size()), trials.data(), nt, res.data(),
                                   best_ix ? best_ix + r : nullptr, nullptr, nullptr);
      K[r] = f.k;
      C[r] = f.c;
      coh[r] = f.coh;
      for (size_t k = 0; k < col.size(); ++k) residual[r * m + col[k]] = res[k];
    }
  });
}

extern "C" {

void orc_topofit(const float* cpx, const double* bperp, int row_inv, double ntw, int64_t n, int64_t m, double* K,
                 double* C, double* coh, float* residual, int64_t* best_ix, int threads) {
  topofit_rows_valid<float>(reinterpret_cast<const Cx<float>*>(cpx), bperp, row_inv, ntw, n, m, K, C, coh,
                            reinterpret_cast<Cx<float>*>(residual), best_ix, threads);
}

void orc_topofit_f64(const double* cpx, const double* bperp, int row_inv, double ntw, int64_t n, int64_t m, double* K,
                     double* C, double* coh, double* residual, int64_t* best_ix, int threads) {
  topofit_rows_valid<double>(reinterpret_cast<const Cx<double>*>(cpx), bperp, row_inv, ntw, n, m, K, C, coh,
                             reinterpret_cast<Cx<double>*>(residual), best_ix, threads);
}

}  // extern "C"

// ----------------------------------------------------------------------
// Whole stage 2 from in-memory inputs: prepare_stage2_inputs minus file
// I/O (native_stage2.rs:415-561) followed by the gamma loop (:242-413).
// ----------------------------------------------------------------------
struct orc_stage2_in {
  int64_t n_ps, n_ifg_full;
  const float* ph_full;      // c64 [n_ps, n_ifg_full]
  const double* bperp_full;  // [n_ifg_full]
  int64_t master_ix;         // 1-based
  const double* bperp_mat;   // NULL or [n_ps, bperp_mat_cols]
  int64_t bperp_mat_cols;
  const double* d_a;  // NULL or [n_ps]
  const float* xy;    // [n_ps, 3]
  double mean_incidence;
  double grid_size, clap_win, clap_low_pass_wavelength, clap_alpha, clap_beta, max_topo_err, lambda_m;
  int small_baseline;
  int psquare;  // filter_weighting == "P-square"
  double gamma_change_convergence;
  int64_t gamma_max_iterations;
  int64_t n_rand;  // 300000 in production, 10000 under the reference's tests
  const int64_t* ifgday_ix;  // [n_ifg, 2] 1-based, small baseline only
  int64_t n_image;
  const double* nr_override;  // NULL, or a precomputed Nr (100) + nr_max_nz_ix at [100]
};

struct orc_stage2_out {
  // sizes the caller must allocate: n = n_ps, m = n_ifg (non-master), g = n_i*n_j
  double* K_ps;       // [n]
  double* C_ps;       // [n]
  double* coh_ps;     // [n]
  double* N_opt;      // [n]
  void* ph_res;       // f32 / f64 [n, m]
  void* ph_patch;     // c64 / c128 [n, m]
  void* ph_grid;      // c64 / c128 [g, m]
  void* ph_weight;    // c64 / c128 [n, m]
  float* grid_ij;     // [n, 2]
  double* low_pass;   // [n_win_ex^2]
  double* Nr;         // [100]
  double* coh_ps_save;
  double* gamma_change_hist;  // [gamma_max_iterations] gamma_change_rms per iteration
  double* coh_hist;           // NULL or [gamma_max_iterations, n] coh per iteration
  double* K_hist;             // NULL or [gamma_max_iterations, n] K per iteration
  double* iter_seconds;       // NULL or [gamma_max_iterations] wall time of each loop iteration
  // scalars
  double Nr_max_nz_ix, gamma_change_save, n_trial_wraps;
  int64_t i_loop, n_i, n_j, n_ifg, n_trials;
};

template <typename R>
static int run_stage2(const orc_stage2_in* in, orc_stage2_out* out, int threads) {
  const int64_t n = in->n_ps;
  const int64_t mf = in->n_ifg_full;
  if (n <= 0 || in->master_ix < 1 || in->master_ix > mf) return -1;
  std::vector<int64_t> no_master;
  for (int64_t k = 0; k < mf; ++k)
    if (in->small_baseline || k != in->master_ix - 1) no_master.push_back(k);
  const int64_t m = static_cast<int64_t>(no_master.size());
  // ph_nm and amplitude (native_stage2.rs:452-467)
  const Cx<float>* phf = reinterpret_cast<const Cx<float>*>(in->ph_full);
  std::vector<Cx<float>> ph_nm(n * m);
  std::vector<float> amp(n * m);
  for (int64_t r = 0; r < n; ++r)
    for (int64_t k = 0; k < m; ++k) {
      Cx<float> v = phf[r * mf + no_master[k]];
      float mag = norm(v);
      float safe = mag == 0.0f ? 1.0f : mag;
      amp[r * m + k] = safe;
      ph_nm[r * m + k] = {v.re / safe, v.im / safe};
    }
  std::vector<double> bperp_nm(m);
  for (int64_t k = 0; k < m; ++k) bperp_nm[k] = static_cast<double>(static_cast<float>(in->bperp_full[no_master[k]]));
  // bperp matrix (native_stage2.rs:563-612)
  std::vector<double> bmat;
  bool have_mat = false;
  if (in->bperp_mat) {
    if (in->bperp_mat_cols == m) {
      bmat.assign(in->bperp_mat, in->bperp_mat + n * m);
    } else if (!in->small_baseline && in->bperp_mat_cols == mf) {
      bmat.resize(n * m);
      for (int64_t r = 0; r < n; ++r)
        for (int64_t k = 0; k < m; ++k) bmat[r * m + k] = in->bperp_mat[r * mf + no_master[k]];
    } else {
      return -2;  // "bp1.bperp_mat has incompatible shape"
    }
    have_mat = true;
  } else if (in->small_baseline) {
    bmat.resize(n * m);
    for (int64_t r = 0; r < n; ++r)
      for (int64_t k = 0; k < m; ++k) bmat[r * m + k] = bperp_nm[k];
    have_mat = true;
  }
  bool row_inv = true;
  if (have_mat && n > 1)
    for (int64_t r = 1; r < n && row_inv; ++r)
      for (int64_t k = 0; k < m; ++k)
        if (bmat[r * m + k] != bmat[k]) { row_inv = false; break; }
  std::vector<double> row_bp = (row_inv && have_mat) ? std::vector<double>(bmat.begin(), bmat.begin() + m) : bperp_nm;
  const double* bperp_use = row_inv ? row_bp.data() : bmat.data();
  // weighting w0 = 1/D_A
  std::vector<double> weighting(n, 1.0);
  if (in->d_a)
    for (int64_t r = 0; r < n; ++r) weighting[r] = in->d_a[r] != 0.0 ? 1.0 / in->d_a[r] : 0.0;
  // grid indices
  grid_indices(in->xy, n, in->grid_size, out->grid_ij);
  int64_t n_i = 1, n_j = 1;
  for (int64_t r = 0; r < n; ++r) {
    n_i = std::max<int64_t>(n_i, static_cast<int64_t>(out->grid_ij[r * 2]));
    n_j = std::max<int64_t>(n_j, static_cast<int64_t>(out->grid_ij[r * 2 + 1]));
  }
  std::vector<int64_t> grid_lin(n);
  for (int64_t r = 0; r < n; ++r)
    grid_lin[r] = (static_cast<int64_t>(out->grid_ij[r * 2]) - 1) * n_j + static_cast<int64_t>(out->grid_ij[r * 2 + 1]) - 1;
  const int64_t g = n_i * n_j;
  if (out->n_i != n_i || out->n_j != n_j) {
    out->n_i = n_i;
    out->n_j = n_j;
    return 1;  // caller must re-allocate ph_grid with the reported sizes
  }
  // low pass, trials
  int64_t nwx = static_cast<int64_t>(std::max(std::round(in->clap_win), 1.0));
  build_low_pass(in->clap_win, in->clap_low_pass_wavelength, in->grid_size, out->low_pass);
  int64_t clap_window = static_cast<int64_t>(std::max(std::round(in->clap_win * 0.75), 1.0));
  double rho = 830000.0;
  double max_k = in->max_topo_err / (in->lambda_m * rho * std::sin(in->mean_incidence) / (4.0 * M_PI));
  double mn = INFINITY, mx = -INFINITY;
  for (double v : bperp_nm) { mn = std::fmin(mn, v); mx = std::fmax(mx, v); }
  double n_trial_wraps = (mx - mn) * max_k / (2.0 * M_PI);
  int64_t tn = static_cast<int64_t>(std::ceil(8.0 * n_trial_wraps));
  std::vector<double> trials;
  for (int64_t v = -tn; v <= tn; ++v) trials.push_back(static_cast<double>(v));
  const int64_t nt = static_cast<int64_t>(trials.size());
  const int64_t low_coh_thresh = in->small_baseline ? 15 : 31;
  out->n_trial_wraps = n_trial_wraps;
  out->n_trials = nt;
  out->n_ifg = m;
  // Nr
  std::vector<double> nr(kCohBins);
  double nr_max_nz_ix = 1.0;
  if (in->nr_override) {
    for (int i = 0; i < kCohBins; ++i) nr[i] = in->nr_override[i];
    nr_max_nz_ix = in->nr_override[kCohBins];
  } else {
    std::vector<int64_t> ia(m), ib(m);
    if (in->small_baseline) {
      for (int64_t k = 0; k < m; ++k) { ia[k] = in->ifgday_ix[k * 2] - 1; ib[k] = in->ifgday_ix[k * 2 + 1] - 1; }
    }
    random_hist(bperp_nm.data(), m, trials.data(), nt, in->n_rand, in->small_baseline, ia.data(), ib.data(),
                in->n_image, nr.data(), &nr_max_nz_ix, threads, nullptr);
  }
  std::vector<double> coh_bins(kCohBins);
  for (int i = 0; i < kCohBins; ++i) coh_bins[i] = kCohBinStart + kCohBinStep * i;

  // loop state
  std::vector<double> K(n, 0.0), C(n, 0.0), coh(n, 0.0), nopt(n, 0.0), coh_save(n, 0.0);
  std::vector<R> ph_res(n * m, R(0));
  std::vector<Cx<R>> ph_patch(n * m), ph_grid(g * m), ph_filt(g * m), ph_weight(n * m);
  std::vector<double> nr_scaled = nr;
  double gamma_change_save = 0.0;
  int64_t i_loop = 1;
  const int64_t max_iter = std::max<int64_t>(in->gamma_max_iterations, 1);
  auto t_iter = std::chrono::steady_clock::now();
  auto record_time = [&]() {
    const auto t_now = std::chrono::steady_clock::now();
    if (out->iter_seconds && i_loop <= in->gamma_max_iterations)
      out->iter_seconds[i_loop - 1] = std::chrono::duration<double>(t_now - t_iter).count();
    t_iter = t_now;
  };
  for (;;) {
    // fill_phase_weight
    parallel_for(n, threads, [&](int64_t b, int64_t e) {
      for (int64_t r = b; r < e; ++r)
        for (int64_t c = 0; c < m; ++c) {
          R bp = static_cast<R>(row_inv ? bperp_use[c] : bperp_use[r * m + c]);
          R ph = -(bp * static_cast<R>(K[r]));
          R sn, cs;
          sincos_r(ph, &sn, &cs);
          Cx<R> src{static_cast<R>(ph_nm[r * m + c].re), static_cast<R>(ph_nm[r * m + c].im)};
          Cx<R> v = cmul(src, Cx<R>{cs, sn});
          R wf = static_cast<R>(weighting[r]);
          ph_weight[r * m + c] = {v.re * wf, v.im * wf};
        }
    });
    // accumulate_grid
    for (auto& v : ph_grid) v = {R(0), R(0)};
    for (int64_t r = 0; r < n; ++r) {
      int64_t gl = grid_lin[r];
      if (gl >= g) continue;
      for (int64_t c = 0; c < m; ++c) {
        ph_grid[gl * m + c].re += ph_weight[r * m + c].re;
        ph_grid[gl * m + c].im += ph_weight[r * m + c].im;
      }
    }
    clap_filter_grid_stack<R>(ph_grid.data(), n_i, n_j, m, clap_window, in->clap_alpha, in->clap_beta, out->low_pass,
                              nwx, ph_filt.data(), threads);
    // extract + normalise
    parallel_for(n, threads, [&](int64_t b, int64_t e) {
      for (int64_t r = b; r < e; ++r)
        for (int64_t c = 0; c < m; ++c) {
          Cx<R> v = ph_filt[grid_lin[r] * m + c];
          R mag = norm(v);
          if (mag != R(0)) v = {v.re / mag, v.im / mag};
          ph_patch[r * m + c] = v;
        }
    });
    fit_rows<R>(ph_patch.data(), ph_nm.data(), bperp_use, row_inv ? 1 : 0, trials.data(), nt, n, m, K.data(), C.data(),
                coh.data(), nopt.data(), ph_res.data(), nullptr, nullptr, nullptr, threads);
    if (out->coh_hist && i_loop <= in->gamma_max_iterations)
      std::copy(coh.begin(), coh.end(), out->coh_hist + (i_loop - 1) * n);
    if (out->K_hist && i_loop <= in->gamma_max_iterations)
      std::copy(K.begin(), K.end(), out->K_hist + (i_loop - 1) * n);
    // rms_difference, native_stage2.rs:2045-2057
    double s = 0.0;
    for (int64_t r = 0; r < n; ++r) {
      double d = coh[r] - coh_save[r];
      s += d * d;
    }
    double gamma_change_rms = std::sqrt(s / static_cast<double>(std::max<int64_t>(n, 1)));
    double gamma_change_change = gamma_change_rms - gamma_change_save;
    gamma_change_save = gamma_change_rms;
    coh_save = coh;
    if (out->gamma_change_hist && i_loop <= in->gamma_max_iterations) out->gamma_change_hist[i_loop - 1] = gamma_change_rms;
    bool stop = std::fabs(gamma_change_change) < in->gamma_change_convergence || i_loop >= max_iter;
    if (stop) {
      record_time();
      break;
    }
    if (in->psquare) {
      std::vector<double> na(kCohBins);
      hist_with_centers(coh.data(), n, coh_bins.data(), kCohBins, na.data());
      double den = 0.0, num = 0.0;
      for (int64_t i = 0; i < low_coh_thresh; ++i) den += nr_scaled[i];
      double scale = 1.0;
      if (den > 0.0) {
        for (int64_t i = 0; i < low_coh_thresh; ++i) num += na[i];
        scale = num / den;
      }
      for (auto& v : nr_scaled) v *= scale;
      psquare_weighting(nr_scaled.data(), na.data(), kCohBins, low_coh_thresh, nr_max_nz_ix, coh.data(), n,
                        weighting.data());
    } else {
      // snr_weighting, native_stage2.rs:1875-1897
      for (int64_t r = 0; r < n; ++r) {
        double gg = 0.0, a2 = 0.0;
        for (int64_t c = 0; c < m; ++c) {
          double a = static_cast<double>(amp[r * m + c]);
          gg += a * std::cos(static_cast<double>(ph_res[r * m + c]));
          a2 += a * a;
        }
        gg /= static_cast<double>(std::max<int64_t>(m, 1));
        a2 /= static_cast<double>(std::max<int64_t>(m, 1));
        double sig = std::sqrt(0.5 * (a2 - gg * gg));
        weighting[r] = sig != 0.0 ? gg / sig : 0.0;
      }
    }
    record_time();
    ++i_loop;
  }
  // outputs
  std::copy(K.begin(), K.end(), out->K_ps);
  std::copy(C.begin(), C.end(), out->C_ps);
  std::copy(coh.begin(), coh.end(), out->coh_ps);
  std::copy(nopt.begin(), nopt.end(), out->N_opt);
  std::copy(coh_save.begin(), coh_save.end(), out->coh_ps_save);
  std::memcpy(out->ph_res, ph_res.data(), sizeof(R) * n * m);
  std::memcpy(out->ph_patch, ph_patch.data(), sizeof(Cx<R>) * n * m);
  std::memcpy(out->ph_grid, ph_grid.data(), sizeof(Cx<R>) * g * m);
  std::memcpy(out->ph_weight, ph_weight.data(), sizeof(Cx<R>) * n * m);
  for (int i = 0; i < kCohBins; ++i) out->Nr[i] = nr_scaled[i];
  out->Nr_max_nz_ix = nr_max_nz_ix;
  out->gamma_change_save = gamma_change_save;
  out->i_loop = i_loop;
  return 0;
}

extern "C" {

int orc_stage2_run(const orc_stage2_in* in, orc_stage2_out* out, int threads) {
  return run_stage2<float>(in, out, threads);
}

int orc_stage2_run_f64(const orc_stage2_in* in, orc_stage2_out* out, int threads) {
  return run_stage2<double>(in, out, threads);
}

}  // extern "C"

// ============================================================ stage 3 ======
// Stage-3 re-estimate (pystamps/pipeline/ported.py:4429-4575, the Python
// reference; the Rust native stage 3 has no re-estimate). numpy semantics:
// _clap_filt_patch in complex128 (ported.py:992-1009); _ps_topofit_single in
// complex64 / float32 (ported.py:2355-2431) with the near-max candidate rule
// (:2433-2448, tolerance 2e-4), per-candidate refinement (:2473-2508) and the
// candidate choice (:2451-2470). numpy's 1-D float sums are pairwise (blocks
// of 8 partial sums, halving above 128 elements); a reduction over the
// non-contiguous axis of a 2-D array adds rows in order. The first element of a
// reduction seeds the accumulator.

namespace s3 {

float pw_f32(const float* a, int64_t n, int64_t stride) {
  if (n < 8) {
    float r = -0.0f;
    for (int64_t i = 0; i < n; ++i) r += a[i * stride];
    return r;
  }
  if (n <= 128) {
    float r[8];
    for (int j = 0; j < 8; ++j) r[j] = a[j * stride];
    int64_t i = 8;
    for (; i < n - (n % 8); i += 8)
      for (int j = 0; j < 8; ++j) r[j] += a[(i + j) * stride];
    float res = ((r[0] + r[1]) + (r[2] + r[3])) + ((r[4] + r[5]) + (r[6] + r[7]));
    for (; i < n; ++i) res += a[i * stride];
    return res;
  }
  int64_t n2 = n / 2;
  n2 -= n2 % 8;
  return pw_f32(a, n2, stride) + pw_f32(a + n2 * stride, n - n2, stride);
}

// np.sum of a contiguous float32 vector
float sum_f32(const float* a, int64_t n) {
  if (n == 0) return 0.0f;
  return a[0] + pw_f32(a + 1, n - 1, 1);
}

// pairwise sum over interleaved complex64 (n = 2 * count floats)
void pw_c64(const float* a, int64_t n, float* rr, float* ri) {
  if (n < 8) {
    float x = -0.0f, y = -0.0f;
    for (int64_t i = 0; i < n; i += 2) {
      x += a[i];
      y += a[i + 1];
    }
    *rr = x;
    *ri = y;
    return;
  }
  if (n <= 128) {
    float r[8];
    for (int j = 0; j < 8; ++j) r[j] = a[j];
    int64_t i = 8;
    for (; i < n - (n % 8); i += 8)
      for (int j = 0; j < 8; ++j) r[j] += a[i + j];
    float x = (r[0] + r[2]) + (r[4] + r[6]);
    float y = (r[1] + r[3]) + (r[5] + r[7]);
    for (; i < n; i += 2) {
      x += a[i];
      y += a[i + 1];
    }
    *rr = x;
    *ri = y;
    return;
  }
  int64_t n2 = n / 2;
  n2 -= n2 % 8;
  float x1, y1, x2, y2;
  pw_c64(a, n2, &x1, &y1);
  pw_c64(a + n2, n - n2, &x2, &y2);
  *rr = x1 + x2;
  *ri = y1 + y2;
}

Cx<float> sum_c64(const std::vector<Cx<float>>& v) {
  if (v.empty()) return {0.0f, 0.0f};
  float x, y;
  pw_c64(reinterpret_cast<const float*>(v.data()) + 2, 2 * static_cast<int64_t>(v.size() - 1), &x, &y);
  return {v[0].re + x, v[0].im + y};
}

// np.exp(-1j * x) for a float32 x: (cos x, -sin x) through cexpf
inline Cx<float> cis_neg(float x) { return {std::cos(x), -std::sin(x)}; }

inline Cx<float> mul(Cx<float> a, Cx<float> b) { return {a.re * b.re - a.im * b.im, a.re * b.im + a.im * b.re}; }

// _clap_filt_patch (ported.py:992-1009) on an n x n complex128 patch
void clap_patch(const std::complex<double>* in, int64_t n, double alpha, double beta, const double* lp,
                std::complex<double>* out) {
  std::vector<std::complex<double>> x(in, in + n * n);
  for (auto& v : x)
    if (std::isnan(v.real()) || std::isnan(v.imag())) v = {0.0, 0.0};
  Fft fft(static_cast<int>(n));
  for (int64_t r = 0; r < n; ++r) fft.run(&x[r * n], 1, false);
  for (int64_t c = 0; c < n; ++c) fft.run(&x[c], static_cast<int>(n), false);
  std::vector<double> h(n * n), hs(n * n), hc(n * n);
  for (int64_t k = 0; k < n * n; ++k) h[k] = std::abs(x[k]);
  const int64_t sh = n / 2, ish = (n + 1) / 2;
  for (int64_t r = 0; r < n; ++r)
    for (int64_t c = 0; c < n; ++c) hs[r * n + c] = h[((r + sh) % n) * n + (c + sh) % n];
  // convolve2d(mode="same", fill 0) with outer(g, g); the kernel is symmetric
  std::vector<double> g = clap_kernel_1d();
  for (int64_t r = 0; r < n; ++r)
    for (int64_t c = 0; c < n; ++c) {
      double s = 0.0;
      for (int64_t a = -3; a <= 3; ++a)
        for (int64_t b = -3; b <= 3; ++b) {
          const int64_t rr = r + a, cc = c + b;
          if (rr < 0 || rr >= n || cc < 0 || cc >= n) continue;
          s += hs[rr * n + cc] * (g[a + 3] * g[b + 3]);
        }
      hc[r * n + c] = s;
    }
  for (int64_t r = 0; r < n; ++r)
    for (int64_t c = 0; c < n; ++c) h[r * n + c] = hc[((r + ish) % n) * n + (c + ish) % n];
  std::vector<double> srt(h);
  std::sort(srt.begin(), srt.end());
  const size_t mid = srt.size() / 2;
  const double med = srt.size() % 2 == 0 ? (srt[mid - 1] + srt[mid]) / 2.0 : srt[mid];
  for (int64_t k = 0; k < n * n; ++k) {
    double v = h[k];
    if (med != 0.0) v /= med;
    v = std::pow(v, alpha) - 1.0;
    if (v < 0.0) v = 0.0;
    x[k] *= v * beta + lp[k];
  }
  for (int64_t r = 0; r < n; ++r) fft.run(&x[r * n], 1, true);
  for (int64_t c = 0; c < n; ++c) fft.run(&x[c], static_cast<int>(n), true);
  const double inv = 1.0 / static_cast<double>(n * n);
  for (int64_t k = 0; k < n * n; ++k) out[k] = x[k] * inv;
}

struct Fit {
  double K, C, coh;
  std::vector<Cx<float>> res;
};

// _ps_topofit_refine_candidate (ported.py:2473-2508) in float32
Fit refine(const std::vector<Cx<float>>& cpx, const std::vector<float>& bp, const std::vector<float>& wgt,
           const std::vector<float>& wb, double den_lin, double coarse_k0) {
  const int64_t m = static_cast<int64_t>(cpx.size());
  float K0 = static_cast<float>(coarse_k0);
  std::vector<Cx<float>> r(m);
  for (int64_t c = 0; c < m; ++c) r[c] = mul(cpx[c], cis_neg(K0 * bp[c]));
  const Cx<float> off = sum_c64(r);
  std::vector<float> t(m);
  for (int64_t c = 0; c < m; ++c) {
    const Cx<float> q = mul(r[c], Cx<float>{off.re, -off.im});
    t[c] = wb[c] * (wgt[c] * std::atan2(q.im, q.re));
  }
  const float mopt = sum_f32(t.data(), m) / static_cast<float>(den_lin);
  K0 = K0 + mopt;
  Fit f;
  f.res.resize(m);
  std::vector<float> ab(m);
  for (int64_t c = 0; c < m; ++c) {
    f.res[c] = mul(cpx[c], cis_neg(K0 * bp[c]));
    ab[c] = std::hypot(f.res[c].re, f.res[c].im);
  }
  const Cx<float> mean = sum_c64(f.res);
  double den2 = static_cast<double>(sum_f32(ab.data(), m));
  if (den2 == 0.0) den2 = 1.0;
  f.K = static_cast<double>(K0);
  f.C = static_cast<double>(std::atan2(mean.im, mean.re));
  f.coh = static_cast<double>(std::hypot(mean.re, mean.im) / static_cast<float>(den2));
  return f;
}

// _ps_topofit_single (ported.py:2355-2431), complex64 / float32 form.
// Returns the candidate count (0: no valid column).
int64_t topofit_single(const Cx<float>* cpx_in, const float* bp_in, int64_t m_in, double n_trial_wraps,
                       double* K, double* C, double* coh, Cx<float>* res_out) {
  for (int64_t c = 0; c < m_in; ++c) res_out[c] = {0.0f, 0.0f};
  std::vector<Cx<float>> cpx;
  std::vector<float> bp;
  std::vector<int64_t> col;
  for (int64_t c = 0; c < m_in; ++c)
    if (cpx_in[c].re != 0.0f || cpx_in[c].im != 0.0f) {
      cpx.push_back(cpx_in[c]);
      bp.push_back(bp_in[c]);
      col.push_back(c);
    }
  const int64_t m = static_cast<int64_t>(cpx.size());
  if (m == 0) {
    *K = *C = *coh = std::numeric_limits<double>::quiet_NaN();
    return 0;
  }
  const int64_t nt = static_cast<int64_t>(std::ceil(8.0 * n_trial_wraps));
  const int64_t T = 2 * nt + 1;
  float mn = bp[0], mx = bp[0];
  for (float v : bp) {
    mn = std::min(mn, v);
    mx = std::max(mx, v);
  }
  double range = static_cast<double>(mx - mn);
  if (range == 0.0) range = 1.0;
  const float rf = static_cast<float>(range), qp = static_cast<float>(M_PI / 4.0);
  std::vector<float> tp(m);
  for (int64_t c = 0; c < m; ++c) tp[c] = bp[c] / rf * qp;
  std::vector<float> ab(m), wgt(m), wb(m), wb2(m);
  for (int64_t c = 0; c < m; ++c) {
    ab[c] = std::hypot(cpx[c].re, cpx[c].im);
    wgt[c] = ab[c];
    wb[c] = wgt[c] * bp[c];
    wb2[c] = wb[c] * wb[c];
  }
  double denom = static_cast<double>(sum_f32(ab.data(), m));
  if (denom == 0.0) denom = 1.0;
  double den_lin = static_cast<double>(sum_f32(wb2.data(), m));
  if (den_lin == 0.0) den_lin = 1.0;
  std::vector<double> ct(T);
  for (int64_t t = 0; t < T; ++t) {
    const float tm = static_cast<float>(t - nt);
    float sx = 0.0f, sy = 0.0f;
    for (int64_t c = 0; c < m; ++c) {  // rows of the (m, T) product added in order
      const Cx<float> p = mul(cis_neg(tp[c] * tm), cpx[c]);
      if (c == 0) {
        sx = p.re;
        sy = p.im;
      } else {
        sx += p.re;
        sy += p.im;
      }
    }
    ct[t] = static_cast<double>(std::hypot(sx, sy) / static_cast<float>(denom));
  }
  // _ps_topofit_near_max_trial_indices (ported.py:2433-2448)
  std::vector<int64_t> cand;
  const double cmax = *std::max_element(ct.begin(), ct.end());
  for (int64_t t = 0; t < T; ++t) {
    bool lm;
    if (T == 1) lm = true;
    else if (t == 0) lm = ct[0] >= ct[1];
    else if (t == T - 1) lm = ct[T - 1] >= ct[T - 2];
    else lm = ct[t] >= ct[t - 1] && ct[t] >= ct[t + 1];
    if (lm && ct[t] >= cmax - 2.0e-4) cand.push_back(t);
  }
  if (cand.empty()) cand.push_back(std::max_element(ct.begin(), ct.end()) - ct.begin());
  std::vector<Fit> fits;
  for (int64_t t : cand)
    fits.push_back(refine(cpx, bp, wgt, wb, den_lin, (M_PI / 4.0) / range * static_cast<double>(t - nt)));
  // _ps_topofit_select_candidate (ported.py:2451-2470)
  size_t pick = 0;
  if (cand.size() > 1) {
    size_t coarse_best = 0;
    for (size_t i = 1; i < cand.size(); ++i)
      if (ct[cand[i]] > ct[cand[coarse_best]]) coarse_best = i;
    const bool endpoints = cand.size() == 2 && cand[0] == 0 && cand[1] == T - 1;
    if (endpoints) {
      pick = coarse_best;
    } else {
      size_t rb = 0;
      for (size_t i = 1; i < fits.size(); ++i)
        if (fits[i].coh > fits[rb].coh) rb = i;
      pick = rb;
    }
  }
  *K = fits[pick].K;
  *C = fits[pick].C;
  *coh = fits[pick].coh;
  for (int64_t k = 0; k < m; ++k) res_out[col[k]] = fits[pick].res[k];
  return static_cast<int64_t>(cand.size());
}

}  // namespace s3

extern "C" {

void orc_s3_clap_patch(const double* in, int64_t n, double alpha, double beta, const double* lp, double* out) {
  s3::clap_patch(reinterpret_cast<const std::complex<double>*>(in), n, alpha, beta, lp,
                 reinterpret_cast<std::complex<double>*>(out));
}

int64_t orc_s3_topofit_single(const float* cpx, const float* bp, int64_t m, double n_trial_wraps, double* K,
                              double* C, double* coh, float* res) {
  return s3::topofit_single(reinterpret_cast<const Cx<float>*>(cpx), bp, m, n_trial_wraps, K, C, coh,
                            reinterpret_cast<Cx<float>*>(res));
}

// The re-estimate loop of ported.py:4489-4550 for the selected rows `sel`.
// ph_grid complex64 [gi, gj, m]; grid_ij [n_ps, 2] 1-based; ph_work complex64
// [n_ps, m]; bperp f64 [n_ps, m]; fit: 0-based columns topofit uses. Outputs:
// ph_patch2 complex128 [n_sel, m], K2/C2/coh2 [n_sel], ph_res2 f32 [n_sel, m].
int orc_s3_reestimate(const float* ph_grid, int64_t gi, int64_t gj, int64_t m, const int64_t* grid_ij,
                      const int64_t* sel, int64_t n_sel, const float* ph_work, const double* bperp,
                      const int64_t* fit, int64_t n_fit, int64_t n_i, int64_t n_j, int64_t n_win, double alpha,
                      double beta, const double* lp, int64_t slc_osf, double n_trial_wraps, double* ph_patch2,
                      double* K2, double* C2, double* coh2, float* ph_res2, int threads) {
  (void)gi;
  const int64_t half = n_win / 2;
  const Cx<float>* grid = reinterpret_cast<const Cx<float>*>(ph_grid);
  const Cx<float>* work = reinterpret_cast<const Cx<float>*>(ph_work);
  std::complex<double>* pp2 = reinterpret_cast<std::complex<double>*>(ph_patch2);
  parallel_for(n_sel, threads, [&](int64_t b, int64_t e) {
    std::vector<std::complex<double>> bit(n_win * n_win), filt(n_win * n_win);
    std::vector<Cx<float>> cpx(n_fit), res(n_fit);
    std::vector<float> bpf(n_fit);
    for (int64_t r = b; r < e; ++r) {
      const int64_t ps = sel[r];
      const int64_t pi = grid_ij[2 * ps], pj = grid_ij[2 * ps + 1];
      int64_t i_min = std::max<int64_t>(pi - half, 1), i_max = i_min + n_win - 1;
      if (i_max > n_i) {
        i_min = i_min - i_max + n_i;
        i_max = n_i;
      }
      int64_t j_min = std::max<int64_t>(pj - half, 1), j_max = j_min + n_win - 1;
      if (j_max > n_j) {
        j_min = j_min - j_max + n_j;
        j_max = n_j;
      }
      std::complex<double>* out = pp2 + r * m;
      if (i_min < 1 || j_min < 1) {
        for (int64_t c = 0; c < m; ++c) out[c] = {0.0, 0.0};
      } else {
        const int64_t bi = pi - i_min, bj = pj - j_min;  // 0-based PS cell in the patch
        const int64_t rad = slc_osf - 1;
        for (int64_t c = 0; c < m; ++c) {
          for (int64_t li = 0; li < n_win; ++li)
            for (int64_t lj = 0; lj < n_win; ++lj) {
              const Cx<float> v = grid[((i_min - 1 + li) * gj + (j_min - 1 + lj)) * m + c];
              bit[li * n_win + lj] = {static_cast<double>(v.re), static_cast<double>(v.im)};
            }
          bit[bi * n_win + bj] = {0.0, 0.0};
          if (c == 0)
            for (int64_t li = std::max<int64_t>(bi - rad, 0); li <= std::min<int64_t>(bi + rad, n_win - 1); ++li)
              for (int64_t lj = std::max<int64_t>(bj - rad, 0); lj <= std::min<int64_t>(bj + rad, n_win - 1); ++lj)
                bit[li * n_win + lj] = {0.0, 0.0};
          s3::clap_patch(bit.data(), n_win, alpha, beta, lp, filt.data());
          out[c] = filt[bi * n_win + bj];
        }
      }
      // psdph = ph_work * conj(ph_patch2) (complex128); any zero -> NaN row
      bool any_zero = false;
      std::vector<std::complex<double>> psd(m);
      for (int64_t c = 0; c < m; ++c) {
        const Cx<float> w = work[ps * m + c];
        psd[c] = std::complex<double>(w.re, w.im) * std::conj(out[c]);
        if (psd[c] == std::complex<double>(0.0, 0.0)) any_zero = true;
      }
      float* pr = ph_res2 + r * m;
      for (int64_t c = 0; c < m; ++c) pr[c] = 0.0f;
      if (any_zero) {
        K2[r] = std::numeric_limits<double>::quiet_NaN();
        coh2[r] = std::numeric_limits<double>::quiet_NaN();
        C2[r] = 0.0;
        continue;
      }
      for (int64_t k = 0; k < n_fit; ++k) {
        const std::complex<double> v = psd[fit[k]] / std::abs(psd[fit[k]]);
        cpx[k] = {static_cast<float>(v.real()), static_cast<float>(v.imag())};
        bpf[k] = static_cast<float>(bperp[ps * m + fit[k]]);
      }
      s3::topofit_single(cpx.data(), bpf.data(), n_fit, n_trial_wraps, &K2[r], &C2[r], &coh2[r], res.data());
      for (int64_t k = 0; k < n_fit; ++k) pr[fit[k]] = std::atan2(res[k].im, res[k].re);
    }
  });
  return 0;
}

}  // extern "C"
