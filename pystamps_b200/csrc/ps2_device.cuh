// Device helpers shared by the stage-2 kernels (sm_100a).
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

namespace ps2 {

constexpr int kWarp = 32;
constexpr unsigned kFull = 0xffffffffu;
constexpr int kCohBins = 100;

// ------------------------------------------------------------ complex ------
// Products are written with explicit _rn intrinsics where the reference rounds
// each product separately (Rust never contracts a*b+c into an FMA); the
// topofit trial sweep, which the reference does not share bit-for-bit anyway,
// uses plain (contractible) arithmetic.
struct c32 {
  float x, y;
};
struct c64d {
  double x, y;
};

__device__ __forceinline__ float2 cmul_rn(float2 a, float2 b) {
  // (a.re*b.re - a.im*b.im, a.re*b.im + a.im*b.re) with every product rounded
  return make_float2(__fsub_rn(__fmul_rn(a.x, b.x), __fmul_rn(a.y, b.y)),
                     __fadd_rn(__fmul_rn(a.x, b.y), __fmul_rn(a.y, b.x)));
}
__device__ __forceinline__ double2 cmul_rn(double2 a, double2 b) {
  return make_double2(__dsub_rn(__dmul_rn(a.x, b.x), __dmul_rn(a.y, b.y)),
                      __dadd_rn(__dmul_rn(a.x, b.y), __dmul_rn(a.y, b.x)));
}
__device__ __forceinline__ float2 cmul(float2 a, float2 b) {
  return make_float2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}
__device__ __forceinline__ double2 cmul(double2 a, double2 b) {
  return make_double2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}
__device__ __forceinline__ float2 conjf2(float2 a) { return make_float2(a.x, -a.y); }
__device__ __forceinline__ double2 conjd2(double2 a) { return make_double2(a.x, -a.y); }

// --------------------------------------------------------- warp reduce -----
template <typename T>
__device__ __forceinline__ T warp_sum(T v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(kFull, v, o);
  return v;
}
__device__ __forceinline__ float warp_min(float v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v = fminf(v, __shfl_xor_sync(kFull, v, o));
  return v;
}
__device__ __forceinline__ float warp_max(float v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v = fmaxf(v, __shfl_xor_sync(kFull, v, o));
  return v;
}
__device__ __forceinline__ double warp_min(double v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v = fmin(v, __shfl_xor_sync(kFull, v, o));
  return v;
}
__device__ __forceinline__ double warp_max(double v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v = fmax(v, __shfl_xor_sync(kFull, v, o));
  return v;
}

// Histogram bin of the equal-spacing Octave rule used for the coherence
// histogram (native_stage2.rs:1593-1607): centres 0.005 + 0.01*i, i < 100.
// d and cutoff0 are computed on the host exactly like the reference.
__device__ __forceinline__ int coh_bin(double v, double cutoff0, double d) {
  if (!isfinite(v)) return -1;
  double a = ceil((v - cutoff0) / d);
  a = fmin(fmax(a, 0.0), double(kCohBins - 1));
  return static_cast<int>(a);
}

}  // namespace ps2
