// Generated by make_sincos_poly.py (minimax sin/cos on [-pi/4, pi/4] after
// Cody-Waite reduction by pi/2; see that script for the design).
// fitted max error: sin 3.6e-09, cos 9.5e-11
#pragma once
namespace ps2 {
constexpr float kSinS1 = -1.666665524e-01f;
constexpr float kSinS2 = 8.332177997e-03f;
constexpr float kSinS3 = -1.951725862e-04f;
constexpr float kCosQ1 = 4.166664556e-02f;
constexpr float kCosQ2 = -1.388736768e-03f;
constexpr float kCosQ3 = 2.443840640e-05f;
constexpr float kHalfPi1 = 1.570796371e+00f;
constexpr float kHalfPi2 = -4.371138829e-08f;
constexpr float kHalfPi3 = -1.776356839e-15f;
constexpr float kTwoOverPi = 6.366197467e-01f;
}  // namespace ps2
