// Generated by make_atan_poly.py (minimax atan on [0, 1]; see that script).
// fitted max error: 4.9e-08
#pragma once
namespace ps2 {
constexpr float kAtanA1 = -3.333165944e-01f;
constexpr float kAtanA2 = 1.996270269e-01f;
constexpr float kAtanA3 = -1.397657394e-01f;
constexpr float kAtanA4 = 9.794210643e-02f;
constexpr float kAtanA5 = -5.777322501e-02f;
constexpr float kAtanA6 = 2.303985879e-02f;
constexpr float kAtanA7 = -4.355323035e-03f;
constexpr float kHalfPiF = 1.570796371e+00f;
constexpr float kPiF = 3.141592741e+00f;
}  // namespace ps2
