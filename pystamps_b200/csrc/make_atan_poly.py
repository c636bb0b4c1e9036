"""Generates atan_poly.h: the polynomial coefficients of the FP32 atan2 of the
topofit refinement (atan2_poly in ps2_kernels.cu).

atan2(y, x) is reduced to t = min(|x|, |y|) / max(|x|, |y|) in [0, 1] and
    atan t = t + t u (A1 + u (A2 + ... + u A7)),   u = t^2  (kAtanA1 .. kAtanA7),
followed by the octant's reflections (pi/2 - r, pi - r, the sign of y). The
coefficients minimise the largest absolute error over t in [0, 1] by
iteratively reweighted least squares on a dense grid (Lawson's algorithm);
the fitted error is 4.9e-8, below the FP32 rounding of the result near pi/4.

    python pystamps_b200/csrc/make_atan_poly.py > pystamps_b200/csrc/atan_poly.h
"""
import numpy as np

N_COEF = 7


def lawson(deg: int = N_COEF, n: int = 6001, iters: int = 400) -> tuple[np.ndarray, float]:
    t = np.linspace(1e-9, 1.0, n)
    u = t * t
    A = np.vander(u, deg, increasing=True) * (t * u)[:, None]
    b = np.arctan(t) - t
    w = np.ones(n)
    c = np.zeros(deg)
    for _ in range(iters):
        c, *_ = np.linalg.lstsq(A * w[:, None], b * w, rcond=None)
        e = np.abs(A @ c - b)
        w = w * np.sqrt(e / e.max()) + 1e-15
        w /= w.max()
    return c, float(np.abs(A @ c - b).max())


def main() -> None:
    c, err = lawson()
    print("// Generated by make_atan_poly.py (minimax atan on [0, 1]; see that script).")
    print(f"// fitted max error: {err:.1e}")
    print("#pragma once")
    print("namespace ps2 {")
    for k, v in enumerate(c):
        print(f"constexpr float kAtanA{k + 1} = {np.float32(v):.9e}f;")
    print(f"constexpr float kHalfPiF = {np.float32(np.pi / 2):.9e}f;")
    print(f"constexpr float kPiF = {np.float32(np.pi):.9e}f;")
    print("}  // namespace ps2")


if __name__ == "__main__":
    main()
