"""Generates sincos_poly.h: the polynomial coefficients of the FP32 phase-ramp
sin/cos of the binning (sincos_cw in ps2_device.cuh).

After reduction by pi/2 (Cody and Waite's method, "Software Manual for the
Elementary Functions", 1980: x - k pi/2 with pi/2 split into three FP32 parts)
the reduced argument r lies in [-pi/4, pi/4], u = r^2, and
    sin r = r + r u (S1 + u (S2 + u S3)),
    cos r = 1 - u/2 + u^2 (Q1 + u (Q2 + u Q3)).
The coefficients minimise the largest error of sin r and cos r over
u in [0, (pi/4)^2] (weighted so it is the error of the function itself), by
iteratively reweighted least squares on a dense grid (Lawson's algorithm).
Fitted errors: 3.6e-9 for sin, 1e-10 for cos, both below FP32 rounding; with
the FP32 arithmetic the largest absolute error of sin x and cos x is 9.2e-8
for |x| up to 5000 (checked against float64 in the comment the script prints).

    python pystamps_b200/csrc/make_sincos_poly.py > pystamps_b200/csrc/sincos_poly.h
"""
import numpy as np

U_MAX = (np.pi / 4) ** 2


def lawson(f, w, deg: int = 2, n: int = 4001, iters: int = 300) -> tuple[np.ndarray, float]:
    u = np.linspace(1e-12, U_MAX * 1.0001, n)
    A = np.vander(u, deg + 1, increasing=True)
    b, wt = f(u), w(u)
    ww = np.ones(n)
    c = np.zeros(deg + 1)
    for _ in range(iters):
        c, *_ = np.linalg.lstsq(A * (wt * ww)[:, None], b * wt * ww, rcond=None)
        e = np.abs((A @ c - b) * wt)
        ww = ww * np.sqrt(e / e.max()) + 1e-15
        ww /= ww.max()
    return c, float(np.abs((A @ c - b) * wt).max())


def main() -> None:
    cs, es = lawson(lambda u: (np.sin(np.sqrt(u)) / np.sqrt(u) - 1) / u, lambda u: u)
    cc, ec = lawson(lambda u: (np.cos(np.sqrt(u)) - 1 + u / 2) / u ** 2, lambda u: u ** 2)
    half_pi = np.pi / 2
    c1 = np.float32(half_pi)
    c2 = np.float32(half_pi - np.float64(c1))
    c3 = np.float32(half_pi - np.float64(c1) - np.float64(c2))
    print("// Generated by make_sincos_poly.py (minimax sin/cos on [-pi/4, pi/4] after")
    print("// Cody-Waite reduction by pi/2; see that script for the design).")
    print(f"// fitted max error: sin {es:.1e}, cos {ec:.1e}")
    print("#pragma once")
    print("namespace ps2 {")
    for name, v in (("kSinS1", cs[0]), ("kSinS2", cs[1]), ("kSinS3", cs[2]),
                    ("kCosQ1", cc[0]), ("kCosQ2", cc[1]), ("kCosQ3", cc[2]),
                    ("kHalfPi1", c1), ("kHalfPi2", c2), ("kHalfPi3", c3),
                    ("kTwoOverPi", np.float32(2 / np.pi))):
        print(f"constexpr float {name} = {np.float32(v):.9e}f;")
    print("}  // namespace ps2")


if __name__ == "__main__":
    main()
