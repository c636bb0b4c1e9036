"""Generates trial_interp_taps.h: the fractional-delay filters the FP32 topofit
uses to evaluate the trial sum between its samples.

The trial sum of a PS, centred on the middle of its phase-ramp band,
    T(m) = sum_c z_c exp(-j phi_c m),   |phi_c| <= pi/8,
(phi_c = (bp_c - mid) (pi/4) / range, mid the middle of the PS's bperp range)
is sampled at every 4th trial, m = 4k. For m = 4k + r, r = 1, 2, 3,
    T(4k + r) ~ sum_{i=-9}^{10} h_r[i] T(4(k + i)),
and the error is at most  sum_c |z_c| * max_{|phi| <= B} |H_r(phi) - exp(-j phi r)|
with H_r(phi) = sum_i h_r[i] exp(-j 4 phi i). The taps minimise that maximum over
B = pi/8 (1 + 1e-3) (a margin over FP32 rounding of the band edge) by
iteratively reweighted least squares on a dense frequency grid (Lawson's
algorithm for a minimax fit). The bound printed below is the achieved maximum
(about 8e-9 of sum |z_c|, under the FP32 rounding of the sum itself).

    python pystamps_b200/csrc/make_trial_interp_taps.py > pystamps_b200/csrc/trial_interp_taps.h
"""
import numpy as np

STRIDE = 4
TAP_LO, N_TAPS = -9, 20
BAND = np.pi / 8 * (1 + 1e-3)


def design(r: int, n_grid: int = 6001, iters: int = 200) -> tuple[np.ndarray, float]:
    phi = np.linspace(-BAND, BAND, n_grid)
    idx = np.arange(TAP_LO, TAP_LO + N_TAPS)
    A = np.exp(-1j * np.outer(phi, STRIDE * idx))
    b = np.exp(-1j * phi * r)
    Ar = np.vstack([A.real, A.imag])
    br = np.concatenate([b.real, b.imag])
    w = np.ones(br.size)
    h = np.zeros(N_TAPS)
    for _ in range(iters):
        h, *_ = np.linalg.lstsq(Ar * w[:, None], br * w, rcond=None)
        e = np.abs(A @ h - b)
        ee = np.concatenate([e, e])
        w = w * np.sqrt(ee / ee.max()) + 1e-15
        w /= w.max()
    h32 = h.astype(np.float32).astype(np.float64)
    return h32, float(np.abs(A @ h32 - b).max())


def main() -> None:
    rows, worst = [], 0.0
    for r in range(1, STRIDE):
        h, err = design(r)
        worst = max(worst, err)
        rows.append(h)
    print("// Generated by make_trial_interp_taps.py (fractional-delay filters for the")
    print("// trial sum sampled at every 4th trial; see that script for the design).")
    print(f"// max |H_r(phi) - exp(-j phi r)| over |phi| <= pi/8 (1 + 1e-3): {worst:.2e}")
    print("#pragma once")
    print("namespace ps2 {")
    print(f"constexpr int kTrialStride = {STRIDE};")
    print(f"constexpr int kInterpTapLo = {TAP_LO};")
    print(f"constexpr int kInterpTaps = {N_TAPS};")
    print(f"__constant__ float kInterpTaps_c[{STRIDE - 1}][{N_TAPS}] = {{")
    for h in rows:
        print("    {" + ", ".join(f"{v:.9e}f" for v in h) + "},")
    print("};")
    print("}  // namespace ps2")


if __name__ == "__main__":
    main()
