"""Precision study: the FP32 path against the plain FP64 path, per gamma iteration.

Both paths run on the GPU from the same prepared patch; the FP64 path is the
FP64 reference (it matches the FP64 restatement of the reference loop to 1e-9).
For each iteration the study reports max / RMS |d gamma| and |d K| (rad/m and,
with K_m = K * lambda * rho * sin(inc) / (4 pi), metres of DEM error), both
free-running (each path on its own state) and, for iteration 1, where the two
states are identical by construction, the arithmetic difference alone.

    python -m pystamps_b200.precision [--workload B] [--iterations 8]
"""
from __future__ import annotations

import argparse
import json
import math

import numpy as np

from . import stage2 as S
from . import synth

ARGMAX_TIE_REL = 1e-6    # best and runner-up trial coherence this close (relative): an argmax tie
NEAR_TIE_FLOOR = 0.5     # FP32 near tie: within ARGMAX_TIE_REL of max(best, 0.5) but not an argmax
                         # tie: an FP32 trial coherence carries an error of roughly fixed size (its
                         # phasor and summation rounding over the columns), so below coherence 0.5 such
                         # rows (an absolute gap under 5e-7) flip as easily; counted separately
WRAP_TIE_RAD = 1e-4      # a refinement residual angle this close to +-pi: a wrap tie


def is_argmax_tie(best, second):
    """Best and runner-up trial coherence within ARGMAX_TIE_REL relative."""
    best = np.asarray(best, np.float64)
    return (best - np.asarray(second, np.float64)) <= ARGMAX_TIE_REL * np.maximum(best, 1e-30)


def is_fp32_tie(best, second):
    """Argmax ties and FP32 near ties: best and runner-up within ARGMAX_TIE_REL
    of max(best, NEAR_TIE_FLOOR). An FP32 evaluation of the trials may pick
    either (for example two trials at 0.23912255 and 0.23912231, 1.007e-6
    relative, of a 2,000,000 x 150 patch)."""
    best = np.asarray(best, np.float64)
    return (best - np.asarray(second, np.float64)) <= ARGMAX_TIE_REL * np.maximum(best, NEAR_TIE_FLOOR)


def trial_values(n_trial_wraps: float) -> np.ndarray:
    """The trial multipliers -ceil(8 n)..ceil(8 n) (native_stage2.rs:1305-1308)."""
    n = math.ceil(8.0 * n_trial_wraps)
    return np.arange(-n, n + 1, dtype=np.float64)


def trial_coherences(ph_nm, ph_patch, bperp, n_trial_wraps: float) -> np.ndarray:
    """FP64 statement of topofit's trial search (native_stage2.rs:1207-1257)
    for a few rows: coherence of every trial, [rows, trials]. psdph =
    conj(ph_patch) * ph_nm; a zero element takes no part (the reference's
    valid columns)."""
    z = np.conj(np.asarray(ph_patch, np.complex128)) * np.asarray(ph_nm, np.complex128)
    bp = np.broadcast_to(np.asarray(bperp, np.float64), z.shape)
    valid = z != 0
    big = np.where(valid, bp, -np.inf).max(axis=1)
    small = np.where(valid, bp, np.inf).min(axis=1)
    rng = big - small
    rng[~np.isfinite(rng) | (rng == 0)] = 1.0
    trials = trial_values(n_trial_wraps)
    denom = np.abs(z).sum(axis=1)
    denom[denom == 0] = 1.0
    theta = (bp / rng[:, None]) * (math.pi / 4)
    s = np.einsum("rc,rct->rt", z, np.exp(-1j * theta[:, :, None] * trials[None, None, :]))
    return np.abs(s) / denom[:, None]


def wrap_distance(ph_nm, ph_patch, bperp, n_trial_wraps: float, best_ix=None) -> np.ndarray:
    """Per row, min over interferograms of pi - |arg(res * conj(offset))| at
    the winning trial (refine_candidate, native_stage2.rs:1259-1303), FP64.
    best_ix: winning trial index per row (default: argmax of
    trial_coherences)."""
    z = np.asarray(ph_nm, np.complex128) * np.conj(np.asarray(ph_patch, np.complex128))
    bp = np.broadcast_to(np.asarray(bperp, np.float64), z.shape)
    rng = bp.max(axis=1) - bp.min(axis=1)
    rng[rng == 0] = 1.0
    if best_ix is None:
        best_ix = np.argmax(trial_coherences(ph_nm, ph_patch, bperp, n_trial_wraps), axis=1)
    k0 = (math.pi / 4) / rng * trial_values(n_trial_wraps)[best_ix]
    res = z * np.exp(-1j * k0[:, None] * bp)
    off = res.sum(axis=1)
    ang = np.angle(res * np.conj(off)[:, None])
    return (math.pi - np.abs(ang)).min(axis=1)


def classify_ties(ph_nm, ph_patch, bperp, n_trial_wraps: float) -> dict:
    """Tie classes of the given rows (few rows: every trial in FP64):
    argmax ties (best and runner-up trial within 1e-6 relative), FP32 near
    ties (within 1e-6 of max(best, 0.5) but not argmax ties) and
    wrap ties (a refinement residual angle within WRAP_TIE_RAD of +-pi). Rows
    that are neither are genuine FP32/FP64 differences."""
    ph_nm = np.atleast_2d(ph_nm)
    ph_patch = np.atleast_2d(ph_patch)
    bp = np.asarray(bperp, np.float64)
    bp = bp[None, :] if bp.ndim == 1 else np.atleast_2d(bp)
    if ph_nm.shape[0] == 0:
        e = np.zeros(0, bool)
        return {"argmax_tie": e, "near_tie": e, "wrap_tie": e, "tie": e}
    coh = trial_coherences(ph_nm, ph_patch, bp, n_trial_wraps)
    srt = np.sort(coh, axis=1)
    best = srt[:, -1]
    second = srt[:, -2] if coh.shape[1] > 1 else np.zeros(coh.shape[0])
    argmax_tie = is_argmax_tie(best, second)
    near_tie = is_fp32_tie(best, second) & ~argmax_tie
    wrap_tie = wrap_distance(ph_nm, ph_patch, bp, n_trial_wraps, np.argmax(coh, axis=1)) < WRAP_TIE_RAD
    return {"argmax_tie": argmax_tie, "near_tie": near_tie, "wrap_tie": wrap_tie,
            "tie": argmax_tie | near_tie | wrap_tie}


def study(prep: S.PreparedPatch, k_to_m: float, iterations: int = 8, device: int = 0) -> list[dict]:
    out = []
    with S.Stage2Context(device) as c32, S.Stage2Context(device) as c64:
        c32.load(prep, "fp32")
        c64.load(prep, "fp64")
        for it in range(1, iterations + 1):
            s32 = c32.iterate(1)[0]
            s64 = c64.iterate(1)[0]
            a = c32.download(["coh_ps", "K_ps"])
            b = c64.download(["coh_ps", "K_ps"])
            dg = np.abs(a["coh_ps"] - b["coh_ps"])
            ok = ~np.isnan(a["K_ps"]) & ~np.isnan(b["K_ps"])
            dk = np.abs(a["K_ps"][ok] - b["K_ps"][ok])
            out.append({
                "iteration": it,
                "gamma_change_fp32": s32["gamma_change_rms"], "gamma_change_fp64": s64["gamma_change_rms"],
                "dgamma_max": float(dg.max()), "dgamma_rms": float(np.sqrt(np.mean(dg * dg))),
                "dgamma_p99": float(np.quantile(dg, 0.99)), "frac_dgamma_le_1e-4": float(np.mean(dg <= 1e-4)),
                "dK_max_rad_per_m": float(dk.max()), "dK_rms_rad_per_m": float(np.sqrt(np.mean(dk * dk))),
                "dK_max_m": float(dk.max() * k_to_m), "dK_rms_m": float(np.sqrt(np.mean(dk * dk)) * k_to_m),
                "frac_dK_le_1e-3_m": float(np.mean(dk * k_to_m <= 1e-3)),
            })
    return out


def main() -> None:
    ap = argparse.ArgumentParser()
    ap.add_argument("--workload", default="B")
    ap.add_argument("--iterations", type=int, default=8)
    a = ap.parse_args()
    w = synth.ALIASES.get(a.workload) or synth.WORKLOADS[a.workload]
    patch = synth.make_workload(w)
    lam = float(patch["parms"]["lambda"])
    k_to_m = lam * S.RHO * math.sin(float(patch["mean_incidence"])) / (4 * math.pi)
    prep = S.prepare_patch(patch)
    rows = study(prep, k_to_m, a.iterations)
    print(json.dumps({"workload": w.name, "n_ps": prep.n_ps, "n_ifg": prep.n_ifg, "k_to_m": k_to_m,
                      "per_iteration": rows}))


if __name__ == "__main__":
    main()
