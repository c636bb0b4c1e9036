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
