"""Generate the golden fixtures in this folder from the runnable Python reference.

Run in a checkout that has the pySTAMPS reference importable (its path is given
with --reference); the fixtures are committed so the tests never need it:

    python tests/golden/make_golden.py --reference /path/to/pystamps

Fixtures (all seeded):

* clap_grid.npz       -- pystamps.pipeline.ported._clap_filt_grid_stack_prepared
                         on the 37x53x3 grid of the reference's own CLAP test
                         (tests/test_stage2_ported.py:910-960) and on a 64x64x4
                         grid with the stage-2 Butterworth low pass; complex64
                         and preserve_precision (complex128) outputs.
* topofit_rows.npz    -- ported._ps_topofit_single in complex128 on 96 random
                         rows of 20 interferograms (row-variant bperp), with the
                         number of near-max candidates per row so the test can
                         skip rows where the Python near-max rule (tolerance
                         2e-4) differs from the Rust first-argmax rule.
* stage2_iter1.npz    -- ported.stage2_estimate_gamma(kernel_backend="python")
                         on a 3,000 PS x 10 ifg synthetic patch, one iteration
                         (gamma_max_iterations=1, so the random-phase histogram
                         does not enter), written as pm1.mat and re-read: the
                         19 pm1 variables as stored (shapes, dtypes) and the
                         parms the patch was written with.
* stage2_3ps.npz      -- the same entry point on the reference's 3-PS fixture
                         (native_stage2.rs:2698-2769: empty CLAP, all rows
                         invalid).
* stage3_units.npz    -- ported._clap_filt_patch on seeded 32x32 patches
                         (alpha 1 and 1.7, one patch with a zeroed cell and a
                         NaN), ported._ps_topofit_single in the stage-3 form
                         (complex64 unit phasors, f32 bperp) on 128 rows, and
                         ported._coh_threshold_from_dist for both selection
                         methods.
* registry_kernels.npz -- the registry kernels stage2_topofit,
                         stage2_topofit_row_invariant,
                         stage2_topofit_coh_row_invariant and stage2_histogram
                         (pystamps/kernels/accelerated.py:410-509) with the
                         python provider, on the reference's own random case, on
                         seeded 400 x 40 rows with zero columns and on 160 rows
                         with two near-equal peaks (several near-max
                         candidates), in complex64 and complex128.
* stage3_select.npz   -- ported.stage3_select_ps after the Python stage 2 on a
                         10,000 PS x 8 ifg patch over a 40 x 40 grid: the
                         select1.mat variables (ix, keep_ix, ph_patch2,
                         ph_res2, K_ps2, C_ps2, coh_ps2, coh_thresh, ...)
                         with the pm1.mat inputs they came from.
"""
from __future__ import annotations

import argparse
import math
import os
import sys
import tempfile
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent


def _import_reference(ref: Path):
    sys.path.insert(0, str(ref))
    from pystamps.pipeline import ported  # noqa: E402

    return ported


def make_clap(ported) -> None:
    rng = np.random.default_rng(0)
    g1 = (rng.standard_normal((37, 53, 3)) + 1j * rng.standard_normal((37, 53, 3))).astype(np.complex64)
    lp1 = np.full((32, 32), 0.01, dtype=np.float64)
    prep1 = ported._prepare_clap_filt_grid_stack(g1.shape, n_win=24, n_pad=8, low_pass=lp1)
    o1 = ported._clap_filt_grid_stack_prepared(g1, alpha=1.0, beta=0.3, prepared=prep1)
    o1d = ported._clap_filt_grid_stack_prepared(g1, alpha=1.0, beta=0.3, prepared=prep1, preserve_precision=True)

    rng = np.random.default_rng(11)
    ph = np.exp(1j * rng.uniform(-np.pi, np.pi, (64, 64, 4)))
    amp = rng.uniform(0.0, 3.0, (64, 64, 1))
    g2 = (ph * amp).astype(np.complex64)
    g2[5, 7, :] = 0
    opts = ported.StageOptions() if hasattr(ported, "StageOptions") else None
    n_win = 32
    freq0 = 1.0 / 800.0
    freq_i = np.arange(-n_win / 2, n_win / 2) / float(50.0 * n_win)
    butter = 1.0 / (1.0 + (freq_i / freq0) ** (2 * 5))
    lp2 = np.fft.fftshift(np.outer(butter, butter)).astype(np.float64)
    del opts
    prep2 = ported._prepare_clap_filt_grid_stack(g2.shape, n_win=24, n_pad=8, low_pass=lp2)
    o2 = ported._clap_filt_grid_stack_prepared(g2, alpha=1.0, beta=0.3, prepared=prep2)
    o2d = ported._clap_filt_grid_stack_prepared(g2, alpha=1.0, beta=0.3, prepared=prep2, preserve_precision=True)
    # alpha != 1 exercises the powf branch
    o3 = ported._clap_filt_grid_stack_prepared(g2, alpha=1.7, beta=0.45, prepared=prep2, preserve_precision=True)
    np.savez_compressed(
        HERE / "clap_grid.npz",
        g1=g1, lp1=lp1, out1=o1, out1_f64=o1d,
        g2=g2, lp2=lp2, out2=o2, out2_f64=o2d, out3_f64=o3,
    )


def make_topofit(ported) -> None:
    rng = np.random.default_rng(21)
    n_row, n_col = 96, 20
    bp_ifg = rng.uniform(-300, 300, n_col)
    grad = 1.0 + 0.02 * rng.uniform(-0.5, 0.5, n_row)
    bperp = (grad[:, None] * bp_ifg[None, :]).astype(np.float64)
    n_trial_wraps = 4.94
    k_true = rng.uniform(-0.04, 0.04, n_row)
    noise = rng.normal(0.0, rng.uniform(0.1, 1.5, n_row)[:, None], (n_row, n_col))
    cpx = np.exp(1j * (k_true[:, None] * bperp + noise)) * rng.uniform(0.5, 1.5, (n_row, n_col))
    cpx = cpx.astype(np.complex128)
    K = np.empty(n_row); C = np.empty(n_row); coh = np.empty(n_row)
    res = np.empty((n_row, n_col), np.complex128)
    n_cand = np.empty(n_row, np.int64)
    for r in range(n_row):
        k, c, h, pr = ported._ps_topofit_single(cpx[r], bperp[r], n_trial_wraps)
        K[r], C[r], coh[r] = k, c, h
        res[r] = pr
        # count near-max candidates exactly as the Python rule does
        bp = bperp[r]
        rngb = float(bp.max() - bp.min()) or 1.0
        tm = ported._stage2_trial_values(n_trial_wraps)
        tp = bp / rngb * (np.pi / 4.0)
        ct = np.abs(np.sum(np.exp(-1j * (tp[:, None] * tm[None, :])) * cpx[r][:, None], axis=0))
        ct = ct / np.sum(np.abs(cpx[r]))
        n_cand[r] = ported._ps_topofit_near_max_trial_indices(ct).size
    np.savez_compressed(HERE / "topofit_rows.npz", cpx=cpx, bperp=bperp, n_trial_wraps=n_trial_wraps,
                        K=K, C=C, coh=coh, residual=res, n_candidates=n_cand)


def _write_patch(ported, patch: Path, p: dict) -> None:
    from scipy.io import savemat

    patch.mkdir(parents=True, exist_ok=True)
    n_ps, n_full = p["ph"].shape
    savemat(patch / "ps1.mat", {
        "n_ps": float(n_ps), "n_ifg": float(n_full), "n_image": float(n_full), "master_ix": float(p["master_ix"]),
        "bperp": p["bperp"].reshape(1, -1), "xy": p["xy"], "mean_incidence": float(p["mean_incidence"]),
    })
    savemat(patch / "ph1.mat", {"ph": p["ph"]})
    if p.get("bperp_mat") is not None:
        savemat(patch / "bp1.mat", {"bperp_mat": np.asarray(p["bperp_mat"], dtype=np.float64)})
    if p.get("D_A") is not None:
        savemat(patch / "da1.mat", {"D_A": np.asarray(p["D_A"], dtype=np.float64).reshape(-1, 1)})
    if p.get("inc") is not None:
        savemat(patch / "inc1.mat", {"inc": np.asarray(p["inc"], dtype=np.float64).reshape(-1, 1)})
    if p.get("la") is not None:
        savemat(patch / "la1.mat", {"la": np.asarray(p["la"], dtype=np.float64).reshape(-1, 1)})
    savemat(patch / "parms.mat", p["parms"])


def _run_python_stage2(ported, p: dict) -> dict:
    from scipy.io import loadmat

    with tempfile.TemporaryDirectory() as tmp:
        os.environ["HOME"] = tmp  # the reference caches its random histogram under ~/.cache
        patch = Path(tmp) / "PATCH_1"
        _write_patch(ported, patch, p)
        ported.stage2_estimate_gamma(patch, kernel_backend="python")
        pm = loadmat(patch / "pm1.mat")
    keys = ["K_ps", "C_ps", "coh_ps", "N_opt", "ph_res", "ph_patch", "ph_grid", "ph_weight", "grid_ij",
            "n_trial_wraps", "i_loop", "coh_ps_save", "gamma_change_save", "low_pass", "grid_size", "Nr",
            "Nr_max_nz_ix", "coh_bins", "step_number"]
    return {k: np.asarray(pm[k]) for k in keys if k in pm}


def make_stage2_iter1(ported) -> None:
    sys.path.insert(0, str(HERE.parents[1]))
    from pystamps_b200 import synth

    p = synth.make_patch(3000, 10, 31, 21, seed=777, max_topo_err=20.0, gamma_max_iterations=1)
    p["inc"] = np.full(p["ph"].shape[0], p["mean_incidence"])
    pm = _run_python_stage2(ported, p)
    np.savez_compressed(
        HERE / "stage2_iter1.npz",
        ph=p["ph"], bperp=p["bperp"], bperp_mat=p["bperp_mat"], D_A=p["D_A"], xy=p["xy"],
        mean_incidence=p["mean_incidence"], max_topo_err=20.0,
        parms_keys=np.asarray(list(p["parms"].keys())),
        parms_values=np.asarray([str(v) for v in p["parms"].values()]),
        **{"pm_" + k: v for k, v in pm.items()},
    )


def make_stage2_3ps(ported) -> None:
    inc = math.radians(23.0)
    p = {
        "ph": np.asarray([[1.0, 0.8 + 0.2j, 0.6 + 0.4j], [1.0, 0.7 + 0.3j, 0.5 + 0.5j], [1.0, 0.9 + 0.1j, 0.4 + 0.6j]],
                         dtype=np.complex64),
        "bperp": np.asarray([0.0, 15.0, 30.0]),
        "master_ix": 1,
        "bperp_mat": np.asarray([[15.0, 30.0]] * 3),
        "D_A": np.ones(3),
        "xy": np.asarray([[1, 0, 0], [2, 5, 5], [3, 10, 10]], dtype=np.float32),
        "mean_incidence": inc,
        "la": np.full(3, inc),
        "parms": {"gamma_max_iterations": 1.0, "filter_grid_size": 50.0},
    }
    pm = _run_python_stage2(ported, p)
    np.savez_compressed(HERE / "stage2_3ps.npz", **{"pm_" + k: v for k, v in pm.items()})


def make_stage3_units(ported) -> None:
    rng = np.random.default_rng(31)
    n_win = 32
    freq0 = 1.0 / 800.0
    freq_i = np.arange(-n_win / 2, n_win / 2) / float(50.0 * n_win)
    butter = 1.0 / (1.0 + (freq_i / freq0) ** (2 * 5))
    lp = np.fft.fftshift(np.outer(butter, butter)).astype(np.float64)
    patches, outs, params = [], [], []
    for k, (alpha, beta) in enumerate([(1.0, 0.3), (1.7, 0.45), (1.0, 0.3), (0.8, 0.5)]):
        amp = rng.uniform(0.0, 4.0, (32, 32))
        g = amp * np.exp(1j * (rng.uniform(-np.pi, np.pi, (32, 32)) + 0.2 * np.arange(32)[None, :]))
        if k == 2:
            g[9, 14] = 0
            g[3, 3] = np.nan
        patches.append(g)
        outs.append(ported._clap_filt_patch(g, alpha, beta, lp))
        params.append((alpha, beta))
    # topofit rows in the stage-3 form: normalised psdph (complex64), f32 bperp
    n_row, n_col = 128, 24
    bp_ifg = rng.uniform(-300, 300, n_col)
    grad = 1.0 + 0.02 * rng.uniform(-0.5, 0.5, n_row)
    bperp = (grad[:, None] * bp_ifg[None, :]).astype(np.float32)
    n_trial_wraps = 7.44
    k_true = rng.uniform(-0.04, 0.04, n_row)
    noise = rng.normal(0.0, rng.uniform(0.1, 1.8, n_row)[:, None], (n_row, n_col))
    cpx = np.exp(1j * (k_true[:, None] * bperp + noise)).astype(np.complex64)
    cpx[5, 3] = 0  # a zero column is skipped by _ps_topofit_single
    K = np.empty(n_row); C = np.empty(n_row); coh = np.empty(n_row)
    res = np.empty((n_row, n_col), np.complex64)
    for r in range(n_row):
        k, c, h, pr = ported._ps_topofit_single(cpx[r], bperp[r], n_trial_wraps)
        K[r], C[r], coh[r] = k, c, h
        res[r] = pr
    # coherence thresholds from the distribution
    n = 30000
    coh_v = np.clip(np.concatenate([rng.beta(2, 5, 21000), rng.beta(8, 2, 9000)]), 0, 1)
    coh_v[::997] = np.nan
    d_a = rng.uniform(0.2, 0.6, n)
    d_s = np.sort(d_a)
    d_max = np.concatenate(([0.0], d_s[2000:n - 2000:2000], [d_s[-1]]))
    centers = np.arange(0.005, 1.0, 0.01)
    nr = np.exp(-0.5 * ((centers - 0.25) / 0.1) ** 2) * 3000
    th = {}
    for meth, mpr in (("DENSITY", 40.0), ("PERCENT", 5.0)):
        t, cf = ported._coh_threshold_from_dist(coh_values=coh_v, D_A=d_a, D_A_max=d_max, coh_bins=centers,
                                                Nr_dist=nr, low_coh_thresh=31, max_percent_rand=mpr,
                                                select_method=meth)
        th[meth] = (mpr, t, np.asarray(cf, dtype=np.float64))
    np.savez_compressed(
        HERE / "stage3_units.npz",
        clap_in=np.stack(patches), clap_out=np.stack(outs), clap_params=np.asarray(params), low_pass=lp,
        topo_cpx=cpx, topo_bperp=bperp, topo_ntw=n_trial_wraps, topo_K=K, topo_C=C, topo_coh=coh, topo_res=res,
        th_coh=coh_v, th_da=d_a, th_damax=d_max, th_centers=centers, th_nr=nr,
        th_density_mpr=th["DENSITY"][0], th_density=th["DENSITY"][1], th_density_cf=th["DENSITY"][2],
        th_percent_mpr=th["PERCENT"][0], th_percent=th["PERCENT"][1], th_percent_cf=th["PERCENT"][2],
    )


def make_stage3_select(ported) -> None:
    from scipy.io import loadmat

    sys.path.insert(0, str(HERE.parents[1]))
    from pystamps_b200 import synth

    p = synth.make_patch(10000, 8, 40, 41, seed=909, max_topo_err=20.0, gamma_max_iterations=4, n_rand=20000)
    p["inc"] = np.full(p["ph"].shape[0], p["mean_incidence"])
    p["parms"].update({"select_method": "DENSITY", "density_rand": 20.0, "slc_osf": 1.0,
                       "gamma_stdev_reject": 0.0})
    with tempfile.TemporaryDirectory() as tmp:
        os.environ["HOME"] = tmp
        patch = Path(tmp) / "PATCH_1"
        _write_patch(ported, patch, p)
        ported.stage2_estimate_gamma(patch, kernel_backend="python")
        ported.stage3_select_ps(patch)
        pm = loadmat(patch / "pm1.mat")
        sel = loadmat(patch / "select1.mat")
    pm_keys = ["K_ps", "C_ps", "coh_ps", "ph_res", "ph_patch", "ph_grid", "grid_ij", "n_trial_wraps", "Nr",
               "coh_bins", "low_pass"]
    sel_keys = ["ix", "keep_ix", "ph_patch2", "ph_res2", "K_ps2", "C_ps2", "coh_ps2", "coh_thresh",
                "coh_thresh_coeffs", "max_percent_rand", "ifg_index"]
    np.savez_compressed(
        HERE / "stage3_select.npz",
        ph=p["ph"], bperp=p["bperp"], bperp_mat=p["bperp_mat"], D_A=p["D_A"], xy=p["xy"],
        **{"pm_" + k: np.asarray(pm[k]) for k in pm_keys if k in pm},
        **{"sel_" + k: np.asarray(sel[k]) for k in sel_keys if k in sel},
    )


def make_registry(ported) -> None:
    """The reference's stage-2 registry kernels with the python provider
    (pystamps/kernels/accelerated.py:410-509): topofit (generic and
    row-invariant, complex64 and complex128 inputs, rows with zero columns and
    an all-zero row), the row-invariant coherence and the histogram."""
    from pystamps.kernels import accelerated as accel

    out = {}
    # the random case of the reference's native-vs-python test (tests/test_kernels_accelerated.py:666-713)
    rng = np.random.default_rng(11)
    out["t0_cpx"] = np.exp(1j * rng.normal(size=(6, 5))).astype(np.complex128)
    out["t0_bp"] = rng.normal(size=(6, 5)).astype(np.float64)
    out["t0_bprow"] = np.tile(np.asarray([-120.0, -40.0, 0.0, 55.0, 90.0]), (6, 1))
    out["t0_ntw"] = np.float64(1.5)
    # larger seeded rows: 400 x 40, row-variant bperp, trial count 81
    rng = np.random.default_rng(77)
    n, m = 400, 40
    bp_ifg = rng.uniform(-300, 300, m)
    bp = (1.0 + 0.02 * rng.uniform(-0.5, 0.5, n))[:, None] * bp_ifg[None, :]
    k = rng.uniform(-0.04, 0.04, n)
    cpx = np.exp(1j * (k[:, None] * bp + rng.normal(0.0, rng.uniform(0.1, 1.5, n)[:, None], (n, m))))
    cpx *= rng.uniform(0.5, 1.5, (n, m))
    cpx[rng.random((n, m)) < 0.03] = 0
    cpx[5] = 0
    out["t1_cpx"] = cpx.astype(np.complex128)
    out["t1_bp"] = bp.astype(np.float64)
    out["t1_ntw"] = np.float64(4.94)
    # rows with two peaks of nearly equal height: antisymmetric bperp per row
    # and two opposite phase ramps, the second weaker by up to 1e-4, so the
    # trials +m and -m are local maxima within 2e-4 of each other (both refined,
    # the better one kept); the last rows put the ramps at the end trials
    # (-n, +n), the case the reference settles by the coarse coherence
    rng = np.random.default_rng(78)
    n, m = 160, 40
    half = np.sort(rng.uniform(5.0, 300.0, m // 2))
    b = np.concatenate([-half[::-1], half])
    bp = (1.0 + 0.02 * rng.uniform(-0.5, 0.5, n))[:, None] * b[None, :]
    q = (np.pi / 4) / (bp.max(axis=1) - bp.min(axis=1))
    n_half = int(np.ceil(8 * 4.94))
    mstar = rng.integers(3, 30, n) + rng.uniform(-0.2, 0.2, n)
    mstar[-8:] = n_half
    a2 = 1.0 - rng.uniform(1e-6, 1e-4, n)
    ph = (q * mstar)[:, None] * bp
    cpx = np.exp(1j * ph) + a2[:, None] * np.exp(-1j * ph)
    cpx += 1e-7 * (rng.standard_normal((n, m)) + 1j * rng.standard_normal((n, m)))
    out["t2_cpx"] = cpx.astype(np.complex128)
    out["t2_bp"] = bp.astype(np.float64)
    out["t2_ntw"] = np.float64(4.94)
    for name in ("t0", "t1", "t2"):
        c128, b64, ntw = out[name + "_cpx"], out[name + "_bp"], float(out[name + "_ntw"])
        brow = out.get(name + "_bprow", np.tile(b64[0], (b64.shape[0], 1)))
        for prec, c, b, br in (("d", c128, b64, brow), ("s", c128.astype(np.complex64), b64.astype(np.float32),
                                                        brow.astype(np.float32))):
            K, C, coh, res = accel.run_stage2_topofit_kernel(c, b, ntw, backend="python")
            out.update({f"{name}{prec}_gen_K": K, f"{name}{prec}_gen_C": C, f"{name}{prec}_gen_coh": coh,
                        f"{name}{prec}_gen_res": res})
            K, C, coh, res = accel.run_stage2_topofit_row_invariant_kernel(c, br, ntw, backend="python")
            out.update({f"{name}{prec}_row_K": K, f"{name}{prec}_row_C": C, f"{name}{prec}_row_coh": coh,
                        f"{name}{prec}_row_res": res})
        out[name + "_cohrow"] = accel.run_stage2_topofit_coh_row_invariant_kernel(c128, brow, ntw, backend="python")
    # histogram: the reference's case, the 100 coherence centres, unequal centres, one centre
    rng = np.random.default_rng(5)
    cases = {
        "h0": (np.asarray([0.1, 0.49, 0.7, 0.9, np.nan]), np.asarray([0.0, 0.5, 1.0])),
        "h1": (np.concatenate([rng.random(10_000), [np.nan, np.inf, -0.3, 1.7, 0.005, 0.995]]),
               0.005 + 0.01 * np.arange(100)),
        "h2": (rng.normal(0.0, 2.0, 5_000), np.asarray([-3.0, -1.0, -0.5, 0.0, 0.25, 2.0, 5.0])),
        "h3": (rng.random(100), np.asarray([0.5])),
    }
    for name, (v, c) in cases.items():
        out[name + "_v"], out[name + "_c"] = v, c
        out[name + "_out"] = accel.run_stage2_histogram_kernel(v, c, backend="python")
    np.savez_compressed(HERE / "registry_kernels.npz", **out)


def main() -> None:
    ap = argparse.ArgumentParser()
    ap.add_argument("--reference", required=True, type=Path)
    ap.add_argument("--only", default="")
    a = ap.parse_args()
    ported = _import_reference(a.reference)
    todo = {"clap": make_clap, "topofit": make_topofit, "iter1": make_stage2_iter1, "3ps": make_stage2_3ps,
            "stage3_units": make_stage3_units, "stage3_select": make_stage3_select, "registry": make_registry}
    for name, fn in todo.items():
        if a.only and name not in a.only.split(","):
            continue
        fn(ported)
        print("wrote", name)


if __name__ == "__main__":
    main()
