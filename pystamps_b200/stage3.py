"""Stage-3 PS selection with the re-estimate on the GPU.

The reference's stage3_select_ps (pystamps/pipeline/ported.py:4328-4620):
coherence thresholds from the random-phase distribution per amplitude-
dispersion bin (_coh_threshold_from_dist, :2274-2348), the initial selection,
the optional bootstrap rejection, then the re-estimate of every selected PS
(:4429-4575) — the hot part, run by ps3_reestimate on the GPU: per PS cell a
32x32 CLAP patch filter with the cell zeroed, then the stage-3 topofit — and
the final keep mask. The threshold statistics are a few histograms over the
PS and run on the host (numpy), as in the reference.
"""
from __future__ import annotations

import ctypes
import math
from pathlib import Path

import numpy as np

from . import _lib
from ._lib import check, ptr

NEAR_MAX_COH_TOL = 2.0e-4  # ported.py:47


class Stage3Error(RuntimeError):
    """Raised for inputs the stage-3 path cannot use."""


# ----------------------------------------------------------- thresholds -----
def hist_with_centers(values, centers) -> np.ndarray:
    """ported._hist_with_centers (ported.py:594-604): nearest-centre counts
    (ties to the lower centre)."""
    centers = np.asarray(centers, dtype=np.float64).reshape(-1)
    values = np.asarray(values, dtype=np.float64).reshape(-1)
    if centers.size == 0:
        return np.asarray([], dtype=np.float64)
    if centers.size == 1:
        return np.asarray([float(values.size)], dtype=np.float64)
    mids = (centers[:-1] + centers[1:]) / 2.0
    ix = np.clip(np.searchsorted(mids, values, side="left"), 0, centers.size - 1)
    return np.bincount(ix, minlength=centers.size).astype(np.float64)


def polyfit_eval_centered(x, y, deg: int, x_eval: float) -> float:
    """Least-squares polynomial on centred and scaled x, evaluated at x_eval
    (ported.py:969-981, MATLAB polyfit with [p, S, mu])."""
    x = np.asarray(x, dtype=np.float64).reshape(-1)
    y = np.asarray(y, dtype=np.float64).reshape(-1)
    if x.size == 0 or y.size == 0:
        return math.nan
    mu0 = float(np.mean(x))
    mu1 = float(np.std(x, ddof=1)) if x.size > 1 else 1.0
    if not np.isfinite(mu1) or mu1 == 0:
        mu1 = 1.0
    coeff = np.polyfit((x - mu0) / mu1, y, deg)
    return float(np.polyval(coeff, (float(x_eval) - mu0) / mu1))


def coh_threshold_from_dist(coh_values, D_A, D_A_max, coh_bins, Nr_dist, low_coh_thresh: int,
                            max_percent_rand: float, select_method: str) -> tuple[np.ndarray, np.ndarray]:
    """Per-PS coherence threshold (ported.py:2274-2348): in each D_A bin the
    random-phase histogram Nr, scaled to the low-coherence part of the PS
    histogram, gives the fraction (PERCENT) or count (DENSITY) of random PS
    above each coherence; a cubic through the six bins around the
    max_percent_rand crossing gives the bin's minimum coherence; a line in
    D_A across bins (if it rises) gives every PS its threshold."""
    coh_values = np.asarray(coh_values, dtype=np.float64).reshape(-1)
    D_A = np.asarray(D_A, dtype=np.float64).reshape(-1)
    D_A_max = np.asarray(D_A_max, dtype=np.float64).reshape(-1)
    Nr_dist = np.asarray(Nr_dist, dtype=np.float64).reshape(-1)
    nb = D_A_max.size - 1
    min_coh = np.full(nb, np.nan)
    D_A_mean = np.full(nb, np.nan)
    for i in range(nb):
        in_bin = (D_A > D_A_max[i]) & (D_A <= D_A_max[i + 1])
        if not np.any(in_bin):
            continue
        chunk = coh_values[in_bin]
        chunk = chunk[np.isfinite(chunk) & (chunk != 0)]
        if chunk.size == 0:
            continue
        D_A_mean[i] = float(np.mean(D_A[in_bin]))
        Na = hist_with_centers(chunk, coh_bins)
        low = min(low_coh_thresh, Na.size)
        den = np.sum(Nr_dist[:low])
        scale = np.sum(Na[:low]) / den if den > 0 else 1.0
        Nr = Nr_dist * scale
        Na1 = Na.copy()
        Na1[Na1 == 0] = 1.0
        if select_method.upper() == "PERCENT":
            pr = np.flip(np.cumsum(np.flip(Nr)) / np.cumsum(np.flip(Na1)) * 100.0)
        else:
            pr = np.flip(np.cumsum(np.flip(Nr)))
        ok = np.where(pr < max_percent_rand)[0]
        if ok.size == 0:
            min_coh[i] = 1.0
            continue
        first = int(ok.min()) + 1
        lo = first - 3
        if lo <= 0:
            continue
        hi = min(first + 2, 100)
        xs = pr[lo - 1:hi]
        ys = np.arange(lo, hi + 1, dtype=np.float64) * 0.01
        if xs.size < 4:
            continue
        min_coh[i] = polyfit_eval_centered(xs, ys, 3, max_percent_rand)
    valid = ~np.isnan(min_coh) & ~np.isnan(D_A_mean)
    if np.sum(valid) < 1:
        thresh = np.full_like(coh_values, 0.3)
        coeffs = np.asarray([], dtype=np.float64)
    else:
        mc, dm = min_coh[valid], D_A_mean[valid]
        if mc.size > 1:
            c = np.polyfit(dm, mc, 1)
            if c[0] > 0:
                thresh = np.polyval(c, D_A)
                coeffs = c.astype(np.float64)
            else:
                thresh = np.full_like(coh_values, float(np.polyval(c, 0.35)))
                coeffs = np.asarray([], dtype=np.float64)
        else:
            thresh = np.full_like(coh_values, float(mc[0]))
            coeffs = np.asarray([], dtype=np.float64)
    thresh[thresh < 0] = 0.0
    return thresh, coeffs


def da_bins(D_A) -> tuple[np.ndarray, np.ndarray]:
    """(D_A used, bin edges): bins of 10,000 PS (2,000 under 50,000 PS); under
    10,000 PS a single bin with D_A = 1 (ported.py:4356-4364)."""
    D_A = np.asarray(D_A, dtype=np.float64).reshape(-1)
    if D_A.size >= 10000:
        s = np.sort(D_A)
        b = 10000 if D_A.size >= 50000 else 2000
        return D_A, np.concatenate(([0.0], s[b:D_A.size - b:b], [s[-1]]))
    return np.ones_like(D_A), np.asarray([0.0, 1.0])


def max_percent_rand(select_method: str, percent_rand: float, density_rand: float, xy, n_bins: int) -> float:
    """ported.py:4368-4378: PERCENT takes percent_rand; DENSITY scales
    density_rand (per km^2) by the patch area per D_A bin."""
    if select_method.upper() == "PERCENT":
        return float(percent_rand)
    xy = np.asarray(xy, dtype=np.float64)
    area = 1.0
    if xy.size:
        area = float(np.prod(np.max(xy[:, 1:3], axis=0) - np.min(xy[:, 1:3], axis=0)) / 1e6)
        if area <= 0:
            area = 1.0
    return float(density_rand) * area / max(1, n_bins)


# ----------------------------------------------------------- re-estimate ----
def reestimate(ph_grid, grid_ij, sel, ph_work, bperp_mat, fit_ifg, *, clap_alpha: float, clap_beta: float,
               low_pass, n_trial_wraps: float, slc_osf: int = 1, clap_win: int = 32, device: int = 0,
               ph_cols=None) -> dict:
    """The stage-3 re-estimate (ported.py:4489-4550) of rows `sel` (0-based)
    on the GPU. grid_ij: pm1.grid_ij of all PS (1-based); ph_work: the
    interferograms without the master column (or, with ph_cols, ph1.ph whole
    and ph_cols its interferogram columns: only the selected rows are then
    gathered); fit_ifg: 0-based columns."""
    sel = np.asarray(sel, dtype=np.int64).reshape(-1)
    gij_all = np.asarray(grid_ij).reshape(-1, 2)
    g = np.ascontiguousarray(ph_grid, dtype=np.complex64)
    if g.ndim != 3:
        raise Stage3Error(f"ph_grid must be [n_i, n_j, n_ifg], got shape {g.shape}")
    m = g.shape[2]
    ph_w = np.asarray(ph_work)
    n_work = ph_w.shape[1] if ph_cols is None else len(ph_cols)
    if n_work != m:
        raise Stage3Error(f"ph has {n_work} interferograms but ph_grid has {m}")
    n = sel.size
    lp = np.ascontiguousarray(low_pass, dtype=np.float64)
    if lp.shape != (clap_win, clap_win):
        raise Stage3Error(f"low_pass must be {clap_win}x{clap_win}, got {lp.shape}")
    rows = ph_w[sel] if ph_cols is None else ph_w[np.ix_(sel, np.asarray(ph_cols, dtype=np.int64))]
    ph_s = np.ascontiguousarray(rows, dtype=np.complex64)
    bp_s = np.ascontiguousarray(np.asarray(bperp_mat)[sel], dtype=np.float32)
    gij = np.ascontiguousarray(np.rint(gij_all[sel]), dtype=np.int64)
    fit = np.ascontiguousarray(fit_ifg, dtype=np.int64)
    d = _lib.S3Desc()
    d.n_sel, d.n_ifg = n, m
    d.ph, d.bperp, d.grid_ij, d.ph_grid = ptr(ph_s), ptr(bp_s), ptr(gij), ptr(g)
    d.grid_rows, d.grid_cols = g.shape[0], g.shape[1]
    d.n_i = int(np.rint(gij_all[:, 0].max())) if gij_all.size else 1
    d.n_j = int(np.rint(gij_all[:, 1].max())) if gij_all.size else 1
    d.fit_ifg, d.n_fit = ptr(fit), fit.size
    d.clap_win, d.clap_alpha, d.clap_beta = clap_win, float(clap_alpha), float(clap_beta)
    d.low_pass, d.slc_osf, d.n_trial_wraps = ptr(lp), int(slc_osf), float(n_trial_wraps)
    out = {"ph_patch2": np.zeros((n, m), np.complex64), "K_ps2": np.empty(n), "C_ps2": np.empty(n),
           "coh_ps2": np.empty(n), "ph_res2": np.zeros((n, m), np.float32)}
    o = _lib.S3Out()
    o.ph_patch2, o.K_ps2, o.C_ps2 = ptr(out["ph_patch2"]), ptr(out["K_ps2"]), ptr(out["C_ps2"])
    o.coh_ps2, o.ph_res2 = ptr(out["coh_ps2"]), ptr(out["ph_res2"])
    check(_lib.lib().ps3_reestimate(ctypes.byref(d), ctypes.byref(o), ctypes.c_int(device)))
    return out


def reestimate_resident(ctx, sel, fit_ifg, *, slc_osf: int = 1, on_device: bool = False) -> dict:
    """The stage-3 re-estimate of rows `sel` (0-based) of a patch that a
    Stage2Context (FP32) has just run through stage 2: the phases, bperp,
    cells, CLAP parameters, trial count and last binned grid (pm1.ph_grid)
    are read where they already are in device memory (ps2_stage3_reestimate),
    so only the selection goes to the device. The phases are the context's
    amplitude-normalised ones; psdph / |psdph| (ported.py:4529-4535) does not
    depend on the amplitude, so the results match `reestimate` on the raw
    phases up to the FP32 rounding of that normalisation.

    on_device=True returns torch CUDA tensors on the context's device."""
    sel = np.ascontiguousarray(np.asarray(sel, dtype=np.int64).reshape(-1))
    fit = np.ascontiguousarray(np.asarray(fit_ifg, dtype=np.int64).reshape(-1))
    p = ctx.prepared
    if p is None:
        raise Stage3Error("the context holds no patch")
    n, m = sel.size, p.n_ifg
    o = _lib.S3Out()
    if on_device:
        import torch

        dev = torch.device("cuda", ctx.device)
        out = {"ph_patch2": torch.zeros((n, m), dtype=torch.complex64, device=dev),
               "K_ps2": torch.empty(n, dtype=torch.float64, device=dev),
               "C_ps2": torch.empty(n, dtype=torch.float64, device=dev),
               "coh_ps2": torch.empty(n, dtype=torch.float64, device=dev),
               "ph_res2": torch.zeros((n, m), dtype=torch.float32, device=dev)}
        addr = {k: v.data_ptr() for k, v in out.items()}
        torch.cuda.current_stream(dev).synchronize()  # the allocations' fills precede the library's stream
    else:
        out = {"ph_patch2": np.zeros((n, m), np.complex64), "K_ps2": np.empty(n), "C_ps2": np.empty(n),
               "coh_ps2": np.empty(n), "ph_res2": np.zeros((n, m), np.float32)}
        addr = {k: ptr(v) for k, v in out.items()}
    o.ph_patch2, o.K_ps2, o.C_ps2 = addr["ph_patch2"], addr["K_ps2"], addr["C_ps2"]
    o.coh_ps2, o.ph_res2 = addr["coh_ps2"], addr["ph_res2"]
    vp = ctypes.c_void_p
    check(_lib.lib().ps2_stage3_reestimate(ctx._ctx, vp(ptr(sel)), ctypes.c_int64(n), vp(ptr(fit)), ctypes.c_int64(fit.size),
                                           ctypes.c_int64(int(slc_osf)), ctypes.byref(o),
                                           ctypes.c_int(1 if on_device else 0)))
    return out


def bootstrap_coh_std(ph_res, sel, fit_ifg) -> np.ndarray:
    """Spread of the residual coherence over 100 bootstrap draws per PS
    (ported.py:4408-4422, numpy default_rng(0), draws in PS order)."""
    cpx = np.exp(1j * np.asarray(ph_res)[:, fit_ifg])
    rng = np.random.default_rng(0)
    out = np.zeros(len(sel))
    for k, i in enumerate(sel):
        s = cpx[i]
        if s.size == 0:
            out[k] = np.inf
            continue
        draw = rng.integers(0, s.size, size=(100, s.size))
        out[k] = float(np.std(np.abs(np.sum(s[draw], axis=1)) / float(s.size)))
    return out


def select_ps(pm: dict, *, ph, bperp_mat, bperp, D_A, xy, master_ix: int, ifg_index, parms: dict,
              device: int = 0) -> dict:
    """stage3_select_ps (ported.py:4328-4620) on in-memory inputs.

    pm: the pm1.mat variables (coh_ps, K_ps, C_ps, ph_patch, ph_res, ph_grid,
    grid_ij, Nr, coh_bins, low_pass, n_trial_wraps); ph: ph1.ph with the master
    column; ifg_index: 1-based interferograms used for the selection
    (_ifg_index_for_selection). Returns the select1.mat variables."""
    coh_ps = np.asarray(pm["coh_ps"], dtype=np.float64).reshape(-1)
    n_ps = coh_ps.size
    coh_bins = np.asarray(pm.get("coh_bins", np.arange(0.005, 1.0, 0.01)), dtype=np.float64).reshape(-1)
    Nr_dist = np.asarray(pm.get("Nr", np.ones(coh_bins.size)), dtype=np.float64).reshape(-1)
    da, da_max = da_bins(D_A if D_A is not None else np.ones(n_ps))
    sb = str(parms.get("small_baseline_flag", "n")).lower() == "y"
    low = 15 if sb else 31
    method = str(parms.get("select_method", "PERCENT"))
    mpr = max_percent_rand(method, float(parms.get("percent_rand", 1.0)), float(parms.get("density_rand", 1.0)),
                           xy, da_max.size - 1)
    thresh_all, coeffs = coh_threshold_from_dist(coh_ps, da, da_max, coh_bins, Nr_dist, low, mpr, method)
    ix0 = np.where(coh_ps > thresh_all)[0]
    fit = np.asarray(ifg_index, dtype=np.int64).reshape(-1) - 1
    K_ps = np.asarray(pm["K_ps"], dtype=np.float64).reshape(-1)
    rej = float(parms.get("gamma_stdev_reject", 0.0))
    if rej > 0 and ix0.size and fit.size:
        ix0 = ix0[bootstrap_coh_std(pm["ph_res"], ix0, fit) < rej]
    ph = np.asarray(ph)
    # the interferograms without the master column, gathered with the selected rows
    # only (no copy of the whole stack)
    ph_cols = None if sb else np.delete(np.arange(ph.shape[1]), int(master_ix) - 1)
    n_work = ph.shape[1] if sb else ph.shape[1] - 1
    bperp = np.asarray(bperp, dtype=np.float64).reshape(-1)
    bperp_work = bperp if sb else np.delete(bperp, int(master_ix) - 1)
    fit = fit[(fit >= 0) & (fit < n_work)]
    lp = np.asarray(pm["low_pass"], dtype=np.float64)
    clap_win = int(round(float(parms.get("clap_win", 32.0)))) or 32
    if lp.shape != (clap_win, clap_win):
        raise Stage3Error(f"pm1.low_pass is {lp.shape}, not {clap_win}x{clap_win}")
    r = reestimate(pm["ph_grid"], pm["grid_ij"], ix0, ph, bperp_mat, fit,
                   clap_alpha=float(parms.get("clap_alpha", 1.0)), clap_beta=float(parms.get("clap_beta", 0.3)),
                   low_pass=lp, n_trial_wraps=float(np.asarray(pm["n_trial_wraps"]).reshape(-1)[0]),
                   slc_osf=max(1, int(round(float(parms.get("slc_osf", 1.0))))), clap_win=clap_win, device=device,
                   ph_cols=ph_cols)
    coh_t = coh_ps.copy()
    coh_t[ix0] = r["coh_ps2"]
    thresh_re, coeffs = coh_threshold_from_dist(coh_t, da, da_max, coh_bins, Nr_dist, low, mpr, method)
    th_sel = thresh_re[ix0]
    th_sel[th_sel < 0] = 0
    thresh_all[ix0] = th_sel
    rng_bp = float(np.max(bperp_work) - np.min(bperp_work))
    if rng_bp <= 0:
        rng_bp = 1.0
    with np.errstate(invalid="ignore"):
        keep = (r["coh_ps2"] > th_sel) & (np.abs(K_ps[ix0] - r["K_ps2"]) < 2 * np.pi / rng_bp)
    return {"ix": ix0 + 1, "keep_ix": keep, "ph_patch2": r["ph_patch2"], "ph_res2": r["ph_res2"],
            "K_ps2": r["K_ps2"], "C_ps2": r["C_ps2"], "coh_ps2": r["coh_ps2"], "coh_thresh": thresh_all[ix0],
            "coh_thresh_coeffs": coeffs, "max_percent_rand": mpr}


# --------------------------------------------------------------- MAT I/O ----
SELECT_DEFAULTS = {"select_method": "PERCENT", "percent_rand": 1.0, "density_rand": 1.0, "gamma_stdev_reject": 0.0,
                   "slc_osf": 1.0, "clap_win": 32.0, "clap_alpha": 1.0, "clap_beta": 0.3,
                   "small_baseline_flag": "n"}


def ifg_index_for_selection(n_ifg: int, master_ix: int, small_baseline: bool, drop=()) -> np.ndarray:
    """_ifg_index_for_selection (ported.py:2755-2764): 1-based interferograms
    kept for the selection, renumbered after the master column is removed."""
    drop = {int(v) for v in np.asarray(drop).reshape(-1)}
    ifg = [i for i in range(1, n_ifg + 1) if i not in drop]
    if not small_baseline:
        ifg = [i for i in ifg if i != master_ix]
        ifg = [i - 1 if i > master_ix else i for i in ifg]
    return np.asarray(ifg, dtype=np.float64)


def stage3_select_ps(patch_dir, device: int = 0) -> str:
    """Drop-in for ported.stage3_select_ps (ported.py:4328-4620): reads
    ps1/ph1/bp1/da1/pm1 and the parms, selects with the re-estimate on the GPU,
    writes select1.mat with the reference's variables and returns its summary
    line."""
    from scipy.io import loadmat, savemat

    from .stage2 import _resolve_parms, _scalar

    patch_dir = Path(patch_dir)
    ps = loadmat(patch_dir / "ps1.mat")
    pm_raw = loadmat(patch_dir / "pm1.mat")
    n_ps = int(round(float(_scalar(ps, "n_ps", 0.0))))
    if n_ps <= 0:
        raise Stage3Error("ps1.mat missing valid n_ps")
    parms = dict(SELECT_DEFAULTS)
    pf = _resolve_parms(patch_dir)
    drop = ()
    if pf is not None:
        raw = loadmat(pf)
        for k, v in SELECT_DEFAULTS.items():
            if k in raw:
                parms[k] = _scalar(raw, k, v)
        if "drop_ifg_index" in raw:
            drop = np.asarray(raw["drop_ifg_index"]).reshape(-1)
    ph = np.asarray(loadmat(patch_dir / "ph1.mat")["ph"])
    if ph.shape[0] != n_ps and ph.shape[1] == n_ps:
        ph = ph.T
    bperp_mat = np.asarray(loadmat(patch_dir / "bp1.mat")["bperp_mat"], dtype=np.float64)
    D_A = None
    if (patch_dir / "da1.mat").exists():
        D_A = np.asarray(loadmat(patch_dir / "da1.mat")["D_A"], dtype=np.float64).reshape(-1)
    master_ix = int(round(float(_scalar(ps, "master_ix", 1.0))))
    sb = str(parms["small_baseline_flag"]).lower() == "y"
    n_ifg = int(round(float(_scalar(ps, "n_ifg", ph.shape[1]))))
    ifg_index = ifg_index_for_selection(n_ifg, master_ix, sb, drop)
    pm = {k: pm_raw[k] for k in ("coh_ps", "K_ps", "C_ps", "ph_patch", "ph_res", "ph_grid", "grid_ij", "Nr",
                                 "coh_bins", "low_pass", "n_trial_wraps") if k in pm_raw}
    out = select_ps(pm, ph=ph, bperp_mat=bperp_mat, bperp=ps["bperp"], D_A=D_A, xy=ps.get("xy"),
                    master_ix=master_ix, ifg_index=ifg_index, parms=parms, device=device)
    col = lambda v, dt: np.asarray(v, dtype=dt).reshape(-1, 1)  # noqa: E731
    savemat(patch_dir / "select1.mat", {
        "ix": col(out["ix"], np.float64), "keep_ix": col(out["keep_ix"], np.bool_),
        "ph_patch2": out["ph_patch2"].astype(np.complex64), "ph_res2": out["ph_res2"],
        "K_ps2": col(out["K_ps2"], np.float64), "C_ps2": col(out["C_ps2"], np.float64),
        "coh_ps2": col(out["coh_ps2"], np.float64), "coh_thresh": col(out["coh_thresh"], np.float64),
        "coh_thresh_coeffs": np.asarray(out["coh_thresh_coeffs"], dtype=np.float64),
        "clap_alpha": float(parms["clap_alpha"]), "clap_beta": float(parms["clap_beta"]),
        "n_win": float(parms["clap_win"]), "max_percent_rand": np.float32(out["max_percent_rand"]),
        "gamma_stdev_reject": float(parms["gamma_stdev_reject"]),
        "small_baseline_flag": str(parms["small_baseline_flag"]), "ifg_index": ifg_index.reshape(1, -1),
    })
    return f"Stage 3 selected {out['ix'].size} PS"
