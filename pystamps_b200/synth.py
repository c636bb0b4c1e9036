"""Seeded synthetic PS stacks with the shapes of the stage-2 workloads.

No public dataset is involved: the reference's golden MATLAB datasets are not
available, so every workload is generated here from a fixed seed
(``seed = 2005 + 1000*config_id + patch_id``).

Generative model (per PS candidate r and non-master interferogram c):

* PS positions uniform over a square of side ``50*cells + 25`` m, which makes
  the reference grid rule (native_stage2.rs:1971-2011) produce exactly
  ``cells x cells`` grid cells at 50 m.
* deformation: a Gaussian random field (2 cm std, 500 m correlation length),
  independent per interferogram, sampled at the PS, as phase 4*pi/lambda*d;
* DEM error: K_m ~ U(-15, 15) m, as phase K_ps*bperp_pixel with
  K_ps = K_m*4*pi/(lambda*rho*sin(inc)), rho = 830 km;
* bperp per interferogram ~ U(-B, B) m; per pixel it carries a 2 % linear
  gradient across the patch, so the bperp matrix is row-variant;
* noise: 30 % stable candidates get wrapped N(0, 0.3) rad, the other 70 % a
  uniform random phase; |ph| = 1; amplitude dispersion D_A ~ U(0.2, 0.6);
* the master image is column 1 (1+0j) and has bperp 0;
* the mean incidence is chosen so that the reference's trial-count rule
  (native_stage2.rs:513-522, 1305-1308) yields the requested trial count.
"""
from __future__ import annotations

import math
from dataclasses import dataclass, field

import numpy as np

RHO = 830_000.0
LAMBDA = 0.0555


@dataclass(frozen=True)
class Workload:
    name: str
    config_id: int
    n_ps: int
    n_ifg: int  # non-master interferograms
    cells: int  # grid cells per side at 50 m
    n_trials: int  # 2*ceil(8*n_trial_wraps)+1
    bperp_max: float = 300.0
    max_topo_err: float = 20.0
    gamma_change_convergence: float = 0.005
    gamma_max_iterations: int = 25
    extra: dict = field(default_factory=dict)


# The named workloads (sizes as stated for each study).
SMALL = Workload("small-20k-ps-20-ifg-64x64", 0, 20_000, 20, 64, 81)
PRECISION = Workload("precision-250k-ps-60-ifg-128x128", 1, 250_000, 60, 128, 161)
DIFFERENTIATION = Workload("differentiation-100k-ps-40-ifg-96x96", 3, 100_000, 40, 96, 121)
FULL_SCALE = Workload("full-scale-2m-ps-150-ifg-256x256", 4, 2_000_000, 150, 256, 161, bperp_max=400.0)
WORKLOADS = {w.name: w for w in (SMALL, PRECISION, DIFFERENTIATION, FULL_SCALE)}
ALIASES = {"A": SMALL, "B": PRECISION, "D": DIFFERENTIATION, "E": FULL_SCALE}

_NW_TARGET = {81: 4.94, 161: 9.94, 121: 7.44}


def nw_target_for_trials(n_trials: int) -> float:
    """A n_trial_wraps value strictly inside the interval that gives n_trials."""
    if n_trials in _NW_TARGET:
        return _NW_TARGET[n_trials]
    half = (n_trials - 1) // 2  # = ceil(8*nw)
    return (half - 0.5) / 8.0


def _grf(rng: np.random.Generator, side_m: float, corr_m: float, std: float, n_fields: int):
    """Gaussian random fields on a square raster (FFT-filtered white noise)."""
    spacing = max(10.0, side_m / 512.0)
    n = int(math.ceil(side_m / spacing)) + 1
    fx = np.fft.fftfreq(n, d=spacing)
    kx, ky = np.meshgrid(fx, fx, indexing="ij")
    # Gaussian covariance with correlation length corr_m -> Gaussian spectrum
    spec = np.exp(-((kx**2 + ky**2) * (math.pi * corr_m) ** 2) / 2.0)
    fields = np.empty((n_fields, n, n), dtype=np.float32)
    for k in range(n_fields):
        white = rng.standard_normal((n, n))
        f = np.fft.ifft2(np.fft.fft2(white) * spec).real
        sd = f.std()
        fields[k] = (f / (sd if sd > 0 else 1.0) * std).astype(np.float32)
    return fields, spacing


def make_patch(
    n_ps: int,
    n_ifg: int,
    cells: int,
    n_trials: int,
    *,
    seed: int,
    bperp_max: float = 300.0,
    max_topo_err: float = 20.0,
    gamma_change_convergence: float = 0.005,
    gamma_max_iterations: int = 25,
    stable_fraction: float = 0.3,
    row_variant: bool = True,
    n_rand: int = 300_000,
) -> dict:
    """Build one in-memory patch (the ps1/ph1/bp1/da1/inc1/parms contents)."""
    rng = np.random.default_rng(seed)
    side = 50.0 * cells + 25.0
    x = rng.uniform(0.0, side, n_ps)
    y = rng.uniform(0.0, side, n_ps)
    xy = np.empty((n_ps, 3), dtype=np.float32)
    xy[:, 0] = np.arange(1, n_ps + 1, dtype=np.float32)
    xy[:, 1] = x.astype(np.float32)
    xy[:, 2] = y.astype(np.float32)

    bperp_ifg = rng.uniform(-bperp_max, bperp_max, n_ifg)
    bperp = np.concatenate(([0.0], bperp_ifg)).astype(np.float32).astype(np.float64)
    bp_range = float(bperp[1:].max() - bperp[1:].min())
    nw = nw_target_for_trials(n_trials)
    sin_inc = 2.0 * bp_range * max_topo_err / (LAMBDA * RHO * nw)
    if not 0.0 < sin_inc < 1.0:
        raise ValueError(f"cannot realise {n_trials} trials with bperp range {bp_range}")
    inc = math.asin(sin_inc)

    if row_variant:
        grad = (1.0 + 0.02 * (x - x.mean()) / side).astype(np.float64)
        bperp_mat = (grad[:, None] * bperp[None, 1:]).astype(np.float32).astype(np.float64)
    else:
        bperp_mat = np.tile(bperp[None, 1:], (n_ps, 1))

    k_m = rng.uniform(-15.0, 15.0, n_ps)
    k_ps = k_m * 4.0 * math.pi / (LAMBDA * RHO * sin_inc)

    fields, spacing = _grf(rng, side, 500.0, 0.02, n_ifg)
    ix = np.clip(np.rint(x / spacing).astype(np.int64), 0, fields.shape[1] - 1)
    iy = np.clip(np.rint(y / spacing).astype(np.int64), 0, fields.shape[2] - 1)
    stable = rng.random(n_ps) < stable_fraction

    ph = np.empty((n_ps, n_ifg + 1), dtype=np.complex64)
    ph[:, 0] = 1.0
    chunk = max(1, min(n_ps, (1 << 22) // max(n_ifg, 1)))
    k32 = k_ps.astype(np.float32)
    for s in range(0, n_ps, chunk):
        e = min(n_ps, s + chunk)
        phase = fields[:, ix[s:e], iy[s:e]].T * np.float32(4.0 * math.pi / LAMBDA)
        phase += k32[s:e, None] * bperp_mat[s:e].astype(np.float32)
        st = stable[s:e]
        noise = rng.uniform(-math.pi, math.pi, (e - s, n_ifg)).astype(np.float32)
        n_st = int(st.sum())
        if n_st:
            noise[st] = rng.normal(0.0, 0.3, (n_st, n_ifg)).astype(np.float32)
        phase += noise
        ph[s:e, 1:].real = np.cos(phase)
        ph[s:e, 1:].imag = np.sin(phase)
    d_a = rng.uniform(0.2, 0.6, n_ps)

    parms = {
        "filter_grid_size": 50.0,
        "clap_win": 32.0,
        "clap_low_pass_wavelength": 800.0,
        "clap_alpha": 1.0,
        "clap_beta": 0.3,
        "max_topo_err": float(max_topo_err),
        "lambda": LAMBDA,
        "small_baseline_flag": "n",
        "filter_weighting": "P-square",
        "gamma_change_convergence": float(gamma_change_convergence),
        "gamma_max_iterations": int(gamma_max_iterations),
    }
    return {
        "ph": ph,
        "bperp": bperp,
        "master_ix": 1,
        "bperp_mat": bperp_mat,
        "D_A": d_a,
        "xy": xy,
        "mean_incidence": inc,
        "parms": parms,
        "n_rand": int(n_rand),
        "truth": {"K_ps": k_ps, "stable": stable},
        "seed": seed,
    }


def make_workload(w: Workload | str, patch_id: int = 0, **overrides) -> dict:
    if isinstance(w, str):
        w = ALIASES.get(w) or WORKLOADS[w]
    kw = dict(
        bperp_max=w.bperp_max,
        max_topo_err=w.max_topo_err,
        gamma_change_convergence=w.gamma_change_convergence,
        gamma_max_iterations=w.gamma_max_iterations,
    )
    kw.update(overrides)
    n_ps = kw.pop("n_ps", w.n_ps)
    n_ifg = kw.pop("n_ifg", w.n_ifg)
    cells = kw.pop("cells", w.cells)
    n_trials = kw.pop("n_trials", w.n_trials)
    return make_patch(n_ps, n_ifg, cells, n_trials, seed=2005 + 1000 * w.config_id + patch_id, **kw)


def batched_workload_shapes(n_patches: int = 64, seed: int = 2005 + 2000) -> list[tuple[int, int, int, int]]:
    """(n_ps, n_ifg, cells, n_trials) for the uneven multi-patch workload.

    PS counts log-uniform in 5k-400k, interferogram counts uniform in 30-120,
    grid side = max(24, ceil(sqrt(n_ps/10))) cells (about 10 PS per cell).
    """
    rng = np.random.default_rng(seed)
    out = []
    for _ in range(n_patches):
        n_ps = int(round(math.exp(rng.uniform(math.log(5_000), math.log(400_000)))))
        n_ifg = int(rng.integers(30, 121))
        cells = max(24, int(math.ceil(math.sqrt(n_ps / 10.0))))
        out.append((n_ps, n_ifg, cells, 161))
    return out
