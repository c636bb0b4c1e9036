"""ORACLE — test infrastructure only (ctypes wrapper of liboracle_stage2.so).

CPU restatement of pySTAMPS' native Rust stage 2
(crates/pystamps-core/src/native_stage2.rs). Only tests/, __graft_entry__.smoke()
and bench.py's CPU-baseline leg import this module, and only as the checker.
The product package (pystamps_b200) never imports it.

Pinned against the reference's own known-answer tests
(native_stage2.rs:2464-2559) in tests/test_oracle_kat.py and against golden
vectors produced by the runnable Python reference in tests/golden/.
"""
from __future__ import annotations

import ctypes
import os
import subprocess
from dataclasses import dataclass
from pathlib import Path

import numpy as np

_HERE = Path(__file__).resolve().parent
_LIB_PATH = _HERE / "liboracle_stage2.so"

COH_BINS = 0.005 + 0.01 * np.arange(100, dtype=np.float64)

_c_f32p = ctypes.POINTER(ctypes.c_float)
_c_f64p = ctypes.POINTER(ctypes.c_double)
_c_i64p = ctypes.POINTER(ctypes.c_int64)
_c_i64 = ctypes.c_int64


def build(force: bool = False) -> Path:
    """Compile the oracle library with its Makefile (g++ only, no GPU)."""
    src = _HERE / "native_stage2.cpp"
    if force or not _LIB_PATH.exists() or _LIB_PATH.stat().st_mtime < src.stat().st_mtime:
        subprocess.run(["make", "-C", str(_HERE), "-B" if force else "liboracle_stage2.so"], check=True,
                       stdout=subprocess.DEVNULL)
    return _LIB_PATH


_lib = None


def lib() -> ctypes.CDLL:
    global _lib
    if _lib is None:
        build()
        _lib = ctypes.CDLL(str(_LIB_PATH))
        _lib.orc_stage2_run.restype = ctypes.c_int
        _lib.orc_stage2_run_f64.restype = ctypes.c_int
    return _lib


def _p(a: np.ndarray, t):
    return a.ctypes.data_as(t)


def _threads(threads: int | None) -> int:
    if threads is None:
        return int(os.environ.get("PS2_ORACLE_THREADS", "0"))
    return int(threads)


# ------------------------------------------------------------ setup pieces --
def rng_uniform(n: int, seed: int = 2005) -> np.ndarray:
    out = np.empty(int(n), dtype=np.float64)
    lib().orc_rng_uniform(ctypes.c_uint32(seed), _c_i64(n), _p(out, _c_f64p))
    return out


def grid_indices(xy: np.ndarray, grid_size: float) -> np.ndarray:
    xy = np.ascontiguousarray(xy, dtype=np.float32)
    out = np.empty((xy.shape[0], 2), dtype=np.float32)
    lib().orc_grid_indices(_p(xy, _c_f32p), _c_i64(xy.shape[0]), ctypes.c_double(grid_size), _p(out, _c_f32p))
    return out


def build_low_pass(clap_win: float = 32.0, low_pass_wavelength: float = 800.0, grid_size: float = 50.0) -> np.ndarray:
    n = int(max(round(clap_win), 1))
    out = np.empty((n, n), dtype=np.float64)
    lib().orc_build_low_pass(ctypes.c_double(clap_win), ctypes.c_double(low_pass_wavelength),
                             ctypes.c_double(grid_size), _p(out, _c_f64p))
    return out


def hist_with_centers(values: np.ndarray, centers: np.ndarray = COH_BINS) -> np.ndarray:
    v = np.ascontiguousarray(values, dtype=np.float64).reshape(-1)
    c = np.ascontiguousarray(centers, dtype=np.float64).reshape(-1)
    out = np.empty(c.size, dtype=np.float64)
    lib().orc_hist_with_centers(_p(v, _c_f64p), _c_i64(v.size), _p(c, _c_f64p), _c_i64(c.size), _p(out, _c_f64p))
    return out


def psquare_lut(nr, na, low_coh_thresh: int, nr_max_nz_ix: float) -> np.ndarray:
    nr = np.ascontiguousarray(nr, dtype=np.float64)
    na = np.ascontiguousarray(na, dtype=np.float64)
    lut = np.empty(nr.size * 10 + 16, dtype=np.float64)
    n = _c_i64(0)
    lib().orc_psquare_lut(_p(nr, _c_f64p), _p(na, _c_f64p), _c_i64(nr.size), _c_i64(low_coh_thresh),
                          ctypes.c_double(nr_max_nz_ix), _p(lut, _c_f64p), ctypes.byref(n))
    return lut[: n.value].copy()


def psquare_weighting(nr, na, low_coh_thresh: int, nr_max_nz_ix: float, coh) -> np.ndarray:
    nr = np.ascontiguousarray(nr, dtype=np.float64)
    na = np.ascontiguousarray(na, dtype=np.float64)
    coh = np.ascontiguousarray(coh, dtype=np.float64)
    w = np.empty(coh.size, dtype=np.float64)
    lib().orc_psquare_weighting(_p(nr, _c_f64p), _p(na, _c_f64p), _c_i64(nr.size), _c_i64(low_coh_thresh),
                                ctypes.c_double(nr_max_nz_ix), _p(coh, _c_f64p), _c_i64(coh.size), _p(w, _c_f64p))
    return w


def trial_values(n_trial_wraps: float) -> np.ndarray:
    n = int(np.ceil(8.0 * n_trial_wraps))
    return np.arange(-n, n + 1, dtype=np.float64)


def random_hist(bperp_nm: np.ndarray, n_trial_wraps: float, n_rand: int = 300_000, threads: int | None = None,
                small_baseline: bool = False, ifgday_ix: np.ndarray | None = None, n_image: int = 0):
    bp = np.ascontiguousarray(bperp_nm, dtype=np.float64)
    nr = np.empty(100, dtype=np.float64)
    mx = ctypes.c_double(0.0)
    if small_baseline:
        ix = np.ascontiguousarray(ifgday_ix, dtype=np.int64)
        ia = np.ascontiguousarray(ix[:, 0] - 1)
        ib = np.ascontiguousarray(ix[:, 1] - 1)
    else:
        ia = ib = np.zeros(1, dtype=np.int64)
    lib().orc_random_hist(_p(bp, _c_f64p), _c_i64(bp.size), ctypes.c_double(n_trial_wraps), _c_i64(n_rand),
                          ctypes.c_int(1 if small_baseline else 0), _p(ia, _c_i64p), _p(ib, _c_i64p),
                          _c_i64(n_image), _p(nr, _c_f64p), ctypes.byref(mx), ctypes.c_int(_threads(threads)))
    return nr, mx.value


# ------------------------------------------------------------- loop pieces --
def fill_phase_weight(ph_nm, bperp, k_ps, w, threads=None) -> np.ndarray:
    ph = np.ascontiguousarray(ph_nm, dtype=np.complex64)
    n, m = ph.shape
    bp = np.ascontiguousarray(bperp, dtype=np.float64)
    row_inv = 1 if bp.ndim == 1 else 0
    k = np.ascontiguousarray(k_ps, dtype=np.float64)
    ww = np.ascontiguousarray(w, dtype=np.float64)
    out = np.empty_like(ph)
    lib().orc_fill_phase_weight(_p(ph, _c_f32p), _p(bp, _c_f64p), ctypes.c_int(row_inv), _p(k, _c_f64p),
                                _p(ww, _c_f64p), _c_i64(n), _c_i64(m), _p(out, _c_f32p), ctypes.c_int(_threads(threads)))
    return out


def accumulate_grid(ph_weight, grid_lin, n_i: int, n_j: int) -> np.ndarray:
    ph = np.ascontiguousarray(ph_weight, dtype=np.complex64)
    gl = np.ascontiguousarray(grid_lin, dtype=np.int64)
    n, m = ph.shape
    out = np.empty((n_i, n_j, m), dtype=np.complex64)
    lib().orc_accumulate_grid(_p(ph, _c_f32p), _p(gl, _c_i64p), _c_i64(n), _c_i64(m), _c_i64(n_i), _c_i64(n_j),
                              _p(out, _c_f32p))
    return out


def clap_filter_grid_stack(ph_grid, alpha: float, beta: float, low_pass, n_win: int = 24, threads=None,
                           fp64: bool = False) -> np.ndarray:
    dt = np.complex128 if fp64 else np.complex64
    g = np.ascontiguousarray(ph_grid, dtype=dt)
    n_i, n_j, m = g.shape
    lp = np.ascontiguousarray(low_pass, dtype=np.float64)
    n_ex = lp.shape[0]
    out = np.empty_like(g)
    if fp64:
        lib().orc_clap_filter_grid_stack_f64(_p(g, _c_f64p), _c_i64(n_i), _c_i64(n_j), _c_i64(m), _c_i64(n_win),
                                             ctypes.c_double(alpha), ctypes.c_double(beta), _p(lp, _c_f64p),
                                             _c_i64(n_ex), _p(out, _c_f64p), ctypes.c_int(_threads(threads)))
    else:
        lib().orc_clap_filter_grid_stack(_p(g, _c_f32p), _c_i64(n_i), _c_i64(n_j), _c_i64(m), _c_i64(n_win),
                                         ctypes.c_double(alpha), ctypes.c_double(beta), _p(lp, _c_f64p),
                                         _c_i64(n_ex), _p(out, _c_f32p), ctypes.c_int(_threads(threads)))
    return out


def extract_patch_phase(ph_filt, grid_lin, threads=None) -> np.ndarray:
    f = np.ascontiguousarray(ph_filt, dtype=np.complex64)
    m = f.shape[-1]
    f2 = f.reshape(-1, m)
    gl = np.ascontiguousarray(grid_lin, dtype=np.int64)
    out = np.empty((gl.size, m), dtype=np.complex64)
    lib().orc_extract_patch_phase(_p(f2, _c_f32p), _p(gl, _c_i64p), _c_i64(gl.size), _c_i64(m), _p(out, _c_f32p),
                                  ctypes.c_int(_threads(threads)))
    return out


@dataclass
class FitRows:
    K: np.ndarray
    C: np.ndarray
    coh: np.ndarray
    N_opt: np.ndarray
    ph_res: np.ndarray
    best_ix: np.ndarray
    best_coh: np.ndarray
    second_coh: np.ndarray


def fit_rows(ph_patch, ph_nm, bperp, n_trial_wraps: float, threads=None) -> FitRows:
    pp = np.ascontiguousarray(ph_patch, dtype=np.complex64)
    nm = np.ascontiguousarray(ph_nm, dtype=np.complex64)
    n, m = nm.shape
    bp = np.ascontiguousarray(bperp, dtype=np.float64)
    row_inv = 1 if bp.ndim == 1 else 0
    K = np.empty(n); C = np.empty(n); coh = np.empty(n); nopt = np.empty(n)
    ph_res = np.empty((n, m), dtype=np.float32)
    bix = np.empty(n, dtype=np.int64); bc = np.empty(n); sc = np.empty(n)
    lib().orc_fit_rows(_p(pp, _c_f32p), _p(nm, _c_f32p), _p(bp, _c_f64p), ctypes.c_int(row_inv),
                       ctypes.c_double(n_trial_wraps), _c_i64(n), _c_i64(m), _p(K, _c_f64p), _p(C, _c_f64p),
                       _p(coh, _c_f64p), _p(nopt, _c_f64p), _p(ph_res, _c_f32p), _p(bix, _c_i64p), _p(bc, _c_f64p),
                       _p(sc, _c_f64p), ctypes.c_int(_threads(threads)))
    return FitRows(K, C, coh, nopt, ph_res, bix, bc, sc)


# ---------------------------------------------------------- whole stage 2 --
class _In(ctypes.Structure):
    _fields_ = [
        ("n_ps", _c_i64), ("n_ifg_full", _c_i64),
        ("ph_full", ctypes.c_void_p), ("bperp_full", ctypes.c_void_p), ("master_ix", _c_i64),
        ("bperp_mat", ctypes.c_void_p), ("bperp_mat_cols", _c_i64), ("d_a", ctypes.c_void_p),
        ("xy", ctypes.c_void_p), ("mean_incidence", ctypes.c_double),
        ("grid_size", ctypes.c_double), ("clap_win", ctypes.c_double),
        ("clap_low_pass_wavelength", ctypes.c_double), ("clap_alpha", ctypes.c_double),
        ("clap_beta", ctypes.c_double), ("max_topo_err", ctypes.c_double), ("lambda_m", ctypes.c_double),
        ("small_baseline", ctypes.c_int), ("psquare", ctypes.c_int),
        ("gamma_change_convergence", ctypes.c_double), ("gamma_max_iterations", _c_i64),
        ("n_rand", _c_i64), ("ifgday_ix", ctypes.c_void_p), ("n_image", _c_i64),
        ("nr_override", ctypes.c_void_p),
    ]


class _Out(ctypes.Structure):
    _fields_ = [
        ("K_ps", ctypes.c_void_p), ("C_ps", ctypes.c_void_p), ("coh_ps", ctypes.c_void_p),
        ("N_opt", ctypes.c_void_p), ("ph_res", ctypes.c_void_p), ("ph_patch", ctypes.c_void_p),
        ("ph_grid", ctypes.c_void_p), ("ph_weight", ctypes.c_void_p), ("grid_ij", ctypes.c_void_p),
        ("low_pass", ctypes.c_void_p), ("Nr", ctypes.c_void_p), ("coh_ps_save", ctypes.c_void_p),
        ("gamma_change_hist", ctypes.c_void_p), ("coh_hist", ctypes.c_void_p), ("K_hist", ctypes.c_void_p),
        ("iter_seconds", ctypes.c_void_p), ("Nr_max_nz_ix", ctypes.c_double), ("gamma_change_save", ctypes.c_double),
        ("n_trial_wraps", ctypes.c_double),
        ("i_loop", _c_i64), ("n_i", _c_i64), ("n_j", _c_i64), ("n_ifg", _c_i64), ("n_trials", _c_i64),
    ]


def stage2_run(patch, *, threads=None, fp64: bool = False, keep_history: bool = False) -> dict:
    """Run the whole restated stage 2 on an in-memory patch.

    ``patch`` is a mapping with the keys produced by
    ``pystamps_b200.synth.make_patch`` (ph, bperp, master_ix, bperp_mat, D_A, xy,
    mean_incidence, parms...). Returns the pm1.mat variables of
    native_stage2.rs:1899-1965 plus per-iteration histories (gamma_change_hist,
    iter_seconds: wall time of each loop iteration, native_stage2.rs:261-406).
    """
    ph = np.ascontiguousarray(patch["ph"], dtype=np.complex64)
    n, mf = ph.shape
    bperp = np.ascontiguousarray(patch["bperp"], dtype=np.float64).reshape(-1)
    bmat = patch.get("bperp_mat")
    bmat = None if bmat is None else np.ascontiguousarray(bmat, dtype=np.float64)
    da = patch.get("D_A")
    da = None if da is None else np.ascontiguousarray(da, dtype=np.float64).reshape(-1)
    xy = np.ascontiguousarray(patch["xy"], dtype=np.float32)
    p = patch["parms"]
    nr_override = patch.get("nr_override")
    nr_ov = None if nr_override is None else np.ascontiguousarray(nr_override, dtype=np.float64)
    ifgday = patch.get("ifgday_ix")
    ifgday = None if ifgday is None else np.ascontiguousarray(ifgday, dtype=np.int64)

    inp = _In()
    inp.n_ps = n
    inp.n_ifg_full = mf
    inp.ph_full = ph.ctypes.data
    inp.bperp_full = bperp.ctypes.data
    inp.master_ix = int(patch.get("master_ix", 1))
    inp.bperp_mat = 0 if bmat is None else bmat.ctypes.data
    inp.bperp_mat_cols = 0 if bmat is None else bmat.shape[1]
    inp.d_a = 0 if da is None else da.ctypes.data
    inp.xy = xy.ctypes.data
    inp.mean_incidence = float(patch["mean_incidence"])
    inp.grid_size = float(p.get("filter_grid_size", 50.0))
    inp.clap_win = float(p.get("clap_win", 32.0))
    inp.clap_low_pass_wavelength = float(p.get("clap_low_pass_wavelength", 800.0))
    inp.clap_alpha = float(p.get("clap_alpha", 1.0))
    inp.clap_beta = float(p.get("clap_beta", 0.3))
    inp.max_topo_err = float(p.get("max_topo_err", 15.0))
    inp.lambda_m = float(p.get("lambda", 0.0555))
    inp.small_baseline = 1 if str(p.get("small_baseline_flag", "n")).lower() == "y" else 0
    inp.psquare = 1 if str(p.get("filter_weighting", "P-square")).lower() == "p-square" else 0
    inp.gamma_change_convergence = float(p.get("gamma_change_convergence", 1e-4))
    inp.gamma_max_iterations = int(round(float(p.get("gamma_max_iterations", 25))))
    inp.n_rand = int(patch.get("n_rand", 300_000))
    inp.ifgday_ix = 0 if ifgday is None else ifgday.ctypes.data
    inp.n_image = int(patch.get("n_image", 0))
    inp.nr_override = 0 if nr_ov is None else nr_ov.ctypes.data

    small = inp.small_baseline == 1
    m = mf if small else mf - 1
    max_it = max(inp.gamma_max_iterations, 1)
    rdt, cdt = (np.float64, np.complex128) if fp64 else (np.float32, np.complex64)
    bufs = dict(
        K_ps=np.empty(n), C_ps=np.empty(n), coh_ps=np.empty(n), N_opt=np.empty(n),
        ph_res=np.empty((n, m), rdt), ph_patch=np.empty((n, m), cdt), ph_weight=np.empty((n, m), cdt),
        grid_ij=np.empty((n, 2), np.float32), low_pass=np.empty((int(round(inp.clap_win)),) * 2),
        Nr=np.empty(100), coh_ps_save=np.empty(n), gamma_change_hist=np.full(max_it, np.nan),
        iter_seconds=np.full(max_it, np.nan),
    )
    if keep_history:
        bufs["coh_hist"] = np.full((max_it, n), np.nan)
        bufs["K_hist"] = np.full((max_it, n), np.nan)
    gij = grid_indices(xy, inp.grid_size)
    n_i = int(max(1, gij[:, 0].max())) if n else 1
    n_j = int(max(1, gij[:, 1].max())) if n else 1
    bufs["ph_grid"] = np.empty((n_i, n_j, m), cdt)
    out = _Out()
    for k, v in bufs.items():
        setattr(out, k, v.ctypes.data)
    out.n_i, out.n_j = n_i, n_j
    fn = lib().orc_stage2_run_f64 if fp64 else lib().orc_stage2_run
    rc = fn(ctypes.byref(inp), ctypes.byref(out), ctypes.c_int(_threads(threads)))
    if rc == -2:
        raise ValueError(f"bp1.bperp_mat has incompatible shape {bmat.shape} for stage-2 ph shape {n}x{m}")
    if rc != 0:
        raise RuntimeError(f"oracle stage2 failed rc={rc}")
    res = dict(bufs)
    it = int(out.i_loop)
    res.update(
        Nr_max_nz_ix=out.Nr_max_nz_ix, gamma_change_save=out.gamma_change_save, n_trial_wraps=out.n_trial_wraps,
        i_loop=it, n_i=n_i, n_j=n_j, n_ifg=int(out.n_ifg), n_trials=int(out.n_trials),
        grid_size=inp.grid_size, coh_bins=COH_BINS.copy(), step_number=1.0,
    )
    res["gamma_change_hist"] = res["gamma_change_hist"][:it]
    res["iter_seconds"] = res["iter_seconds"][:it]
    if keep_history:
        res["coh_hist"] = res["coh_hist"][:it]
        res["K_hist"] = res["K_hist"][:it]
    return res


def topofit(cpxphase, bperp, n_trial_wraps: float, threads=None, fp64: bool | None = None):
    """Registry-level topofit (zero columns skipped, all-zero rows -> NaN)."""
    if fp64 is None:
        fp64 = np.asarray(cpxphase).dtype == np.complex128
    dt = np.complex128 if fp64 else np.complex64
    cpx = np.ascontiguousarray(cpxphase, dtype=dt)
    n, m = cpx.shape
    bp = np.ascontiguousarray(bperp, dtype=np.float64)
    row_inv = 1 if bp.ndim == 1 else 0
    K = np.empty(n); C = np.empty(n); coh = np.empty(n)
    res = np.empty_like(cpx)
    bix = np.empty(n, dtype=np.int64)
    fn = lib().orc_topofit_f64 if fp64 else lib().orc_topofit
    pt = _c_f64p if fp64 else _c_f32p
    fn(_p(cpx, pt), _p(bp, _c_f64p), ctypes.c_int(row_inv), ctypes.c_double(n_trial_wraps), _c_i64(n), _c_i64(m),
       _p(K, _c_f64p), _p(C, _c_f64p), _p(coh, _c_f64p), _p(res, pt), _p(bix, _c_i64p), ctypes.c_int(_threads(threads)))
    return K, C, coh, res, bix


# ------------------------------------------------------ stage-3 re-estimate --
def s3_clap_patch(patch, alpha: float, beta: float, low_pass) -> np.ndarray:
    """ported._clap_filt_patch (ported.py:992-1009), complex128."""
    x = np.ascontiguousarray(patch, dtype=np.complex128)
    n = x.shape[0]
    lp = np.ascontiguousarray(low_pass, dtype=np.float64)
    out = np.empty_like(x)
    lib().orc_s3_clap_patch(_p(x, _c_f64p), _c_i64(n), ctypes.c_double(alpha), ctypes.c_double(beta),
                            _p(lp, _c_f64p), _p(out, _c_f64p))
    return out


def s3_topofit_single(cpx, bperp, n_trial_wraps: float):
    """ported._ps_topofit_single (ported.py:2355-2431) in the complex64 / float32
    form stage 3 uses. Returns (K, C, coh, residual complex64, candidate count)."""
    c = np.ascontiguousarray(cpx, dtype=np.complex64)
    b = np.ascontiguousarray(bperp, dtype=np.float32)
    K = ctypes.c_double(); C = ctypes.c_double(); h = ctypes.c_double()
    res = np.empty_like(c)
    lib().orc_s3_topofit_single.restype = ctypes.c_int64
    nc = lib().orc_s3_topofit_single(_p(c, _c_f32p), _p(b, _c_f32p), _c_i64(c.size), ctypes.c_double(n_trial_wraps),
                                     ctypes.byref(K), ctypes.byref(C), ctypes.byref(h), _p(res, _c_f32p))
    return K.value, C.value, h.value, res, int(nc)


def s3_reestimate(ph_grid, grid_ij, sel, ph_work, bperp, fit_ix, *, alpha: float, beta: float, low_pass,
                  n_trial_wraps: float, slc_osf: int = 1, n_win: int = 32, threads=None) -> dict:
    """The stage-3 re-estimate loop (ported.py:4489-4550) for rows `sel`."""
    g = np.ascontiguousarray(ph_grid, dtype=np.complex64)
    gi, gj, m = g.shape
    ij = np.ascontiguousarray(np.asarray(grid_ij).reshape(-1, 2), dtype=np.int64)
    s = np.ascontiguousarray(sel, dtype=np.int64)
    w = np.ascontiguousarray(ph_work, dtype=np.complex64)
    bp = np.ascontiguousarray(bperp, dtype=np.float64)
    f = np.ascontiguousarray(fit_ix, dtype=np.int64)
    lp = np.ascontiguousarray(low_pass, dtype=np.float64)
    n_i, n_j = int(ij[:, 0].max()), int(ij[:, 1].max())
    pp2 = np.empty((s.size, m), dtype=np.complex128)
    K = np.empty(s.size); C = np.empty(s.size); coh = np.empty(s.size)
    res = np.empty((s.size, m), dtype=np.float32)
    lib().orc_s3_reestimate(_p(g, _c_f32p), _c_i64(gi), _c_i64(gj), _c_i64(m), _p(ij, _c_i64p), _p(s, _c_i64p),
                            _c_i64(s.size), _p(w, _c_f32p), _p(bp, _c_f64p), _p(f, _c_i64p), _c_i64(f.size),
                            _c_i64(n_i), _c_i64(n_j), _c_i64(n_win), ctypes.c_double(alpha), ctypes.c_double(beta),
                            _p(lp, _c_f64p), _c_i64(slc_osf), ctypes.c_double(n_trial_wraps), _p(pp2, _c_f64p),
                            _p(K, _c_f64p), _p(C, _c_f64p), _p(coh, _c_f64p), _p(res, _c_f32p),
                            ctypes.c_int(_threads(threads)))
    return {"ph_patch2": pp2, "K_ps2": K, "C_ps2": C, "coh_ps2": coh, "ph_res2": res}
