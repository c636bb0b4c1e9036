"""Stage-2 gamma estimation on the GPU: the host side of the cuda backend.

This mirrors the reference's stage-2 driver boundary:

* ``prepare_patch`` restates ``prepare_stage2_inputs``
  (crates/pystamps-core/src/native_stage2.rs:415-561) for in-memory arrays:
  master-column removal, unit normalisation, f32 grid indices, low pass,
  trial count, random-phase histogram (on the GPU in FP64).
* ``Stage2Context`` owns one device-resident patch and runs the gamma loop
  (native_stage2.rs:261-406) through ``libps2cuda``.
* ``stage2_estimate_gamma(patch_dir, kernel_backend="cuda")`` is the
  drop-in for ``pystamps.pipeline.ported.stage2_estimate_gamma``
  (pystamps/pipeline/ported.py:3683) and ``run_stage2_native_with_options``:
  it reads ps1/ph1/bp1/da1/inc1/la1/parms MAT files and writes pm1.mat with the
  variables of write_pm1 (native_stage2.rs:1899-1965).

Errors are raised as ``Stage2Error`` with the reference's wording
("stage 2 native implementation error: ...", crates/pystamps-core/src/lib.rs:47-48).
"""
from __future__ import annotations

import ctypes
import math
import os
from dataclasses import dataclass, field
from pathlib import Path

import numpy as np

from . import _lib
from ._lib import PRECISION_FP32, PRECISION_FP64, check, lib, ptr

COH_BINS = 0.005 + 0.01 * np.arange(100, dtype=np.float64)
RHO = 830_000.0
DEFAULT_MEAN_INCIDENCE = math.radians(23.0)
DEFAULT_PARMS = {
    "filter_grid_size": 50.0,
    "clap_win": 32.0,
    "clap_low_pass_wavelength": 800.0,
    "clap_alpha": 1.0,
    "clap_beta": 0.3,
    "max_topo_err": 15.0,
    "lambda": 0.0555,
    "small_baseline_flag": "n",
    "filter_weighting": "P-square",
    "gamma_change_convergence": 1.0e-4,
    "gamma_max_iterations": 25,
}


class Stage2Error(ValueError):
    def __init__(self, message: str):
        super().__init__(f"stage 2 native implementation error: {message}")


# ------------------------------------------------------------ preparation --
def _saturate_i32(v: np.ndarray) -> np.ndarray:
    """Rust's float-to-i32 `as` cast: truncation toward zero, saturating at
    the i32 range (NaN never reaches it here)."""
    return np.clip(np.trunc(v.astype(np.float64)), -2.0 ** 31, 2.0 ** 31 - 1).astype(np.int64)


def grid_indices(xy: np.ndarray, grid_size: float) -> np.ndarray:
    """stage2_grid_indices (native_stage2.rs:1971-2011), f32 arithmetic.

    The reference's f32 min and max ignore NaN (`f32::min`, `f32::max`): a NaN
    coordinate takes no part in the minimum and its bin becomes 1
    (`NaN.ceil().max(1.0)`); a bin beyond the i32 range saturates like `as i32`.
    """
    xy = np.asarray(xy, dtype=np.float32)
    n = xy.shape[0]
    out = np.zeros((n, 2), dtype=np.float32)
    if n == 0:
        return out
    eps = np.float32(1.0e-6)
    scale = np.float32(grid_size)
    bins = []
    for col in (2, 1):  # i from y, j from x
        v = xy[:, col]
        with np.errstate(invalid="ignore", over="ignore"):
            lo = np.fmin(np.float32(np.inf), np.fmin.reduce(v))
            f = np.fmax(np.ceil(((v - lo) + eps) / scale), np.float32(1.0))
        bins.append(_saturate_i32(f).astype(np.float32))
    for k, b in enumerate(bins):
        top = int(max(1, _saturate_i32(b).max()))
        if top > 1:
            b[_saturate_i32(b) == top] = np.float32(top - 1)
        out[:, k] = b
    return out


def build_low_pass(clap_win: float, low_pass_wavelength: float, grid_size: float) -> np.ndarray:
    """build_low_pass (native_stage2.rs:2013-2043): fftshifted 5th-order Butterworth."""
    n = int(max(round(clap_win), 1))
    f0 = 1.0 / low_pass_wavelength
    butter = np.empty(n)
    for i in range(n):
        f = (float(i) - n / 2.0) / (grid_size * n)
        x = f / f0
        x2 = x * x
        x4 = x2 * x2
        x8 = x4 * x4
        butter[i] = 1.0 / (1.0 + x2 * x8)
    sh = n // 2
    idx = (np.arange(n) + sh) % n
    return np.outer(butter[idx], butter[idx])


def trial_count(n_trial_wraps: float) -> int:
    return 2 * int(math.ceil(8.0 * n_trial_wraps)) + 1


def random_coherence_histogram(bperp_nm, n_trial_wraps: float, n_rand: int = 300_000, small_baseline: bool = False,
                               ifgday_ix=None, n_image: int = 0):
    """Nr on the GPU in FP64 (random_coherence_histogram, native_stage2.rs:1310-1356)."""
    bp = np.ascontiguousarray(bperp_nm, dtype=np.float64)
    nr = np.zeros(100, dtype=np.float64)
    mx = ctypes.c_double(0.0)
    ix = None if ifgday_ix is None else np.ascontiguousarray(ifgday_ix, dtype=np.int64)
    check(lib().ps2_random_coherence_histogram(
        ctypes.c_void_p(ptr(bp)), ctypes.c_int64(bp.size), ctypes.c_double(n_trial_wraps), ctypes.c_int64(n_rand),
        ctypes.c_int32(1 if small_baseline else 0), ctypes.c_void_p(ptr(ix)), ctypes.c_int64(n_image),
        ctypes.c_void_p(ptr(nr)), ctypes.byref(mx)))
    return nr, mx.value


@dataclass
class PreparedPatch:
    n_ps: int
    n_ifg: int
    ph_nm: np.ndarray          # complex64 [N, M]
    amp: np.ndarray            # f32 [N, M]
    bperp: np.ndarray          # f32 [N, M] or [M]
    row_invariant: bool
    bperp_nm: np.ndarray       # f64 [M]
    grid_ij: np.ndarray        # f32 [N, 2]
    grid_lin: np.ndarray       # i64 [N]
    n_i: int
    n_j: int
    weight0: np.ndarray        # f64 [N]
    low_pass: np.ndarray       # f64 [32, 32]
    n_trial_wraps: float
    nr: np.ndarray             # f64 [100]
    nr_max_nz_ix: float
    low_coh_thresh: int
    psquare: bool
    gamma_change_convergence: float
    gamma_max_iterations: int
    clap_window: int
    clap_alpha: float
    clap_beta: float
    grid_size: float
    extra: dict = field(default_factory=dict)


def _parm(parms: dict, key: str):
    v = parms.get(key, DEFAULT_PARMS[key])
    return v


def prepare_patch(patch: dict, *, nr: np.ndarray | None = None, nr_max_nz_ix: float | None = None) -> PreparedPatch:
    """prepare_stage2_inputs (native_stage2.rs:415-561) for in-memory inputs.

    ``patch`` holds ph (complex [N, n_ifg_full]), bperp ([n_ifg_full]),
    master_ix (1-based), optional bperp_mat, D_A, xy ([N, 3]: id, x, y),
    mean_incidence (radians, already resolved from inc1/la1/ps1), parms and
    optionally n_rand / ifgday_ix / n_image. ``nr`` skips the histogram.
    """
    parms = dict(DEFAULT_PARMS)
    parms.update(patch.get("parms", {}))
    ph_full = np.asarray(patch["ph"], dtype=np.complex64)
    if ph_full.ndim != 2 or ph_full.shape[0] == 0:
        raise Stage2Error("ps1.mat missing valid n_ps")
    n_ps, n_full = ph_full.shape
    master_ix = int(round(float(patch.get("master_ix", 1))))
    if master_ix < 1 or master_ix > n_full:
        raise Stage2Error(f"ps1.master_ix must be 1-based within ph1 width {n_full}; got {master_ix}")
    bperp_full = np.asarray(patch["bperp"], dtype=np.float64).reshape(-1).astype(np.float32).astype(np.float64)
    if bperp_full.size != n_full:
        raise Stage2Error(f"ps1.bperp has length {bperp_full.size} but ph1.ph has {n_full} interferograms")
    small = str(_parm(parms, "small_baseline_flag")).strip().lower() == "y"
    cols = np.arange(n_full, dtype=np.int64) if small else np.array([k for k in range(n_full) if k != master_ix - 1],
                                                                     dtype=np.int64)
    m = cols.size
    # unit phases and magnitudes (|ph|, 1 where it is 0) in one threaded native
    # pass: hypotf, the zero guard and the divisions of :452-467
    ph_full = np.ascontiguousarray(ph_full)
    ph_nm = np.empty((n_ps, m), dtype=np.complex64)
    safe = np.empty((n_ps, m), dtype=np.float32)
    check(lib().ps2_prepare_phase(ctypes.c_void_p(ph_full.ctypes.data), ctypes.c_int64(n_ps), ctypes.c_int64(n_full),
                                  ctypes.c_void_p(cols.ctypes.data), ctypes.c_int64(m),
                                  ctypes.c_void_p(ph_nm.ctypes.data), ctypes.c_void_p(safe.ctypes.data),
                                  ctypes.c_int(0)))
    bperp_nm = bperp_full[cols]
    # bp1.bperp_mat (native_stage2.rs:563-612)
    bmat = patch.get("bperp_mat")
    if bmat is not None:
        bmat = np.asarray(bmat, dtype=np.float64)
        if bmat.ndim != 2 or bmat.shape[0] != n_ps:
            if bmat.ndim == 2 and bmat.shape[1] == n_ps:
                bmat = bmat.T
            else:
                raise Stage2Error(f"bp1.bperp_mat is missing or invalid: shape {bmat.shape}")
        if bmat.shape[1] == m:
            pass
        elif not small and bmat.shape[1] == n_full:
            pass  # the master column is skipped by the native pass below
        else:
            raise Stage2Error(
                f"bp1.bperp_mat has incompatible shape {bmat.shape[0]}x{bmat.shape[1]} for stage-2 ph shape {n_ps}x{m}")
    if bmat is None:  # (small baselines: every row is bperp_nm, row-invariant)
        row_inv = True
        bperp = np.ascontiguousarray(bperp_nm.astype(np.float32))
    else:
        # f32 rows and the row-invariance test (native_stage2.rs:2413-2428) in one pass
        bmat = np.ascontiguousarray(bmat, dtype=np.float64)
        sel = cols if bmat.shape[1] != m else None
        bp32 = np.empty((n_ps, m), dtype=np.float32)
        inv = ctypes.c_int32(0)
        check(lib().ps2_prepare_bperp(ctypes.c_void_p(bmat.ctypes.data), ctypes.c_int64(n_ps),
                                      ctypes.c_int64(bmat.shape[1]),
                                      ctypes.c_void_p(sel.ctypes.data if sel is not None else 0), ctypes.c_int64(m),
                                      ctypes.c_void_p(bp32.ctypes.data), ctypes.byref(inv), ctypes.c_int(0)))
        row_inv = n_ps <= 1 or inv.value == 1
        bperp = np.ascontiguousarray(bp32[0]) if row_inv else bp32
    d_a = patch.get("D_A")
    if d_a is None or np.asarray(d_a).size != n_ps:
        d_a = np.ones(n_ps)
    d_a = np.asarray(d_a, dtype=np.float64).reshape(-1)
    with np.errstate(divide="ignore"):
        weight0 = np.where(d_a != 0.0, 1.0 / np.where(d_a != 0.0, d_a, 1.0), 0.0)
    xy = np.asarray(patch["xy"], dtype=np.float32)
    if xy.shape != (n_ps, 3):
        if xy.shape == (3, n_ps):
            xy = xy.T
        else:
            raise Stage2Error(f"ps1.xy has incompatible shape {xy.shape[0]}x{xy.shape[1]}; expected {n_ps}x3")
    gij = grid_indices(xy, float(_parm(parms, "filter_grid_size")))
    n_i = int(max(1, gij[:, 0].max()))
    n_j = int(max(1, gij[:, 1].max()))
    grid_lin = ((gij[:, 0].astype(np.int64) - 1) * n_j + (gij[:, 1].astype(np.int64) - 1)).astype(np.int64)
    clap_win = float(_parm(parms, "clap_win"))
    low_pass = build_low_pass(clap_win, float(_parm(parms, "clap_low_pass_wavelength")),
                              float(_parm(parms, "filter_grid_size")))
    inc = float(patch.get("mean_incidence", DEFAULT_MEAN_INCIDENCE))
    max_k = float(_parm(parms, "max_topo_err")) / (float(_parm(parms, "lambda")) * RHO * math.sin(inc) / (4.0 * math.pi))
    ntw = float((bperp_nm.max() - bperp_nm.min()) * max_k / (2.0 * math.pi))
    low_coh_thresh = 15 if small else 31
    if nr is None:
        nr, nr_max_nz_ix = random_coherence_histogram(
            bperp_nm, ntw, int(patch.get("n_rand", 300_000)), small,
            patch.get("ifgday_ix"), int(patch.get("n_image", 0)))
    elif nr_max_nz_ix is None:
        nz = np.flatnonzero(np.asarray(nr) > 0)
        nr_max_nz_ix = float(nz[-1] + 1) if nz.size else 1.0
    fw = str(_parm(parms, "filter_weighting")).strip().lower()
    return PreparedPatch(
        n_ps=n_ps, n_ifg=m, ph_nm=ph_nm, amp=np.ascontiguousarray(safe), bperp=bperp, row_invariant=row_inv,
        bperp_nm=bperp_nm, grid_ij=gij, grid_lin=grid_lin, n_i=n_i, n_j=n_j, weight0=weight0, low_pass=low_pass,
        n_trial_wraps=ntw, nr=np.asarray(nr, dtype=np.float64), nr_max_nz_ix=float(nr_max_nz_ix),
        low_coh_thresh=low_coh_thresh, psquare=(fw == "p-square"),
        gamma_change_convergence=float(_parm(parms, "gamma_change_convergence")),
        gamma_max_iterations=int(round(float(_parm(parms, "gamma_max_iterations")))),
        clap_window=int(max(round(clap_win * 0.75), 1)), clap_alpha=float(_parm(parms, "clap_alpha")),
        clap_beta=float(_parm(parms, "clap_beta")), grid_size=float(_parm(parms, "filter_grid_size")),
    )


# ------------------------------------------------------------------ context --
class Stage2Context:
    """One device-resident patch and its gamma loop (libps2cuda context)."""

    def __init__(self, device: int = 0):
        self._lib = lib()
        self._ctx = ctypes.c_void_p()
        check(self._lib.ps2_create(ctypes.byref(self._ctx), ctypes.c_int(device)))
        self.device = int(device)
        self.prepared: PreparedPatch | None = None
        self.precision = PRECISION_FP32
        self._keep = []

    def close(self) -> None:
        if self._ctx:
            self._lib.ps2_destroy(self._ctx)
            self._ctx = ctypes.c_void_p()

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def load(self, p: PreparedPatch, precision: str | int = "fp32", device_arrays: dict | None = None) -> None:
        """Upload a prepared patch. ``device_arrays`` (torch CUDA tensors for
        ph_nm / bperp / grid_lin / weight0 / low_pass / nr / amp) replace the
        host arrays and are copied device-to-device."""
        prec = precision if isinstance(precision, int) else (PRECISION_FP64 if str(precision) == "fp64" else PRECISION_FP32)
        src = {
            "ph_nm": np.ascontiguousarray(p.ph_nm, dtype=np.complex64),
            "amp": np.ascontiguousarray(p.amp, dtype=np.float32),
            "bperp": np.ascontiguousarray(p.bperp, dtype=np.float32),
            "grid_lin": np.ascontiguousarray(p.grid_lin, dtype=np.int64),
            "weight0": np.ascontiguousarray(p.weight0, dtype=np.float64),
            "low_pass": np.ascontiguousarray(p.low_pass, dtype=np.float64),
            "nr": np.ascontiguousarray(p.nr, dtype=np.float64),
        }
        on_dev = 0
        if device_arrays:
            src.update(device_arrays)
            on_dev = 1
        self._keep = list(src.values())
        d = _lib.PatchDesc()
        d.n_ps = p.n_ps
        d.n_ifg = p.n_ifg
        d.ph_nm = ptr(src["ph_nm"])
        d.amp = ptr(src["amp"]) if not p.psquare else 0
        d.bperp = ptr(src["bperp"])
        d.bperp_row_invariant = 1 if p.row_invariant else 0
        d.grid_lin = ptr(src["grid_lin"])
        d.n_i = p.n_i
        d.n_j = p.n_j
        d.weight0 = ptr(src["weight0"])
        d.low_pass = ptr(src["low_pass"])
        d.n_win_ex = int(np.asarray(p.low_pass).shape[0])
        d.clap_window = p.clap_window
        d.clap_alpha = p.clap_alpha
        d.clap_beta = p.clap_beta
        d.n_trial_wraps = p.n_trial_wraps
        d.nr = ptr(src["nr"])
        d.nr_max_nz_ix = p.nr_max_nz_ix
        d.low_coh_thresh = p.low_coh_thresh
        d.psquare = 1 if p.psquare else 0
        d.gamma_change_convergence = p.gamma_change_convergence
        d.gamma_max_iterations = p.gamma_max_iterations
        d.precision = prec
        d.pointers_on_device = on_dev
        check(self._lib.ps2_load_patch(self._ctx, ctypes.byref(d)))
        self.prepared = p
        self.precision = prec
        self._keep = []

    def autotune(self) -> tuple[int, list[float]]:
        """Pick the fastest launch shapes for this patch (ps2_autotune: topofit
        lanes per PS, CLAP warps and blocks per SM, binning blocks per SM);
        returns the topofit lanes and the time of each lane candidate."""
        lanes = ctypes.c_int32(0)
        ms = (ctypes.c_double * 4)()
        check(self._lib.ps2_autotune(self._ctx, ctypes.byref(lanes), ms))
        return int(lanes.value), list(ms)

    def reset(self) -> None:
        check(self._lib.ps2_reset(self._ctx))

    def launch_shapes(self, set_to=None) -> list[int]:
        """[topofit lanes, CLAP warps per block, CLAP blocks per SM, binning
        blocks per SM, CLAP form (0 window stack, 1 fused window blocks)]
        (ps2_launch_shapes; 0 = built-in rule); set_to pins them."""
        get = (ctypes.c_int32 * 5)()
        st = None if set_to is None else (ctypes.c_int32 * 5)(*[int(v) for v in set_to])
        check(self._lib.ps2_launch_shapes(self._ctx, get, st))
        return list(get) if set_to is None else [int(v) for v in set_to]

    def step(self) -> dict:
        """One iteration under the stop rule (ps2_step)."""
        st = _lib.IterStats()
        check(self._lib.ps2_step(self._ctx, ctypes.byref(st)))
        return st.as_dict()

    def export_state(self) -> bytes:
        """The loop state after the last iteration (ps2_export_state): an opaque
        checkpoint for this patch, loaded the same way, in this precision."""
        n = ctypes.c_int64(0)
        check(self._lib.ps2_export_state(self._ctx, None, ctypes.byref(n)))
        buf = ctypes.create_string_buffer(n.value)
        check(self._lib.ps2_export_state(self._ctx, buf, ctypes.byref(n)))
        return buf.raw[:n.value]

    def import_state(self, state: bytes) -> None:
        """Resume from a checkpoint of export_state (ps2_import_state): the next
        step/iterate/run continues with the iteration after the checkpoint."""
        check(self._lib.ps2_import_state(self._ctx, ctypes.c_char_p(state), ctypes.c_int64(len(state))))

    def run(self) -> dict:
        st = _lib.IterStats()
        check(self._lib.ps2_run_to_convergence(self._ctx, ctypes.byref(st)))
        return st.as_dict()

    def iterate(self, n: int) -> list[dict]:
        arr = (_lib.IterStats * int(n))()
        check(self._lib.ps2_iterate(self._ctx, ctypes.c_int64(n), arr))
        return [s.as_dict() for s in arr]

    def timing(self) -> tuple[float, list[float]]:
        tot = ctypes.c_double(0.0)
        per = (ctypes.c_double * 4)()
        check(self._lib.ps2_last_timing(self._ctx, ctypes.byref(tot), per))
        return tot.value, list(per)

    def launch_count(self) -> int:
        return int(self._lib.ps2_last_launch_count(self._ctx))

    def download(self, keys=None, out=None) -> dict:
        """pm1.mat variables (native_stage2.rs:1899-1965) in the caller's row order.
        out: optional arrays to fill for the per-PS vectors (K_ps, C_ps,
        coh_ps, N_opt, coh_ps_save: float64, C-contiguous, n_ps long), for
        callers that reuse (for example pinned) host buffers across patches."""
        p = self.prepared
        n, m = p.n_ps, p.n_ifg
        fp64 = self.precision == PRECISION_FP64
        want = set(keys) if keys else {"K_ps", "C_ps", "coh_ps", "N_opt", "ph_res", "ph_patch", "ph_grid",
                                        "ph_weight", "coh_ps_save", "Nr"}
        given = out or {}
        out = {}
        o = _lib.Outputs()
        for k in ("K_ps", "C_ps", "coh_ps", "N_opt", "coh_ps_save"):
            if k in want:
                g = given.get(k)
                if g is not None:
                    if not (isinstance(g, np.ndarray) and g.dtype == np.float64 and g.shape == (n,)
                            and g.flags.c_contiguous and g.flags.writeable):
                        raise ValueError(f"download: out[{k!r}] must be a writeable C-contiguous float64 array "
                                         f"of length {n}")
                    out[k] = g
                else:
                    out[k] = np.empty(n, dtype=np.float64)
                setattr(o, k, ptr(out[k]))
        cdt, rdt = (np.complex128, np.float64) if fp64 else (np.complex64, np.float32)
        suffix = "_f64" if fp64 else ""
        if "ph_res" in want:
            out["ph_res"] = np.empty((n, m), dtype=rdt)
            setattr(o, "ph_res" + suffix, ptr(out["ph_res"]))
        if "ph_patch" in want:
            out["ph_patch"] = np.empty((n, m), dtype=cdt)
            setattr(o, "ph_patch" + suffix, ptr(out["ph_patch"]))
        if "ph_weight" in want:
            out["ph_weight"] = np.empty((n, m), dtype=cdt)
            setattr(o, "ph_weight" + suffix, ptr(out["ph_weight"]))
        if "ph_grid" in want:
            out["ph_grid"] = np.empty((p.n_i, p.n_j, m), dtype=cdt)
            setattr(o, "ph_grid" + suffix, ptr(out["ph_grid"]))
        if "Nr" in want:
            out["Nr"] = np.empty(100, dtype=np.float64)
            o.Nr = ptr(out["Nr"])
        gcs = np.zeros(1, dtype=np.float64)
        il = np.zeros(1, dtype=np.int64)
        o.gamma_change_save = ptr(gcs)
        o.i_loop = ptr(il)
        check(self._lib.ps2_download(self._ctx, ctypes.byref(o)))
        out["gamma_change_save"] = float(gcs[0])
        out["i_loop"] = int(il[0])
        out.update(
            step_number=1.0, n_trial_wraps=float(np.float32(p.n_trial_wraps)), grid_ij=p.grid_ij,
            grid_size=p.grid_size, low_pass=p.low_pass, Nr_max_nz_ix=p.nr_max_nz_ix, coh_bins=COH_BINS.copy(),
        )
        return out


def run_stage2(patch: dict | PreparedPatch, *, precision: str = "fp32", device: int = 0, nr=None,
               nr_max_nz_ix=None, keys=None) -> dict:
    """Prepare (if needed), run to convergence and download one patch."""
    p = patch if isinstance(patch, PreparedPatch) else prepare_patch(patch, nr=nr, nr_max_nz_ix=nr_max_nz_ix)
    with Stage2Context(device) as ctx:
        ctx.load(p, precision)
        last = ctx.run()
        res = ctx.download(keys)
        res["stats"] = last
        res["ms"] = ctx.timing()
    return res


# ---------------------------------------------------------------- MAT I/O --
def _resolve_parms(patch_dir: Path) -> Path | None:
    for cand in (patch_dir / "parms.mat", patch_dir.parent / "parms.mat", patch_dir.parent.parent / "parms.mat"):
        if cand.exists():
            return cand
    return None


def _scalar(d: dict, key: str, default):
    v = d.get(key)
    if v is None:
        return default
    a = np.asarray(v)
    if a.dtype.kind in "US":
        return str(a.reshape(-1)[0]).strip() if a.size else default
    if a.size == 0:
        return default
    return a.reshape(-1)[0].item()


def _mean_incidence(patch_dir: Path, ps: dict) -> float:
    """stage2_trial_wrap_mean_incidence (native_stage2.rs:2130-2153)."""
    from scipy.io import loadmat

    for fname, var, off in (("inc1.mat", "inc", 0.0), ("la1.mat", "la", 0.052)):
        f = patch_dir / fname
        if f.exists():
            try:
                vals = np.asarray(loadmat(f).get(var), dtype=np.float64).reshape(-1)
            except Exception:
                continue
            ok = vals[np.isfinite(vals) & ((vals != 0.0) | (var == "la"))]
            if ok.size:
                return float(ok.sum() / ok.size + off)
    mi = ps.get("mean_incidence")
    if mi is not None:
        return float(np.asarray(mi, dtype=np.float64).reshape(-1)[0]) + 0.052
    return DEFAULT_MEAN_INCIDENCE


def load_patch_dir(patch_dir: Path) -> dict:
    from scipy.io import loadmat

    patch_dir = Path(patch_dir)
    try:
        ps = loadmat(patch_dir / "ps1.mat")
    except Exception as err:
        raise Stage2Error(f"unable to read ps1.mat: {err}")
    try:
        ph = loadmat(patch_dir / "ph1.mat")
    except Exception as err:
        raise Stage2Error(f"unable to read ph1.mat: {err}")
    n_ps = int(round(float(_scalar(ps, "n_ps", 0.0))))
    if n_ps == 0:
        raise Stage2Error("ps1.mat missing valid n_ps")
    phv = np.asarray(ph.get("ph"))
    if phv.ndim != 2:
        raise Stage2Error("ph1.ph is missing or invalid")
    if phv.shape[0] != n_ps and phv.shape[1] == n_ps:
        phv = phv.T
    if phv.shape[0] != n_ps:
        raise Stage2Error(f"ph1.ph has incompatible shape {phv.shape[0]}x{phv.shape[1]} for n_ps={n_ps}")
    pf = _resolve_parms(patch_dir)
    parms = {}
    if pf is not None:
        try:
            raw = loadmat(pf)
            for k in DEFAULT_PARMS:
                if k in raw:
                    parms[k] = _scalar(raw, k, DEFAULT_PARMS[k])
        except Exception:
            parms = {}
    patch = {
        "ph": phv.astype(np.complex64),
        "bperp": np.asarray(ps.get("bperp"), dtype=np.float64).reshape(-1),
        "master_ix": float(_scalar(ps, "master_ix", 1.0)),
        "xy": np.asarray(ps.get("xy"), dtype=np.float32),
        "mean_incidence": _mean_incidence(patch_dir, ps),
        "parms": parms,
    }
    if (patch_dir / "bp1.mat").exists():
        try:
            patch["bperp_mat"] = np.asarray(loadmat(patch_dir / "bp1.mat").get("bperp_mat"), dtype=np.float64)
        except Exception as err:
            raise Stage2Error(f"unable to read bp1.mat: {err}")
    if (patch_dir / "da1.mat").exists():
        da = loadmat(patch_dir / "da1.mat").get("D_A")
        if da is not None:
            patch["D_A"] = np.asarray(da, dtype=np.float64).reshape(-1)
    if "ifgday_ix" in ps:
        ix = np.asarray(ps["ifgday_ix"], dtype=np.float64)
        patch["ifgday_ix"] = np.rint(ix if ix.shape[-1] == 2 else ix.T).astype(np.int64)
        patch["n_image"] = int(np.rint(ix).max())
    return patch


def write_pm1(path: Path, res: dict) -> None:
    """write_pm1 (native_stage2.rs:1899-1965) as a MATLAB v5 file."""
    from scipy.io import savemat

    col = lambda v: np.asarray(v, dtype=np.float64).reshape(-1, 1)  # noqa: E731
    row = lambda v: np.asarray(v, dtype=np.float64).reshape(1, -1)  # noqa: E731
    savemat(path, {
        "K_ps": col(res["K_ps"]), "C_ps": col(res["C_ps"]), "coh_ps": col(res["coh_ps"]), "N_opt": col(res["N_opt"]),
        "ph_res": np.asarray(res["ph_res"], dtype=np.float32),
        "ph_patch": np.asarray(res["ph_patch"], dtype=np.complex64), "step_number": 1.0,
        "ph_grid": np.asarray(res["ph_grid"], dtype=np.complex64),
        "n_trial_wraps": np.float32(res["n_trial_wraps"]), "grid_ij": np.asarray(res["grid_ij"], dtype=np.float32),
        "grid_size": float(res["grid_size"]), "low_pass": np.asarray(res["low_pass"], dtype=np.float64),
        "i_loop": float(res["i_loop"]), "ph_weight": np.asarray(res["ph_weight"], dtype=np.complex64),
        "Nr": row(res["Nr"]), "Nr_max_nz_ix": float(res["Nr_max_nz_ix"]), "coh_bins": row(res["coh_bins"]),
        "coh_ps_save": col(res["coh_ps_save"]), "gamma_change_save": float(res["gamma_change_save"]),
    })


def stage2_estimate_gamma(patch_dir, backend: str = "auto", kernel_backend: str = "cuda", native_threads: int = 0,
                          device: int = 0, precision: str = "fp32") -> str:
    """Drop-in for ported.stage2_estimate_gamma / run_stage2_native_with_threads
    with the cuda kernel backend: reads the patch, runs the loop on the GPU,
    writes pm1.mat and returns the reference's summary line."""
    kb = (kernel_backend or "cuda").strip().lower()
    if kb in ("gpu",):
        kb = "cuda"
    if kb not in ("cuda", "auto"):
        raise ValueError(f"Unsupported stage-2 kernel backend '{kernel_backend}' for this package. Use: cuda")
    patch_dir = Path(patch_dir)
    patch = load_patch_dir(patch_dir)
    if os.environ.get("PYSTAMPS_STAGE2_NATIVE_DEBUG_PM") is None:
        res = run_stage2(patch, precision=precision, device=device)
    else:
        # the reference's per-iteration dumps (native_stage2.rs:259, 337-356,
        # 385-404): pm1_iter_NN.mat after every iteration
        p = prepare_patch(patch)
        with Stage2Context(device) as ctx:
            ctx.load(p, precision)
            while True:
                st = ctx.step()
                res = ctx.download()
                write_pm1(patch_dir / f"pm1_iter_{res['i_loop']:02d}.mat", res)
                if st["stop"]:
                    break
    write_pm1(patch_dir / "pm1.mat", res)
    return f"Stage 2 computed coherence for {res['K_ps'].size} candidates in {res['i_loop']} iterations using the cuda backend"
