"""The ``cuda`` provider for the reference's stage-2 kernel registry.

Same names, argument meaning and return values as the registry wrappers in
pystamps/kernels/accelerated.py:429-509 (``run_stage2_grid_accumulate_kernel``,
``run_stage2_topofit_kernel``, ``run_stage2_topofit_row_invariant_kernel``,
``run_stage2_topofit_coh_row_invariant_kernel``, ``run_stage2_histogram_kernel``)
with ``backend="cuda"``, and the registry's topofit rule (near-max candidates,
ported._ps_topofit_single); ``run_native_topofit_rows`` is the native driver's
first-argmax rule that the gamma loop uses. Each call goes
through the C ABI of libps2cuda (host buffers in, host buffers out). There is
no CPU fallback: a missing library or device raises
``BackendUnavailableError``.
"""
from __future__ import annotations

import ctypes

import numpy as np

from ._lib import BackendUnavailableError, check, lib, ptr  # noqa: F401

_BACKENDS = ("cuda", "gpu", "auto")


def _backend(backend: str) -> None:
    if (backend or "auto").strip().lower() not in _BACKENDS:
        raise ValueError(f"Unsupported kernel backend '{backend}' for the cuda provider")


def run_stage2_grid_accumulate_kernel(ph_weight, grid_lin, n_i: int, n_j: int, *, backend: str = "cuda",
                                      threads: int = 0, out=None):
    """accumulate_weighted_grid (src/lib.rs:1013-1087): complex64 [n_i, n_j, M]."""
    _backend(backend)
    ph = np.ascontiguousarray(ph_weight, dtype=np.complex64)
    if ph.ndim != 2:
        raise ValueError("ph_weight must be a 2-D complex array")
    gl = np.ascontiguousarray(np.asarray(grid_lin).reshape(-1), dtype=np.int64)
    if gl.size != ph.shape[0]:
        raise ValueError("grid_lin length must match ph_weight rows")
    res = np.empty((int(n_i), int(n_j), ph.shape[1]), dtype=np.complex64)
    check(lib().ps2_grid_accumulate(ctypes.c_void_p(ptr(ph)), ctypes.c_void_p(ptr(gl)), ctypes.c_int64(ph.shape[0]),
                                    ctypes.c_int64(ph.shape[1]), ctypes.c_int64(n_i), ctypes.c_int64(n_j),
                                    ctypes.c_void_p(ptr(res))))
    if out is not None:
        out[...] = res
        return out
    return res


NEAR_MAX_COH_TOL = 2.0e-4  # ported._STAGE2_TOPOFIT_NEAR_MAX_COH_TOL (pystamps/pipeline/ported.py:47)


def _near_max(cpx, bp_arr, row_inv: bool, n_trial_wraps: float, tol: float, single: bool, residual: bool = True):
    rdt, cdt = (np.float32, np.complex64) if single else (np.float64, np.complex128)
    cpx = np.ascontiguousarray(cpx, dtype=cdt)
    n, m = cpx.shape
    bp = np.ascontiguousarray(bp_arr, dtype=rdt)
    K = np.empty(n)
    C = np.empty(n)
    coh = np.empty(n)
    res = np.empty((n, m), dtype=np.complex64) if residual else None
    check(lib().ps2_topofit_near_max(ctypes.c_void_p(ptr(cpx)), ctypes.c_void_p(ptr(bp)), ctypes.c_int32(int(row_inv)),
                                     ctypes.c_int32(0 if single else 1), ctypes.c_double(n_trial_wraps),
                                     ctypes.c_int64(n), ctypes.c_int64(m), ctypes.c_double(tol),
                                     ctypes.c_void_p(ptr(K)), ctypes.c_void_p(ptr(C)), ctypes.c_void_p(ptr(coh)),
                                     ctypes.c_void_p(ptr(res))))
    return K, C, coh, res


def _cpx2d(cpxphase):
    cpx = np.asarray(cpxphase)
    if cpx.ndim != 2:
        raise ValueError("cpxphase must be a 2-D complex array")
    return cpx


def _single(cpx, bp) -> bool:
    """The reference's precision choice (_ps_topofit_single: single precision
    when either input is)."""
    return cpx.dtype == np.complex64 or np.asarray(bp).dtype == np.float32


def _row_invariant_vector(bperp, n_row: int):
    """_stage2_row_invariant_bperp_matrix (pystamps/kernels/accelerated.py:
    284-306): the row vector the row-invariant kernels use (row 0 of a matrix)."""
    bp = np.asarray(bperp)
    real_dtype = np.float32 if bp.dtype == np.float32 else np.float64
    if bp.ndim == 1:
        return np.ascontiguousarray(bp.reshape(-1), dtype=real_dtype)
    if bp.ndim == 2:
        if bp.shape[0] not in {1, int(n_row)}:
            raise BackendUnavailableError(
                f"Row-invariant stage-2 bperp has incompatible shape {bp.shape} for n_row={n_row}")
        return np.ascontiguousarray(bp.reshape(-1) if bp.shape[0] == 1 else bp[0, :], dtype=real_dtype)
    raise BackendUnavailableError("Row-invariant stage-2 bperp must be a 1-D vector or 2-D matrix")


def run_stage2_topofit_kernel(cpxphase, bperp, n_trial_wraps: float, *, backend: str = "cuda", threads: int = 0,
                              cpu_fallback=None, near_max_tol: float = NEAR_MAX_COH_TOL):
    """The registry's "stage2_topofit" (pystamps/kernels/accelerated.py:446-460):
    _ps_topofit_batch_generic (pystamps/pipeline/ported.py:2516-2532), i.e.
    _ps_topofit_single per row: zero columns skipped, near-max candidates
    within near_max_tol (2e-4; the PyO3 twin, src/lib.rs:525-586, uses 5e-3)
    refined and chosen as the reference chooses. Single precision when either
    input is (complex64 / float32), double otherwise. bperp [n, m] (or a
    vector, then the row-invariant kernel). Returns (K, C, coh, residual
    complex64)."""
    _backend(backend)
    cpx = _cpx2d(cpxphase)
    n, m = cpx.shape
    bp = np.asarray(bperp)
    if bp.ndim == 1:
        return run_stage2_topofit_row_invariant_kernel(cpx, bp, n_trial_wraps, backend=backend,
                                                       near_max_tol=near_max_tol)
    if bp.shape != (n, m):
        raise ValueError(f"bperp has shape {bp.shape}; expected {(n, m)}")
    return _near_max(cpx, bp, False, n_trial_wraps, near_max_tol, _single(cpx, bp))


def run_stage2_topofit_row_invariant_kernel(cpxphase, bperp, n_trial_wraps: float, *, backend: str = "cuda",
                                            threads: int = 0, cpu_fallback=None,
                                            near_max_tol: float = NEAR_MAX_COH_TOL):
    """The registry's "stage2_topofit_row_invariant" (accelerated.py:463-477):
    _ps_topofit_batch_row_invariant (ported.py:2535-2552), the first bperp row
    for every row."""
    _backend(backend)
    cpx = _cpx2d(cpxphase)
    vec = _row_invariant_vector(bperp, cpx.shape[0])
    if vec.size != cpx.shape[1]:
        raise ValueError(f"bperp has {vec.size} columns; expected {cpx.shape[1]}")
    return _near_max(cpx, vec, True, n_trial_wraps, near_max_tol, _single(cpx, vec))


def run_stage2_topofit_coh_row_invariant_kernel(cpxphase, bperp, n_trial_wraps: float, *, backend: str = "cuda",
                                                threads: int = 0, cpu_fallback=None,
                                                near_max_tol: float = NEAR_MAX_COH_TOL):
    """The registry's "stage2_topofit_coh_row_invariant" (accelerated.py:480-493):
    _ps_topofit_batch_row_invariant_coh (ported.py:2555-2620), which works in
    complex128 / float64 whatever the input precision. Returns coh f64 [n].
    Rows with some zero columns: the reference's vectorised single-candidate
    path takes the bperp range over all columns, here it is taken over the
    non-zero ones as _ps_topofit_single does; the two agree when no element is
    zero (the random-phase rows this kernel serves)."""
    _backend(backend)
    cpx = _cpx2d(cpxphase)
    vec = _row_invariant_vector(bperp, cpx.shape[0]).astype(np.float64)
    if vec.size != cpx.shape[1]:
        raise ValueError(f"bperp has {vec.size} columns; expected {cpx.shape[1]}")
    return _near_max(cpx, vec, True, n_trial_wraps, near_max_tol, False, residual=False)[2]


def run_stage2_histogram_kernel(values, centers, *, backend: str = "cuda"):
    """The registry's "stage2_histogram" (accelerated.py:496-509 over
    _stage2_histogram_with_centers_cpu, :235-265): counts per centre of the
    finite values, f64."""
    _backend(backend)
    v = np.asarray(values, dtype=np.float64).reshape(-1)
    v = np.ascontiguousarray(v[np.isfinite(v)])
    c = np.ascontiguousarray(np.asarray(centers, dtype=np.float64).reshape(-1))
    out = np.zeros(c.size, dtype=np.float64)
    check(lib().ps2_histogram_with_centers(ctypes.c_void_p(ptr(v)), ctypes.c_int64(v.size), ctypes.c_void_p(ptr(c)),
                                           ctypes.c_int64(c.size), ctypes.c_void_p(ptr(out))))
    return out


def run_native_topofit_rows(cpxphase, bperp, n_trial_wraps: float):
    """The native driver's topofit over rows (native_stage2.rs:659-720,
    1207-1303: first-argmax peak, FP32) through ps2_topofit: the rule the gamma
    loop uses. Zero columns are skipped; an all-zero row gives NaN. Returns
    (K, C, coh, residual complex64)."""
    cpx = np.ascontiguousarray(_cpx2d(cpxphase), dtype=np.complex64)
    n, m = cpx.shape
    bp = np.asarray(bperp)
    row_inv = 1 if bp.ndim == 1 or (bp.ndim == 2 and bp.shape[0] == 1) else 0
    bp = np.ascontiguousarray(bp.reshape(-1) if row_inv else bp, dtype=np.float32)
    if (row_inv and bp.size != m) or (not row_inv and bp.shape != (n, m)):
        raise ValueError("bperp must be [n, m] or [m]")
    K = np.empty(n)
    C = np.empty(n)
    coh = np.empty(n)
    res = np.empty((n, m), dtype=np.complex64)
    check(lib().ps2_topofit(ctypes.c_void_p(ptr(cpx)), ctypes.c_void_p(ptr(bp)), ctypes.c_int32(row_inv),
                            ctypes.c_double(n_trial_wraps), ctypes.c_int64(n), ctypes.c_int64(m),
                            ctypes.c_void_p(ptr(K)), ctypes.c_void_p(ptr(C)), ctypes.c_void_p(ptr(coh)),
                            ctypes.c_void_p(ptr(res))))
    return K, C, coh, res


def run_stage2_clap_filter_kernel(ph_grid, alpha: float, beta: float, low_pass, n_win: int = 24, *,
                                  backend: str = "cuda"):
    """clap_filter_grid_stack (native_stage2.rs:742-922): complex64 [n_i, n_j, M]."""
    _backend(backend)
    g = np.ascontiguousarray(ph_grid, dtype=np.complex64)
    if g.ndim != 3:
        raise ValueError("ph_grid must be [n_i, n_j, n_ifg]")
    lp = np.ascontiguousarray(low_pass, dtype=np.float64)
    out = np.empty_like(g)
    check(lib().ps2_clap_filter_grid(ctypes.c_void_p(ptr(g)), ctypes.c_int64(g.shape[0]), ctypes.c_int64(g.shape[1]),
                                     ctypes.c_int64(g.shape[2]), ctypes.c_int64(n_win), ctypes.c_double(alpha),
                                     ctypes.c_double(beta), ctypes.c_void_p(ptr(lp)), ctypes.c_int64(lp.shape[0]),
                                     ctypes.c_void_p(ptr(out))))
    return out


def run_stage2_random_hist_kernel(bperp_nm, n_trial_wraps: float, n_rand: int = 300_000, *, backend: str = "cuda",
                                  small_baseline: bool = False, ifgday_ix=None, n_image: int = 0):
    """(Nr, Nr_max_nz_ix) of random_coherence_histogram (native_stage2.rs:1310-1356)."""
    _backend(backend)
    from .stage2 import random_coherence_histogram

    return random_coherence_histogram(bperp_nm, n_trial_wraps, n_rand, small_baseline, ifgday_ix, n_image)
