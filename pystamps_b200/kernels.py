"""The ``cuda`` provider for the reference's stage-2 kernel registry.

Same names, argument meaning and return values as the registry wrappers in
pystamps/kernels/accelerated.py:429-509 (``run_stage2_grid_accumulate_kernel``,
``run_stage2_topofit_kernel``, ...) with ``backend="cuda"``; each call goes
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


def run_stage2_topofit_kernel(cpxphase, bperp, n_trial_wraps: float, *, backend: str = "cuda", threads: int = 0,
                              cpu_fallback=None):
    """ps_topofit over rows (src/lib.rs:1159-1247) with the native driver's
    first-argmax peak (native_stage2.rs:1207-1257). Returns (K, C, coh,
    residual complex64)."""
    _backend(backend)
    cpx = np.ascontiguousarray(cpxphase, dtype=np.complex64)
    if cpx.ndim != 2:
        raise ValueError("cpxphase must be a 2-D complex array")
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


run_stage2_topofit_row_invariant_kernel = run_stage2_topofit_kernel


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
