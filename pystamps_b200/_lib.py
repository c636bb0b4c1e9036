"""ctypes binding of libps2cuda.so (the C ABI in include/ps2cuda.h).

The library is built in-tree (pystamps_b200/libps2cuda.so) by
``pystamps_b200.build.build()``. There is no CPU fallback: when the library or
a CUDA device is missing, every entry point raises ``BackendUnavailableError``.
"""
from __future__ import annotations

import ctypes
import os
from pathlib import Path

_HERE = Path(__file__).resolve().parent
LIB_PATH = _HERE / "libps2cuda.so"

PS2_OK = 0
ERRORS = {
    -1: "invalid argument",
    -2: "CUDA error",
    -3: "no patch loaded",
    -4: "unsupported",
    -5: "out of device memory",
}
PRECISION_FP32 = 0
PRECISION_FP64 = 1
COH_BINS = 100

c_i64 = ctypes.c_int64
c_i32 = ctypes.c_int32
c_dbl = ctypes.c_double
c_vp = ctypes.c_void_p

# Every symbol the header declares (tests check the library exports them all).
EXPORTED = (
    "ps2_create", "ps2_destroy", "ps2_last_error", "ps2_load_patch", "ps2_iterate", "ps2_run_to_convergence",
    "ps2_reset", "ps2_download", "ps2_last_timing", "ps2_last_launch_count", "ps2_grid_accumulate", "ps2_topofit",
    "ps2_clap_filter_grid", "ps2_random_coherence_histogram", "ps2_clap_filter_grid_noalloc", "ps2_autotune",
    "ps2_coherence_forward", "ps2_coherence_backward", "ps2_batch_run", "ps3_reestimate",
    "ps2_stage3_reestimate", "ps2_shard_bin", "ps2_shard_filter", "ps2_shard_fit", "ps2_shard_finalize",
    "ps2_prepare_phase", "ps2_prepare_bperp", "ps2_topofit_near_max", "ps2_histogram_with_centers",
    "ps2_export_state", "ps2_import_state", "ps2_step", "ps2_launch_shapes",
)


class BackendUnavailableError(RuntimeError):
    """The CUDA stage-2 backend cannot run (library or device missing)."""


class Stage2CudaError(RuntimeError):
    """A ps2_* call returned an error status."""

    def __init__(self, code: int, message: str):
        self.code = code
        super().__init__(f"stage 2 cuda implementation error ({ERRORS.get(code, code)}): {message}")


class PatchDesc(ctypes.Structure):
    _fields_ = [
        ("n_ps", c_i64), ("n_ifg", c_i64), ("ph_nm", c_vp), ("amp", c_vp), ("bperp", c_vp),
        ("bperp_row_invariant", c_i32), ("grid_lin", c_vp), ("n_i", c_i64), ("n_j", c_i64),
        ("weight0", c_vp), ("low_pass", c_vp), ("n_win_ex", c_i64), ("clap_window", c_i64),
        ("clap_alpha", c_dbl), ("clap_beta", c_dbl), ("n_trial_wraps", c_dbl), ("nr", c_vp),
        ("nr_max_nz_ix", c_dbl), ("low_coh_thresh", c_i64), ("psquare", c_i32),
        ("gamma_change_convergence", c_dbl), ("gamma_max_iterations", c_i64), ("precision", c_i32),
        ("pointers_on_device", c_i32),
    ]


class IterStats(ctypes.Structure):
    _fields_ = [
        ("i_loop", c_i64), ("gamma_change_rms", c_dbl), ("gamma_change_delta", c_dbl), ("stop", c_i32),
        ("n_invalid", c_i32),
    ]

    def as_dict(self) -> dict:
        return {k: getattr(self, k) for k, _ in self._fields_}


class Outputs(ctypes.Structure):
    _fields_ = [
        ("K_ps", c_vp), ("C_ps", c_vp), ("coh_ps", c_vp), ("N_opt", c_vp), ("ph_res", c_vp), ("ph_patch", c_vp),
        ("ph_grid", c_vp), ("ph_weight", c_vp), ("coh_ps_save", c_vp), ("Nr", c_vp), ("gamma_change_save", c_vp),
        ("i_loop", c_vp), ("ph_res_f64", c_vp), ("ph_patch_f64", c_vp), ("ph_grid_f64", c_vp),
        ("ph_weight_f64", c_vp),
    ]


class S3Desc(ctypes.Structure):
    _fields_ = [
        ("n_sel", c_i64), ("n_ifg", c_i64), ("ph", c_vp), ("bperp", c_vp), ("grid_ij", c_vp), ("ph_grid", c_vp),
        ("grid_rows", c_i64), ("grid_cols", c_i64), ("n_i", c_i64), ("n_j", c_i64), ("fit_ifg", c_vp),
        ("n_fit", c_i64), ("clap_win", c_i64), ("clap_alpha", ctypes.c_double), ("clap_beta", ctypes.c_double),
        ("low_pass", c_vp), ("slc_osf", c_i64), ("n_trial_wraps", ctypes.c_double),
    ]


class S3Out(ctypes.Structure):
    _fields_ = [("ph_patch2", c_vp), ("K_ps2", c_vp), ("C_ps2", c_vp), ("coh_ps2", c_vp), ("ph_res2", c_vp)]


_lib = None


def lib() -> ctypes.CDLL:
    """Load the in-tree library; raise if it is absent (no fallback)."""
    global _lib
    if _lib is not None:
        return _lib
    path = Path(os.environ.get("PS2CUDA_LIB", str(LIB_PATH)))
    if not path.exists():
        raise BackendUnavailableError(
            f"{path} is missing: build it with `python -c 'import pystamps_b200.build as b; b.build()'`")
    L = ctypes.CDLL(str(path))
    L.ps2_last_error.restype = ctypes.c_char_p
    L.ps2_destroy.restype = None
    L.ps2_last_launch_count.restype = c_i64
    for name in EXPORTED:
        fn = getattr(L, name)
        if name not in ("ps2_last_error", "ps2_destroy", "ps2_last_launch_count"):
            fn.restype = ctypes.c_int
    _lib = L
    return L


def check(rc: int) -> None:
    if rc != PS2_OK:
        msg = lib().ps2_last_error().decode(errors="replace")
        raise Stage2CudaError(rc, msg)


def ptr(a) -> int:
    """Address of a numpy array or a torch tensor (host or device)."""
    if a is None:
        return 0
    if hasattr(a, "data_ptr"):
        return int(a.data_ptr())
    return int(a.ctypes.data)
