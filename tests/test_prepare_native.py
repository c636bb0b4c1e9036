"""The library's host passes of the stage-2 preparation (ps2_prepare_phase,
ps2_prepare_bperp; prepare_stage2_inputs, native_stage2.rs:447-467, 563-612)
give the numpy statement of the same steps bit for bit, edge values included.
Host code only: no device is touched."""
import ctypes

import numpy as np
import pytest

VP = ctypes.c_void_p


def _bits(a):
    return a.view(np.uint32 if a.dtype in (np.float32, np.complex64) else np.uint64)


def _numpy_phase(ph, cols):
    sub = ph[:, cols]
    re = np.ascontiguousarray(sub.real, dtype=np.float32)
    im = np.ascontiguousarray(sub.imag, dtype=np.float32)
    mag = np.hypot(re, im).astype(np.float32)
    safe = np.where(mag == 0.0, np.float32(1.0), mag).astype(np.float32)
    out = np.empty(sub.shape, np.complex64)
    with np.errstate(invalid="ignore"):
        out.real = re / safe
        out.imag = im / safe
    return out, safe


@pytest.mark.parametrize("threads", [1, 3, 0])
def test_phase_pass_matches_numpy(cuda_lib, threads):
    rng = np.random.default_rng(7)
    n, nf = 5000, 17
    scale = np.exp(rng.uniform(-45, 45, (n, nf)))
    ph = ((rng.standard_normal((n, nf)) * scale).astype(np.float32)
          + 1j * (rng.standard_normal((n, nf)) * scale).astype(np.float32)).astype(np.complex64)
    ph[::7, 3] = 0
    ph[::9, 4] = -0.0 + 0j
    ph[::11, 5] = np.nan
    ph[::13, 6] = np.inf + 1j
    ph[::17, 8] = 1e-45 - 1e-45j
    cols = np.array([k for k in range(nf) if k != 2], dtype=np.int64)
    ref, amp_ref = _numpy_phase(ph, cols)
    out = np.empty(ref.shape, np.complex64)
    amp = np.empty(ref.shape, np.float32)
    assert cuda_lib.ps2_prepare_phase(VP(ph.ctypes.data), ctypes.c_int64(n), ctypes.c_int64(nf),
                                      VP(cols.ctypes.data), ctypes.c_int64(cols.size), VP(out.ctypes.data),
                                      VP(amp.ctypes.data), ctypes.c_int(threads)) == 0
    np.testing.assert_array_equal(_bits(out), _bits(ref))
    np.testing.assert_array_equal(_bits(amp), _bits(amp_ref))


def test_bperp_pass_matches_numpy(cuda_lib):
    rng = np.random.default_rng(8)
    n, width = 4000, 12
    cols = np.arange(1, width, dtype=np.int64)
    inv = ctypes.c_int32(-1)
    for bm, expect_inv in ((rng.uniform(-400, 400, (n, width)), False),
                           (np.tile(rng.uniform(-400, 400, width), (n, 1)), True)):
        out = np.empty((n, cols.size), np.float32)
        assert cuda_lib.ps2_prepare_bperp(VP(bm.ctypes.data), ctypes.c_int64(n), ctypes.c_int64(width),
                                          VP(cols.ctypes.data), ctypes.c_int64(cols.size), VP(out.ctypes.data),
                                          ctypes.byref(inv), ctypes.c_int(0)) == 0
        np.testing.assert_array_equal(_bits(out), _bits(bm[:, cols].astype(np.float32)))
        assert bool(inv.value) == expect_inv == bool(np.all(bm[:, cols] == bm[0:1, cols]))
    bm = np.tile(rng.uniform(-400, 400, width), (n, 1))
    bm[n // 2, 3] = np.nan  # NaN never equals the first row
    out = np.empty((n, width), np.float32)
    assert cuda_lib.ps2_prepare_bperp(VP(bm.ctypes.data), ctypes.c_int64(n), ctypes.c_int64(width), VP(0),
                                      ctypes.c_int64(width), VP(out.ctypes.data), ctypes.byref(inv),
                                      ctypes.c_int(2)) == 0
    assert inv.value == 0


def test_host_passes_reject_bad_columns(cuda_lib):
    ph = np.zeros((4, 3), np.complex64)
    out = np.empty((4, 3), np.complex64)
    amp = np.empty((4, 3), np.float32)
    bad = np.array([0, 3, 1], dtype=np.int64)
    assert cuda_lib.ps2_prepare_phase(VP(ph.ctypes.data), ctypes.c_int64(4), ctypes.c_int64(3), VP(bad.ctypes.data),
                                      ctypes.c_int64(3), VP(out.ctypes.data), VP(amp.ctypes.data), ctypes.c_int(1)) != 0
    assert b"outside" in cuda_lib.ps2_last_error()
    bm = np.zeros((4, 3))
    inv = ctypes.c_int32(0)
    assert cuda_lib.ps2_prepare_bperp(VP(bm.ctypes.data), ctypes.c_int64(4), ctypes.c_int64(3), VP(0),
                                      ctypes.c_int64(2), VP(out.ctypes.data), ctypes.byref(inv), ctypes.c_int(1)) != 0
