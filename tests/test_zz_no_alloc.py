"""CLAP through the entry point that allocates no GPU memory.

Some callers of this library cannot call cudaMalloc: a host that runs under
another allocator's memory budget (a framework's caching pool, a Rust or JVM
host that hands in device buffers it already owns) or code that must avoid the
device-wide synchronisation of cudaMalloc/cudaFree. ps2_clap_filter_grid_noalloc
serves them from a fixed 32 MiB scratch array inside the library; the caller
passes device input and output buffers. This file is named so that pytest
collects it last.
"""
import ctypes

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _noalloc(lib, d_in, shape, low_pass, d_out, alpha=1.0, beta=0.3):
    n_i, n_j, m = shape
    return lib.ps2_clap_filter_grid_noalloc(
        ctypes.c_void_p(d_in.data_ptr()), ctypes.c_int64(n_i), ctypes.c_int64(n_j), ctypes.c_int64(m),
        ctypes.c_int64(24), ctypes.c_double(alpha), ctypes.c_double(beta),
        ctypes.c_void_p(low_pass.ctypes.data), ctypes.c_int64(32), ctypes.c_void_p(d_out.data_ptr()),
        ctypes.c_void_p(None))


def test_noalloc_clap_matches_the_allocating_entry_point_on_two_calls(cuda_lib):
    import torch

    from pystamps_b200 import kernels, stage2

    low_pass = np.ascontiguousarray(stage2.build_low_pass(32.0, 800.0, 50.0))
    rng = np.random.default_rng(12)
    # two calls in a row on different grids: the second reuses the scratch the first left behind
    for shape in [(64, 64, 20), (40, 37, 7)]:
        g = (rng.standard_normal(shape) + 1j * rng.standard_normal(shape)).astype(np.complex64)
        g[3, 5, 0] = np.nan
        ref = kernels.run_stage2_clap_filter_kernel(g, 1.0, 0.3, low_pass)
        d_in = torch.from_numpy(np.ascontiguousarray(g).view(np.float32)).cuda()
        d_out = torch.full_like(d_in, 7.0)
        rc = _noalloc(cuda_lib, d_in, shape, low_pass, d_out)
        assert rc == 0, cuda_lib.ps2_last_error()
        torch.cuda.synchronize()
        out = d_out.cpu().numpy().view(np.complex64).reshape(shape)
        scale = np.abs(ref).max()
        # the tolerance of the CLAP parity tests (relative to the largest output)
        assert np.abs(out - ref).max() <= 2e-6 * scale


def test_noalloc_clap_rejects_sizes_beyond_its_scratch(cuda_lib):
    import torch

    low_pass = np.zeros((32, 32))
    shape = (256, 256, 150)
    d_in = torch.zeros(4, dtype=torch.float32, device="cuda")
    rc = _noalloc(cuda_lib, d_in, shape, low_pass, d_in)
    assert rc == -4
    assert b"more than the fixed" in cuda_lib.ps2_last_error()
