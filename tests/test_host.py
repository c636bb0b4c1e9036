"""Host-side preparation (prepare_stage2_inputs restated for the GPU path) against the oracle."""
import math

import numpy as np
import pytest

from pystamps_b200 import stage2, synth


@pytest.fixture(scope="module", autouse=True)
def _host_library(cuda_lib):
    """prepare_patch runs its row passes in the library's host code (no device)."""
    return cuda_lib


@pytest.fixture(scope="module")
def small_patch():
    return synth.make_patch(3000, 10, 31, 21, seed=11, n_rand=2000)


def test_grid_indices_bit_exact_with_oracle(oracle, small_patch):
    xy = small_patch["xy"]
    np.testing.assert_array_equal(stage2.grid_indices(xy, 50.0), oracle.grid_indices(xy, 50.0))
    rng = np.random.default_rng(3)
    xy2 = np.column_stack([np.arange(5000), rng.uniform(-3e4, 3e4, 5000), rng.uniform(-1e3, 9e4, 5000)]).astype(np.float32)
    for g in (50.0, 37.5, 100.0):
        np.testing.assert_array_equal(stage2.grid_indices(xy2, g), oracle.grid_indices(xy2, g))


def test_grid_indices_nan_and_infinite_coordinates(oracle):
    """Rust's f32::min/max skip NaN (native_stage2.rs:1973-1989): a NaN
    coordinate is left out of the minimum and gets bin 1; an infinite one
    saturates the i32 bin like `as i32`."""
    rng = np.random.default_rng(5)
    xy = np.column_stack([np.arange(400), rng.uniform(0, 3000, 400), rng.uniform(0, 2000, 400)]).astype(np.float32)
    xy[3, 1] = np.nan
    xy[7, 2] = np.nan
    xy[9, 1:] = np.nan
    g = stage2.grid_indices(xy, 50.0)
    np.testing.assert_array_equal(g, oracle.grid_indices(xy, 50.0))
    assert g[3, 1] == 1 and g[7, 0] == 1 and g[9, 0] == 1 and g[9, 1] == 1
    ok = np.isfinite(xy[:, 1]) & np.isfinite(xy[:, 2])
    np.testing.assert_array_equal(g[ok], stage2.grid_indices(xy[ok], 50.0))
    # every coordinate NaN: min stays +inf, every bin 1
    allnan = xy.copy()
    allnan[:, 1:] = np.nan
    np.testing.assert_array_equal(stage2.grid_indices(allnan, 50.0), np.ones((400, 2), np.float32))
    np.testing.assert_array_equal(oracle.grid_indices(allnan, 50.0), np.ones((400, 2), np.float32))
    inf = xy[:20].copy()
    inf[4, 2] = np.inf
    gi = stage2.grid_indices(inf, 50.0)
    np.testing.assert_array_equal(gi, oracle.grid_indices(inf, 50.0))
    assert gi[4, 0] == np.float32(2 ** 31 - 2)


def test_prepare_patch_with_nan_coordinates_matches_oracle_cells(oracle):
    patch = synth.make_patch(2000, 8, 24, 21, seed=12, n_rand=1000)
    xy = np.array(patch["xy"], dtype=np.float32)
    xy[[5, 50, 500], 1] = np.nan
    patch = dict(patch, xy=xy)
    prep = stage2.prepare_patch(patch, nr=np.ones(100), nr_max_nz_ix=100.0)
    g = oracle.grid_indices(xy, 50.0)
    assert np.all(prep.grid_ij[[5, 50, 500], 1] == 1)
    np.testing.assert_array_equal(prep.grid_ij, g)


def test_grid_boundary_bin_single_precision():
    xy = np.array([[1.0, -23497.43359375, 0.0], [2.0, -21497.43359375, 0.0], [3.0, -20497.43359375, 0.0]],
                  dtype=np.float32)
    assert int(stage2.grid_indices(xy, 50.0)[1, 1]) == 40


def test_low_pass_bit_exact_with_oracle(oracle):
    np.testing.assert_array_equal(stage2.build_low_pass(32.0, 800.0, 50.0), oracle.build_low_pass(32.0, 800.0, 50.0))


@pytest.mark.parametrize("name", ["A", "B", "D", "E"])
def test_synthetic_workloads_realise_their_shapes(name):
    w = synth.ALIASES[name]
    # a thin version of the workload: same extent, trial rule and baselines
    p = synth.make_workload(w, n_ps=4000, n_ifg=w.n_ifg)
    prep = stage2.prepare_patch(p, nr=np.ones(100))
    assert (prep.n_i, prep.n_j) == (w.cells, w.cells)
    assert stage2.trial_count(prep.n_trial_wraps) == w.n_trials
    assert prep.n_ifg == w.n_ifg
    assert not prep.row_invariant


def test_prepare_matches_oracle_setup(oracle, small_patch):
    prep = stage2.prepare_patch(small_patch, nr=np.ones(100))
    r = oracle.stage2_run(dict(small_patch, parms=dict(small_patch["parms"], gamma_max_iterations=1)))
    assert prep.n_trial_wraps == r["n_trial_wraps"]
    np.testing.assert_array_equal(prep.grid_ij, r["grid_ij"])
    assert (prep.n_i, prep.n_j) == (r["n_i"], r["n_j"])
    assert prep.low_coh_thresh == 31 and prep.psquare
    np.testing.assert_array_equal(prep.weight0, 1.0 / small_patch["D_A"])


def test_prepare_normalises_and_keeps_zero(small_patch):
    p = dict(small_patch)
    ph = p["ph"].copy()
    ph[0, 3] = 0
    ph[1, 2] = 3.0 - 4.0j
    p["ph"] = ph
    prep = stage2.prepare_patch(p, nr=np.ones(100))
    assert prep.ph_nm[0, 2] == 0 and prep.amp[0, 2] == 1.0
    assert prep.ph_nm[1, 1] == np.complex64(0.6 - 0.8j) and prep.amp[1, 1] == 5.0


def test_prepare_error_paths(small_patch):
    bad = dict(small_patch, bperp_mat=np.ones((small_patch["ph"].shape[0], 1)))
    with pytest.raises(stage2.Stage2Error, match="bp1.bperp_mat has incompatible shape"):
        stage2.prepare_patch(bad, nr=np.ones(100))
    with pytest.raises(stage2.Stage2Error, match="master_ix"):
        stage2.prepare_patch(dict(small_patch, master_ix=99), nr=np.ones(100))
    with pytest.raises(stage2.Stage2Error, match="stage 2 native implementation error"):
        stage2.prepare_patch(dict(small_patch, bperp=np.zeros(3)), nr=np.ones(100))


def test_row_invariant_bperp_detected(small_patch):
    p = dict(small_patch, bperp_mat=np.tile(small_patch["bperp"][1:], (small_patch["ph"].shape[0], 1)))
    prep = stage2.prepare_patch(p, nr=np.ones(100))
    assert prep.row_invariant and prep.bperp.shape == (10,)


def test_mat_roundtrip_patch_dir(tmp_path, small_patch):
    from scipy.io import savemat

    d = tmp_path / "PATCH_1"
    d.mkdir()
    n = small_patch["ph"].shape[0]
    savemat(d / "ps1.mat", {"n_ps": float(n), "master_ix": 1.0, "bperp": small_patch["bperp"].reshape(1, -1),
                            "xy": small_patch["xy"]})
    savemat(d / "ph1.mat", {"ph": small_patch["ph"]})
    savemat(d / "bp1.mat", {"bperp_mat": small_patch["bperp_mat"]})
    savemat(d / "da1.mat", {"D_A": small_patch["D_A"].reshape(-1, 1)})
    savemat(d / "inc1.mat", {"inc": np.full((n, 1), small_patch["mean_incidence"])})
    savemat(d / "parms.mat", dict(small_patch["parms"]))
    p = stage2.load_patch_dir(d)
    assert p["ph"].shape == small_patch["ph"].shape
    # the reference averages the per-PS incidences (sum / count)
    inc = np.full(n, small_patch["mean_incidence"])
    assert p["mean_incidence"] == inc.sum() / n
    a = stage2.prepare_patch(p, nr=np.ones(100))
    b = stage2.prepare_patch(dict(small_patch, mean_incidence=inc.sum() / n), nr=np.ones(100))
    assert a.n_trial_wraps == b.n_trial_wraps
    np.testing.assert_array_equal(a.grid_lin, b.grid_lin)
