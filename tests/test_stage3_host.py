"""Stage 3 on the CPU: the oracle's restatement of the re-estimate and the
host threshold statistics (pystamps_b200.stage3) against the golden vectors
produced by the Python reference (tests/golden/make_golden.py)."""
import numpy as np
import pytest


@pytest.fixture(scope="module")
def units(golden):
    return golden("stage3_units.npz")


@pytest.fixture(scope="module")
def sel(golden):
    return golden("stage3_select.npz")


def test_oracle_patch_clap_matches_reference(oracle, units):
    for k in range(units["clap_in"].shape[0]):
        a, b = units["clap_params"][k]
        out = oracle.s3_clap_patch(units["clap_in"][k], a, b, units["low_pass"])
        ref = units["clap_out"][k]
        assert np.abs(out - ref).max() <= 1e-13 * np.abs(ref).max(), k


def test_oracle_stage3_topofit_matches_reference(oracle, units):
    ntw = float(units["topo_ntw"])
    for r in range(units["topo_cpx"].shape[0]):
        K, C, coh, res, _ = oracle.s3_topofit_single(units["topo_cpx"][r], units["topo_bperp"][r], ntw)
        assert abs(K - units["topo_K"][r]) <= 1e-6 * max(abs(units["topo_K"][r]), 1e-3), r
        assert abs(coh - units["topo_coh"][r]) <= 1e-6, r
        assert np.abs(res - units["topo_res"][r]).max() <= 1e-5, r


def test_oracle_reestimate_matches_reference_select(oracle, sel):
    ix0 = sel["sel_ix"].ravel().astype(np.int64) - 1
    fit = sel["sel_ifg_index"].ravel().astype(np.int64) - 1
    out = oracle.s3_reestimate(sel["pm_ph_grid"], np.rint(sel["pm_grid_ij"]).astype(np.int64), ix0,
                               sel["ph"][:, 1:], sel["bperp_mat"], fit, alpha=1.0, beta=0.3,
                               low_pass=sel["pm_low_pass"], n_trial_wraps=float(sel["pm_n_trial_wraps"].ravel()[0]))
    pp = sel["sel_ph_patch2"]
    assert np.abs(out["ph_patch2"] - pp).max() <= 1e-6 * np.abs(pp).max()
    K = sel["sel_K_ps2"].ravel()
    np.testing.assert_array_equal(np.isnan(out["K_ps2"]), np.isnan(K))
    ok = ~np.isnan(K)
    assert np.max(np.abs(out["K_ps2"][ok] - K[ok]) / np.maximum(np.abs(K[ok]), 1e-3)) <= 1e-5
    assert np.nanmax(np.abs(out["coh_ps2"] - sel["sel_coh_ps2"].ravel())) <= 1e-6
    assert np.abs(out["ph_res2"] - sel["sel_ph_res2"]).max() <= 1e-4


@pytest.mark.parametrize("method", ["density", "percent"])
def test_threshold_from_distribution_matches_reference(units, method):
    from pystamps_b200 import stage3

    t, cf = stage3.coh_threshold_from_dist(units["th_coh"], units["th_da"], units["th_damax"], units["th_centers"],
                                           units["th_nr"], 31, float(units[f"th_{method}_mpr"]), method.upper())
    np.testing.assert_allclose(t, units[f"th_{method}"], rtol=1e-12, atol=1e-12)
    np.testing.assert_allclose(cf, units[f"th_{method}_cf"].reshape(-1), rtol=1e-12, atol=1e-12)


def test_da_bins_and_max_percent_rand(sel):
    from pystamps_b200 import stage3

    da, edges = stage3.da_bins(sel["D_A"])
    assert edges[0] == 0.0 and edges[-1] == np.max(sel["D_A"]) and edges.size == 5  # 10,000 PS: edges every 2,000
    da1, e1 = stage3.da_bins(np.full(50, 0.3))
    assert np.all(da1 == 1.0) and list(e1) == [0.0, 1.0]
    mpr = stage3.max_percent_rand("DENSITY", 1.0, 20.0, sel["xy"], edges.size - 1)
    assert mpr == pytest.approx(float(sel["sel_max_percent_rand"].ravel()[0]), rel=1e-6)
    assert stage3.max_percent_rand("PERCENT", 7.0, 20.0, sel["xy"], 5) == 7.0


def test_hist_with_centers_ties_go_to_the_lower_centre():
    from pystamps_b200 import stage3

    c = np.array([0.0, 1.0, 2.0])
    np.testing.assert_array_equal(stage3.hist_with_centers([0.5, 0.49, 1.5, 5.0, -3.0], c), [3.0, 1.0, 1.0])
