"""The oracle against the reference's own known-answer tests and golden vectors.

KATs: crates/pystamps-core/src/native_stage2.rs:2464-2559 (RNG, P-square,
histogram rule, 100-bin random-coherence histogram); trial values and the f32
grid boundary bin from tests/test_stage2_ported.py:703-707 and
tests/test_stage2_trial_wraps.py:111-128. Golden vectors: tests/golden/*.npz,
produced by tests/golden/make_golden.py from the Python reference.
"""
import math

import numpy as np
import pytest

RNG_KAT = [
    (0, 0.092958990583191195), (1, 0.37373775840752277), (2, 0.44877057937117765), (9, 0.574897127600281),
    (10, 0.067322284274237226), (31, 0.43152622807181651), (32, 0.88306283014597708),
    (33, 0.074287163034898504), (1000, 0.35920165460545467), (99_999, 0.020806164093088213),
    (1_000_000, 0.4917673475125352),
]
PSQUARE_KAT = [1.8308507589276466e-06, 0.011860147976383777, 0.011860147976383777, 4.288734335628797e-06,
               8.21030522409814e-06, 1.0, 1.0]
NR_KAT = [
    0.0, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0, 1.0, 0.0, 0.0, 1.0, 1.0, 4.0, 5.0,
    0.0, 2.0, 7.0, 5.0, 14.0, 14.0, 15.0, 10.0, 29.0, 21.0, 26.0, 29.0, 44.0, 42.0, 57.0,
    54.0, 63.0, 71.0, 68.0, 71.0, 87.0, 87.0, 76.0, 98.0, 111.0, 100.0, 137.0, 123.0,
    139.0, 154.0, 148.0, 149.0, 162.0, 195.0, 212.0, 202.0, 200.0, 203.0, 228.0, 209.0,
    222.0, 227.0, 223.0, 239.0, 201.0, 199.0, 231.0, 203.0, 192.0, 184.0, 187.0, 188.0,
    185.0, 180.0, 183.0, 186.0, 163.0, 152.0, 147.0, 155.0, 158.0, 171.0, 169.0, 155.0,
    139.0, 140.0, 144.0, 126.0, 125.0, 125.0, 115.0, 110.0, 116.0, 104.0, 95.0, 75.0, 74.0,
    85.0, 73.0, 56.0, 61.0, 37.0, 26.0,
]


def test_rng_matches_reference_kat(oracle):
    v = oracle.rng_uniform(1_000_001)
    for ix, exp in RNG_KAT:
        assert abs(v[ix] - exp) <= 1e-15


def test_psquare_weighting_kat(oracle):
    nr = np.arange(100, dtype=np.float64)
    na = np.arange(100, 200, dtype=np.float64)
    coh = np.array([0.0, 0.0049, 0.005, 0.3144, 0.3145, 0.9999, 1.1])
    w = oracle.psquare_weighting(nr, na, 31, 45.0, coh)
    np.testing.assert_allclose(w, PSQUARE_KAT, rtol=0, atol=1e-12)


def test_psquare_table_has_1001_entries(oracle):
    lut = oracle.psquare_lut(np.ones(100), np.ones(100), 0, 100.0)
    assert lut.shape == (1001,)


def test_histogram_equal_spacing_rule(oracle):
    out = oracle.hist_with_centers(np.array([0.01, 0.02, 0.03, np.nan]), np.array([0.005, 0.015, 0.025, 0.035]))
    assert out.tolist() == [1.0, 1.0, 1.0, 0.0]


def test_random_coherence_histogram_kat(oracle):
    nr, mx = oracle.random_hist(np.array([-20.0, -5.0, 0.0, 13.0, 27.0]), 0.5, n_rand=10_000)
    assert nr.tolist() == NR_KAT
    assert mx == 100.0


def test_trial_values(oracle):
    np.testing.assert_array_equal(oracle.trial_values(0.725669801235199), np.arange(-6.0, 7.0))


def test_grid_indices_keep_single_precision_boundary_bin(oracle):
    xy = np.array([[1.0, -23497.43359375, 0.0], [2.0, -21497.43359375, 0.0], [3.0, -20497.43359375, 0.0]],
                  dtype=np.float32)
    g = oracle.grid_indices(xy, 50.0)
    assert int(g[1, 1]) == 40
    x64 = xy.astype(np.float64)[:, 1]
    assert int(np.ceil((x64 - x64.min() + 1e-6) / 50.0)[1]) == 41


def test_accumulate_grid_single_precision_order(oracle):
    # tests/test_stage2_ported.py:864-883
    w = np.array([[1e-6 + 2e-6j, -3e-6 + 4e-6j], [5e-6 - 6e-6j, 7e-6 + 8e-6j], [9e-6 + 1e-6j, -2e-6 - 3e-6j]],
                 dtype=np.complex64)
    out = oracle.accumulate_grid(w, np.zeros(3, dtype=np.int64), 1, 1)
    exp = np.zeros(2, dtype=np.complex64)
    for r in range(3):
        exp = (exp + w[r]).astype(np.complex64)
    np.testing.assert_array_equal(out.reshape(-1), exp)


@pytest.mark.parametrize("case", ["1", "2"])
def test_clap_matches_python_reference_bit_for_bit(oracle, golden, case):
    d = golden("clap_grid.npz")
    g, lp = d["g" + case], d["lp" + case]
    out = oracle.clap_filter_grid_stack(g, 1.0, 0.3, lp)
    np.testing.assert_array_equal(out, d["out" + case])
    out64 = oracle.clap_filter_grid_stack(g, 1.0, 0.3, lp, fp64=True)
    scale = np.abs(d["out" + case + "_f64"]).max()
    assert np.abs(out64 - d["out" + case + "_f64"]).max() <= 1e-14 * scale


def test_clap_alpha_not_one_matches_python_reference(oracle, golden):
    d = golden("clap_grid.npz")
    out = oracle.clap_filter_grid_stack(d["g2"], 1.7, 0.45, d["lp2"], fp64=True)
    assert np.abs(out - d["out3_f64"]).max() <= 1e-14 * np.abs(d["out3_f64"]).max()


def test_topofit_matches_python_reference_f64(oracle, golden):
    d = golden("topofit_rows.npz")
    K, C, coh, res, _ = oracle.topofit(d["cpx"], d["bperp"], float(d["n_trial_wraps"]))
    single = d["n_candidates"] == 1  # rows where near-max (Python) == first-argmax (Rust)
    assert single.sum() >= 90
    np.testing.assert_allclose(K[single], d["K"][single], rtol=0, atol=1e-12)
    np.testing.assert_allclose(C[single], d["C"][single], rtol=0, atol=1e-12)
    np.testing.assert_allclose(coh[single], d["coh"][single], rtol=0, atol=1e-12)
    np.testing.assert_allclose(res[single], d["residual"][single], rtol=0, atol=1e-12)


def test_low_pass_matches_python_reference(oracle, golden):
    d = golden("stage2_iter1.npz")
    np.testing.assert_allclose(oracle.build_low_pass(), d["pm_low_pass"], rtol=1e-14, atol=1e-300)


def _iter1_patch(d):
    return dict(ph=d["ph"], bperp=d["bperp"], master_ix=1, bperp_mat=d["bperp_mat"], D_A=d["D_A"], xy=d["xy"],
                mean_incidence=float(d["mean_incidence"]),
                parms=dict(max_topo_err=20.0, gamma_max_iterations=1, gamma_change_convergence=0.005),
                nr_override=np.concatenate([np.zeros(100), [1.0]]))


def test_first_iteration_matches_python_reference(oracle, golden):
    """One gamma iteration of the whole loop against ported.stage2_estimate_gamma.

    The first iteration does not depend on the random-phase histogram. The two
    implementations differ by design in the ph_weight ramp precision (f64 in
    Python, f32 in Rust) and the near-max peak rule, so agreement is stated
    as tolerances and fractions."""
    d = golden("stage2_iter1.npz")
    r = oracle.stage2_run(_iter1_patch(d))
    assert r["i_loop"] == 1
    np.testing.assert_array_equal(r["grid_ij"], d["pm_grid_ij"])
    assert float(np.float32(r["n_trial_wraps"])) == float(d["pm_n_trial_wraps"].reshape(-1)[0])
    np.testing.assert_array_equal(r["N_opt"], d["pm_N_opt"].reshape(-1))
    for key, tol in (("ph_weight", 2e-6), ("ph_grid", 2e-5), ("ph_patch", 1e-5)):
        a, b = r[key], d["pm_" + key].reshape(r[key].shape)
        assert np.abs(a - b).max() <= tol, key
    dk = np.abs(r["K_ps"] - d["pm_K_ps"].reshape(-1))
    dc = np.abs(r["coh_ps"] - d["pm_coh_ps"].reshape(-1))
    assert np.mean(dk <= 1e-5) >= 0.995
    assert np.mean(dc <= 1e-4) >= 0.995


def test_three_ps_fixture_matches_python_reference(oracle, golden):
    """native_stage2.rs:2698-2769: 1x1 grid, empty CLAP, every row invalid."""
    d = golden("stage2_3ps.npz")
    p = dict(ph=np.array([[1.0, 0.8 + 0.2j, 0.6 + 0.4j], [1.0, 0.7 + 0.3j, 0.5 + 0.5j], [1.0, 0.9 + 0.1j, 0.4 + 0.6j]],
                         dtype=np.complex64),
             bperp=np.array([0.0, 15.0, 30.0]), master_ix=1, bperp_mat=np.array([[15.0, 30.0]] * 3), D_A=np.ones(3),
             xy=np.array([[1, 0, 0], [2, 5, 5], [3, 10, 10]], dtype=np.float32),
             mean_incidence=math.radians(23.0) + 0.052, parms=dict(gamma_max_iterations=1), n_rand=10_000)
    r = oracle.stage2_run(p)
    for k in ("K_ps", "C_ps", "coh_ps", "N_opt", "coh_ps_save"):
        np.testing.assert_allclose(r[k], d["pm_" + k].reshape(-1), rtol=1e-5, atol=1e-7, equal_nan=True)
    np.testing.assert_array_equal(r["ph_res"], d["pm_ph_res"].reshape(r["ph_res"].shape))
    np.testing.assert_array_equal(r["grid_ij"], d["pm_grid_ij"])
    assert r["i_loop"] == int(d["pm_i_loop"].reshape(-1)[0])


def test_bad_bp_shape_is_a_stage2_error(oracle):
    # native_stage2.rs:2617-2626
    p = dict(ph=np.ones((3, 3), np.complex64), bperp=np.array([0.0, 15.0, 30.0]), master_ix=1,
             bperp_mat=np.array([[10.0], [20.0], [30.0]]), xy=np.zeros((3, 3), np.float32),
             mean_incidence=0.4, parms=dict(gamma_max_iterations=1), n_rand=100)
    with pytest.raises(ValueError, match="incompatible shape"):
        oracle.stage2_run(p)


def test_fp64_oracle_tracks_fp32_oracle(oracle):
    from pystamps_b200 import synth

    p = synth.make_patch(2000, 12, 24, 41, seed=5, gamma_max_iterations=3, n_rand=2000)
    r32 = oracle.stage2_run(p)
    r64 = oracle.stage2_run(p, fp64=True)
    assert r32["i_loop"] == r64["i_loop"]
    ok = np.abs(r32["coh_ps"] - r64["coh_ps"]) <= 1e-3
    assert ok.mean() >= 0.99
