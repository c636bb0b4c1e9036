"""CUDA path (through the C ABI) against the oracle on the same seeded inputs.

Bit-exact: grid accumulation, grid indices, the random-phase histogram.
Within tolerance (FP32 vs the reference's f32/f64 mix): CLAP, topofit, the
whole gamma loop. Topofit rows whose best and runner-up trial coherences are
within 1e-6 relative are argmax ties, and within 1e-6 of max(best, 0.5) FP32
near ties: they are counted and reported, not held to the K tolerance.
"""
import math

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

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

# tolerances (FP32 path vs oracle)
GAMMA_TOL = 1e-4      # max |d gamma| for PS whose topofit peak is not a near-tie
K_REL_TOL = 1e-4      # |dK| / max(|K|, 1e-3 rad/m)


@pytest.fixture(scope="module")
def K(cuda_lib):
    from pystamps_b200 import kernels

    return kernels


@pytest.fixture(scope="module")
def S(cuda_lib):
    from pystamps_b200 import stage2

    return stage2


def test_grid_accumulate_bit_exact(K, oracle):
    rng = np.random.default_rng(1)
    for n, m, ni, nj in ((5000, 37, 20, 30), (1, 1, 1, 1), (777, 150, 9, 7), (64, 3, 1, 1)):
        w = (rng.standard_normal((n, m)) + 1j * rng.standard_normal((n, m))).astype(np.complex64)
        gl = rng.integers(0, ni * nj, n)
        if n > 10:
            gl[::97] = -1  # rows outside the grid are skipped
            gl[5] = ni * nj
        np.testing.assert_array_equal(K.run_stage2_grid_accumulate_kernel(w, gl, ni, nj),
                                      oracle.accumulate_grid(w, gl, ni, nj))


def test_grid_accumulate_reference_vector(K):
    w = np.array([[1e-6 + 2e-6j, -3e-6 + 4e-6j], [5e-6 - 6e-6j, 7e-6 + 8e-6j], [9e-6 + 1e-6j, -2e-6 - 3e-6j]],
                 dtype=np.complex64)
    exp = np.zeros(2, dtype=np.complex64)
    for r in range(3):
        exp = (exp + w[r]).astype(np.complex64)
    np.testing.assert_array_equal(K.run_stage2_grid_accumulate_kernel(w, np.zeros(3), 1, 1).reshape(-1), exp)


@pytest.mark.parametrize("case", ["1", "2"])
def test_clap_against_golden(K, golden, case):
    d = golden("clap_grid.npz")
    out = K.run_stage2_clap_filter_kernel(d["g" + case], 1.0, 0.3, d["lp" + case])
    ref = d["out" + case + "_f64"]
    scale = np.abs(ref).max()
    err = np.abs(out - ref) / scale
    assert err.max() <= 2e-6, err.max()


def test_clap_alpha_not_one_against_golden(K, golden):
    d = golden("clap_grid.npz")
    out = K.run_stage2_clap_filter_kernel(d["g2"], 1.7, 0.45, d["lp2"])
    ref = d["out3_f64"]
    assert (np.abs(out - ref) / np.abs(ref).max()).max() <= 5e-6


def test_clap_edges_nan_and_empty(K, oracle):
    rng = np.random.default_rng(4)
    lp = oracle.build_low_pass()
    for shape in ((24, 24, 2), (25, 31, 5), (64, 40, 3), (18, 18, 2)):
        g = (rng.standard_normal(shape) + 1j * rng.standard_normal(shape)).astype(np.complex64)
        g[0, 0, 0] = np.nan
        out = K.run_stage2_clap_filter_kernel(g, 1.0, 0.3, lp)
        ref = oracle.clap_filter_grid_stack(g, 1.0, 0.3, lp)
        sc = max(np.abs(ref).max(), 1e-30)
        assert np.all(np.isfinite(out))
        assert (np.abs(out - ref) / sc).max() <= 2e-6, shape
    with pytest.raises(Exception, match="underflows"):
        K.run_stage2_clap_filter_kernel(np.ones((20, 30, 2), np.complex64), 1.0, 0.3, lp)


def _tie_mask(oracle_best, oracle_second):
    from pystamps_b200.precision import is_fp32_tie

    return is_fp32_tie(oracle_best, oracle_second)


def test_topofit_against_oracle(K, oracle, golden):
    d = golden("topofit_rows.npz")
    cpx = d["cpx"].astype(np.complex64)
    bp = d["bperp"]
    ntw = float(d["n_trial_wraps"])
    Kg, Cg, hg, rg = K.run_native_topofit_rows(cpx, bp, ntw)
    Ko, Co, ho, ro, _ = oracle.topofit(cpx, bp, ntw)
    np.testing.assert_allclose(Kg, Ko, rtol=K_REL_TOL, atol=1e-7)
    np.testing.assert_allclose(hg, ho, rtol=0, atol=1e-5)
    np.testing.assert_allclose(np.angle(np.exp(1j * (Cg - Co))), 0, atol=1e-4)
    assert np.abs(rg - ro).max() <= 1e-4


def test_topofit_zero_columns_and_empty_rows(K, oracle):
    rng = np.random.default_rng(8)
    n, m = 300, 45
    cpx = np.exp(1j * rng.uniform(-np.pi, np.pi, (n, m))).astype(np.complex64)
    cpx[rng.random((n, m)) < 0.1] = 0
    cpx[7] = 0  # all-zero row -> NaN
    bp = rng.uniform(-300, 300, (n, m))
    Kg, Cg, hg, rg = K.run_native_topofit_rows(cpx, bp, 3.3)
    Ko, Co, ho, ro, _ = oracle.topofit(cpx, bp.astype(np.float32).astype(np.float64), 3.3)
    assert np.isnan(Kg[7]) and np.isnan(hg[7]) and np.isnan(Cg[7])
    ok = ~np.isnan(Ko)
    np.testing.assert_allclose(hg[ok], ho[ok], atol=1e-5)
    same = np.abs(Kg[ok] - Ko[ok]) <= 1e-4 * np.maximum(np.abs(Ko[ok]), 1e-3)
    assert same.mean() >= 0.99
    assert np.all(rg[cpx == 0] == 0)


# n_half = ceil(8 ntw): 40 and 88 take the full trial sweep, 41 .. 87 the
# sampled one (every 4th trial exact, fractional-delay filters between)
@pytest.mark.parametrize("m,ntw", [(20, 4.94), (60, 9.94), (150, 9.94), (3, 0.4), (33, 1.0), (60, 5.1),
                                   (150, 10.8), (150, 10.9), (47, 7.6), (3, 9.94), (5, 10.8)])
def test_topofit_random_rows_argmax_and_ties(K, oracle, m, ntw):
    rng = np.random.default_rng(m)
    n = 4000
    bp = rng.uniform(-300, 300, m)[None, :] * (1 + 0.02 * rng.uniform(-0.5, 0.5, (n, 1)))
    k = rng.uniform(-0.04, 0.04, n)
    cpx = (np.exp(1j * (k[:, None] * bp + rng.normal(0, 0.8, (n, m))))).astype(np.complex64)
    bp32 = bp.astype(np.float32).astype(np.float64)
    Kg, Cg, hg, _ = K.run_native_topofit_rows(cpx, bp32, ntw)
    fr = oracle.fit_rows(np.ones((n, m), np.complex64), cpx, bp32, ntw)
    tie = _tie_mask(fr.best_coh, fr.second_coh)
    good = ~tie
    dK = np.abs(Kg - fr.K) / np.maximum(np.abs(fr.K), 1e-3)
    assert (dK[good] <= K_REL_TOL).mean() >= 0.999, (dK[good] > K_REL_TOL).sum()
    assert np.abs(hg - fr.coh)[good].max() <= GAMMA_TOL


@pytest.mark.parametrize("m,ntw", [(150, 9.94), (60, 5.1), (150, 10.8), (40, 7.6)])
def test_topofit_peaks_at_the_end_trials(K, oracle, m, ntw):
    """Rows whose best trial is the first or the last one (m = -n_half or
    +n_half), where the sampled sweep's filters read samples beyond the trial
    range, and rows one trial inside them: the same argmax and refined values
    as the oracle."""
    rng = np.random.default_rng(int(10 * ntw) + m)
    n = 2000
    n_half = math.ceil(8 * ntw)
    bp = rng.uniform(-300, 300, (n, m))
    rngbp = bp.max(axis=1) - bp.min(axis=1)
    step = math.pi / 4 / rngbp  # K of one trial step, per row
    edge = rng.choice([-n_half, n_half, -(n_half - 1), n_half - 1], n)
    k = (edge + rng.uniform(-0.2, 0.2, n)) * step
    cpx = np.exp(1j * (k[:, None] * bp + rng.normal(0, 0.3, (n, m)))).astype(np.complex64)
    bp32 = bp.astype(np.float32).astype(np.float64)
    Kg, Cg, hg, _ = K.run_native_topofit_rows(cpx, bp32, ntw)
    fr = oracle.fit_rows(np.ones((n, m), np.complex64), cpx, bp32, ntw)
    good = ~_tie_mask(fr.best_coh, fr.second_coh)
    dK = np.abs(Kg - fr.K) / np.maximum(np.abs(fr.K), 1e-3)
    assert (dK[good] <= K_REL_TOL).all(), (dK[good] > K_REL_TOL).sum()
    assert np.abs(hg - fr.coh)[good].max() <= GAMMA_TOL


def test_random_hist_kat(S):
    nr, mx = S.random_coherence_histogram(np.array([-20.0, -5.0, 0.0, 13.0, 27.0]), 0.5, 10_000)
    assert nr.tolist() == NR_KAT
    assert mx == 100.0


def test_random_hist_matches_oracle(S, oracle):
    rng = np.random.default_rng(2)
    bp = rng.uniform(-300, 300, 20)
    a, am = S.random_coherence_histogram(bp, 4.94, 30_000)
    b, bm = oracle.random_hist(bp, 4.94, n_rand=30_000)
    np.testing.assert_array_equal(a, b)
    assert am == bm


def test_random_hist_small_baseline_matches_oracle(S, oracle):
    rng = np.random.default_rng(3)
    ix = np.array([[1, 2], [1, 3], [2, 3], [2, 4], [3, 5], [4, 5]], dtype=np.int64)
    bp = rng.uniform(-200, 200, 6)
    a, _ = S.random_coherence_histogram(bp, 2.0, 20_000, True, ix, 5)
    b, _ = oracle.random_hist(bp, 2.0, n_rand=20_000, small_baseline=True, ifgday_ix=ix, n_image=5)
    np.testing.assert_array_equal(a, b)


def _loop_compare(S, oracle, patch, precision="fp32"):
    nr, mx = oracle.random_hist(patch["bperp"][1:], S.prepare_patch(patch, nr=np.ones(100)).n_trial_wraps,
                                n_rand=patch.get("n_rand", 300_000))
    g = S.run_stage2(patch, precision=precision, nr=nr, nr_max_nz_ix=mx)
    o = oracle.stage2_run(dict(patch, nr_override=np.concatenate([nr, [mx]])), fp64=(precision == "fp64"),
                          keep_history=True)
    o["Nr_base"] = nr
    return g, o


def _teacher_forced(S, oracle, patch, iterations=5):
    """Every GPU iteration against the oracle's iteration applied to the GPU's
    own previous state (K, coh, scaled Nr): the loop is checked step by step,
    free of the P-square table's step discontinuity (round(1000*coh)).
    Returns the number of argmax ties met."""
    prep = S.prepare_patch(patch)
    bp = prep.bperp.astype(np.float64)
    n_ties = 0
    with S.Stage2Context() as ctx:
        ctx.load(prep)
        prev = None
        for it in range(1, iterations + 1):
            ctx.iterate(1)
            g = ctx.download()
            if prev is None:
                w = prep.weight0
                K0 = np.zeros(prep.n_ps)
            else:
                na_prev = oracle.hist_with_centers(prev["coh_ps"])
                w = oracle.psquare_weighting(prev["Nr"], na_prev, 31, prep.nr_max_nz_ix, prev["coh_ps"])
                K0 = prev["K_ps"]
            # Nr scaling in this iteration's P-square update (native_stage2.rs:364-374)
            base = prep.nr if prev is None else prev["Nr"]
            na_cur = oracle.hist_with_centers(g["coh_ps"])
            den = base[:31].sum()
            scale = na_cur[:31].sum() / den if den > 0 else 1.0
            np.testing.assert_allclose(g["Nr"], base * scale, rtol=1e-14)
            pw = oracle.fill_phase_weight(prep.ph_nm, bp, K0, w)
            fin = np.isfinite(pw)
            np.testing.assert_array_equal(np.isfinite(g["ph_weight"]), fin)
            assert np.abs(g["ph_weight"] - pw)[fin].max() <= 5e-7 * max(1.0, np.abs(pw[fin]).max()), it
            # binning is bit-exact given the same weighted phases
            np.testing.assert_array_equal(g["ph_grid"], oracle.accumulate_grid(g["ph_weight"], prep.grid_lin,
                                                                               prep.n_i, prep.n_j))
            filt = oracle.clap_filter_grid_stack(g["ph_grid"], prep.clap_alpha, prep.clap_beta, prep.low_pass)
            patch_o = oracle.extract_patch_phase(filt, prep.grid_lin)
            # unit phasors of CLAP output: FP32 vs FP64 FFT error, amplified in weak cells
            dp = np.abs(g["ph_patch"] - patch_o)
            assert dp.max() <= 2e-4 and np.quantile(dp, 0.999) <= 1e-5, (it, dp.max())
            fr = oracle.fit_rows(g["ph_patch"], prep.ph_nm, bp, prep.n_trial_wraps)
            tie = _tie_mask(fr.best_coh, fr.second_coh)
            n_ties += int(tie.sum())
            good = ~tie & ~np.isnan(fr.K)
            np.testing.assert_array_equal(np.isnan(g["K_ps"]), np.isnan(fr.K))
            if good.any():  # with very few interferograms every row can be a tie
                assert np.abs(g["coh_ps"] - fr.coh)[good].max() <= 1e-5, it
                dK = np.abs(g["K_ps"] - fr.K) / np.maximum(np.abs(fr.K), 1e-3)
                assert dK[good].max() <= K_REL_TOL, it
            np.testing.assert_array_equal(g["N_opt"], fr.N_opt)
            prev = g
    return n_ties


def test_stage2_loop_teacher_forced(S, oracle):
    from pystamps_b200 import synth

    patch = synth.make_patch(6000, 16, 32, 41, seed=101, n_rand=20_000)
    n_ties = _teacher_forced(S, oracle, patch)
    print(f"argmax ties over 5 iterations: {n_ties}")


def test_stage2_loop_teacher_forced_row_invariant_invalid_rows(S, oracle):
    from pystamps_b200 import synth

    patch = synth.make_patch(3000, 12, 24, 41, seed=7, n_rand=5000, row_variant=False)
    ph = patch["ph"].copy()
    ph[10:20, 3] = 0  # zero phase -> psdph zero -> invalid rows (native_stage2.rs:686-697)
    patch["ph"] = ph
    _teacher_forced(S, oracle, patch, iterations=4)


def _sensitivity(oracle, patch, g, o):
    """Median |dgamma| of the GPU run against the oracle, and of the oracle's
    own FP64 variant against its FP32 run: the free-running loop amplifies
    ulp-level differences through the P-square table step, so the reference
    algorithm's own precision sensitivity calibrates the tolerance."""
    o64 = oracle.stage2_run(dict(patch, nr_override=np.concatenate([o["Nr_base"], [o["Nr_max_nz_ix"]]])), fp64=True)
    return np.median(np.abs(g["coh_ps"] - o["coh_ps"])), np.median(np.abs(o64["coh_ps"] - o["coh_ps"]))


def _perturbed_spread(oracle, patch, o, eps=1e-6, seeds=(1, 2, 3)):
    """The reference algorithm's own divergence: the oracle run again with its
    input phases rotated by eps * N(0, 1) rad (about the size of the per-
    iteration FP32 differences the teacher-forced tests bound), against its
    unperturbed run. Returns the largest median and 90th percentile of
    |d gamma| over the seeds."""
    med, p90 = 0.0, 0.0
    nr = np.concatenate([o["Nr_base"], [o["Nr_max_nz_ix"]]])
    for sd in seeds:
        rng = np.random.default_rng(sd)
        ph = patch["ph"] * np.exp(1j * eps * rng.standard_normal(patch["ph"].shape)).astype(patch["ph"].dtype)
        op = oracle.stage2_run(dict(patch, ph=ph, nr_override=nr))
        d = np.abs(op["coh_ps"] - o["coh_ps"])
        med, p90 = max(med, float(np.median(d))), max(p90, float(np.quantile(d, 0.9)))
    return med, p90


@pytest.mark.parametrize("seed", [101, 103])
def test_stage2_loop_free_running_against_oracle(S, oracle, seed):
    """Whole loop to convergence, GPU and oracle each on their own state.

    Per-iteration parity is what the teacher-forced tests pin. Run freely, the
    two trajectories separate: a PS whose best and runner-up trials are within
    rounding of each other takes a different K, and round(1000 coh) in the
    P-square table moves weights by whole table steps, after which the binned
    grid and every neighbour's filtered phase differ. How far depends on the
    seed (median |d gamma| from 1e-7 to 3e-4 on this shape), and the oracle run
    against itself with its input phases rotated by 1e-6 rad separates by as
    much (seeds 101 and 103: median 5e-4, 90th percentile 3e-3, twice the
    GPU's). The bounds: same iteration count, cells and invalid rows; the
    GPU's median and 90th percentile |d gamma| within 1.5x the largest of
    three such perturbed oracle runs (plus 1e-6 and 1e-5, the scale of one
    iteration's FP32 differences, for seeds whose perturbed runs do not
    separate)."""
    from pystamps_b200 import synth

    patch = synth.make_patch(6000, 16, 32, 41, seed=seed, n_rand=20_000)
    g, o = _loop_compare(S, oracle, patch)
    np.testing.assert_array_equal(g["grid_ij"], o["grid_ij"])
    assert g["i_loop"] == o["i_loop"]
    d = np.abs(g["coh_ps"] - o["coh_ps"])
    d_gpu, d_ref = _sensitivity(oracle, patch, g, o)
    p_med, p_p90 = _perturbed_spread(oracle, patch, o)
    print(f"seed {seed}: median |dgamma| {d_gpu:.2e} (oracle FP32 vs FP64 {d_ref:.2e}, oracle vs oracle with "
          f"1e-6 rad input rotations {p_med:.2e}), p90 {np.quantile(d, 0.9):.2e} (perturbed oracle {p_p90:.2e})")
    assert d_gpu <= 1.5 * p_med + 1e-6, (d_gpu, p_med)
    assert np.quantile(d, 0.9) <= 1.5 * p_p90 + 1e-5, (np.quantile(d, 0.9), p_p90)
    np.testing.assert_array_equal(np.isnan(g["K_ps"]), np.isnan(o["K_ps"]))
    np.testing.assert_allclose(g["Nr"], o["Nr"], rtol=5e-2)  # cumulative scaling of a chaotic history


def test_stage2_invalid_rows_and_row_invariant(S, oracle):
    from pystamps_b200 import synth

    patch = synth.make_patch(3000, 12, 24, 41, seed=7, n_rand=5000, row_variant=False)
    ph = patch["ph"].copy()
    ph[10:20, 3] = 0
    patch["ph"] = ph
    g, o = _loop_compare(S, oracle, patch)
    np.testing.assert_array_equal(np.isnan(g["K_ps"]), np.isnan(o["K_ps"]))
    assert np.all(np.isnan(g["K_ps"][10:20])) and np.all(g["coh_ps"][10:20] == 0)
    assert g["i_loop"] == o["i_loop"]
    d_gpu, d_ref = _sensitivity(oracle, patch, g, o)
    assert d_gpu <= 3 * d_ref + 1e-5, (d_gpu, d_ref)


def test_stage2_snr_weighting_path(S, oracle):
    from pystamps_b200 import synth

    patch = synth.make_patch(3000, 12, 24, 41, seed=9, n_rand=5000, gamma_max_iterations=4)
    patch["parms"] = dict(patch["parms"], filter_weighting="SNR")
    g, o = _loop_compare(S, oracle, patch)
    assert g["i_loop"] == o["i_loop"]
    d_gpu, d_ref = _sensitivity(oracle, patch, g, o)
    assert d_gpu <= 3 * d_ref + 1e-5, (d_gpu, d_ref)


def test_stage2_fp64_path_matches_fp64_oracle(S, oracle):
    from pystamps_b200 import synth

    patch = synth.make_patch(4000, 16, 32, 41, seed=33, n_rand=10_000, gamma_max_iterations=5)
    g, o = _loop_compare(S, oracle, patch, precision="fp64")
    assert g["i_loop"] == o["i_loop"]
    # FP64 against FP64: the table discontinuity is reached only at ~1e-15
    assert np.mean(np.abs(g["coh_ps"] - o["coh_ps"]) <= 1e-9) >= 0.99
    assert np.mean(np.abs(g["K_ps"] - o["K_ps"]) <= 1e-9) >= 0.99


def test_stage2_deterministic_and_bounded_at_precision_size(S):
    """Size-independent properties at the 250k-PS x 60-ifg x 128^2 shape."""
    from pystamps_b200 import synth

    patch = synth.make_workload("B")
    prep = S.prepare_patch(patch)
    with S.Stage2Context() as ctx:
        ctx.load(prep)
        st = ctx.run()
        a = ctx.download(["K_ps", "coh_ps", "ph_grid"])
        ctx.reset()
        st2 = ctx.run()
        b = ctx.download(["K_ps", "coh_ps", "ph_grid"])
    assert st == st2
    np.testing.assert_array_equal(a["coh_ps"], b["coh_ps"])
    np.testing.assert_array_equal(a["ph_grid"], b["ph_grid"])
    coh = a["coh_ps"]
    assert np.all((coh >= 0) & (coh <= 1 + 1e-6))
    valid = ~np.isnan(a["K_ps"])
    rng_bp = float(prep.bperp_nm.max() - prep.bperp_nm.min())
    kmax = (math.pi / 4) / rng_bp * (8 * prep.n_trial_wraps + 1) * 1.5
    assert np.all(np.abs(a["K_ps"][valid]) <= kmax)
    # FP32 vs the plain FP64 GPU path on the same input
    with S.Stage2Context() as ctx:
        ctx.load(prep, "fp64")
        st64 = ctx.run()
        c = ctx.download(["coh_ps", "K_ps"])
    assert st64["i_loop"] == st["i_loop"]
    d = np.abs(c["coh_ps"] - coh)
    assert np.median(d) <= GAMMA_TOL


def test_graph_loop_matches_individual_launches(S, monkeypatch):
    """The loop to convergence as one conditional-WHILE graph launch gives the
    same bits as the same kernels launched one by one."""
    from pystamps_b200 import synth

    patch = synth.make_patch(5000, 20, 32, 41, seed=55, n_rand=5000)
    prep = S.prepare_patch(patch)
    monkeypatch.setenv("PS2_NO_GRAPH", "1")
    a = S.run_stage2(prep, keys=["K_ps", "coh_ps", "ph_grid", "Nr"])
    monkeypatch.setenv("PS2_NO_GRAPH", "0")
    with S.Stage2Context() as ctx:
        ctx.load(prep)
        st = ctx.run()
        b = ctx.download(["K_ps", "coh_ps", "ph_grid", "Nr"])
        launches = ctx.launch_count()
    assert st["i_loop"] == a["i_loop"] > 1
    assert launches >= 5 * st["i_loop"]
    for k in ("K_ps", "coh_ps", "ph_grid", "Nr"):
        np.testing.assert_array_equal(a[k], b[k])
