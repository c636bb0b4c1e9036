"""Stage-3 re-estimate on the GPU (ps3_reestimate through the C ABI) against
the Python reference's select1.mat (golden) and against the oracle on a larger
synthetic selection.

Tolerances (FP32 patch filter vs the reference's complex128): ph_patch2 within
2e-6 of the largest |ph_patch2|; K_ps2 within 1e-4 relative and coh_ps2 within
1e-5, except rows where the reference's candidate rule sits on an edge: a
trial coherence within 1e-5 of the near-max threshold (max - 2e-4) or of a
neighbour (local-maximum test), or two candidates whose refined coherences are
within 1e-5 — those rows are counted and reported, like argmax ties in stage 2.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

EDGE = 1e-5


def _edge_rows(oracle, cpx_rows, bp_rows, ntw):
    """Rows whose candidate set or choice is within EDGE of flipping (FP64
    evaluation of the reference's trial coherences)."""
    n_half = int(np.ceil(8 * ntw))
    tm = np.arange(-n_half, n_half + 1, dtype=np.float64)
    edge = np.zeros(len(cpx_rows), dtype=bool)
    for r, (c, b) in enumerate(zip(cpx_rows, bp_rows)):
        c = c.astype(np.complex128)
        b = b.astype(np.float64)
        rng = (b.max() - b.min()) or 1.0
        ct = np.abs(np.exp(-1j * np.outer(b / rng * np.pi / 4, tm)).T @ c) / np.abs(c).sum()
        thr = ct.max() - 2e-4
        near_thr = np.abs(ct - thr) < EDGE
        near_nb = np.zeros_like(near_thr)
        near_nb[1:] |= np.abs(ct[1:] - ct[:-1]) < EDGE
        near_nb[:-1] |= np.abs(ct[:-1] - ct[1:]) < EDGE
        cand = ct >= thr
        edge[r] = bool(np.any(near_thr) or np.any(near_nb & cand) or cand.sum() > 1)
    return edge


def _psd_rows(ph_work, pp2, fit):
    psd = ph_work.astype(np.complex128) * np.conj(pp2.astype(np.complex128))
    psd = psd / np.abs(psd)
    return psd[:, fit].astype(np.complex64)


def test_reestimate_matches_reference_select(cuda_lib, golden, oracle):
    from pystamps_b200 import stage3

    sel = golden("stage3_select.npz")
    ix0 = sel["sel_ix"].ravel().astype(np.int64) - 1
    fit = sel["sel_ifg_index"].ravel().astype(np.int64) - 1
    ntw = float(sel["pm_n_trial_wraps"].ravel()[0])
    ph_work = sel["ph"][:, 1:]
    out = stage3.reestimate(sel["pm_ph_grid"], sel["pm_grid_ij"], ix0, ph_work, sel["bperp_mat"], fit,
                            clap_alpha=1.0, clap_beta=0.3, low_pass=sel["pm_low_pass"], n_trial_wraps=ntw)
    pp = sel["sel_ph_patch2"]
    err_pp = np.abs(out["ph_patch2"] - pp).max() / np.abs(pp).max()
    K = sel["sel_K_ps2"].ravel()
    np.testing.assert_array_equal(np.isnan(out["K_ps2"]), np.isnan(K))
    edge = _edge_rows(oracle, _psd_rows(ph_work[ix0], pp, fit), sel["bperp_mat"][ix0][:, fit], ntw)
    ok = ~np.isnan(K) & ~edge
    dK = np.abs(out["K_ps2"] - K) / np.maximum(np.abs(K), 1e-3)
    dc = np.abs(out["coh_ps2"] - sel["sel_coh_ps2"].ravel())
    print(f"ph_patch2 {err_pp:.2e}; edge rows {int(edge.sum())} of {edge.size}; non-edge max dK {dK[ok].max():.2e} "
          f"max dcoh {dc[ok].max():.2e}; all rows dK > 1e-4: {int((dK > 1e-4).sum())}")
    assert err_pp <= 2e-6
    assert dK[ok].max() <= 1e-4
    assert dc[ok].max() <= 1e-5
    res = np.abs(out["ph_res2"] - sel["sel_ph_res2"])[ok]
    assert np.quantile(res, 0.999) <= 1e-4


def test_select_ps_matches_reference(cuda_lib, golden):
    from pystamps_b200 import stage3

    sel = golden("stage3_select.npz")
    pm = {k[3:]: sel[k] for k in sel.files if k.startswith("pm_")}
    parms = {"select_method": "DENSITY", "density_rand": 20.0, "slc_osf": 1.0, "gamma_stdev_reject": 0.0,
             "clap_alpha": 1.0, "clap_beta": 0.3, "clap_win": 32.0, "small_baseline_flag": "n"}
    out = stage3.select_ps(pm, ph=sel["ph"], bperp_mat=sel["bperp_mat"], bperp=sel["bperp"], D_A=sel["D_A"],
                           xy=sel["xy"], master_ix=1, ifg_index=sel["sel_ifg_index"].ravel(), parms=parms)
    np.testing.assert_array_equal(out["ix"], sel["sel_ix"].ravel().astype(np.int64))
    np.testing.assert_allclose(out["coh_thresh"], sel["sel_coh_thresh"].ravel(), rtol=1e-6)
    keep_ref = sel["sel_keep_ix"].ravel().astype(bool)
    flips = int((out["keep_ix"] != keep_ref).sum())
    print(f"keep_ix: {int(out['keep_ix'].sum())} kept vs {int(keep_ref.sum())}, {flips} differ")
    assert flips <= max(3, keep_ref.size // 2000)


def test_reestimate_matches_oracle_on_a_larger_selection(cuda_lib, oracle):
    from pystamps_b200 import stage2 as S
    from pystamps_b200 import stage3, synth

    patch = synth.make_workload("A")  # 20,000 PS x 20 ifg, 64 x 64 cells
    prep = S.prepare_patch(patch)
    with S.Stage2Context() as c:
        c.load(prep, "fp32")
        c.run()
        pm = c.download(["coh_ps", "K_ps", "ph_grid"])
    rng = np.random.default_rng(5)
    sel_rows = np.sort(rng.choice(prep.n_ps, 3000, replace=False))
    gij = np.rint(prep.grid_ij).astype(np.int64)
    fit = np.arange(prep.n_ifg)
    ntw = float(np.float32(prep.n_trial_wraps))
    bp = np.asarray(prep.bperp, dtype=np.float64)
    bp = np.broadcast_to(bp, (prep.n_ps, prep.n_ifg)) if bp.ndim == 1 else bp
    g = stage3.reestimate(pm["ph_grid"], gij, sel_rows, prep.ph_nm, bp, fit, clap_alpha=1.0, clap_beta=0.3,
                          low_pass=prep.low_pass, n_trial_wraps=ntw)
    o = oracle.s3_reestimate(pm["ph_grid"], gij, sel_rows, prep.ph_nm, bp, fit, alpha=1.0, beta=0.3,
                             low_pass=prep.low_pass, n_trial_wraps=ntw)
    err_pp = np.abs(g["ph_patch2"] - o["ph_patch2"]).max() / np.abs(o["ph_patch2"]).max()
    assert err_pp <= 2e-6, err_pp
    edge = _edge_rows(oracle, _psd_rows(prep.ph_nm[sel_rows], o["ph_patch2"], fit), bp[sel_rows], ntw)
    ok = ~np.isnan(o["K_ps2"]) & ~edge
    dK = np.abs(g["K_ps2"] - o["K_ps2"]) / np.maximum(np.abs(o["K_ps2"]), 1e-3)
    dc = np.abs(g["coh_ps2"] - o["coh_ps2"])
    print(f"edge rows {int(edge.sum())} of {edge.size}; non-edge max dK {dK[ok].max():.2e} max dcoh {dc[ok].max():.2e}")
    assert dK[ok].max() <= 1e-4
    assert dc[ok].max() <= 1e-5
    # every selected PS of a cell shares one patch: same ph_patch2 row
    cells = gij[sel_rows, 0] * 1000 + gij[sel_rows, 1]
    _, first = np.unique(cells, return_index=True)
    for i in first[:50]:
        same = np.where(cells == cells[i])[0]
        assert np.all(g["ph_patch2"][same] == g["ph_patch2"][i])


def test_stage3_select_ps_on_a_patch_directory(cuda_lib, golden, tmp_path):
    """MAT files in, select1.mat out, like the reference's stage3_select_ps."""
    from scipy.io import loadmat, savemat

    from pystamps_b200 import stage3

    sel = golden("stage3_select.npz")
    n = sel["ph"].shape[0]
    savemat(tmp_path / "ps1.mat", {"n_ps": float(n), "n_ifg": float(sel["ph"].shape[1]), "master_ix": 1.0,
                                   "bperp": sel["bperp"].reshape(1, -1), "xy": sel["xy"]})
    savemat(tmp_path / "ph1.mat", {"ph": sel["ph"]})
    savemat(tmp_path / "bp1.mat", {"bperp_mat": sel["bperp_mat"]})
    savemat(tmp_path / "da1.mat", {"D_A": sel["D_A"].reshape(-1, 1)})
    savemat(tmp_path / "parms.mat", {"select_method": "DENSITY", "density_rand": 20.0, "slc_osf": 1.0,
                                     "gamma_stdev_reject": 0.0, "clap_alpha": 1.0, "clap_beta": 0.3,
                                     "clap_win": 32.0, "small_baseline_flag": "n"})
    savemat(tmp_path / "pm1.mat", {k[3:]: sel[k] for k in sel.files if k.startswith("pm_")})
    msg = stage3.stage3_select_ps(tmp_path)
    out = loadmat(tmp_path / "select1.mat")
    assert msg == f"Stage 3 selected {sel['sel_ix'].size} PS"
    np.testing.assert_array_equal(out["ix"].ravel(), sel["sel_ix"].ravel())
    np.testing.assert_array_equal(out["ifg_index"].ravel(), sel["sel_ifg_index"].ravel())
    assert int((out["keep_ix"].ravel().astype(bool) != sel["sel_keep_ix"].ravel().astype(bool)).sum()) <= 3
    np.testing.assert_allclose(out["coh_thresh"].ravel(), sel["sel_coh_thresh"].ravel(), rtol=1e-6)
    assert float(out["max_percent_rand"].ravel()[0]) == pytest.approx(float(sel["sel_max_percent_rand"].ravel()[0]))


@pytest.mark.gpu
@pytest.mark.parametrize("row_variant,slc_osf", [(True, 1), (False, 2)])
def test_resident_reestimate_matches_host_entry(cuda_lib, row_variant, slc_osf):
    """ps2_stage3_reestimate on the context that ran stage 2 gives the same
    bits as ps3_reestimate on the downloaded grid and the context's phases."""
    import torch

    from pystamps_b200 import stage2 as S
    from pystamps_b200 import stage3, synth

    patch = synth.make_workload("A", row_variant=row_variant)
    prep = S.prepare_patch(patch)
    assert prep.row_invariant == (not row_variant)
    rng = np.random.default_rng(11)
    sel_rows = rng.choice(prep.n_ps, 2500, replace=False)  # unsorted: any row order
    fit = np.sort(rng.choice(prep.n_ifg, prep.n_ifg - 3, replace=False))
    gij = np.rint(prep.grid_ij).astype(np.int64)
    bp = np.asarray(prep.bperp, dtype=np.float64)
    bp = np.broadcast_to(bp, (prep.n_ps, prep.n_ifg)) if bp.ndim == 1 else bp
    with S.Stage2Context() as c:
        c.load(prep, "fp32")
        c.run()
        pm = c.download(["ph_grid"])
        r = stage3.reestimate_resident(c, sel_rows, fit, slc_osf=slc_osf)
        rd = stage3.reestimate_resident(c, sel_rows, fit, slc_osf=slc_osf, on_device=True)
        with pytest.raises(Exception, match="outside"):
            stage3.reestimate_resident(c, np.array([prep.n_ps]), fit)
        with pytest.raises(Exception, match="outside"):
            stage3.reestimate_resident(c, sel_rows[:4], np.array([prep.n_ifg]))
    h = stage3.reestimate(pm["ph_grid"], gij, sel_rows, prep.ph_nm, bp, fit, clap_alpha=prep.clap_alpha,
                          clap_beta=prep.clap_beta, low_pass=prep.low_pass, n_trial_wraps=prep.n_trial_wraps,
                          slc_osf=slc_osf)
    for k in ("ph_patch2", "ph_res2", "K_ps2", "C_ps2", "coh_ps2"):
        np.testing.assert_array_equal(r[k], h[k], err_msg=k)
        np.testing.assert_array_equal(rd[k].cpu().numpy(), h[k], err_msg=k)
    assert torch.isfinite(rd["coh_ps2"]).any()


@pytest.mark.gpu
def test_resident_reestimate_rejects_fp64_and_unrun_contexts(cuda_lib):
    from pystamps_b200 import stage2 as S
    from pystamps_b200 import stage3, synth

    prep = S.prepare_patch(synth.make_patch(1500, 12, 26, 41, seed=3, n_rand=2000, gamma_max_iterations=2))
    with S.Stage2Context() as c:
        c.load(prep, "fp32")
        with pytest.raises(Exception, match="has not run"):
            stage3.reestimate_resident(c, np.arange(10), np.arange(prep.n_ifg))
        c.load(prep, "fp64")
        c.run()
        with pytest.raises(Exception, match="FP64"):
            stage3.reestimate_resident(c, np.arange(10), np.arange(prep.n_ifg))
