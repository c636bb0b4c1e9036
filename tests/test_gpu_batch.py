"""Several patches per GPU on concurrent streams, and the topofit autotuner."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def uneven_patches(cuda_lib):
    from pystamps_b200 import stage2, synth

    shapes = [(9000, 24, 32), (2500, 31, 24), (14000, 40, 40), (4000, 18, 26), (6000, 33, 30), (3000, 27, 24)]
    out = []
    for k, (n, m, cells) in enumerate(shapes):
        p = synth.make_patch(n, m, cells, 41, seed=4000 + k, n_rand=3000, gamma_max_iterations=6)
        out.append(stage2.prepare_patch(p))
    return out


def test_concurrent_streams_match_one_at_a_time(uneven_patches):
    from pystamps_b200 import batch, stage2

    multi = batch.run_patches(uneven_patches, streams=3)
    for p, r in zip(uneven_patches, multi):
        single = stage2.run_stage2(p, keys=batch.SUMMARY_KEYS)
        assert r["i_loop"] == single["i_loop"]
        for k in batch.SUMMARY_KEYS:
            np.testing.assert_array_equal(r[k], single[k])


def test_autotune_picks_a_shape_with_the_same_iteration(uneven_patches, oracle):
    from pystamps_b200 import stage2

    p = uneven_patches[2]
    with stage2.Stage2Context() as ctx:
        ctx.load(p)
        lanes, ms = ctx.autotune()
        assert lanes in (4, 8, 16, 32) and all(t > 0 for t in ms)
        ctx.iterate(1)
        g = ctx.download(["coh_ps", "K_ps", "ph_patch"])
    fr = oracle.fit_rows(g["ph_patch"], p.ph_nm, p.bperp.astype(np.float64), p.n_trial_wraps)
    tie = (fr.best_coh - fr.second_coh) <= 1e-6 * np.maximum(fr.best_coh, 1e-30)
    good = ~tie & ~np.isnan(fr.K)
    assert np.abs(g["coh_ps"] - fr.coh)[good].max() <= 1e-5
