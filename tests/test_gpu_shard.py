"""One patch split over shards (ranks emulated as contexts of one process on
one GPU): the per-PS results equal those of one context over the whole patch,
iteration for iteration."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("n_shards,row_variant,precision,clap_form",
                         [(3, True, "fp32", 0), (2, False, "fp32", 0), (4, True, "fp64", 0), (3, True, "fp32", 1),
                          (2, True, "fp64", 1)])
def test_shards_match_one_context(cuda_lib, n_shards, row_variant, precision, clap_form):
    """clap_form 1: every context runs the fused CLAP (window blocks): a shard
    computes the whole blocks that hold its windows."""
    from pystamps_b200 import shard, stage2, synth

    patch = synth.make_patch(6000, 12, 30, 41, seed=77, n_rand=3000, gamma_max_iterations=6, row_variant=row_variant)
    prep = stage2.prepare_patch(patch)
    keys = ("K_ps", "C_ps", "coh_ps", "N_opt", "ph_grid")
    shapes = [0, 0, 0, 0, clap_form]
    with stage2.Stage2Context() as c:
        c.load(prep, precision)
        c.launch_shapes(shapes)
        st = c.run()
        one = c.download(keys)
    got = shard.run_sharded_local(prep, n_shards, precision=precision, keys=keys, shapes=shapes)
    assert got["i_loop"] == one["i_loop"] == st["i_loop"]
    for k in ("K_ps", "C_ps", "coh_ps", "N_opt"):
        np.testing.assert_array_equal(got[k], one[k], err_msg=k)
    np.testing.assert_array_equal(got["ph_grid"], one["ph_grid"])
    assert abs(got["stats"]["gamma_change_rms"] - st["gamma_change_rms"]) <= 1e-12 * max(1.0, st["gamma_change_rms"])


def test_one_shard_is_the_whole_patch(cuda_lib):
    from pystamps_b200 import shard, stage2, synth

    prep = stage2.prepare_patch(synth.make_patch(3000, 8, 24, 21, seed=78, n_rand=2000, gamma_max_iterations=4))
    with stage2.Stage2Context() as c:
        c.load(prep)
        c.run()
        one = c.download(("K_ps", "coh_ps"))
    got = shard.run_sharded_local(prep, 1, keys=("K_ps", "coh_ps"))
    np.testing.assert_array_equal(got["K_ps"], one["K_ps"])
    np.testing.assert_array_equal(got["coh_ps"], one["coh_ps"])


def test_shard_calls_reject_bad_arguments(cuda_lib):
    import ctypes

    from pystamps_b200 import _lib, shard, stage2, synth

    prep = stage2.prepare_patch(synth.make_patch(2000, 6, 24, 21, seed=79, n_rand=1000, gamma_max_iterations=2))
    r = shard.ShardRank(prep, 0, prep.n_i * prep.n_j)
    try:
        L = _lib.lib()
        assert L.ps2_shard_bin(r.ctx._ctx, ctypes.c_void_p(0)) != 0
        g = r.bin()
        assert L.ps2_shard_filter(r.ctx._ctx, ctypes.c_void_p(g.data_ptr()), ctypes.c_int64(5), ctypes.c_int64(2)) != 0
        assert L.ps2_shard_filter(r.ctx._ctx, ctypes.c_void_p(g.data_ptr()), ctypes.c_int64(0),
                                  ctypes.c_int64(prep.n_i * prep.n_j + 1)) != 0
        r.filter(g)
        st = r.fit()
        assert st[:100].sum() == prep.n_ps
        bad = st.copy()
        bad[3] = -1.0
        with pytest.raises(Exception, match="histogram"):
            r.finalize(bad, prep.n_ps)
        with pytest.raises(Exception, match="n_total"):
            r.finalize(st, prep.n_ps - 1)
    finally:
        r.close()
