"""ps2_batch_run: uneven patches run together give exactly the results each
patch gets alone (same kernels per unit, same per-block partial sums)."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

KEYS = ("K_ps", "C_ps", "coh_ps", "N_opt", "ph_grid", "ph_patch", "Nr", "coh_ps_save")


def _patches():
    from pystamps_b200 import stage2 as S
    from pystamps_b200 import synth

    # (n_ps, n_ifg, cells per side, trials): lane classes 4 and 8, a grid with
    # no CLAP windows (18 cells), uneven sizes and iteration counts
    shapes = [(30_000, 40, 48, 81), (4_000, 110, 24, 121), (12_000, 20, 18, 41), (60_000, 97, 64, 161),
              (8_000, 33, 30, 81), (25_000, 64, 40, 121)]
    out = []
    for k, (n, m, cells, t) in enumerate(shapes):
        p = synth.make_patch(n, m, cells, t, seed=7100 + k, gamma_max_iterations=8)
        out.append(S.prepare_patch(p))
    return out


def test_batch_matches_each_patch_alone(cuda_lib):
    from pystamps_b200 import batch
    from pystamps_b200 import stage2 as S

    preps = _patches()
    alone = []
    for p in preps:
        with S.Stage2Context() as c:
            c.load(p, "fp32")
            st = c.run()
            r = c.download(KEYS)
            r["stats"] = st
            alone.append(r)
    with batch.Batch(preps) as b:
        stats = b.run()
        together = b.download(KEYS)
        n_launch = b.launch_count()
    iters = [r["i_loop"] for r in alone]
    assert len(set(iters)) > 1, iters  # the patches stop at different iterations
    for k, (a, t, st) in enumerate(zip(alone, together, stats)):
        assert t["i_loop"] == a["i_loop"], k
        assert st["i_loop"] == a["stats"]["i_loop"] and st["stop"] == 1
        for key in KEYS:
            np.testing.assert_array_equal(t[key], a[key], err_msg=f"patch {k} {key}")
    # per iteration: reset, bin, clap, overlap, topofit per lane class (2 here), finalize,
    # and the graph's loop-condition kernel
    assert n_launch == 8 * max(iters)


def test_batch_with_both_clap_forms_matches_each_patch_alone(cuda_lib):
    """Patches of one batch may use different CLAP forms (the context's launch
    shape): window stack or fused window blocks, each as it runs alone."""
    from pystamps_b200 import batch
    from pystamps_b200 import stage2 as S

    preps = _patches()[:4]
    forms = [1, 0, 1, 1]
    alone = []
    for p, f in zip(preps, forms):
        with S.Stage2Context() as c:
            c.load(p, "fp32")
            c.launch_shapes([0, 0, 0, 0, f])
            c.run()
            alone.append(c.download(KEYS))
    with batch.Batch(preps) as b:
        for c, f in zip(b.ctxs, forms):
            c.launch_shapes([0, 0, 0, 0, f])
        b.run()
        together = b.download(KEYS)
    for k, (a, t) in enumerate(zip(alone, together)):
        for key in KEYS:
            np.testing.assert_array_equal(t[key], a[key], err_msg=f"patch {k} {key}")


def test_batch_rerun_after_reset_is_identical(cuda_lib):
    from pystamps_b200 import batch

    preps = _patches()[:3]
    with batch.Batch(preps) as b:
        b.run()
        first = b.download(("K_ps", "coh_ps"))
        b.reset()
        b.run()
        second = b.download(("K_ps", "coh_ps"))
    for a, c in zip(first, second):
        np.testing.assert_array_equal(a["K_ps"], c["K_ps"])
        np.testing.assert_array_equal(a["coh_ps"], c["coh_ps"])


def test_batch_rejects_bad_input(cuda_lib):
    from pystamps_b200 import _lib, batch
    from pystamps_b200 import stage2 as S

    preps = _patches()[:2]
    with S.Stage2Context() as c64:
        c64.load(preps[0], "fp64")
        import ctypes

        arr = (ctypes.c_void_p * 1)(c64._ctx.value)
        with pytest.raises(_lib.Stage2CudaError):
            _lib.check(_lib.lib().ps2_batch_run(arr, ctypes.c_int64(1), None))
    with batch.Batch(preps[:1]) as b:
        import ctypes

        arr = (ctypes.c_void_p * 2)(b.ctxs[0]._ctx.value, b.ctxs[0]._ctx.value)
        with pytest.raises(_lib.Stage2CudaError):
            _lib.check(_lib.lib().ps2_batch_run(arr, ctypes.c_int64(2), None))


def test_batch_eager_loop_matches_graph_loop(cuda_lib, monkeypatch):
    from pystamps_b200 import batch

    preps = _patches()[:3]
    with batch.Batch(preps) as b:
        b.run()
        graph = b.download(("K_ps", "coh_ps", "N_opt"))
        b.reset()
        monkeypatch.setenv("PS2_NO_GRAPH", "1")
        b.run()
        eager = b.download(("K_ps", "coh_ps", "N_opt"))
        assert b.launch_count() == 7 * max(r["i_loop"] for r in eager)
    for a, c in zip(graph, eager):
        assert a["i_loop"] == c["i_loop"]
        for k in ("K_ps", "coh_ps", "N_opt"):
            np.testing.assert_array_equal(a[k], c[k])
