"""Checkpoint / resume of the gamma loop and the per-iteration pm1 dumps.

A loop interrupted after iteration k (ps2_export_state), restored into a new
context holding the same patch (ps2_import_state) and run to convergence gives
the same bits as the loop run once without interruption; the reference's
PYSTAMPS_STAGE2_NATIVE_DEBUG_PM dumps (native_stage2.rs:259, 337-356, 385-404)
are written one per iteration by the patch-directory drop-in.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

KEYS = ["K_ps", "C_ps", "coh_ps", "N_opt", "ph_grid", "ph_patch", "ph_weight", "coh_ps_save", "Nr"]


@pytest.fixture(scope="module")
def S(cuda_lib):
    from pystamps_b200 import stage2

    return stage2


@pytest.fixture(scope="module")
def patch():
    from pystamps_b200 import synth

    return synth.make_patch(5000, 20, 32, 41, seed=55, n_rand=5000)


@pytest.fixture(scope="module")
def prep(S, patch):
    return S.prepare_patch(patch)


@pytest.mark.parametrize("precision", ["fp32", "fp64"])
def test_resume_from_checkpoint_is_bit_identical(S, prep, precision):
    with S.Stage2Context() as c:
        c.load(prep, precision)
        full = c.run()
        ref = c.download(KEYS)
    assert full["i_loop"] >= 3
    for k_stop in (1, full["i_loop"] - 1):
        with S.Stage2Context() as a:
            a.load(prep, precision)
            for _ in range(k_stop):
                assert not a.step()["stop"]
            blob = a.export_state()
        with S.Stage2Context() as b:
            b.load(prep, precision)
            b.import_state(blob)
            last = b.run()
            got = b.download(KEYS)
        assert last["i_loop"] == full["i_loop"]
        assert last["gamma_change_rms"] == full["gamma_change_rms"]
        for k in KEYS:
            np.testing.assert_array_equal(got[k], ref[k], err_msg=f"{k} after resuming at {k_stop}")
        assert got["gamma_change_save"] == ref["gamma_change_save"]


def test_import_rejects_other_patches_and_truncated_states(S, prep):
    from pystamps_b200 import synth
    from pystamps_b200._lib import Stage2CudaError

    other = S.prepare_patch(synth.make_patch(3000, 20, 32, 41, seed=56, n_rand=2000))
    with S.Stage2Context() as a:
        a.load(prep)
        a.step()
        blob = a.export_state()
        with pytest.raises(Stage2CudaError, match="truncated"):
            a.import_state(blob[:-8])
        with pytest.raises(Stage2CudaError, match="not a loop state"):
            a.import_state(b"x" * len(blob))
    with S.Stage2Context() as b:
        b.load(other)
        with pytest.raises(Stage2CudaError, match="the state is of a 5000 x 20 patch"):
            b.import_state(blob)
    with S.Stage2Context() as c:
        c.load(prep, "fp64")
        with pytest.raises(Stage2CudaError, match="FP32"):
            c.import_state(blob)


def test_step_matches_run_to_convergence(S, prep):
    with S.Stage2Context() as c:
        c.load(prep)
        full = c.run()
        ref = c.download(KEYS)
    with S.Stage2Context() as c:
        c.load(prep)
        n = 0
        while True:
            st = c.step()
            n += 1
            if st["stop"]:
                break
        got = c.download(KEYS)
    assert n == full["i_loop"] == st["i_loop"]
    for k in KEYS:
        np.testing.assert_array_equal(got[k], ref[k], err_msg=k)


def test_debug_pm_dumps_one_file_per_iteration(S, patch, tmp_path, monkeypatch):
    from scipy.io import loadmat

    from test_gpu_pm1 import REQUIRED, write_patch

    d = tmp_path / "PATCH_1"
    write_patch(d, patch)
    monkeypatch.delenv("PYSTAMPS_STAGE2_NATIVE_DEBUG_PM", raising=False)
    S.stage2_estimate_gamma(d)
    plain = loadmat(d / "pm1.mat")
    monkeypatch.setenv("PYSTAMPS_STAGE2_NATIVE_DEBUG_PM", "1")
    S.stage2_estimate_gamma(d)
    n = int(plain["i_loop"].reshape(-1)[0])
    dumps = sorted(p.name for p in d.glob("pm1_iter_*.mat"))
    assert n >= 2 and dumps == [f"pm1_iter_{i:02d}.mat" for i in range(1, n + 1)]
    last = loadmat(d / dumps[-1])
    final = loadmat(d / "pm1.mat")
    for k in REQUIRED:
        np.testing.assert_array_equal(last[k], final[k], err_msg=k)
        np.testing.assert_array_equal(final[k], plain[k], err_msg=k)
    assert int(loadmat(d / "pm1_iter_01.mat")["i_loop"].reshape(-1)[0]) == 1


def test_download_into_caller_buffers(S, prep):
    """download(out=...) fills the caller's float64 arrays (reused, e.g. pinned,
    host buffers) with the values a plain download returns; wrong buffers are refused."""
    keys = ["K_ps", "C_ps", "coh_ps", "N_opt"]
    with S.Stage2Context() as c:
        c.load(prep)
        c.iterate(2)
        ref = c.download(keys)
        bufs = {k: np.full(prep.n_ps, 7.0) for k in keys}
        got = c.download(keys, out=bufs)
        for k in keys:
            assert got[k] is bufs[k]
            np.testing.assert_array_equal(bufs[k], ref[k], err_msg=k)
        with pytest.raises(ValueError, match="float64 array"):
            c.download(["K_ps"], out={"K_ps": np.zeros(prep.n_ps, np.float32)})
