"""Edge shapes of the stage-2 loop, each checked iteration by iteration
against the oracle (the teacher-forced comparison of test_gpu_parity): the
fewest interferograms the trial count allows, the most the kernels take (256,
16 lanes per PS), a grid too small for any CLAP window (filtered phase 0, all
rows invalid, as in the reference's 3-PS fixture), and the size limits."""
import numpy as np
import pytest

from test_gpu_parity import _teacher_forced

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def S(cuda_lib):
    from pystamps_b200 import stage2

    return stage2


def test_two_interferograms(S, oracle):
    from pystamps_b200 import synth

    patch = synth.make_patch(4000, 2, 30, 21, seed=41, n_rand=4000)
    _teacher_forced(S, oracle, patch, iterations=3)


def test_256_interferograms(S, oracle):
    from pystamps_b200 import synth

    patch = synth.make_patch(1500, 256, 26, 41, seed=42, n_rand=2000)
    _teacher_forced(S, oracle, patch, iterations=2)


def test_single_cell_grid_has_no_windows(S, oracle):
    from pystamps_b200 import synth

    patch = synth.make_patch(300, 8, 1, 21, seed=43, n_rand=2000, gamma_max_iterations=2)
    prep = S.prepare_patch(patch)
    assert (prep.n_i, prep.n_j) == (1, 1)
    with S.Stage2Context() as c:
        c.load(prep)
        c.run()
        g = c.download(["K_ps", "coh_ps", "ph_patch"])
    assert np.all(g["ph_patch"] == 0)
    assert np.all(np.isnan(g["K_ps"])) and np.all(g["coh_ps"] == 0)


def test_size_limits_are_reported(S):
    from pystamps_b200 import synth
    from pystamps_b200._lib import Stage2CudaError

    patch = synth.make_patch(500, 257, 24, 21, seed=44, n_rand=1000)
    prep = S.prepare_patch(patch, nr=np.ones(100), nr_max_nz_ix=100.0)
    with S.Stage2Context() as c:
        with pytest.raises(Stage2CudaError, match="257"):
            c.load(prep)
