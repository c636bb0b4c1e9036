"""The autotuner's launch shapes: CLAP warps per block and resident blocks per
SM and binning's resident blocks per SM change only how the work is spread
over the GPU, so every choice gives the same bits; the CLAP form (window stack
and overlap-add pass, or blocks of 4 x 4 windows summed into FP64 partials and
a combine pass) associates each cell's FP64 sum of window values differently,
and those sums are exact for the window values of a patch, so it gives the same
bits too. The chosen shapes are kept per (interferogram bucket, PS bucket) for
later loads."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

KEYS = ["ph_grid", "ph_patch", "K_ps", "coh_ps", "C_ps"]


@pytest.fixture(scope="module")
def prep(cuda_lib):
    from pystamps_b200 import stage2, synth

    return stage2.prepare_patch(synth.make_patch(20_000, 40, 40, 81, seed=77, n_rand=3000))


@pytest.mark.parametrize("precision", ["fp32", "fp64"])
def test_clap_and_binning_shapes_are_bit_identical(prep, precision):
    from pystamps_b200 import stage2

    shapes = [[0, 4, 0, 0, 0], [0, 0, 1, 0, 0], [0, 4, 1, 2, 0], [0, 0, 0, 4, 0], [0, 0, 0, 1, 0],
              [0, 0, 0, 0, 1], [0, 4, 1, 0, 1], [0, 8, 0, 3, 1]]
    if precision == "fp64":
        shapes = [[0, 0, 1, 0, 0], [0, 0, 0, 2, 0], [0, 4, 1, 1, 0], [0, 0, 0, 0, 1], [0, 4, 1, 0, 1]]
    with stage2.Stage2Context() as ctx:
        ctx.load(prep, precision)
        ctx.launch_shapes([0, 0, 0, 0, 0])
        ctx.iterate(2)
        ref = ctx.download(KEYS)
        for sh in shapes:
            ctx.launch_shapes(sh)
            assert ctx.launch_shapes() == sh
            ctx.reset()
            ctx.iterate(2)
            got = ctx.download(KEYS)
            for k in KEYS:
                np.testing.assert_array_equal(got[k], ref[k], err_msg=f"{k} with shapes {sh}")


def test_autotune_keeps_its_choice_for_the_bucket(prep):
    from pystamps_b200 import stage2
    from pystamps_b200._lib import Stage2CudaError

    with stage2.Stage2Context() as ctx:
        ctx.load(prep)
        lanes, ms = ctx.autotune()
        chosen = ctx.launch_shapes()
    assert lanes in (4, 8, 16, 32) and chosen[0] == lanes and all(t > 0 for t in ms)
    assert chosen[1] in (4, 8) and chosen[2] in (0, 1) and chosen[3] in (0, 2, 3) and chosen[4] in (0, 1)
    with stage2.Stage2Context() as ctx:
        ctx.load(prep)  # same bucket: the table's shapes
        assert ctx.launch_shapes() == chosen
        with pytest.raises(Stage2CudaError, match="lanes 0/4/8/16/32"):
            ctx.launch_shapes([3, 0, 0, 0, 0])
        with pytest.raises(Stage2CudaError, match="CLAP form 0/1"):
            ctx.launch_shapes([0, 0, 0, 0, 2])
    with stage2.Stage2Context() as ctx:
        ctx.load(prep, "fp64")
        with pytest.raises(Stage2CudaError, match="FP64 CLAP runs 4 warps"):
            ctx.launch_shapes([0, 8, 0, 0, 0])
