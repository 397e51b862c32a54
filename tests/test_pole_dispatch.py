"""Host logic of the pole step's form choice (no GPU): the measured crossover between the tensor-core and the
CUDA-core kernels, and the tensor-core geometry the bench's roofline counts MMAs with."""
from blocksvibe_b200 import recursion as RC, roofline as RL


def test_crossover_picks_the_measured_faster_form():
    assert RC.pole_mma_gain(34, 5, 6) > RC.POLE_MIN_GAIN          # cfg2 batched: 30 of 32 columns
    assert RC.pole_mma_gain(34, 5, 1) < 1                         # one lambda order per recursion: 5 columns
    assert RC.pole_mma_gain(34, 3, 10) < 1                        # three structures: the CUDA cores win
    assert RC.pole_mma_gain(34, 1, 64) == 0                       # no tensor-core form for S = 1
    assert RC.pole_mma_gain(42, 5, 6) > RC.pole_mma_gain(34, 5, 6)
    # a second, nearly empty chunk halves the gain
    assert RC.pole_mma_gain(34, 5, 7) < 0.6 * RC.pole_mma_gain(34, 5, 6)


def test_ratio_table_grows_with_structures():
    for row in RC.POLE_FULL_CHUNK_RATIO.values():
        assert list(row) == sorted(row)


def test_mma_geometry_mirrors_the_kernel():
    # (U, MT): K digits per entry and 128-position tiles (pole_mma.cuh PoleMmaGeom)
    assert RL.pole_mma_geometry(10) == (64, 1)
    assert RL.pole_mma_geometry(26) == (128, 1)
    assert RL.pole_mma_geometry(30) == (128, 2)
    assert RL.pole_mma_geometry(34) == (160, 2)
    assert RL.pole_mma_geometry(46) == (192, 2)
    lev = {"t_slot": [0] * 10}
    issued, useful = RL.pole_mma_macs(lev, 150, 5, 34)              # S^2 B = 150 numbers: 30 columns
    assert issued == 2 * 10 * 5 * 5 * 5 * 2 * 128 * 32 * 32
    assert useful == 2 * 10 * 25 * 30 * 136 ** 2
