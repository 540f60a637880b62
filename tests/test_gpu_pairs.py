"""Paired tiles in the staged y and z sweeps (option tma_pairs: 1, the default, pairs the z sweep;
2, used here, both): two warp groups share each stage, which holds two adjacent 32-column tiles
copied as one 64-column TMA box, and the group that finishes reading a stage second refills it.
Every line is solved by the same code from the same values, so fields and gradients must be the
same bits as with one tile per stage; the cases cover an odd number of z tiles (the last pair half
empty), y planes with an odd number of tiles (the y sweep then stays unpaired), three substrates
(tiles that start mid-voxel) and the plain-320 line shape.  The bounded wait on a pair's copy runs
out like any other."""

import numpy as np
import pytest

from parabiofvm_b200._abi import BfvmError
from gpu_runner import gpu_runner
from test_gpu_parity import _box

pytestmark = pytest.mark.gpu

BFVM_ERR_TIMEOUT = 7


@pytest.mark.parametrize("grid,S", [((42, 300, 290), 4), ((50, 300, 290), 4), ((52, 300, 290), 3),
                                    ((64, 320, 320), 16)])
def test_pairs_identical_to_single_tiles(grid, S):
    w = _box(grid, S, seed=sum(grid) + S)
    paired = gpu_runner(w)
    single = gpu_runner(w)
    paired.s.set_option("tma_pairs", 2)
    single.s.set_option("tma_pairs", 0)
    paired.run_steps(3, 0)
    single.run_steps(3, 0)
    np.testing.assert_array_equal(paired.densities(), single.densities())
    np.testing.assert_array_equal(paired.gradients(), single.gradients())
    for axis in (1, 2):
        paired.s.sweep(axis)
        single.s.sweep(axis)
        np.testing.assert_array_equal(paired.densities(), single.densities())
    paired.close()
    single.close()


@pytest.mark.parametrize("axis", [1, 2])
def test_paired_wait_runs_out(axis):
    w = _box((42, 300, 290), 4, seed=5 + axis)
    g = gpu_runner(w)
    fresh = gpu_runner(w)
    for r in (g, fresh):
        r.s.set_option("tma_pairs", 2)
    g.s.set_option("wait_limit_cycles", 2_000_000)
    g.s.set_option("test_drop_tile_copy", 1)  # the second tile of the first pair
    with pytest.raises(BfvmError) as e:
        g.s.sweep(axis)
        g.s.synchronize()
    assert e.value.status == BFVM_ERR_TIMEOUT, str(e.value)
    g.s.synchronize()
    g.s.set_option("test_drop_tile_copy", -1)
    g.s.set_option("wait_limit_cycles", 4_000_000_000)
    g.s.store_densities(w.densities)
    g.run_steps(2, 0)
    fresh.run_steps(2, 0)
    np.testing.assert_array_equal(g.densities(), fresh.densities())
    g.close()
    fresh.close()
