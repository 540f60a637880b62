"""bfvm_autotune: it measures the staged sweeps' launch shapes on a scratch copy, leaves the
field untouched, and the tuned solver steps bit for bit like the untuned one."""

import numpy as np
import pytest

from parabiofvm_b200.workloads import make_solver, synthetic

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("edge,S", [(64, 8), (50, 3)])
def test_autotune_keeps_results(edge, S):
    w = synthetic(edge, S, 1500, seed=edge + S, clustered=True, sigma=100.0, interior_fraction=0.01)
    ref = make_solver(w)
    ref.run_steps(4, 0)
    want = ref.load_densities().copy(), ref.load_gradients().copy(), ref.load_internalized().copy()
    ref.close()

    g = make_solver(w)
    before = g.load_densities().copy()
    choices = g.autotune()
    np.testing.assert_array_equal(g.load_densities(), before)  # the field is not touched
    assert len(choices) == 3
    for groups, stages in choices:
        assert (groups, stages) == (0, 0) or (1 <= groups <= 8 and 2 <= stages <= 4)
    g.run_steps(4, 0)
    for got, exp in zip((g.load_densities(), g.load_gradients(), g.load_internalized()), want):
        np.testing.assert_array_equal(got, exp)
    g.close()

    # a later solver of the same shape takes the cached shapes; its results are the same too
    h = make_solver(w)
    h.run_steps(4, 0)
    np.testing.assert_array_equal(h.load_densities(), want[0])
    h.close()
