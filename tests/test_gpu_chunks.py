"""Lines longer than the staged sweep takes whole (more than 512 voxels), cut into chunks of at
most 512 that it takes: a carries pass (each chunk's end values from the elements near its ends,
folded into the chunks' carries) and the staged sweep of the chunks entered with their carries.
Checked against the FP32 oracle at the multi-block bar along each axis, with Dirichlet faces and
interior nodes, two to four chunks per line, substrate counts that need 16-byte-aligned x chunk
bounds, and against the ensemble sweep that takes these lines without chunks."""

import numpy as np
import pytest

from gpu_runner import gpu_runner
from scenarios import make_oracle, rel_err
from test_gpu_parity import _box

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("grid,S", [((1600, 8, 8), 4), ((1030, 10, 6), 6), ((10, 1100, 10), 2), ((8, 8, 2048), 4),
                                    ((12, 12, 777), 3), ((700, 600, 4), 4), ((6, 6, 1031), 4), ((1031, 6, 5), 4)])
def test_chunked_lines_against_the_oracle(grid, S):
    """Equal chunks swept in one launch (1600 = 4 x 400, 1030 = 5 x 206 with 16-byte-aligned x
    bounds at 6 substrates, 777 = 3 x 259, ...) and, for a prime length (1031), chunks of unequal
    length swept one launch each."""
    w = _box(grid, S, seed=sum(grid) * S + 1)
    o = make_oracle(w, np.float32)
    g = gpu_runner(w)
    o.diffusion()
    g.diffusion()
    assert rel_err(g.densities(), o.densities()) < 1e-5
    o.run_steps(2, 1)
    g.run_steps(2, 1)
    assert rel_err(g.densities(), o.densities()) < 1e-5
    np.testing.assert_allclose(g.gradients(), o.gradients(), rtol=0, atol=2e-5 * float(np.abs(o.gradients()).max()))
    g.close()


@pytest.mark.parametrize("grid,S", [((1024, 16, 16), 4), ((16, 1024, 16), 4), ((16, 16, 1024), 8)])
def test_chunked_lines_against_the_ensemble_sweep(grid, S):
    """The same steps with the staged path off (option tma_sweeps 0: the ensemble sweep, whole lines
    in one CTA) agree to rounding, and the chunked path repeats its own bits."""
    w = _box(grid, S, seed=7 * sum(grid) + S)
    a = gpu_runner(w)
    b = gpu_runner(w)
    c = gpu_runner(w)
    b.s.set_option("tma_sweeps", 0)
    for r in (a, b, c):
        r.run_steps(3, 0)
    assert rel_err(a.densities(), b.densities()) < 1e-5
    np.testing.assert_array_equal(a.densities(), c.densities())
    for r in (a, b, c):
        r.close()
