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


@pytest.mark.parametrize("grid,S,dims", [((2000, 1, 1), 4, 1), ((1100, 40, 1), 4, 2), ((1200, 30, 1), 8, 2)])
def test_chunked_lines_in_1d_and_2d(grid, S, dims):
    """1-D and 2-D meshes with long x lines: the chunks' x rows, with Dirichlet 1.0 on substrate 0
    at both x faces, against the FP32 oracle over a few full steps."""
    from parabiofvm_b200.workloads import Workload

    rng = np.random.default_rng(sum(grid) + S)
    w = Workload(dims=dims, bbox_min=(0, 0, 0), bbox_max=(20 * grid[0], 20 * grid[1], 20),
                 voxel_shape=(20, 20, 20),
                 diffusion_coefficients=list(np.exp(rng.uniform(np.log(1e3), np.log(1e5), S))),
                 decay_rates=list(rng.uniform(0.01, 1.0, S)), time_step=0.01, initial_conditions=[0.0] * S)
    w.densities = rng.uniform(0, 1, grid[0] * grid[1] * S).astype(np.float32)
    vals = np.zeros(S)
    conds = np.zeros(S, dtype=bool)
    vals[0], conds[0] = 1.0, True
    for is_max in (False, True):
        w.boundary[(0, is_max)] = (vals, conds)
    o = make_oracle(w, np.float32)
    g = gpu_runner(w)
    o.run_steps(3, 0)
    g.run_steps(3, 0)
    assert rel_err(g.densities(), o.densities()) < 1e-5
    g.close()


def test_chunk_length_option():
    """Lines of 300 cut into chunks of at most 160 (option chunk_elements) agree to rounding with
    the same lines swept whole, and the option is checked."""
    from parabiofvm_b200 import BfvmError

    w = _box((300, 60, 40), 8, seed=99)
    whole = gpu_runner(w)
    cut = gpu_runner(w)
    cut.s.set_option("chunk_elements", 160)
    whole.run_steps(3, 0)
    cut.run_steps(3, 0)
    assert rel_err(cut.densities(), whole.densities()) < 1e-5
    for bad in (63, 513, -1):
        with pytest.raises(BfvmError):
            cut.s.set_option("chunk_elements", bad)
    cut.s.set_option("chunk_elements", 0)
    whole.close()
    cut.close()
