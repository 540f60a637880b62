"""The Dirichlet face conditions written by position inside the staged sweeps (option
face_dirichlet): each staged sweep of the step writes the face conditions into the values it
stores, and the scatter kernel after it keeps the interior elements.  The result must be the same
bits as the scatter of the whole list (face_dirichlet 0, the default), and match the oracle, for
every precedence case where faces meet: edges and corners with different values per face and
substrate, faces that condition only some substrates, and meshes whose interior Dirichlet voxels
lie on a face (where the sweeps leave the faces to the scatter)."""

import numpy as np
import pytest

from gpu_runner import gpu_runner
from parabiofvm_b200.workloads import Workload
from scenarios import make_oracle, rel_err

pytestmark = pytest.mark.gpu


def _faces_workload(grid, S, dims, seed, interior=0.01, interior_on_faces=False, cond_p=0.6):
    """A seeded mesh with a different value on every (face, substrate) and a random subset of
    conditioned substrates per face, plus interior Dirichlet voxels (inside the mesh unless
    interior_on_faces)."""
    rng = np.random.default_rng(seed)
    shape = tuple(grid[:dims]) + (1,) * (3 - dims)
    w = Workload(dims=dims, bbox_min=(0, 0, 0), bbox_max=tuple(20 * g for g in shape), voxel_shape=(20, 20, 20),
                 diffusion_coefficients=list(np.exp(rng.uniform(np.log(1e3), np.log(1e5), S))),
                 decay_rates=list(rng.uniform(0.01, 1.0, S)), time_step=0.01, initial_conditions=[0.0] * S)
    V = shape[0] * shape[1] * shape[2]
    w.densities = rng.uniform(0, 1, V * S).astype(np.float32)
    for d in range(dims):
        for is_max in (False, True):
            f = 2 * d + int(is_max)
            vals = 10.0 * (f + 1) + np.arange(S)
            conds = rng.uniform(size=S) < cond_p
            w.boundary[(d, is_max)] = (vals, conds)
    if interior > 0 and dims == 3:
        lo = 0 if interior_on_faces else 1
        inner = [g - 2 * lo for g in shape]
        n = max(1, int(interior * inner[0] * inner[1] * inner[2]))
        pick = rng.choice(inner[0] * inner[1] * inner[2], size=n, replace=False)
        w.interior_voxels = np.stack([pick % inner[0] + lo, (pick // inner[0]) % inner[1] + lo,
                                      pick // (inner[0] * inner[1]) + lo], axis=1).astype(np.int32)
        w.interior_values = rng.uniform(0, 1, (n, S))
        w.interior_conditions = rng.uniform(size=(n, S)) < 0.8
    return w


def _pair(w):
    by_pos = gpu_runner(w)
    scatter = gpu_runner(w)
    by_pos.s.set_option("face_dirichlet", 1)
    scatter.s.set_option("face_dirichlet", 0)
    return by_pos, scatter


@pytest.mark.parametrize("grid,S,dims,on_faces", [((48, 40, 36), 16, 3, False), ((40, 40, 40), 5, 3, False),
                                                  ((70, 33, 20), 4, 3, False), ((36, 36, 36), 8, 3, True),
                                                  ((600, 24, 24), 4, 3, False), ((100, 90, 1), 6, 2, False),
                                                  ((300, 1, 1), 8, 1, False)])
def test_faces_by_position_identical_to_scatter(grid, S, dims, on_faces):
    """Steps, the LOD step alone, and the step with the gradient: the same bits both ways.  The
    cases cover substrate counts that leave lanes of an x tile idle (5), lines that straddle 32-column
    tiles (70 x 4), interior voxels on the faces (the scatter then writes the faces), lines longer than
    the staged sweep takes (600: the x sweep is not staged and the whole list follows it), 2D and 1D."""
    w = _faces_workload(grid, S, dims, seed=sum(grid) + S, interior_on_faces=on_faces)
    a, b = _pair(w)
    for first, n in ((0, 2), (2, 3)):
        a.run_steps(n, first)
        b.run_steps(n, first)
        np.testing.assert_array_equal(a.densities(), b.densities())
        np.testing.assert_array_equal(a.gradients(), b.gradients())
    a.diffusion()
    b.diffusion()
    np.testing.assert_array_equal(a.densities(), b.densities())
    a.s.diffusion_gradient()
    b.s.diffusion_gradient()
    np.testing.assert_array_equal(a.densities(), b.densities())
    np.testing.assert_array_equal(a.gradients(), b.gradients())
    a.close()
    b.close()


@pytest.mark.parametrize("grid,S", [((24, 20, 18), 4), ((30, 26, 22), 16)])
def test_faces_by_position_against_the_oracle(grid, S):
    """Single-block lines (at most 32 voxels): the staged sweeps reproduce the reference's Thomas
    solve bit for bit, so the LOD step with the faces written by position equals the FP32 oracle's
    bit for bit, precedence at edges and corners included."""
    w = _faces_workload(grid, S, 3, seed=3 * sum(grid) + S)
    o = make_oracle(w, np.float32)
    g = gpu_runner(w)
    g.s.set_option("face_dirichlet", 1)
    for _ in range(2):
        o.diffusion()
        g.diffusion()
        np.testing.assert_array_equal(g.densities(), o.densities())
    g.close()


def test_faces_by_position_multi_block_against_the_oracle():
    """Multi-block lines (96 x 80 x 72): within the multi-block bar of the FP32 oracle after three
    LOD steps."""
    w = _faces_workload((96, 80, 72), 8, 3, seed=11)
    o = make_oracle(w, np.float32)
    g = gpu_runner(w)
    g.s.set_option("face_dirichlet", 1)
    for _ in range(3):
        o.diffusion()
        g.diffusion()
    assert rel_err(g.densities(), o.densities()) < 1e-5
    g.close()
