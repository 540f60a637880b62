"""The reference's own test cases (test/test.cpp) on the CUDA library, through the C ABI.

Same cases and golden values as tests/test_oracle_goldens.py, with the GPU solver as the runner.
The meshes are small enough that every line fits one register block, so the GPU arithmetic is the
reference's operation for operation and the 4-ULP EXPECT_FLOAT_EQ bound applies unchanged.
"""

import pytest

import reference_cases as rc
from gpu_runner import gpu_runner

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("dims", [1, 2, 3])
def test_diffusion_uniform(dims):
    rc.case_diffusion_uniform(gpu_runner, dims)


@pytest.mark.parametrize("dims", [1, 2, 3])
def test_diffusion_random(dims):
    rc.case_diffusion_random(gpu_runner, dims)


@pytest.mark.parametrize("dims", [1, 2, 3])
def test_dirichlet_one_cond(dims):
    rc.case_dirichlet_one_cond(gpu_runner, dims)


@pytest.mark.parametrize("dims", [1, 2, 3])
def test_dirichlet_multiple_cond(dims):
    rc.case_dirichlet_multiple_cond(gpu_runner, dims)


@pytest.mark.parametrize("dims", [1, 2, 3])
def test_gradient(dims):
    rc.case_gradient(gpu_runner, dims)


@pytest.mark.parametrize("dims", [1, 2, 3])
def test_dirichlet_boundaries(dims):
    rc.case_dirichlet_boundaries(gpu_runner, dims)


@pytest.mark.parametrize("internalized", [True, False])
@pytest.mark.parametrize("recompute", [True, False])
@pytest.mark.parametrize("dims", [1, 2, 3])
def test_agents_simple(dims, internalized, recompute):
    rc.case_agents_simple(gpu_runner, dims, internalized, recompute)


@pytest.mark.parametrize("internalized", [True, False])
@pytest.mark.parametrize("recompute", [True, False])
@pytest.mark.parametrize("big", [False, True])
def test_agents_conflict(big, internalized, recompute):
    rc.case_agents_conflict(gpu_runner, internalized, recompute, big=big)


@pytest.mark.parametrize("size", [(200, 200), (200, 20000), (20000, 200), (20000, 20000)])
def test_diffusion_2d_sizes(size):
    """test/test_device.cpp:35-67: 2D uniform diffusion at 10..1000 voxels per side."""
    import numpy as np

    import scenarios as sc
    scn = sc.default_microenv(sc.mesh(2, (size[0], size[1], 0), (20, 20, 0)))
    r = gpu_runner(scn)
    r.diffusion()
    d = r.densities().reshape(-1, 2)
    # every line longer than one block goes through the block carries: 1e-5 relative, not 4 ULPs
    np.testing.assert_allclose(d[:, 0], sc.golden(85), rtol=1e-5)
    np.testing.assert_allclose(d[:, 1], sc.golden(86), rtol=1e-5)
