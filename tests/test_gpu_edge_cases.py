"""Edge cases and error behaviour of the C ABI on the GPU."""

import numpy as np
import pytest

import scenarios as sc
from gpu_runner import gpu_runner
from parabiofvm_b200 import BfvmError, Solver
from scenarios import make_oracle, synthetic

pytestmark = pytest.mark.gpu


def test_axis_of_one_voxel():
    """A 3D mesh one voxel thick: that axis keeps only the decay part (diffusion_solver.cpp:76-85)."""
    scn = sc.Scenario(dims=3, bbox_min=(0, 0, 0), bbox_max=(200, 160, 20), voxel_shape=(20, 20, 20),
                      diffusion_coefficients=[1000.0, 10.0], decay_rates=[0.3, 1.0], time_step=0.1,
                      initial_conditions=[1.0, 2.0])
    scn.densities = np.random.default_rng(0).uniform(0, 1, scn.voxel_count * 2)
    o = make_oracle(scn)
    g = gpu_runner(scn)
    o.diffusion()
    g.diffusion()
    np.testing.assert_array_equal(g.densities(), o.densities())


@pytest.mark.parametrize("S", [1, 5, 17, 33])
def test_substrate_counts(S):
    scn = synthetic(20, S, 300, seed=S, clustered=True, sigma=40.0, interior_fraction=0.02)
    o = make_oracle(scn)
    g = gpu_runner(scn)
    for k in range(3):
        o.run_steps(1, k)
        g.run_steps(1, k)
    np.testing.assert_array_equal(g.densities(), o.densities())
    np.testing.assert_array_equal(g.internalized(), o.internalized())


def test_agent_outside_mesh_reports_error():
    scn = synthetic(10, 2, 50, seed=1)
    scn.agents.positions[3] = [-500.0, 10.0, 10.0]
    g = gpu_runner(scn)
    g.secretion(True)
    with pytest.raises(BfvmError) as e:
        g.s.synchronize()
    assert e.value.status == 6
    g.s.synchronize()  # the flag is cleared once reported


def test_no_agents_is_a_no_op():
    scn = synthetic(10, 2, 0, seed=1)
    g = gpu_runner(scn)
    before = g.densities()
    g.secretion(True)
    np.testing.assert_array_equal(g.densities(), before)


def test_all_agents_in_one_voxel():
    scn = synthetic(10, 2, 3000, seed=2)
    scn.agents.positions[:] = [55.0, 55.0, 55.0]
    o = make_oracle(scn)
    g = gpu_runner(scn)
    for rc in (True, False):
        o.secretion(rc)
        g.secretion(rc)
    np.testing.assert_array_equal(g.densities(), o.densities())
    np.testing.assert_array_equal(g.internalized(), o.internalized())


def test_invalid_arguments():
    with pytest.raises(BfvmError):
        Solver(4, (0, 0, 0), (100, 100, 100), (20, 20, 20), [1.0], [0.1], 0.01)
    with pytest.raises(BfvmError):
        Solver(3, (0, 0, 0), (100, 100, 100), (0, 20, 20), [1.0], [0.1], 0.01)
    s = Solver(3, (0, 0, 0), (100, 100, 100), (20, 20, 20), [1.0], [0.1], 0.01)
    with pytest.raises(BfvmError):
        s.set_interior_dirichlet([[9, 0, 0]], [[1.0]], [[1]])
    with pytest.raises(BfvmError):
        s.set_boundary_dirichlet(3, 0, [1.0], [1])
    with pytest.raises(BfvmError):
        s.release(0)
    s.close()


def test_agent_count_change_rebins():
    scn = synthetic(12, 2, 100, seed=3, clustered=True, sigma=30.0)
    o = make_oracle(scn)
    g = gpu_runner(scn)
    o.secretion(True)
    g.secretion(True)
    a = scn.agents
    keep = slice(0, 60)
    args = [x[keep] for x in (a.secretion_rates, a.saturation_densities, a.uptake_rates, a.net_export_rates)]
    intern = g.internalized().reshape(-1, 2)[keep]
    g.s.store_agents(*args, intern, a.fraction_released[keep], a.volumes[keep], a.positions[keep])
    o.set_agents(*args, intern, a.fraction_released[keep], a.volumes[keep], a.positions[keep])
    o.secretion(True)
    g.secretion(False)  # a new agent count forces the binning to be rebuilt
    np.testing.assert_array_equal(g.densities(), o.densities())


def test_positions_alone_enter_binning_at_recompute():
    """bfvm_store_agent_positions: the new positions take effect at the next recompute, exactly as
    a full bfvm_store_agents of the same arrays with the moved positions would."""
    from parabiofvm_b200.workloads import make_solver

    scn = synthetic(24, 3, 800, seed=11, clustered=True, sigma=60.0)
    a = scn.agents
    moved = np.ascontiguousarray(a.positions[::-1], np.float32)

    g = make_solver(scn)
    g.secretion(True)
    g.store_agent_positions(moved)
    g.secretion(False)  # still binned by the old positions
    g.secretion(True)
    got = g.load_densities(), g.load_internalized()
    g.close()

    h = make_solver(scn)
    h.secretion(True)
    h.store_agents(a.secretion_rates, a.saturation_densities, a.uptake_rates, a.net_export_rates,
                   h.load_internalized(), a.fraction_released, a.volumes, moved)
    h.secretion(False)
    h.secretion(True)
    want = h.load_densities(), h.load_internalized()
    h.close()
    np.testing.assert_array_equal(got[0], want[0])
    np.testing.assert_array_equal(got[1], want[1])


def test_positions_alone_reject_a_count_change():
    from parabiofvm_b200._abi import check
    from parabiofvm_b200.workloads import make_solver

    scn = synthetic(12, 2, 50, seed=3)
    g = make_solver(scn)
    with pytest.raises(BfvmError) as e:
        check(g._lib.bfvm_store_agent_positions(g._h, 49, None))
    assert e.value.status == 1
    g.close()
