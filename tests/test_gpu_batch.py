"""Batched ensembles (bfvm_batch_*): every instance of a batch must end exactly where the same
solver stepped alone ends, bit for bit, whatever the other instances are."""

import numpy as np
import pytest

from parabiofvm_b200 import Batch
from parabiofvm_b200.workloads import make_solver, synthetic

pytestmark = pytest.mark.gpu


def _ensemble():
    ws = [
        synthetic(24, 3, 300, seed=1, clustered=True, sigma=50.0, interior_fraction=0.02),
        synthetic(37, 5, 800, seed=2, clustered=True, sigma=80.0),
        synthetic(50, 4, 2000, seed=3, interior_fraction=0.01),
        synthetic(40, 2, 0, seed=4, dims=2),
        synthetic(33, 8, 500, seed=5, clustered=True, sigma=40.0, internalized=False),
        synthetic(64, 1, 100, seed=6),
        synthetic(48, 3, 0, seed=7, dims=1),
        synthetic(40, 8, 60, seed=8, interior_fraction=0.01),
    ]
    return ws


def _state(s):
    out = [s.load_densities().copy(), s.load_gradients().copy()]
    if s.agents_count:
        out.append(s.load_internalized().copy())
    return out


@pytest.mark.parametrize("steps,first", [(12, 0), (3, 1)])
def test_batch_matches_each_solver_alone(steps, first):
    ws = _ensemble()
    alone = []
    for w in ws:
        s = make_solver(w)
        s.run_steps(steps, first)
        s.synchronize()
        alone.append(_state(s))
        s.close()
    solvers = [make_solver(w) for w in ws]
    b = Batch(solvers)
    b.run_steps(steps, first)
    b.synchronize()
    for i, s in enumerate(solvers):
        got = _state(s)
        for g, a in zip(got, alone[i]):
            np.testing.assert_array_equal(g, a, err_msg=f"instance {i}")
    # a second call continues from there, with the graphs already built
    b.run_steps(2, first + steps)
    b.synchronize()
    b.close()
    for s in solvers:
        s.close()


def test_batch_follows_changes_to_an_instance():
    ws = _ensemble()[:3]
    solvers = [make_solver(w) for w in ws]
    ref = [make_solver(w) for w in ws]
    b = Batch(solvers)
    b.run_steps(2, 0)
    # new agents on one instance (a different count: its buffers are reallocated)
    a = synthetic(37, 5, 400, seed=9, clustered=True, sigma=80.0).agents
    solvers[1].store_agents(a.secretion_rates, a.saturation_densities, a.uptake_rates, a.net_export_rates,
                            a.internalized, a.fraction_released, a.volumes, a.positions)
    b.run_steps(3, 2)
    b.synchronize()
    for r in ref:
        r.run_steps(2, 0)
    ref[1].store_agents(a.secretion_rates, a.saturation_densities, a.uptake_rates, a.net_export_rates,
                        a.internalized, a.fraction_released, a.volumes, a.positions)
    for r in ref:
        r.run_steps(3, 2)
        r.synchronize()
    for s, r in zip(solvers, ref):
        for g, e in zip(_state(s), _state(r)):
            np.testing.assert_array_equal(g, e)
    b.close()
    for s in solvers + ref:
        s.close()


def test_solver_alone_then_batched_then_alone():
    """A solver with internalized substrates keeps its agent terms in the binning's sorted order,
    alone and in a batch (whose ensemble update reads them sorted too).  Joining and leaving a batch
    keeps the results bit for bit those of a solver that only ever stepped alone."""
    ws = _ensemble()[:3]
    solvers = [make_solver(w) for w in ws]
    ref = make_solver(ws[0])
    solvers[0].run_steps(12, 0)
    b = Batch(solvers)
    b.run_steps(12, 12)
    b.synchronize()
    b.close()
    solvers[0].release(5)
    solvers[0].run_steps(12, 24)
    ref.run_steps(24, 0)
    ref.release(5)
    ref.run_steps(12, 24)
    for g, e in zip(_state(solvers[0]), _state(ref)):
        np.testing.assert_array_equal(g, e)
    for s in solvers + [ref]:
        s.close()


def test_autotuned_batch_matches_each_solver_alone():
    """bfvm_batch_autotune times the ensemble kernels' launch choices on scratch copies: it leaves
    the instances' state as it was, and the batch stepped with the chosen launches still ends
    exactly where each solver stepped alone ends."""
    ws = _ensemble()
    alone = []
    for w in ws:
        s = make_solver(w)
        s.run_steps(11, 0)
        alone.append(_state(s))
        s.close()
    solvers = [make_solver(w) for w in ws]
    b = Batch(solvers)
    b.run_steps(1, 0)
    choices = b.autotune()
    assert set(choices["sweep_ctas_per_sm"]) <= {1, 2} and set(choices["sweep_ctas_per_slot"]) <= {1, 2, 4}
    assert choices["gradient_planes"] in (32, 64, 128) and choices["gradient_load_batch"] in (4, 8)
    b.run_steps(10, 1)
    b.synchronize()
    for i, s in enumerate(solvers):
        for g, a in zip(_state(s), alone[i]):
            np.testing.assert_array_equal(g, a, err_msg=f"instance {i}")
    b.close()
    for s in solvers:
        s.close()


def test_batch_members_changed_between_steps():
    """Between batch steps, two members release an agent's internalized substrates (found through
    the agent's rank while the terms are sorted) and a third has its internalized amounts loaded
    and stored back, across a recompute step that rebins and sorts again: the members end where
    solvers stepped alone with the same calls end, bit for bit.  Covers the four-substrate sorted
    update with and without voxels shared by agents (meshes 2 and 7)."""
    ws = _ensemble()
    solvers = [make_solver(w) for w in ws]
    ref = [make_solver(w) for w in ws]
    b = Batch(solvers)

    def changes(group):
        group[2].release(3)
        group[7].release(11)
        a = ws[1].agents
        amounts = group[1].load_internalized().copy()
        group[1].store_agents(a.secretion_rates, a.saturation_densities, a.uptake_rates, a.net_export_rates,
                              amounts, a.fraction_released, a.volumes, a.positions)

    b.run_steps(6, 0)
    b.synchronize()
    changes(solvers)
    b.run_steps(8, 6)
    b.synchronize()
    for r in ref:
        r.run_steps(6, 0)
    changes(ref)
    for r in ref:
        r.run_steps(8, 6)
        r.synchronize()
    for i, (s, r) in enumerate(zip(solvers, ref)):
        for g, e in zip(_state(s), _state(r)):
            np.testing.assert_array_equal(g, e, err_msg=f"instance {i}")
    b.close()
    for s in solvers + ref:
        s.close()


def test_batch_faces_written_by_the_sweeps():
    """The ensemble sweeps write the face conditions of each mesh whose interior Dirichlet voxels
    stay off the faces, and the overwrites after them take only the interior elements.  Meshes with
    a different value on every (face, substrate), random subsets of conditioned substrates per
    face (so every precedence case where faces meet occurs), interior voxels on the faces (that
    mesh keeps its whole list), lines that straddle tiles, 2-D and 1-D: each ends bit for bit where
    the same solver stepped alone ends."""
    from test_gpu_faces import _faces_workload

    ws = [_faces_workload((24, 20, 18), 4, 3, seed=1), _faces_workload((30, 26, 22), 16, 3, seed=2),
          _faces_workload((36, 36, 36), 8, 3, seed=3, interior_on_faces=True),
          _faces_workload((70, 33, 20), 5, 3, seed=4), _faces_workload((40, 30, 1), 6, 2, seed=5),
          _faces_workload((50, 1, 1), 3, 1, seed=6)]
    alone = []
    for w in ws:
        s = make_solver(w)
        s.run_steps(4, 0)
        alone.append(_state(s))
        s.close()
    solvers = [make_solver(w) for w in ws]
    b = Batch(solvers)
    b.run_steps(4, 0)
    b.synchronize()
    for i, s in enumerate(solvers):
        for g, a in zip(_state(s), alone[i]):
            np.testing.assert_array_equal(g, a, err_msg=f"instance {i}")
    b.close()
    for s in solvers:
        s.close()


def test_all_3d_batch_matches_each_solver_alone():
    """A batch of 3-D meshes only runs the gradient kernel without the 1-D and 2-D forms (the
    batch-256 case): meshes of 1 to 8 substrates (the four-substrate march and the one-element
    march), z extents that do not divide the planes per work unit, agents binned on a recompute
    step; each ends bit for bit where the same solver stepped alone ends."""
    ws = [synthetic(24, 3, 300, seed=11, clustered=True, sigma=50.0, interior_fraction=0.02),
          synthetic(37, 5, 800, seed=12, clustered=True, sigma=80.0),
          synthetic(50, 4, 2000, seed=13, interior_fraction=0.01),
          synthetic(33, 1, 500, seed=14, internalized=False),
          synthetic(70, 7, 3000, seed=15, clustered=True, sigma=60.0),
          synthetic(45, 8, 60, seed=16)]
    alone = []
    for w in ws:
        s = make_solver(w)
        s.run_steps(12, 0)
        alone.append(_state(s))
        s.close()
    solvers = [make_solver(w) for w in ws]
    b = Batch(solvers)
    b.run_steps(12, 0)
    b.synchronize()
    for i, s in enumerate(solvers):
        for g, a in zip(_state(s), alone[i]):
            np.testing.assert_array_equal(g, a, err_msg=f"instance {i}")
    b.close()
    for s in solvers:
        s.close()
