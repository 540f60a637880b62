"""z-slabs on one GPU: a mesh split into slabs (bfvm_create_slab), each slab its own solver, stepped
through parabiofvm_b200.slabs.step with LocalExchange (the exchanges as copies between the
solvers), against the same mesh held by one solver and stepped by bfvm_run_steps.

The slabs' z sweep solves every line in two passes around the exchanged carries, so it agrees
with the single solver to float rounding, not bit for bit; everything else (x and y sweeps,
Dirichlet, secretion, the gradient given the same field) is the same arithmetic.  One slab is the
single solver exactly.
"""

import numpy as np
import pytest

from parabiofvm_b200.workloads import make_solver, synthetic
from scenarios import rel_err, rel_l2


def _workload(edge_xy, planes, S, agents, seed):
    w = synthetic(edge_xy, S, agents, seed=seed, clustered=True, sigma=80.0, interior_fraction=0.02)
    # stretch the mesh along z: more planes than the x and y edge
    dx = w.voxel_shape[2]
    w.bbox_max = (w.bbox_max[0], w.bbox_max[1], planes * dx)
    rng = np.random.default_rng(seed + 1)
    w.densities = rng.uniform(0, 1, w.voxel_count * S).astype(np.float32)
    if w.interior_voxels is not None:
        keep = w.interior_voxels[:, 2] < planes - 1
        w.interior_voxels = w.interior_voxels[keep]
        w.interior_values = w.interior_values[keep]
        w.interior_conditions = w.interior_conditions[keep]
        extra = rng.integers(1, [edge_xy - 1, edge_xy - 1, planes - 1], size=(40, 3)).astype(np.int32)
        w.interior_voxels = np.concatenate([w.interior_voxels, extra])
        w.interior_values = np.concatenate([w.interior_values, rng.uniform(0, 1, (40, S))])
        w.interior_conditions = np.concatenate([w.interior_conditions, rng.random((40, S)) < 0.5])
    if w.agents is not None:
        pz = rng.uniform(0, planes * dx, w.agents.count).astype(np.float32)
        w.agents.positions[:, 2] = np.minimum(pz, np.nextafter(np.float32(planes * dx), np.float32(0)))
    return w


def _run(w, bounds, steps):
    import torch

    from parabiofvm_b200 import slabs as sl

    stream = torch.cuda.Stream()
    parts = [sl.make_slab(w, bounds, k, stream=stream) for k in range(len(bounds) - 1)]
    ex = sl.LocalExchange()
    sl.run_steps(parts, ex, steps)
    torch.cuda.synchronize()
    S = w.S
    dens = np.concatenate([p.load_densities() for p in parts])
    grads = [p.load_gradients().reshape(3, -1) for p in parts]
    grad = np.concatenate(grads, axis=1).reshape(-1)
    intern = np.zeros((w.agents.count if w.agents is not None else 0, S), np.float32)
    for p in parts:
        if p.agents_count:
            intern[p.agent_index] = p.load_internalized().reshape(-1, S)
    assert sum(p.agents_count for p in parts) == (w.agents.count if w.agents is not None else 0)
    for p in parts:
        p.close()
    return dens, grad, intern


def _single(w, steps):
    s = make_solver(w)
    s.run_steps(steps)
    out = (s.load_densities(), s.load_gradients(), s.load_internalized().reshape(-1, w.S) if w.agents else None)
    s.close()
    return out


@pytest.mark.gpu
def test_one_slab_is_the_single_solver():
    w = _workload(16, 70, 4, 300, seed=3)
    dens, grad, intern = _run(w, [0, 70], 3)
    ref = _single(w, 3)
    np.testing.assert_array_equal(dens, ref[0])
    np.testing.assert_array_equal(grad, ref[1])
    np.testing.assert_array_equal(intern, ref[2])


@pytest.mark.gpu
@pytest.mark.parametrize("planes,bounds", [
    (48, [0, 20, 48]),             # one block per slab, virtual fronts of 12 and 4
    (100, [0, 37, 70, 100]),       # two blocks, two blocks, one block
    (100, [0, 64, 100]),           # a slab of whole blocks (no virtual front)
    (130, [0, 2, 66, 68, 130]),    # slabs of two planes
])
def test_slabs_match_the_single_solver(planes, bounds):
    w = _workload(16, planes, 4, 400, seed=planes + len(bounds))
    steps = 3  # a recompute step, then two with the binning reused
    dens, grad, intern = _run(w, bounds, steps)
    ref = _single(w, steps)
    # the z sweep's carries cross the slab edges in float: a few ulps per step
    assert rel_err(dens, ref[0]) < 2e-5
    assert rel_l2(dens, ref[0]) < 2e-6
    # a gradient is a difference of two field values times 1/h or 1/(2h), so it can differ by at
    # most twice the field's largest difference over h, plus its own rounding
    du = float(np.abs(dens.astype(np.float64) - ref[0]).max())
    dg = float(np.abs(grad.astype(np.float64) - ref[1]).max())
    assert dg <= 2 * du / w.voxel_shape[2] + 1e-6 * float(np.abs(ref[1]).max())
    assert rel_l2(grad, ref[1]) < 2e-5
    # an agent's internalized amount changes by voxel volume x den/(1+den) x its voxel's density
    # each step: the field's differences reach it multiplied by up to the voxel volume per step
    di = float(np.abs(intern.astype(np.float64) - ref[2]).max())
    vox = w.voxel_shape[0] * w.voxel_shape[1] * w.voxel_shape[2]
    assert di <= 2 * steps * vox * du + 1e-6 * float(np.abs(ref[2]).max()), (di, du)
    assert rel_l2(intern, ref[2]) < 2e-5


@pytest.mark.gpu
@pytest.mark.parametrize("planes,bounds", [(100, [0, 37, 70, 100]), (130, [0, 2, 66, 68, 130])])
def test_slabs_against_the_oracle(planes, bounds):
    """The split mesh stepped against the FP32 oracle directly (not only against the single CUDA
    solver): the field at the multi-block bar after three full steps, and the agents' internalized
    amounts."""
    from scenarios import make_oracle

    w = _workload(16, planes, 4, 400, seed=planes + 7 * len(bounds))
    dens, grad, intern = _run(w, bounds, 3)
    o = make_oracle(w, np.float32)
    o.run_steps(3, 0)
    assert rel_err(dens, o.densities()) < 2e-5
    assert rel_l2(grad, o.gradients()) < 2e-5
    assert rel_l2(intern, o.internalized().reshape(-1, w.S)) < 2e-5


@pytest.mark.gpu
def test_slab_substrates_not_multiple_of_four_in_x():
    # X * S = 15 * 3: not a multiple of 4, which the staged slab sweep needs
    from parabiofvm_b200 import slabs as sl
    from parabiofvm_b200._abi import BfvmError

    w = synthetic(15, 3, 0, seed=5)
    with pytest.raises(BfvmError, match="multiple of 4"):
        sl.make_slab(w, [0, 7, 15], 0)


@pytest.mark.gpu
def test_whole_mesh_calls_are_refused_on_a_split_mesh():
    from parabiofvm_b200 import Batch
    from parabiofvm_b200 import slabs as sl
    from parabiofvm_b200._abi import BfvmError

    w = _workload(8, 40, 4, 0, seed=9)
    s = sl.make_slab(w, [0, 20, 40], 1)
    for call in (s.diffusion, s.gradient, lambda: s.run_steps(1), lambda: s.sweep(2)):
        with pytest.raises(BfvmError) as e:
            call()
        assert e.value.status == 5
    s.sweep(0)  # the x and y sweeps stay within the slab
    s.sweep(1)
    with pytest.raises(BfvmError) as e:
        s.diffusion_end(s.exchange.new_zeros(2 * s.lines * 2))
    assert e.value.status == 5  # end without begin
    with pytest.raises(BfvmError):
        Batch([s])
    s.synchronize()
    s.close()


@pytest.mark.gpu
@pytest.mark.parametrize("planes,bounds,D", [
    (100, [0, 37, 70, 100], [50.0, 1e3, 1e5, 1e6]),  # slow decay: the sums keep every plane
    (300, [0, 150, 300], [50.0, 1e3, 5e3, 1e4]),      # fast decay: the sums keep the edge planes
    (300, [0, 100, 200, 300], [1e3, 3e4, 1e5, 2e5]),
    (120, [0, 50, 120], [1e3, 1e5]),                  # 2 substrates: the one-line-per-thread kernel
])
def test_reduce_pass_publishes_the_zero_carry_solve(planes, bounds, D):
    """The exchange that bfvm_slab_diffusion_begin writes, A = the forward value at the slab's last
    plane and B = its first solution, both from zero carries, against the float64 Thomas solve of
    the slab's part of every z line (src/solver/host/diffusion_solver.cpp:72-142) on the field the
    x and y sweeps left (no Dirichlet conditions, so that field is the z sweep's right-hand side)."""
    from parabiofvm_b200 import slabs as sl
    from test_slabs_cpu import slab_solve, thomas_coefficients

    w = synthetic(8, len(D), 0, seed=planes + len(bounds), boundary_substrate0=False)
    w.diffusion_coefficients = list(D)
    w.bbox_max = (w.bbox_max[0], w.bbox_max[1], planes * w.voxel_shape[2])
    w.densities = np.random.default_rng(planes).uniform(0, 1, w.voxel_count * w.S).astype(np.float32)
    bp, c = thomas_coefficients(planes, w.voxel_shape[2], 3, w.time_step, w.diffusion_coefficients, w.decay_rates)
    for k in range(len(bounds) - 1):
        i0, i1 = bounds[k], bounds[k + 1]
        s = sl.make_slab(w, bounds, k)
        s.sweep(0)
        s.sweep(1)
        d = s.load_densities().reshape(i1 - i0, -1).astype(np.float64)
        s.close()
        s = sl.make_slab(w, bounds, k)
        s.diffusion_begin()
        s.synchronize()  # the exchange is written on the slab's own stream
        ex = s.exchange.cpu().numpy().reshape(2, -1).astype(np.float64)
        s.close()
        x, f = slab_solve(d, bp, c, i0, i1)
        # every weight is positive (c < 0 in the reference's sign convention) and the field too, so
        # the float sums carry a relative error of a few ulps per term at most
        if i1 < planes:
            assert np.all(np.abs(ex[0] - f[-1]) <= 8e-6 * f[-1]), k
        else:
            assert not ex[0].any()
        if i0 > 0:
            assert np.all(np.abs(ex[1] - x[0]) <= 8e-6 * x[0]), k
        else:
            assert not ex[1].any()
