"""Bulk supply and uptake (src/solver/host/bulk_solver.cpp:20-33):
D = (D + dt*S*T) / (1 + dt*(U+S)) per voxel and substrate, with tabulated rates.

* CPU: the oracle against a float32 numpy restatement in the reference's operation order;
* GPU: the CUDA kernel against the oracle, bit for bit, for one rate row and for per-voxel rates.
"""

import numpy as np
import pytest

from scenarios import Scenario, make_oracle

f32 = np.float32


def _scene(seed=0, S=3):
    scn = Scenario(dims=3, bbox_min=(0, 0, 0), bbox_max=(140, 100, 60), voxel_shape=(20, 20, 20),
                   diffusion_coefficients=[10.0] * S, decay_rates=[0.1] * S, time_step=0.25,
                   initial_conditions=[0.0] * S)
    scn.densities = np.random.default_rng(seed).uniform(0, 5, scn.voxel_count * S).astype(f32)
    return scn


def _rates(scn, per_voxel, seed=1):
    rng = np.random.default_rng(seed)
    n = scn.voxel_count * scn.S if per_voxel else scn.S
    return (rng.uniform(0, 2, n).astype(f32), rng.uniform(0, 1, n).astype(f32), rng.uniform(0, 10, n).astype(f32))


def _restated(dens, dt, supply, uptake, target, S):
    d = dens.astype(f32).reshape(-1, S)
    sr, ur, tr = (np.broadcast_to(a.reshape(-1, S), d.shape) for a in (supply, uptake, target))
    dt = f32(dt)
    return ((d + (dt * sr) * tr) / (f32(1) + dt * (ur + sr))).reshape(-1)


@pytest.mark.parametrize("per_voxel", [False, True])
def test_oracle_bulk_matches_restatement(per_voxel):
    scn = _scene()
    o = make_oracle(scn)
    rates = _rates(scn, per_voxel)
    o.bulk(*rates, per_voxel)
    np.testing.assert_array_equal(o.densities(), _restated(scn.densities, scn.time_step, *rates, scn.S))


@pytest.mark.gpu
@pytest.mark.parametrize("per_voxel", [False, True])
def test_gpu_bulk_bit_exact(per_voxel):
    from parabiofvm_b200.workloads import make_solver

    scn = _scene(seed=4)
    rates = _rates(scn, per_voxel, seed=5)
    o = make_oracle(scn)
    g = make_solver(scn)
    g.set_bulk_rates(*rates, per_voxel)
    for _ in range(3):
        o.bulk(*rates, per_voxel)
        g.bulk()
    np.testing.assert_array_equal(g.load_densities(), o.densities())
    g.close()


@pytest.mark.gpu
def test_gpu_bulk_needs_rates():
    from parabiofvm_b200 import BfvmError
    from parabiofvm_b200.workloads import make_solver

    scn = _scene()
    g = make_solver(scn)
    with pytest.raises(BfvmError) as e:
        g.bulk()
    assert e.value.status == 5
    g.set_bulk_rates(*_rates(scn, False), False)
    g.bulk()
    g.set_bulk_rates(None, None, None, False)  # removed again
    with pytest.raises(BfvmError):
        g.bulk()
    g.close()
