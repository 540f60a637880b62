"""The C++20 host API (parabiofvm_b200/host: microenvironment_builder, agent container, solver) as
a paraBioFVM user drives it, from tests/cpp/facade_cases.cpp.

* host behaviour (no GPU): mesh shape, voxel lookup, builder output, agent removal;
* on the GPU: the uniform 3D diffusion case against the goldens of test/test.cpp:111-112, a
  scene with Dirichlet conditions and agents, stepped and released, against the oracle, and agents
  added and removed on the GPU copy against the round trip through the host.
"""

import json
import os
import subprocess

import numpy as np
import pytest

from scenarios import Agents, Scenario, assert_float_eq, golden, make_oracle, rel_err

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
LIBDIR = os.path.join(ROOT, "parabiofvm_b200", "_lib")


@pytest.fixture(scope="module")
def program(tmp_path_factory):
    from parabiofvm_b200 import build

    build.build_host()
    exe = str(tmp_path_factory.mktemp("facade") / "facade_cases")
    cmd = ["g++", "-std=c++20", "-O1", "-Wall", "-Wextra", "-Werror",
           "-I" + os.path.join(ROOT, "parabiofvm_b200", "host", "include"),
           os.path.join(ROOT, "tests", "cpp", "facade_cases.cpp"), "-o", exe,
           "-L" + LIBDIR, "-lbiofvm_b200", "-lbfvm_cuda", "-Wl,-rpath," + LIBDIR]
    r = subprocess.run(cmd, capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    return exe


def run(program, mode):
    r = subprocess.run([program, mode], capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stderr
    return json.loads(r.stdout)


def test_host_behaviour(program):
    out = run(program, "host")
    # cartesian_mesh: ceil((max - min) / voxel) per axis (src/mesh.cpp:7-25)
    assert out["grid"] == [11, 5, 2]
    assert out["voxel_count"] == 110 and out["voxel_volume"] == 20 * 20 * 30
    assert out["voxel_position"] == [2, 2, 3]  # truncating (45, 59, 91) / (20, 20, 30)
    assert out["voxel_center"] == [30, 50, 105]
    # builder: a 2D mesh, initial conditions everywhere, faces only where a condition is set
    assert out["grid2"] == [5, 3, 1]
    assert out["initial"] == [3, 4]
    assert out["faces"] == [0, 1, 1, 0]  # x-min, x-max, y-min, y-max
    assert out["xmax_face"] == [0, 10, 0, 1]
    assert out["ymin_face"] == [0, 8, 0, 1]
    assert out["interior_voxels"] == [1, 2, 3, 1]
    assert out["interior_conditions"] == [1, 0, 1, 1]  # empty conditions mean all substrates
    # removing agent 1 of 4 moves the last agent (id 3) into slot 1 with its data
    assert out["agents"] == 3 and out["moved_id"] == 3 and out["moved_index"] == 1
    assert out["moved_volume"] == 103 and out["moved_secretion"] == [3, 13]
    assert out["moved_voxel"] == [1, 0, 0]
    assert out["host_resident"] == 1  # microenvironment::data_residency starts at host


@pytest.mark.gpu
def test_uniform_diffusion_goldens(program):
    out = run(program, "uniform3d")
    d = np.asarray(out["densities"], np.float32).reshape(-1, 2)
    assert_float_eq(d[:, 0], golden(111), "C++ API D3 uniform s0")
    assert_float_eq(d[:, 1], golden(112), "C++ API D3 uniform s1")


@pytest.mark.gpu
def test_steps_with_dirichlet_and_agents_match_oracle(program):
    out = run(program, "step")
    S, A = 3, 40
    scn = Scenario(dims=3, bbox_min=(0, 0, 0), bbox_max=(120, 100, 80), voxel_shape=(20, 20, 20),
                   diffusion_coefficients=[1000.0, 100.0, 10.0], decay_rates=[0.1, 0.5, 1.0], time_step=0.01,
                   initial_conditions=[1.0, 0.5, 0.0], compute_internalized=True)
    scn.boundary[(0, False)] = (np.array([1.0, 0.0, 0.0]), np.array([True, False, False]))
    scn.boundary[(2, True)] = (np.array([0.0, 0.0, 2.0]), np.array([False, False, True]))
    scn.interior_voxels = np.asarray(out["interior_voxels"], np.int32).reshape(-1, 3)
    scn.interior_values = np.asarray(out["interior_values"]).reshape(-1, S)
    scn.interior_conditions = np.asarray(out["interior_conditions"]).reshape(-1, S) > 0
    f = lambda k: np.asarray(out[k], np.float32).reshape(A, S)  # noqa: E731
    scn.agents = Agents(secretion_rates=f("secretion_rates"), saturation_densities=f("saturation_densities"),
                        uptake_rates=f("uptake_rates"), net_export_rates=f("net_export_rates"),
                        internalized=np.zeros((A, S), np.float32), fraction_released=f("fraction_released"),
                        volumes=np.asarray(out["volumes"], np.float32),
                        positions=np.asarray(out["positions"], np.float32).reshape(A, 3))
    o = make_oracle(scn)
    for step in range(3):
        o.diffusion()
        o.gradient()
        o.secretion(step % 10 == 0)
    o.release(5)
    assert rel_err(np.asarray(out["densities"]), o.densities()) < 1e-6
    assert rel_err(np.asarray(out["gradients"]), o.gradients()) < 1e-6
    assert rel_err(np.asarray(out["internalized"]), o.internalized()) < 1e-6


@pytest.mark.gpu
def test_bulk_from_builder_callbacks(program):
    """The builder's three bulk callbacks, tabulated by bulk.initialize, two bulk.solve steps."""
    out = run(program, "bulk")
    f32 = np.float32
    X, Y, S = 7, 5, 3
    v = np.arange(X * Y)
    x, y = (v % X).astype(f32), (v // X).astype(f32)
    s = np.arange(S, dtype=f32)
    supply = f32(0.1) * (x[:, None] + f32(1)) + f32(0.01) * s[None, :]
    uptake = np.broadcast_to(f32(0.05) * (y[:, None] + f32(1)), (X * Y, S)).astype(f32)
    target = (f32(1) + x[:, None] + f32(2) * y[:, None] + s[None, :]).astype(f32)
    scn = Scenario(dims=2, bbox_min=(0, 0, 0), bbox_max=(140, 100, 0), voxel_shape=(20, 20, 20),
                   diffusion_coefficients=[10.0, 20.0, 30.0], decay_rates=[0.1, 0.2, 0.3], time_step=0.5,
                   initial_conditions=[2.0, 0.5, 0.0])
    o = make_oracle(scn)
    for _ in range(2):
        o.bulk(supply, uptake, target, True)
    np.testing.assert_array_equal(np.asarray(out["densities"], np.float32), o.densities())


@pytest.mark.gpu
def test_agents_added_and_removed_on_the_gpu_copy(program):
    """Agents released, removed and added between steps (src/agent_data.cpp:10-53) through
    cell.add_agents / cell.remove_agents, against the reference's round trip of every agent array
    (load_data_from_solver, the change on the host, store_data_to_solver): identical results."""
    dev = run(program, "lifecycle_device")
    host = run(program, "lifecycle_host")
    assert dev["agents"] == host["agents"] == 40 - 1 + 6 - 3
    for k in ("volumes", "densities", "gradients", "internalized"):
        np.testing.assert_array_equal(np.asarray(dev[k], np.float32), np.asarray(host[k], np.float32), err_msg=k)
