"""Test scenarios shared by the oracle tests and the GPU parity tests.

``Scenario`` describes one microenvironment (mesh, substrates, Dirichlet conditions, agents,
initial field) independently of the solver that runs it; ``make_oracle`` and ``make_gpu`` build it
on the CPU oracle or on the CUDA library.

The fixtures restate the reference's test fixtures (paths relative to the paraBioFVM root):
``default_microenv`` (test/utils.cpp:10-31), ``biorobots_microenv`` (:33-54),
``interactions_microenv`` (:56-86), ``add_dirichlet_at`` (:88-109), ``add_boundary_dirichlet``
(:111-132), ``set_default_agent_values`` (:204-222).  ``float_eq`` is GoogleTest's
``EXPECT_FLOAT_EQ`` (equal within 4 units in the last place of a float).
"""

from __future__ import annotations

import json
import os

import numpy as np

from parabiofvm_b200.workloads import Agents, Scenario, Workload, synthetic  # noqa: F401

_GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "reference_goldens.json")
_golden_cache = None


def golden(line: int) -> float:
    """Golden value written in the reference's test/test.cpp at ``line``."""
    global _golden_cache
    if _golden_cache is None:
        with open(_GOLDEN) as f:
            _golden_cache = json.load(f)
    return _golden_cache["scalars"]["test/test.cpp"][str(line)]["value"]


def golden_vector(test: str):
    global _golden_cache
    if _golden_cache is None:
        golden(59)
    return _golden_cache["vectors"][test]["values"]


def _ulp_key(x: np.ndarray) -> np.ndarray:
    """Map float32 bit patterns onto a monotonic integer line (GoogleTest's biased form)."""
    i = np.asarray(x, dtype=np.float32).view(np.int32).astype(np.int64)
    return np.where(i < 0, -(i & 0x7FFFFFFF), i)


def ulp_distance(a, b) -> np.ndarray:
    return np.abs(_ulp_key(np.asarray(a, np.float32)) - _ulp_key(np.asarray(b, np.float32)))


def float_eq(a, b, max_ulps: int = 4) -> bool:
    """GoogleTest EXPECT_FLOAT_EQ: both sides as float, at most 4 ULPs apart (NaN never equal)."""
    a = np.asarray(a, np.float32)
    b = np.asarray(b, np.float32)
    if np.isnan(a).any() or np.isnan(b).any():
        return False
    return bool((ulp_distance(a, b) <= max_ulps).all())


def assert_float_eq(actual, expected, what: str = "", max_ulps: int = 4):
    actual = np.asarray(actual, np.float32)
    expected = np.broadcast_to(np.asarray(expected, np.float32), actual.shape)
    d = ulp_distance(actual, expected)
    if np.isnan(actual).any() or (d > max_ulps).any():
        i = int(np.argmax(d))
        raise AssertionError(f"{what}: {actual.reshape(-1)[i]!r} != {expected.reshape(-1)[i]!r} "
                             f"({int(d.reshape(-1)[i])} ulps at flat index {i})")


def mesh(dims, bbox_max, voxel_shape, bbox_min=(0, 0, 0)):
    return dict(dims=dims, bbox_min=tuple(bbox_min), bbox_max=tuple(bbox_max), voxel_shape=tuple(voxel_shape))


def default_microenv(m) -> Scenario:
    """test/utils.cpp:10-31: 2 substrates, dt=5, D={4,2}, decay={5,3}, initial 1."""
    return Scenario(**m, diffusion_coefficients=[4.0, 2.0], decay_rates=[5.0, 3.0], time_step=5.0,
                    initial_conditions=[1.0, 1.0])


def biorobots_microenv(m) -> Scenario:
    """test/utils.cpp:33-54: 2 substrates, dt=0.01, D=1000, decay={0.1,0.4}, initial 0."""
    return Scenario(**m, diffusion_coefficients=[1000.0, 1000.0], decay_rates=[0.1, 0.4], time_step=0.01,
                    initial_conditions=[0.0, 0.0])


def interactions_microenv(m) -> Scenario:
    """test/utils.cpp:56-86: 5 substrates."""
    return Scenario(**m, diffusion_coefficients=[100000.0, 100.0, 1000.0, 1000.0, 1000.0],
                    decay_rates=[0.1, 0.1, 0.1, 0.01, 0.1], time_step=0.01,
                    initial_conditions=[1.0, 0.0, 0.0, 0.0, 0.0])


def add_dirichlet_at(scn: Scenario, indices, values):
    """test/utils.cpp:88-109: interior Dirichlet on substrate 0 only."""
    n = len(indices)
    vox = np.array([list(ix)[: scn.dims] for ix in indices], dtype=np.int32).reshape(n, scn.dims)
    vals = np.zeros((n, scn.S), dtype=np.float64)
    conds = np.zeros((n, scn.S), dtype=bool)
    vals[:, 0] = values
    conds[:, 0] = True
    scn.interior_voxels, scn.interior_values, scn.interior_conditions = vox, vals, conds


def add_boundary_dirichlet(scn: Scenario, dim_idx: int, is_min: bool, value: float):
    """test/utils.cpp:111-132: substrate 0 gets ``value``; the others 42 with the condition off."""
    key = (dim_idx, not is_min)
    if key not in scn.boundary:
        scn.boundary[key] = (np.full(scn.S, 42.0), np.zeros(scn.S, dtype=bool))
    vals, conds = scn.boundary[key]
    vals[0] = value
    conds[0] = True


def set_default_agent_values(rows: list, rates_offset, volume, position, dims):
    """test/utils.cpp:204-222 for a 2-substrate scenario; appends one agent row."""
    rows.append(dict(sec=[rates_offset + 100, 0], upt=[rates_offset + 200, 0], sat=[rates_offset + 300, 0],
                     nex=[rates_offset + 400, 0], vol=volume, pos=list(position)[:dims]))


def agents_from_rows(rows, S, dims) -> Agents:
    A = len(rows)
    f = lambda key: np.array([r[key] for r in rows], dtype=np.float64).reshape(A, S)  # noqa: E731
    return Agents(secretion_rates=f("sec"), saturation_densities=f("sat"), uptake_rates=f("upt"),
                  net_export_rates=f("nex"), internalized=np.zeros((A, S)), fraction_released=np.zeros((A, S)),
                  volumes=np.array([r["vol"] for r in rows], dtype=np.float64),
                  positions=np.array([r["pos"] for r in rows], dtype=np.float64).reshape(A, dims))


def make_oracle(scn: Scenario, dtype=np.float32):
    from oracle import Oracle

    o = Oracle(scn.dims, scn.bbox_min, scn.bbox_max, scn.voxel_shape, scn.diffusion_coefficients,
               scn.decay_rates, scn.time_step, scn.initial_conditions, scn.compute_internalized, dtype=dtype)
    for (dim, is_max), (vals, conds) in scn.boundary.items():
        o.set_boundary_dirichlet(dim, is_max, vals, conds)
    if scn.interior_voxels is not None:
        o.set_interior_dirichlet(scn.interior_voxels, scn.interior_values, scn.interior_conditions)
    if scn.densities is not None:
        o.set_densities(scn.densities)
    if scn.agents is not None:
        a = scn.agents
        o.set_agents(a.secretion_rates, a.saturation_densities, a.uptake_rates, a.net_export_rates,
                     a.internalized, a.fraction_released, a.volumes, a.positions)
    o.initialize()
    return o


def make_gpu(scn: Scenario, device: int = 0):
    from parabiofvm_b200.workloads import make_solver

    return make_solver(scn, device)


def index_field(scn: Scenario) -> np.ndarray:
    """Densities equal to their flat index (test/test.cpp:125-131, 162-169, 203-212)."""
    return np.arange(scn.voxel_count * scn.S, dtype=np.float64)


def rel_err(actual, ref, floor_frac=1e-6):
    """Max relative error with a floor: |a-r| / max(|r|, floor_frac * max|r|)."""
    a = np.asarray(actual, np.float64).reshape(-1)
    r = np.asarray(ref, np.float64).reshape(-1)
    floor = max(float(np.abs(r).max()) * floor_frac, 1e-30)
    return float((np.abs(a - r) / np.maximum(np.abs(r), floor)).max())


def rel_l2(actual, ref):
    a = np.asarray(actual, np.float64).reshape(-1)
    r = np.asarray(ref, np.float64).reshape(-1)
    return float(np.linalg.norm(a - r) / max(np.linalg.norm(r), 1e-300))
