"""Microenvironment descriptions and seeded synthetic workloads.

``Workload`` holds everything needed to build a microenvironment (mesh, substrates, Dirichlet
conditions, agents, initial field) independently of the solver that runs it; ``synthetic`` draws
the seeded workloads used by the benchmark and the tests; ``make_solver`` builds one on the GPU.
"""

from __future__ import annotations

import copy
import dataclasses
from typing import Optional

import numpy as np

@dataclasses.dataclass
class Agents:
    secretion_rates: np.ndarray      # [A][S]
    saturation_densities: np.ndarray  # [A][S]
    uptake_rates: np.ndarray         # [A][S]
    net_export_rates: np.ndarray     # [A][S]
    internalized: np.ndarray         # [A][S]
    fraction_released: np.ndarray    # [A][S]
    volumes: np.ndarray              # [A]
    positions: np.ndarray            # [A][dims]

    @property
    def count(self):
        return int(self.volumes.shape[0])


@dataclasses.dataclass
class Workload:
    dims: int
    bbox_min: tuple
    bbox_max: tuple
    voxel_shape: tuple
    diffusion_coefficients: list
    decay_rates: list
    time_step: float
    initial_conditions: list
    compute_internalized: bool = False
    # (dim, is_max) -> (values[S], conditions[S])
    boundary: dict = dataclasses.field(default_factory=dict)
    interior_voxels: Optional[np.ndarray] = None   # [N][dims] int32
    interior_values: Optional[np.ndarray] = None   # [N][S]
    interior_conditions: Optional[np.ndarray] = None  # [N][S] bool
    agents: Optional[Agents] = None
    densities: Optional[np.ndarray] = None  # explicit initial field (flat, [z][y][x][s])

    @property
    def S(self):
        return len(self.diffusion_coefficients)

    @property
    def grid(self):
        g = [1, 1, 1]
        for d in range(self.dims):
            g[d] = (self.bbox_max[d] - self.bbox_min[d] + self.voxel_shape[d] - 1) // self.voxel_shape[d]
        return tuple(g)

    @property
    def voxel_count(self):
        g = self.grid
        return g[0] * g[1] * g[2]

    @property
    def voxel_volume(self):
        return self.voxel_shape[0] * self.voxel_shape[1] * self.voxel_shape[2]

    def copy(self):
        return copy.deepcopy(self)



# the tests call the same structure a scenario
Scenario = Workload


def make_solver(w: Workload, device: int = 0):
    """Create a GPU solver holding workload ``w`` (field, Dirichlet conditions, agents)."""
    from . import Solver

    s = Solver(w.dims, w.bbox_min, w.bbox_max, w.voxel_shape, w.diffusion_coefficients, w.decay_rates, w.time_step,
               compute_internalized=w.compute_internalized, device=device)
    for (dim, is_max), (vals, conds) in w.boundary.items():
        s.set_boundary_dirichlet(dim, is_max, vals, conds)
    if w.interior_voxels is not None:
        s.set_interior_dirichlet(w.interior_voxels, w.interior_values, w.interior_conditions)
    field = w.densities
    if field is None:
        field = np.tile(np.asarray(w.initial_conditions, np.float32), w.voxel_count)
    s.store_densities(field)
    if w.agents is not None:
        a = w.agents
        s.store_agents(a.secretion_rates, a.saturation_densities, a.uptake_rates, a.net_export_rates,
                       a.internalized, a.fraction_released, a.volumes, a.positions)
    return s


def synthetic(grid_edge, S, agents, seed, dx=20, dt=0.01, clustered=False, n_clusters=32, sigma=200.0,
              interior_fraction=0.0, boundary_substrate0=True, internalized=True, dims=3):
    """A seeded synthetic microenvironment.

    Diffusion coefficients log-uniform in [1e3, 1e5] um^2/min, decay rates uniform in [0.01, 1]
    /min, initial densities uniform [0, 1), Dirichlet value 1.0 for substrate 0 on every face,
    agents with volume 1000 um^3, secretion U(0,10), saturation U(0,1), uptake U(0,1), net export 0;
    uniform positions or ``n_clusters`` Gaussian clusters of width ``sigma`` (rejected into the box).
    A fraction of interior voxels can be marked Dirichlet with values U(0,1) on every substrate.
    """
    rng = np.random.default_rng(seed)
    L = grid_edge * dx
    bmax = (L, L if dims >= 2 else dx, L if dims >= 3 else dx)
    scn = Workload(dims=dims, bbox_min=(0, 0, 0), bbox_max=bmax, voxel_shape=(dx, dx, dx),
                   diffusion_coefficients=list(np.exp(rng.uniform(np.log(1e3), np.log(1e5), S))),
                   decay_rates=list(rng.uniform(0.01, 1.0, S)), time_step=dt,
                   initial_conditions=[0.0] * S, compute_internalized=internalized)
    scn.densities = rng.uniform(0.0, 1.0, scn.voxel_count * S).astype(np.float32)
    if boundary_substrate0:
        for d in range(dims):
            for is_max in (False, True):
                vals = np.zeros(S)
                conds = np.zeros(S, dtype=bool)
                vals[0] = 1.0
                conds[0] = True
                scn.boundary[(d, is_max)] = (vals, conds)
    if interior_fraction > 0:
        g = scn.grid
        inner = [max(g[d] - 2, 0) if d < dims else 1 for d in range(3)]
        n_inner = inner[0] * inner[1] * inner[2]
        n = int(round(interior_fraction * n_inner))
        pick = rng.choice(n_inner, size=n, replace=False)
        coords = []
        rem = pick
        for d in range(dims):
            coords.append(rem % inner[d] + 1)
            rem = rem // inner[d]
        scn.interior_voxels = np.stack(coords, axis=1).astype(np.int32)
        scn.interior_values = rng.uniform(0, 1, (n, S))
        scn.interior_conditions = np.ones((n, S), dtype=bool)
    if agents > 0:
        if clustered:
            centres = rng.uniform(0, L, (n_clusters, dims))
            pos = np.empty((0, dims))
            while pos.shape[0] < agents:
                c = centres[rng.integers(0, n_clusters, agents)]
                p = c + rng.normal(0.0, sigma, (agents, dims))
                p = p[((p >= 0) & (p < L)).all(axis=1)]
                pos = np.concatenate([pos, p])
            pos = pos[:agents]
        else:
            pos = rng.uniform(0, L, (agents, dims))
        # keep positions strictly inside the box in float32 (the voxel index truncates)
        pos = np.minimum(pos.astype(np.float32), np.nextafter(np.float32(L), np.float32(0)))
        scn.agents = Agents(secretion_rates=rng.uniform(0, 10, (agents, S)),
                            saturation_densities=rng.uniform(0, 1, (agents, S)),
                            uptake_rates=rng.uniform(0, 1, (agents, S)),
                            net_export_rates=np.zeros((agents, S)),
                            internalized=np.zeros((agents, S)),
                            fraction_released=rng.uniform(0, 1, (agents, S)),
                            volumes=np.full(agents, 1000.0),
                            positions=pos.astype(np.float64))
    return scn


