"""One mesh split along z into slabs, one solver per slab (bfvm_create_slab, bfvm_slab_*).

A mesh too large for one GPU, or one stepped faster by several, is cut into slabs of whole z
planes.  Each slab is a solver of its own (normally on its own GPU, one process per GPU):
- The x and y sweeps, the Dirichlet overwrites and secretion never cross a z plane, so every slab
  runs them alone.
- The z sweep and the z gradient cross slab edges.  A step therefore has two exchanges, which this
  module performs between the library's calls:
  - an all-gather of 2 floats per z line from every slab (the reduced system of the z sweep);
  - each slab's first and last plane to its neighbours (the gradient's halo).

``GroupExchange`` runs both over a torch.distributed process group: NCCL between GPUs, or gloo for
tests on the CPU.  ``LocalExchange`` joins slabs held by one process, for example several slabs
emulated on one GPU.  ``step`` is the driver's step (diffusion, gradient, secretion) over the slabs
of this process.
"""

from __future__ import annotations

import ctypes

import numpy as np

from . import _abi
from ._abi import check
from . import Solver, _f32, _fp


def plan_slabs(planes: int, count: int) -> list[int]:
    """Plane boundaries [count + 1] of an even split: the first planes % count slabs get one more."""
    if count < 1 or planes < 2 * count:
        raise ValueError(f"{planes} planes cannot be split into {count} slabs of at least 2 planes")
    base, extra = divmod(planes, count)
    bounds = [0]
    for k in range(count):
        bounds.append(bounds[-1] + base + (1 if k < extra else 0))
    return bounds


def slab_coefficients(planes, voxel_z, diffusion_coefficients, decay_rates, time_step, bounds):
    """The [count][3][S] coefficients (Gamma, beta, Lambda) that couple the slabs of a z line
    (bfvm_slab_coefficients; host only)."""
    lib = _abi.load()
    D = _f32(diffusion_coefficients)
    lam = _f32(decay_rates, D.size)
    b = np.ascontiguousarray(bounds, np.int32)
    count = b.size - 1
    out = np.empty((count, 3, D.size), np.float32)
    check(lib.bfvm_slab_coefficients(int(planes), int(voxel_z), D.size, float(time_step), _fp(D), _fp(lam), count,
                                     b.ctypes.data_as(ctypes.POINTER(ctypes.c_int32)), _fp(out)))
    return out


def slab_reduce_weights(planes, voxel_z, diffusion_coefficients, decay_rates, time_step, first_plane, end_plane):
    """The reduce pass's weights of the slab holding planes [first_plane, end_plane)
    (bfvm_slab_reduce_weights; host only): the first plane of A's sum, A's weights [planes][S] and
    B's weights [planes][S] (from the slab's first plane)."""
    lib = _abi.load()
    D = _f32(diffusion_coefficients)
    lam = _f32(decay_rates, D.size)
    w = np.zeros((2 * (end_plane - first_plane), D.size), np.float32)  # both sums may keep every plane
    af, na, nb = ctypes.c_int32(), ctypes.c_int32(), ctypes.c_int32()
    check(lib.bfvm_slab_reduce_weights(int(planes), int(voxel_z), D.size, float(time_step), _fp(D), _fp(lam),
                                       int(first_plane), int(end_plane), _fp(w), ctypes.byref(af), ctypes.byref(na),
                                       ctypes.byref(nb)))
    return int(af.value), w[:na.value].copy(), w[na.value:na.value + nb.value].copy()


def agent_slabs(positions, bbox_min_z, voxel_z, bounds):
    """The slab of each agent, from its z position, by the float arithmetic the slab's own voxel
    lookup uses ((pos - slab min) / dz, truncated); -1 where no slab takes the agent."""
    pz = np.asarray(positions, np.float32)[:, 2]
    out = np.full(pz.shape, -1, np.int64)
    for k in range(len(bounds) - 1):
        lo = np.float32(bbox_min_z + bounds[k] * voxel_z)
        t = (pz - lo) / np.float32(voxel_z)
        nz = bounds[k + 1] - bounds[k]
        # t in (-1, 0) truncates to plane 0 in the lookup, which belongs to slab 0 only
        ok = ((t > -1.0) if k == 0 else (t >= 0.0)) & (t < nz) & (out < 0)
        out[ok] = k
    return out


class Slab(Solver):
    """Slab `slab` of a mesh split at plane boundaries `bounds` (see plan_slabs), on `device`.

    Besides the Solver calls that stay within the slab (Dirichlet, agents, secretion, release),
    it owns the device buffers of the exchanges: `exchange` [2][lines] (this slab's part of the
    z sweep's reduced system) and `edges` [2][lines] (its first and last plane), lines = X*Y*S.
    Its work runs on the torch stream `stream` (a new one if None); `step` enqueues the exchanges
    there too, so the slabs that one process holds share one stream.
    Agents added or removed on a slab (add_agents, remove_agents) must lie in its planes; the
    slab's `agent_index` (set by make_slab) is the caller's to keep in step with such changes.
    """

    def __init__(self, bbox_min, bbox_max, voxel_shape, diffusion_coefficients, decay_rates, time_step, bounds, slab,
                 compute_internalized=False, device=0, stream=None):
        import torch

        self._lib = _abi.load()
        self.dims = 3
        self.S = len(diffusion_coefficients)
        self.bounds = [int(b) for b in bounds]
        self.count = len(self.bounds) - 1
        self.index = int(slab)
        self.mesh_bbox_min = tuple(int(t) for t in bbox_min)
        self.voxel_shape = tuple(int(t) for t in voxel_shape)
        i3 = lambda v: (ctypes.c_int32 * 3)(*[int(t) for t in v])  # noqa: E731
        D = _f32(diffusion_coefficients)
        lam = _f32(decay_rates, self.S)
        b = np.ascontiguousarray(self.bounds, np.int32)
        h = ctypes.c_void_p()
        check(self._lib.bfvm_create_slab(ctypes.byref(h), int(device), i3(bbox_min), i3(bbox_max), i3(voxel_shape),
                                         self.S, float(time_step), _fp(D), _fp(lam), int(bool(compute_internalized)),
                                         self.count, b.ctypes.data_as(ctypes.POINTER(ctypes.c_int32)), self.index))
        self._h = h
        g = (ctypes.c_int32 * 3)()
        V = ctypes.c_int64()
        check(self._lib.bfvm_get_shape(self._h, g, ctypes.byref(V), None, None))
        self.grid = tuple(int(t) for t in g)
        self.voxel_count = int(V.value)
        self.agents_count = 0
        self.first_plane = self.bounds[self.index]
        self.lines = self.grid[0] * self.grid[1] * self.S
        self.device = torch.device("cuda", int(device))
        self.stream = stream if stream is not None else torch.cuda.Stream(self.device)
        with torch.cuda.stream(self.stream):
            self.exchange = torch.empty(2 * self.lines, dtype=torch.float32, device=self.device)
            self.edges = torch.empty((2, self.lines), dtype=torch.float32, device=self.device)
        self.set_stream(self.stream.cuda_stream)

    # -- the whole mesh's description, restricted to this slab ------------------------------------------
    def set_mesh_boundary_dirichlet(self, dim, is_max, values, conditions):
        """A face condition of the whole mesh: x and y faces on every slab, the z-min face on slab 0
        only, the z-max face on the last slab only."""
        if dim == 2 and ((is_max and self.index != self.count - 1) or (not is_max and self.index != 0)):
            return
        self.set_boundary_dirichlet(dim, is_max, values, conditions)

    def set_mesh_interior_dirichlet(self, voxels, values, conditions):
        """Interior conditions of the whole mesh: those whose voxel lies in this slab, moved to its
        planes."""
        vox = np.asarray(voxels, np.int32).reshape(-1, 3)
        z = vox[:, 2]
        mine = (z >= self.first_plane) & (z < self.first_plane + self.grid[2])
        local = vox[mine].copy()
        local[:, 2] -= self.first_plane
        self.set_interior_dirichlet(local, np.asarray(values, np.float32).reshape(len(vox), self.S)[mine],
                                    np.asarray(conditions, np.uint8).reshape(len(vox), self.S)[mine])

    def select_agents(self, positions):
        """Indices of the mesh's agents (by position) whose voxel this slab holds."""
        slab = agent_slabs(positions, self.mesh_bbox_min[2], self.voxel_shape[2], self.bounds)
        return np.nonzero(slab == self.index)[0]

    def store_mesh_densities(self, densities):
        """This slab's planes of a whole-mesh field [Z][Y][X][S]."""
        plane = self.lines
        d = np.asarray(densities, np.float32).reshape(-1)
        self.store_densities(d[self.first_plane * plane:(self.first_plane + self.grid[2]) * plane])

    # -- the step, between exchanges -----------------------------------------------------------------
    def diffusion_begin(self):
        check(self._lib.bfvm_slab_diffusion_begin(self._h, ctypes.c_void_p(self.exchange.data_ptr())))

    def diffusion_end(self, gathered):
        if gathered.numel() != self.count * 2 * self.lines:
            raise ValueError("the gathered exchange must hold [slab_count][2][X*Y*S] floats")
        check(self._lib.bfvm_slab_diffusion_end(self._h, ctypes.c_void_p(gathered.data_ptr())))

    def edge_planes(self):
        check(self._lib.bfvm_slab_edge_planes(self._h, ctypes.c_void_p(self.edges[0].data_ptr()),
                                              ctypes.c_void_p(self.edges[1].data_ptr())))

    def gradient_with(self, below, above):
        ptr = lambda t: None if t is None else ctypes.c_void_p(t.data_ptr())  # noqa: E731
        check(self._lib.bfvm_slab_gradient_solve(self._h, ptr(below), ptr(above)))


class LocalExchange:
    """The exchanges between the slabs of a mesh when one process holds all of them (several slabs
    emulated on one GPU, or a single slab)."""

    def gather(self, slabs):
        import torch

        return torch.cat([s.exchange for s in slabs])

    def halos(self, slabs):
        out = []
        for k, _ in enumerate(slabs):
            below = slabs[k - 1].edges[1] if k > 0 else None
            above = slabs[k + 1].edges[0] if k + 1 < len(slabs) else None
            out.append((below, above))
        return out


class GroupExchange:
    """The exchanges between ranks of a torch.distributed group, one slab per rank, rank = slab
    index.  With NCCL the buffers are device tensors; gloo takes CPU tensors (tests)."""

    def __init__(self, group=None):
        import torch.distributed as dist

        self.dist = dist
        self.group = group
        self.rank = dist.get_rank(group)
        self.world = dist.get_world_size(group)
        self._gathered = None
        self._halo = None

    def gather(self, slabs):
        import torch

        (s,) = slabs
        if s.index != self.rank or s.count != self.world:
            raise ValueError("GroupExchange holds slab `rank` of `world size` slabs on each rank")
        n = s.exchange.numel()
        if self._gathered is None or self._gathered.numel() != self.world * n:
            self._gathered = torch.empty(self.world * n, dtype=s.exchange.dtype, device=s.exchange.device)
        if self.dist.get_backend(self.group) == "nccl":
            self.dist.all_gather_into_tensor(self._gathered, s.exchange, group=self.group)
        else:
            parts = list(self._gathered.view(self.world, n).unbind(0))
            self.dist.all_gather(parts, s.exchange, group=self.group)
        return self._gathered

    def halos(self, slabs):
        import torch

        (s,) = slabs
        if self._halo is None or self._halo.shape != s.edges.shape:
            self._halo = torch.empty_like(s.edges)
        below = self._halo[0] if self.rank > 0 else None
        above = self._halo[1] if self.rank + 1 < self.world else None
        ops = []
        if below is not None:
            ops.append(self.dist.P2POp(self.dist.irecv, below, self._peer(self.rank - 1), self.group))
            ops.append(self.dist.P2POp(self.dist.isend, s.edges[0], self._peer(self.rank - 1), self.group))
        if above is not None:
            ops.append(self.dist.P2POp(self.dist.irecv, above, self._peer(self.rank + 1), self.group))
            ops.append(self.dist.P2POp(self.dist.isend, s.edges[1], self._peer(self.rank + 1), self.group))
        if ops:
            for req in self.dist.batch_isend_irecv(ops):
                req.wait()
        return [(below, above)]

    def _peer(self, rank):
        return rank if self.group is None else self.dist.get_global_rank(self.group, rank)


def step(slabs, exchange, recompute):
    """One step of the reference driver (src/main.cpp:76-96) on a split mesh: diffusion with the
    z sweep's exchange, the gradient with the halo exchange, then secretion.  `slabs` are the slabs
    this process holds, in slab order, all on one stream."""
    import contextlib

    streams = {id(getattr(s, "stream", None)) for s in slabs}
    if len(streams) != 1:
        raise ValueError("the slabs that one process holds must share one stream")
    stream = getattr(slabs[0], "stream", None)
    if stream is None:
        ctx = contextlib.nullcontext()  # slabs without a device (tests of the exchange on the CPU)
    else:
        import torch

        ctx = torch.cuda.stream(stream)
    with ctx:
        _step(slabs, exchange, recompute)


def _step(slabs, exchange, recompute):
    for s in slabs:
        s.diffusion_begin()
    gathered = exchange.gather(slabs)
    for s in slabs:
        s.diffusion_end(gathered)
    for s in slabs:
        s.edge_planes()
    for s, (below, above) in zip(slabs, exchange.halos(slabs)):
        s.gradient_with(below, above)
    for s in slabs:
        s.secretion(recompute)


def run_steps(slabs, exchange, steps, first_step=0):
    """`steps` steps, recompute on every 10th as bfvm_run_steps does."""
    for i in range(steps):
        step(slabs, exchange, (first_step + i) % 10 == 0)


def make_slab(w, bounds, index, device=0, stream=None):
    """Slab `index` of workload `w` (a parabiofvm_b200.workloads.Workload, dims 3) split at
    `bounds`: its Dirichlet conditions, its planes of the initial field, and the agents whose voxel
    it holds (their indices in the workload are `agent_index`)."""
    s = Slab(w.bbox_min, w.bbox_max, w.voxel_shape, w.diffusion_coefficients, w.decay_rates, w.time_step, bounds,
             index, compute_internalized=w.compute_internalized, device=device, stream=stream)
    for (dim, is_max), (vals, conds) in w.boundary.items():
        s.set_mesh_boundary_dirichlet(dim, is_max, vals, conds)
    if w.interior_voxels is not None:
        s.set_mesh_interior_dirichlet(w.interior_voxels, w.interior_values, w.interior_conditions)
    field = w.densities
    if field is None:
        field = np.tile(np.asarray(w.initial_conditions, np.float32), w.voxel_count)
    s.store_mesh_densities(field)
    s.agent_index = np.zeros(0, np.int64)
    if w.agents is not None:
        a = w.agents
        idx = s.select_agents(a.positions)
        s.agent_index = idx
        pick = lambda v: None if v is None else np.asarray(v)[idx]  # noqa: E731
        s.store_agents(pick(a.secretion_rates), pick(a.saturation_densities), pick(a.uptake_rates),
                       pick(a.net_export_rates), pick(a.internalized), pick(a.fraction_released), pick(a.volumes),
                       pick(a.positions))
    return s
