"""B200-native microenvironment step for paraBioFVM models.

``Solver`` is a thin Python face of the C ABI (include/bfvm.h): one microenvironment on one GPU
with the reference solver's operations -- diffusion (LOD Thomas sweeps with the Dirichlet
overwrites), Dirichlet, gradient, secretion/uptake, release of internalized substrates -- plus a
graph-captured multi-step driver.  Arrays use the reference's layouts (src/traits.h): densities
[z][y][x][s]; gradients [x][s][1], [y][x][s][2] or [3][z][y][x][s]; agents [agent][substrate].
"""

from __future__ import annotations

import ctypes

import numpy as np

from . import _abi
from ._abi import BfvmError, check

__all__ = ["Solver", "Batch", "BfvmError", "library_path"]


def library_path() -> str:
    return _abi.LIB_PATH


def _f32(a, n=None):
    arr = np.ascontiguousarray(a, dtype=np.float32).reshape(-1)
    if n is not None and arr.size != n:
        raise ValueError(f"expected {n} values, got {arr.size}")
    return arr


def _fp(a):
    return a.ctypes.data_as(ctypes.POINTER(ctypes.c_float))


def plan_agent_removal(agents, indices):
    """Host part of Solver.remove_agents (bfvm_plan_agent_removal, no device): the agents left
    after agent_data::remove of indices[0], indices[1], ... and the moves (dst, src) of agent rows
    that leave the stored order the reference leaves."""
    idx = np.ascontiguousarray(indices, dtype=np.int32).reshape(-1)
    P32 = ctypes.POINTER(ctypes.c_int32)
    dst = np.zeros(max(idx.size, 1), np.int32)
    src = np.zeros(max(idx.size, 1), np.int32)
    remaining = ctypes.c_int32()
    moves = ctypes.c_int32()
    check(_abi.load().bfvm_plan_agent_removal(int(agents), idx.size, idx.ctypes.data_as(P32), ctypes.byref(remaining),
                                              ctypes.byref(moves), dst.ctypes.data_as(P32), src.ctypes.data_as(P32)))
    return int(remaining.value), dst[:moves.value].copy(), src[:moves.value].copy()


class Solver:
    """A microenvironment resident on one GPU (bfvm_create ... bfvm_destroy)."""

    def __init__(self, dims, bbox_min, bbox_max, voxel_shape, diffusion_coefficients, decay_rates, time_step,
                 compute_internalized=False, device=0):
        self._lib = _abi.load()
        self.dims = int(dims)
        self.S = len(diffusion_coefficients)
        i3 = lambda v: (ctypes.c_int32 * 3)(*[int(t) for t in list(v) + [0] * (3 - len(v))])  # noqa: E731
        D = _f32(diffusion_coefficients)
        lam = _f32(decay_rates, self.S)
        h = ctypes.c_void_p()
        check(self._lib.bfvm_create(ctypes.byref(h), int(device), self.dims, i3(bbox_min), i3(bbox_max),
                                    i3(voxel_shape), self.S, float(time_step), _fp(D), _fp(lam),
                                    int(bool(compute_internalized))))
        self._h = h
        g = (ctypes.c_int32 * 3)()
        V = ctypes.c_int64()
        check(self._lib.bfvm_get_shape(self._h, g, ctypes.byref(V), None, None))
        self.grid = tuple(int(t) for t in g)
        self.voxel_count = int(V.value)
        self.agents_count = 0

    # -- lifecycle ------------------------------------------------------------------------------
    def close(self):
        if getattr(self, "_h", None):
            self._lib.bfvm_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    # -- Dirichlet ------------------------------------------------------------------------------
    def set_boundary_dirichlet(self, dim, is_max, values, conditions):
        if values is None:
            check(self._lib.bfvm_set_boundary_dirichlet(self._h, int(dim), int(bool(is_max)), None, None))
            return
        v = _f32(values, self.S)
        c = np.ascontiguousarray(conditions, dtype=np.uint8).reshape(-1)
        check(self._lib.bfvm_set_boundary_dirichlet(self._h, int(dim), int(bool(is_max)), _fp(v),
                                                    c.ctypes.data_as(ctypes.POINTER(ctypes.c_uint8))))

    def set_interior_dirichlet(self, voxels, values, conditions):
        vox = np.ascontiguousarray(voxels, dtype=np.int32).reshape(-1)
        n = vox.size // self.dims
        v = _f32(values, n * self.S)
        c = np.ascontiguousarray(conditions, dtype=np.uint8).reshape(-1)
        if c.size != n * self.S:
            raise ValueError("conditions must have count * substrates entries")
        check(self._lib.bfvm_set_interior_dirichlet(self._h, n, vox.ctypes.data_as(ctypes.POINTER(ctypes.c_int32)),
                                                    _fp(v), c.ctypes.data_as(ctypes.POINTER(ctypes.c_uint8))))

    # -- data movement ----------------------------------------------------------------------------
    def store_densities(self, densities):
        self._dens_keep = _f32(densities, self.voxel_count * self.S)
        check(self._lib.bfvm_store_densities(self._h, _fp(self._dens_keep)))

    def load_densities(self, out=None):
        out = np.empty(self.voxel_count * self.S, np.float32) if out is None else out
        check(self._lib.bfvm_load_densities(self._h, _fp(out)))
        return out

    def store_densities_device(self, tensor):
        """The field from a device tensor (float32, voxels x substrates) on the solver's stream."""
        if tensor.numel() != self.voxel_count * self.S or not tensor.is_contiguous():
            raise ValueError("expected a contiguous device tensor of voxels x substrates floats")
        check(self._lib.bfvm_store_densities_device(self._h, ctypes.c_void_p(tensor.data_ptr())))

    def load_densities_device(self, tensor):
        if tensor.numel() != self.voxel_count * self.S or not tensor.is_contiguous():
            raise ValueError("expected a contiguous device tensor of voxels x substrates floats")
        check(self._lib.bfvm_load_densities_device(self._h, ctypes.c_void_p(tensor.data_ptr())))

    def load_gradients(self, out=None):
        out = np.empty(self.voxel_count * self.S * self.dims, np.float32) if out is None else out
        check(self._lib.bfvm_load_gradients(self._h, _fp(out)))
        return out

    def store_agents(self, secretion_rates, saturation_densities, uptake_rates, net_export_rates, internalized,
                     fraction_released, volumes, positions):
        vol = _f32(volumes)
        n = vol.size
        arrs = [_f32(a, n * self.S) for a in (secretion_rates, saturation_densities, uptake_rates, net_export_rates,
                                                internalized)]
        frac = None if fraction_released is None else _f32(fraction_released, n * self.S)
        pos = _f32(positions, n * self.dims)
        self._agents_keep = arrs + [frac, vol, pos]
        check(self._lib.bfvm_store_agents(self._h, n, *[_fp(a) for a in arrs], _fp(frac) if frac is not None else None,
                                          _fp(vol), _fp(pos)))
        self.agents_count = n

    def store_agent_positions(self, positions):
        """Positions alone of the stored agents (the per-step input of moving agents); they enter
        the voxel binning at the next recompute."""
        pos = _f32(positions, self.agents_count * self.dims)
        self._positions_keep = pos
        check(self._lib.bfvm_store_agent_positions(self._h, self.agents_count, _fp(pos)))

    def store_agent_positions_async(self, positions):
        """Positions through the solver's copy stream, overlapping the work queued after this call;
        `positions` must be a float32 array that stays valid (pinned for overlap) until synchronize."""
        pos = np.asarray(positions)
        if pos.dtype != np.float32 or not pos.flags.c_contiguous or pos.size != self.agents_count * self.dims:
            raise ValueError("expected a contiguous float32 array of agents x dims")
        check(self._lib.bfvm_store_agent_positions_async(self._h, self.agents_count, _fp(pos)))

    def load_internalized_async(self, out):
        """Internalized substrates into `out` (float32, agents x substrates, pinned for overlap)
        through the copy stream; complete after synchronize."""
        if out.dtype != np.float32 or not out.flags.c_contiguous or out.size != self.agents_count * self.S:
            raise ValueError("expected a contiguous float32 array of agents x substrates")
        check(self._lib.bfvm_load_internalized_async(self._h, _fp(out)))

    def load_internalized(self, out=None):
        out = np.empty(self.agents_count * self.S, np.float32) if out is None else out
        check(self._lib.bfvm_load_internalized(self._h, _fp(out)))
        return out

    # -- solvers --------------------------------------------------------------------------------
    def diffusion(self):
        check(self._lib.bfvm_diffusion_solve(self._h))

    def sweep(self, axis):
        check(self._lib.bfvm_diffusion_sweep(self._h, int(axis)))

    def dirichlet(self):
        check(self._lib.bfvm_dirichlet_solve(self._h))

    def gradient(self):
        check(self._lib.bfvm_gradient_solve(self._h))

    def diffusion_gradient(self):
        """diffusion() then gradient(), the gradient computed inside the z sweep where it can be."""
        check(self._lib.bfvm_diffusion_gradient_solve(self._h))

    def secretion(self, recompute):
        check(self._lib.bfvm_secretion_solve(self._h, int(bool(recompute))))

    def set_bulk_rates(self, supply_rates, uptake_rates, supply_target_densities, per_voxel):
        """Tabulated bulk supply/uptake rates: [voxel][s] when per_voxel, else one [s] row."""
        if supply_rates is None:
            check(self._lib.bfvm_set_bulk_rates(self._h, 0, None, None, None))
            return
        n = self.voxel_count * self.S if per_voxel else self.S
        arrs = [_f32(a, n) for a in (supply_rates, uptake_rates, supply_target_densities)]
        check(self._lib.bfvm_set_bulk_rates(self._h, int(bool(per_voxel)), *[_fp(a) for a in arrs]))

    def bulk(self):
        check(self._lib.bfvm_bulk_solve(self._h))

    def release(self, index):
        check(self._lib.bfvm_release_internalized(self._h, int(index)))

    def add_agents(self, count, secretion_rates=None, saturation_densities=None, uptake_rates=None,
                   net_export_rates=None, internalized=None, fraction_released=None, volumes=None, positions=None):
        """Append `count` agents on the GPU (agent_data::add per agent), with these rows for them;
        an array left None stays 0.  The stored agents do not pass through the host."""
        count = int(count)
        rows = [self.S] * 6 + [1, self.dims]
        arrs = [None if a is None else _f32(a, count * r)
                for a, r in zip((secretion_rates, saturation_densities, uptake_rates, net_export_rates, internalized,
                                 fraction_released, volumes, positions), rows)]
        self._added_keep = arrs
        check(self._lib.bfvm_add_agents(self._h, count, *[None if a is None else _fp(a) for a in arrs]))
        self.agents_count += count

    def remove_agents(self, indices):
        """agent_data::remove of indices[0], indices[1], ... in order, on the GPU: each moves the
        then-last agent into the freed slot."""
        idx = np.ascontiguousarray(indices, dtype=np.int32).reshape(-1)
        check(self._lib.bfvm_remove_agents(self._h, idx.size, idx.ctypes.data_as(ctypes.POINTER(ctypes.c_int32))))
        self.agents_count -= idx.size

    def run_steps(self, steps, first_step=0):
        check(self._lib.bfvm_run_steps(self._h, int(steps), int(first_step)))

    def synchronize(self):
        check(self._lib.bfvm_synchronize(self._h))

    def autotune(self):
        """Measure the staged sweeps' launch shapes and keep the fastest; returns [(groups, stages)]
        per axis ((0, 0) where the staged path does not apply)."""
        out = (ctypes.c_int32 * 6)()
        check(self._lib.bfvm_autotune(self._h, out))
        return [(out[2 * d], out[2 * d + 1]) for d in range(self.dims)]

    def set_option(self, name, value):
        check(self._lib.bfvm_set_option(self._h, name.encode(), int(value)))

    # -- device access ------------------------------------------------------------------------------
    def set_stream(self, stream_ptr):
        check(self._lib.bfvm_set_stream(self._h, ctypes.c_void_p(int(stream_ptr)) if stream_ptr else None))

    def device_densities(self):
        p = ctypes.POINTER(ctypes.c_float)()
        n = ctypes.c_int64()
        check(self._lib.bfvm_device_densities(self._h, ctypes.byref(p), ctypes.byref(n)))
        return ctypes.cast(p, ctypes.c_void_p).value, int(n.value)

    def device_gradients(self):
        p = ctypes.POINTER(ctypes.c_float)()
        n = ctypes.c_int64()
        check(self._lib.bfvm_device_gradients(self._h, ctypes.byref(p), ctypes.byref(n)))
        return ctypes.cast(p, ctypes.c_void_p).value, int(n.value)

    @property
    def launch_count(self):
        n = ctypes.c_int64()
        check(self._lib.bfvm_launch_count(self._h, ctypes.byref(n)))
        return int(n.value)


class Batch:
    """Independent solvers of one device stepped together (bfvm_batch_*): each instance runs
    exactly its own bfvm_run_steps, as branches of one CUDA graph."""

    def __init__(self, solvers):
        self._lib = _abi.load()
        self.solvers = list(solvers)
        arr = (ctypes.c_void_p * len(self.solvers))(*[s._h.value for s in self.solvers])
        h = ctypes.c_void_p()
        check(self._lib.bfvm_batch_create(ctypes.byref(h), len(self.solvers), arr))
        self._h = h

    def run_steps(self, steps, first_step=0):
        check(self._lib.bfvm_batch_run_steps(self._h, int(steps), int(first_step)))

    def synchronize(self):
        check(self._lib.bfvm_batch_synchronize(self._h))

    def autotune(self):
        """Time the ensemble kernels' launch choices (bfvm_batch_autotune) and keep the fastest;
        returns them."""
        c = (ctypes.c_int32 * 8)()
        check(self._lib.bfvm_batch_autotune(self._h, c))
        return {"sweep_ctas_per_sm": list(c[0:3]), "sweep_ctas_per_slot": list(c[3:6]), "gradient_planes": c[6],
                "gradient_load_batch": c[7]}

    def close(self):
        if getattr(self, "_h", None) is not None and self._h.value:
            self._lib.bfvm_batch_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
