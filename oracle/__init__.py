"""CPU oracle for the microenvironment step -- test infrastructure only.

A ctypes binding to ``oracle/build/liboracle.so``, the C++ restatement of the reference's host
solvers (``src/solver/host/{diffusion,dirichlet,gradient,cell}_solver.cpp``; see the header of
``bfvm_oracle.cpp`` for the line-by-line map).  Only the tests, ``__graft_entry__.smoke()`` and the
CPU-baseline leg of ``bench.py`` use it, always as the checker or the CPU baseline; the product
library never imports it.

``Oracle(dtype=np.float32)`` follows the reference's FP32 build; ``np.float64`` follows its
``-DDOUBLE_PRECISION`` build (``USE_DOUBLES``, include/BioFVM/types.h:13-17).
"""

from __future__ import annotations

import ctypes
import os
import subprocess

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB_PATH = os.path.join(_HERE, "build", "liboracle.so")
_lib = None


def build() -> str:
    """Compile the oracle with its Makefile (seconds); returns the library path."""
    subprocess.run(["make", "-s", "-C", _HERE], check=True)
    return _LIB_PATH


def _load():
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(_LIB_PATH):
        build()
    lib = ctypes.CDLL(_LIB_PATH)
    vp = ctypes.c_void_p
    ip = ctypes.POINTER(ctypes.c_int)
    u8p = ctypes.POINTER(ctypes.c_uint8)
    for suf, ct in (("f32", ctypes.c_float), ("f64", ctypes.c_double)):
        tp = ctypes.POINTER(ct)
        sig = {
            "create": (vp, [ctypes.c_int, ip, ip, ip, ctypes.c_int, ct, tp, tp, tp, ctypes.c_int]),
            "destroy": (None, [vp]),
            "grid_shape": (None, [vp, ip]),
            "set_boundary_dirichlet": (None, [vp, ctypes.c_int, ctypes.c_int, tp, u8p]),
            "set_interior_dirichlet": (None, [vp, ctypes.c_int, ip, tp, u8p]),
            "initialize": (None, [vp]),
            "set_densities": (None, [vp, tp]),
            "get_densities": (None, [vp, tp]),
            "get_gradients": (None, [vp, tp]),
            "set_agents": (None, [vp, ctypes.c_int, tp, tp, tp, tp, tp, tp, tp, tp]),
            "add_agents": (None, [vp, ctypes.c_int, tp, tp, tp, tp, tp, tp, tp, tp]),
            "remove_agent": (None, [vp, ctypes.c_int]),
            "get_internalized": (None, [vp, tp]),
            "diffusion": (None, [vp]),
            "dirichlet": (None, [vp]),
            "gradient": (None, [vp]),
            "secretion": (None, [vp, ctypes.c_int]),
            "release": (None, [vp, ctypes.c_int]),
            "run_steps": (None, [vp, ctypes.c_int, ctypes.c_int]),
            "is_conflict": (ctypes.c_int, [vp]),
            "bulk": (None, [vp, tp, tp, tp, ctypes.c_int]),
        }
        for name, (res, args) in sig.items():
            fn = getattr(lib, f"oracle_{suf}_{name}")
            fn.restype = res
            fn.argtypes = args
    lib.oracle_set_threads.argtypes = [ctypes.c_int]
    lib.oracle_set_threads.restype = None
    lib.oracle_max_threads.restype = ctypes.c_int
    _lib = lib
    return lib


def set_threads(n: int) -> None:
    _load().oracle_set_threads(int(n))


def max_threads() -> int:
    return int(_load().oracle_max_threads())


def _ptr(a: np.ndarray, ct):
    return a.ctypes.data_as(ctypes.POINTER(ct))


class Oracle:
    """One microenvironment plus its host solvers, in the reference's memory layouts.

    Densities are ``[z][y][x][s]`` (src/traits.h:76-83).  Gradients are ``[x][s][1]`` in 1D,
    ``[y][x][s][2]`` in 2D and ``[3][z][y][x][s]`` in 3D (src/traits.h:22-28, 50-56, 85-92).
    """

    def __init__(self, dims, bbox_min, bbox_max, voxel_shape, diffusion_coefficients, decay_rates,
                 time_step, initial_conditions=None, compute_internalized=False, dtype=np.float32):
        self.dtype = np.dtype(dtype)
        self._ct = ctypes.c_float if self.dtype == np.float32 else ctypes.c_double
        self._suf = "f32" if self.dtype == np.float32 else "f64"
        self._lib = _load()
        self.dims = int(dims)
        self.S = len(diffusion_coefficients)
        if initial_conditions is None:
            initial_conditions = [0.0] * self.S
        i3 = lambda v: (ctypes.c_int * 3)(*[int(t) for t in v])  # noqa: E731
        D = np.ascontiguousarray(diffusion_coefficients, dtype=self.dtype)
        lam = np.ascontiguousarray(decay_rates, dtype=self.dtype)
        ic = np.ascontiguousarray(initial_conditions, dtype=self.dtype)
        self._h = self._fn("create")(self.dims, i3(bbox_min), i3(bbox_max), i3(voxel_shape), self.S,
                                     self._ct(time_step), _ptr(D, self._ct), _ptr(lam, self._ct),
                                     _ptr(ic, self._ct), int(bool(compute_internalized)))
        g = (ctypes.c_int * 3)()
        self._fn("grid_shape")(self._h, g)
        self.grid = tuple(int(t) for t in g)
        self.voxel_count = self.grid[0] * self.grid[1] * self.grid[2]
        self.agents_count = 0

    def _fn(self, name):
        return getattr(self._lib, f"oracle_{self._suf}_{name}")

    def close(self):
        if getattr(self, "_h", None):
            self._fn("destroy")(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    # -- Dirichlet -----------------------------------------------------------------------------
    def set_boundary_dirichlet(self, dim, is_max, values, conditions):
        if values is None:
            self._fn("set_boundary_dirichlet")(self._h, dim, int(is_max), None, None)
            return
        v = np.ascontiguousarray(values, dtype=self.dtype)
        c = np.ascontiguousarray(conditions, dtype=np.uint8)
        self._fn("set_boundary_dirichlet")(self._h, dim, int(is_max), _ptr(v, self._ct), _ptr(c, ctypes.c_uint8))

    def set_interior_dirichlet(self, voxels, values, conditions):
        vox = np.ascontiguousarray(voxels, dtype=np.int32).reshape(-1)
        n = vox.size // self.dims
        v = np.ascontiguousarray(values, dtype=self.dtype).reshape(-1)
        c = np.ascontiguousarray(conditions, dtype=np.uint8).reshape(-1)
        self._fn("set_interior_dirichlet")(self._h, n, _ptr(vox, ctypes.c_int), _ptr(v, self._ct),
                                           _ptr(c, ctypes.c_uint8))

    # -- state ---------------------------------------------------------------------------------
    def initialize(self):
        self._fn("initialize")(self._h)

    def set_densities(self, arr):
        a = np.ascontiguousarray(arr, dtype=self.dtype).reshape(-1)
        assert a.size == self.voxel_count * self.S
        self._fn("set_densities")(self._h, _ptr(a, self._ct))

    def densities(self):
        out = np.empty(self.voxel_count * self.S, dtype=self.dtype)
        self._fn("get_densities")(self._h, _ptr(out, self._ct))
        return out

    def gradients(self):
        out = np.empty(self.voxel_count * self.S * self.dims, dtype=self.dtype)
        self._fn("get_gradients")(self._h, _ptr(out, self._ct))
        return out

    def set_agents(self, secretion_rates, saturation_densities, uptake_rates, net_export_rates,
                   internalized, fraction_released, volumes, positions):
        arrs = [np.ascontiguousarray(a, dtype=self.dtype).reshape(-1) for a in
                (secretion_rates, saturation_densities, uptake_rates, net_export_rates, internalized,
                 fraction_released, volumes, positions)]
        n = arrs[6].size
        self._keep = arrs
        self.agents_count = n
        self._fn("set_agents")(self._h, n, *[_ptr(a, self._ct) for a in arrs])

    def add_agents(self, count, secretion_rates=None, saturation_densities=None, uptake_rates=None,
                   net_export_rates=None, internalized=None, fraction_released=None, volumes=None, positions=None):
        """agent_data::add `count` times (src/agent_data.cpp:10-25), the new rows set to these values;
        an array left None stays 0."""
        count = int(count)
        arrs = [None if a is None else np.ascontiguousarray(a, dtype=self.dtype).reshape(-1) for a in
                (secretion_rates, saturation_densities, uptake_rates, net_export_rates, internalized,
                 fraction_released, volumes, positions)]
        self._fn("add_agents")(self._h, count, *[None if a is None else _ptr(a, self._ct) for a in arrs])
        self.agents_count += count

    def remove_agent(self, index):
        """agent_data::remove (src/agent_data.cpp:27-53): the last agent moves into the freed slot."""
        self._fn("remove_agent")(self._h, int(index))
        self.agents_count -= 1

    def internalized(self):
        out = np.empty(self.agents_count * self.S, dtype=self.dtype)
        self._fn("get_internalized")(self._h, _ptr(out, self._ct))
        return out

    # -- solvers -------------------------------------------------------------------------------
    def diffusion(self):
        self._fn("diffusion")(self._h)

    def dirichlet(self):
        self._fn("dirichlet")(self._h)

    def gradient(self):
        self._fn("gradient")(self._h)

    def secretion(self, recompute):
        self._fn("secretion")(self._h, int(bool(recompute)))

    def release(self, index):
        self._fn("release")(self._h, int(index))

    def run_steps(self, steps, first_step=0):
        self._fn("run_steps")(self._h, int(steps), int(first_step))

    def bulk(self, supply_rates, uptake_rates, supply_target_densities, per_voxel):
        """Bulk supply/uptake with tabulated rates: [voxel][s] when per_voxel, else [s]."""
        n = self.voxel_count * self.S if per_voxel else self.S
        arrs = [np.ascontiguousarray(a, dtype=self.dtype).reshape(-1) for a in
                (supply_rates, uptake_rates, supply_target_densities)]
        assert all(a.size == n for a in arrs)
        self._fn("bulk")(self._h, *[_ptr(a, self._ct) for a in arrs], int(bool(per_voxel)))

    @property
    def is_conflict(self):
        return bool(self._fn("is_conflict")(self._h))
