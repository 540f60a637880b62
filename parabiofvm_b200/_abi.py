"""ctypes declarations of the C ABI in include/bfvm.h (libbfvm_cuda.so).

The library is built in-tree by ``parabiofvm_b200/build.py``.  There is no CPU fallback: if the
library is missing or cannot be loaded, ``load()`` raises.
"""

from __future__ import annotations

import ctypes
import os

PKG = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(PKG, "_lib", "libbfvm_cuda.so")
HEADER = os.path.join(os.path.dirname(PKG), "include", "bfvm.h")

_lib = None

c_int = ctypes.c_int
c_int32 = ctypes.c_int32
c_int64 = ctypes.c_int64
c_float = ctypes.c_float
c_void_p = ctypes.c_void_p
P = ctypes.POINTER

SIGNATURES = {
    "bfvm_last_error": (ctypes.c_char_p, []),
    "bfvm_status_string": (ctypes.c_char_p, [c_int]),
    "bfvm_version": (c_int, []),
    "bfvm_create": (c_int, [P(c_void_p), c_int, c_int, P(c_int32), P(c_int32), P(c_int32), c_int32, c_float,
                            P(c_float), P(c_float), c_int]),
    "bfvm_destroy": (c_int, [c_void_p]),
    "bfvm_get_shape": (c_int, [c_void_p, P(c_int32), P(c_int64), P(c_int32), P(c_int32)]),
    "bfvm_set_stream": (c_int, [c_void_p, c_void_p]),
    "bfvm_set_boundary_dirichlet": (c_int, [c_void_p, c_int, c_int, P(c_float), P(ctypes.c_uint8)]),
    "bfvm_set_interior_dirichlet": (c_int, [c_void_p, c_int32, P(c_int32), P(c_float), P(ctypes.c_uint8)]),
    "bfvm_store_densities": (c_int, [c_void_p, P(c_float)]),
    "bfvm_load_densities": (c_int, [c_void_p, P(c_float)]),
    "bfvm_load_gradients": (c_int, [c_void_p, P(c_float)]),
    "bfvm_store_densities_device": (c_int, [c_void_p, c_void_p]),
    "bfvm_load_densities_device": (c_int, [c_void_p, c_void_p]),
    "bfvm_store_agents": (c_int, [c_void_p, c_int32] + [P(c_float)] * 8),
    "bfvm_store_agent_positions": (c_int, [c_void_p, c_int32, P(c_float)]),
    "bfvm_load_internalized": (c_int, [c_void_p, P(c_float)]),
    "bfvm_store_agent_positions_async": (c_int, [c_void_p, c_int32, P(c_float)]),
    "bfvm_load_internalized_async": (c_int, [c_void_p, P(c_float)]),
    "bfvm_diffusion_solve": (c_int, [c_void_p]),
    "bfvm_diffusion_sweep": (c_int, [c_void_p, c_int]),
    "bfvm_dirichlet_solve": (c_int, [c_void_p]),
    "bfvm_gradient_solve": (c_int, [c_void_p]),
    "bfvm_diffusion_gradient_solve": (c_int, [c_void_p]),
    "bfvm_secretion_solve": (c_int, [c_void_p, c_int]),
    "bfvm_release_internalized": (c_int, [c_void_p, c_int32]),
    "bfvm_add_agents": (c_int, [c_void_p, c_int32] + [P(c_float)] * 8),
    "bfvm_remove_agents": (c_int, [c_void_p, c_int32, P(c_int32)]),
    "bfvm_plan_agent_removal": (c_int, [c_int32, c_int32, P(c_int32), P(c_int32), P(c_int32), P(c_int32),
                                        P(c_int32)]),
    "bfvm_set_bulk_rates": (c_int, [c_void_p, c_int, P(c_float), P(c_float), P(c_float)]),
    "bfvm_bulk_solve": (c_int, [c_void_p]),
    "bfvm_run_steps": (c_int, [c_void_p, c_int32, c_int32]),
    "bfvm_synchronize": (c_int, [c_void_p]),
    "bfvm_set_option": (c_int, [c_void_p, ctypes.c_char_p, c_int64]),
    "bfvm_autotune": (c_int, [c_void_p, P(c_int32)]),
    "bfvm_device_densities": (c_int, [c_void_p, P(P(c_float)), P(c_int64)]),
    "bfvm_device_gradients": (c_int, [c_void_p, P(P(c_float)), P(c_int64)]),
    "bfvm_launch_count": (c_int, [c_void_p, P(c_int64)]),
    "bfvm_batch_create": (c_int, [P(c_void_p), c_int32, P(c_void_p)]),
    "bfvm_batch_destroy": (c_int, [c_void_p]),
    "bfvm_batch_run_steps": (c_int, [c_void_p, c_int32, c_int32]),
    "bfvm_batch_synchronize": (c_int, [c_void_p]),
    "bfvm_batch_autotune": (c_int, [c_void_p, P(c_int32)]),
    "bfvm_create_slab": (c_int, [P(c_void_p), c_int, P(c_int32), P(c_int32), P(c_int32), c_int32, c_float,
                                 P(c_float), P(c_float), c_int, c_int32, P(c_int32), c_int32]),
    "bfvm_slab_info": (c_int, [c_void_p, P(c_int32), P(c_int32), P(c_int32), P(c_int32)]),
    "bfvm_slab_diffusion_begin": (c_int, [c_void_p, c_void_p]),
    "bfvm_slab_diffusion_end": (c_int, [c_void_p, c_void_p]),
    "bfvm_slab_edge_planes": (c_int, [c_void_p, c_void_p, c_void_p]),
    "bfvm_slab_gradient_solve": (c_int, [c_void_p, c_void_p, c_void_p]),
    "bfvm_slab_coefficients": (c_int, [c_int32, c_int32, c_int32, c_float, P(c_float), P(c_float), c_int32,
                                       P(c_int32), P(c_float)]),
    "bfvm_slab_reduce_weights": (c_int, [c_int32, c_int32, c_int32, c_float, P(c_float), P(c_float), c_int32,
                                         c_int32, P(c_float), P(c_int32), P(c_int32), P(c_int32)]),
    "bfvm_sur_create": (c_int, [P(c_void_p), c_int, P(c_int32), c_int32, c_int32, ctypes.c_uint64]),
    "bfvm_sur_destroy": (c_int, [c_void_p]),
    "bfvm_sur_set_stream": (c_int, [c_void_p, c_void_p]),
    "bfvm_sur_parameter_count": (c_int, [c_void_p, P(c_int64)]),
    "bfvm_sur_load": (c_int, [c_void_p, P(c_float)]),
    "bfvm_sur_save": (c_int, [c_void_p, P(c_float)]),
    "bfvm_sur_infer": (c_int, [c_void_p, c_int32] + [c_void_p] * 4),
    "bfvm_sur_gradients": (c_int, [c_void_p, c_int32] + [c_void_p] * 5 + [P(c_float)]),
    "bfvm_sur_load_gradients": (c_int, [c_void_p, P(c_float)]),
    "bfvm_sur_train_step": (c_int, [c_void_p, c_int32] + [c_void_p] * 5 + [c_float, P(c_float)]),
    "bfvm_sur_synchronize": (c_int, [c_void_p]),
    "bfvm_sur_agent_rates": (c_int, [P(c_int32), P(c_int32), P(c_int32), c_int32, c_float, c_int32]
                             + [c_void_p] * 8 + [c_void_p, c_void_p]),
    "bfvm_sur_random_field": (c_int, [P(c_int32), c_int32, c_int32, P(c_float), c_void_p, c_void_p]),
    "bfvm_sur_conv3d": (c_int, [P(c_int32), c_void_p, c_void_p, c_void_p, c_void_p, c_int32, c_void_p, c_void_p,
                                c_void_p, c_void_p, c_int32, c_void_p, c_void_p]),
    "bfvm_sur_conv3d_wgrad": (c_int, [P(c_int32)] + [c_void_p] * 5),
    "bfvm_secretion_solve_noalloc": (c_int, [c_void_p, c_int, P(c_int32), P(c_int32), P(c_int32), c_int32, c_float,
                                             c_int32] + [c_void_p] * 8 + [c_void_p]),
}


class BfvmError(RuntimeError):
    def __init__(self, status, message):
        super().__init__(f"{message} (status {status})")
        self.status = status


def load():
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise RuntimeError(f"CUDA library {LIB_PATH} is not built; run `python parabiofvm_b200/build.py`")
    lib = ctypes.CDLL(LIB_PATH)
    for name, (res, args) in SIGNATURES.items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    _lib = lib
    return lib


def check(status: int):
    if status != 0:
        lib = load()
        raise BfvmError(status, lib.bfvm_last_error().decode() or lib.bfvm_status_string(status).decode())


def header_functions(path: str = HEADER):
    """Names of the functions declared in include/bfvm.h."""
    import re

    with open(path) as f:
        text = f.read()
    return sorted(set(re.findall(r"^\s*(?:const\s+)?\w+\**\s+\**(bfvm_\w+)\s*\(", text, flags=re.M)))
