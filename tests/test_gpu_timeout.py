"""The bounded waits of the staged sweeps, run out on purpose without faulting the GPU.

Every wait of a staged sweep on a tile copy is bounded (option "wait_limit_cycles").  The test-only
option "test_drop_tile_copy" arms the stage barrier of one tile without issuing its copies, so no
copy is ever in flight toward that stage and its wait runs out after the (short) limit.  The kernel
then gives up the tile, lets its other copies land, and returns; the next synchronising call
reports BFVM_ERR_TIMEOUT instead of the reference's abort() (src/solver/device/CUDA/
device_context.h:12-21).  With the options cleared and the field stored again, the same solver
steps bit for bit like a fresh one: the context and the solver survive the timeout.
"""

import numpy as np
import pytest

from parabiofvm_b200._abi import BfvmError
from parabiofvm_b200.workloads import make_solver, synthetic

pytestmark = pytest.mark.gpu

BFVM_ERR_TIMEOUT = 7


@pytest.mark.parametrize("axis", [0, 1, 2])
def test_sweep_wait_runs_out_and_solver_recovers(axis):
    from parabiofvm_b200 import _abi

    assert _abi.load().bfvm_status_string(BFVM_ERR_TIMEOUT).decode().lower().find("time") >= 0
    w = synthetic(64, 4, 3000, seed=31 + axis, clustered=True, sigma=100.0, interior_fraction=0.01)
    s = make_solver(w)
    fresh = make_solver(w)
    s.set_option("wait_limit_cycles", 2_000_000)  # about a millisecond
    s.set_option("test_drop_tile_copy", 0)
    with pytest.raises(BfvmError) as e:
        s.sweep(axis)
        s.synchronize()
    assert e.value.status == BFVM_ERR_TIMEOUT, str(e.value)
    # the error is reported once; the solver keeps working
    s.synchronize()
    s.set_option("test_drop_tile_copy", -1)
    s.set_option("wait_limit_cycles", 4_000_000_000)
    s.store_densities(w.densities)
    s.run_steps(3, 0)
    fresh.run_steps(3, 0)
    np.testing.assert_array_equal(s.load_densities(), fresh.load_densities())
    np.testing.assert_array_equal(s.load_gradients(), fresh.load_gradients())
    s.close()
    fresh.close()


def test_wait_limit_option_is_checked():
    w = synthetic(16, 2, 0, seed=1)
    s = make_solver(w)
    for bad in (0, 9999, 40_000_000_001):
        with pytest.raises(BfvmError):
            s.set_option("wait_limit_cycles", bad)
    with pytest.raises(BfvmError):
        s.set_option("test_drop_tile_copy", -2)
    s.close()
